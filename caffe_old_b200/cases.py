"""Case descriptions and structured-mesh node generators.

A case mirrors the keys CAFFE reads from ``case/case.info`` (``Solver.*``,
``Boundaries.<face>.{type,refVector,refValue}``, ``ImmersedBoundaries.Sphere.*``;
see src/Solvers/Solver.cpp:8, src/Solvers/Simple.cpp:61-67,104-108,
src/Solvers/Piso.cpp:9, src/Domains/Field/FlowBoundaryConditions.cpp:25-40 and
src/Solvers/IbPiso.cpp:37-38) plus the linear-solver selection that the
reference leaves to PETSc defaults.

Face order everywhere is east, west, north, south, top, bottom (+i, -i, +j, -j,
+k, -k), as in HexaFvmMesh::Direction (src/Domains/HexaFvmMesh/HexaFvmMesh.h:44).

Node arrays are float64 of shape (nK+1, nJ+1, nI+1, 3), i fastest, the order
StructuredMesh reads a Tecplot BLOCK file in (StructuredMesh.cpp:48-60).
"""
from __future__ import annotations

import dataclasses
import math
from typing import Sequence

import numpy as np

FACES = ("east", "west", "north", "south", "top", "bottom")
FLOW_TYPES = {"inlet": 0, "outlet": 1, "wall": 2, "empty": 3, "zeroGradient": 4}
SOLVER_KINDS = {"simple": 0, "piso": 1, "ibpiso": 2}
CONVECTION = {"upwind": 0, "central": 1}
# Krylov methods.  bicgstab_sgs is the reference's own choice (PETSc KSPBCGS with
# PCSOR, src/Math/SparseMatrix.cpp:95-100); the GPU path implements the others.
KSP_METHODS = {"bicgstab_sgs": 0, "bicgstab_jacobi": 1, "cg_jacobi": 2}
# Precision / preconditioner form of the pressure-correction solve on the GPU.
P_FORMS = {"fp64": 0, "mixed": 1, "learned": 2, "learned_mixed": 3}


@dataclasses.dataclass
class CaseSpec:
    kind: str = "simple"
    bc: tuple = ("wall",) * 6
    ref_vec: tuple = ((0.0, 0.0, 0.0),) * 6
    ref_val: tuple = (0.0,) * 6
    rho: float = 1.0
    mu: float = 0.01
    time_accurate: bool = False
    omega_u: float = 0.7
    omega_p: float = 0.3
    n_inner: int = 1
    n_pcorr: int = 1
    convection: str = "upwind"
    nonorth: bool = False
    mom_method: str = "bicgstab_jacobi"
    p_method: str = "bicgstab_jacobi"
    mom_rtol: float = 1e-8
    p_rtol: float = 1e-8
    maxit: int = 20000
    ib_radius: float = 0.0
    ib_center: tuple = (0.0, 0.0, 0.0)
    u_init: tuple = (0.0, 0.0, 0.0)
    p_init: float = 0.0
    dt: float = 1.0
    p_form: str = "fp64"
    # absolute floors of the linear solves, ||b - A x|| <= max(rtol ||b||, atol) (PETSc's test)
    mom_atol: float = 0.0
    p_atol: float = 0.0

    def replace(self, **kw) -> "CaseSpec":
        return dataclasses.replace(self, **kw)

    def validate(self) -> None:
        if self.kind not in SOLVER_KINDS:
            raise ValueError(f"unknown solver kind {self.kind!r}")
        if len(self.bc) != 6 or any(b not in FLOW_TYPES for b in self.bc):
            raise ValueError(f"invalid boundary types {self.bc!r}")
        if self.convection not in CONVECTION:
            raise ValueError(f"unknown convection scheme {self.convection!r}")
        for m in (self.mom_method, self.p_method):
            if m not in KSP_METHODS:
                raise ValueError(f"unknown Krylov method {m!r}")
        if self.p_form not in P_FORMS:
            raise ValueError(f"unknown pressure-solve form {self.p_form!r}")
        if self.kind == "ibpiso" and self.ib_radius <= 0.0:
            raise ValueError("ibpiso needs a sphere radius > 0")
        if not (self.mom_atol >= 0.0 and self.p_atol >= 0.0):
            raise ValueError("absolute tolerances must be >= 0")


# ---------------------------------------------------------------------------
# node generators
# ---------------------------------------------------------------------------
def cartesian_nodes(n_cells: Sequence[int], lengths: Sequence[float]) -> np.ndarray:
    """Uniform box with the node coordinates of StructuredMesh::initializeCartesianMesh
    (src/Domains/HexaFvmMesh/StructuredMesh.cpp:131-148): x = i*hx with hx = L/(nNodes-1)."""
    nI, nJ, nK = (int(v) for v in n_cells)
    hx, hy, hz = (float(lengths[q]) / float(n) for q, n in enumerate((nI, nJ, nK)))
    i = np.arange(nI + 1, dtype=np.float64) * hx
    j = np.arange(nJ + 1, dtype=np.float64) * hy
    k = np.arange(nK + 1, dtype=np.float64) * hz
    out = np.empty((nK + 1, nJ + 1, nI + 1, 3), dtype=np.float64)
    out[..., 0] = i[None, None, :]
    out[..., 1] = j[None, :, None]
    out[..., 2] = k[:, None, None]
    return out


def skewed_nodes(n_cells: Sequence[int], lengths: Sequence[float], shear_deg: float = 30.0,
                 jitter: float = 0.1, seed: int = 0) -> np.ndarray:
    """Box sheared in the x-z plane (x += z tan(shear)), with a seeded uniform jitter of
    up to ``jitter`` times the local spacing on interior nodes only (boundary nodes stay
    on the sheared box faces)."""
    nodes = cartesian_nodes(n_cells, lengths)
    nI, nJ, nK = (int(v) for v in n_cells)
    h = np.array([float(lengths[q]) / float(n) for q, n in enumerate((nI, nJ, nK))])
    rng = np.random.default_rng(seed)
    if jitter > 0.0 and nI > 1 and nJ > 1 and nK > 1:
        inner = nodes[1:-1, 1:-1, 1:-1]
        inner += rng.uniform(-jitter, jitter, size=inner.shape) * h[None, None, None, :]
    nodes[..., 0] += nodes[..., 2] * math.tan(math.radians(shear_deg))
    return nodes


# ---------------------------------------------------------------------------
# the five benchmark configurations, at full or reduced size
# ---------------------------------------------------------------------------
def lid_cavity_bcs(lid_face: str = "north", lid_velocity=(1.0, 0.0, 0.0), two_d: bool = False):
    bc = ["wall"] * 6
    ref = [(0.0, 0.0, 0.0)] * 6
    ref[FACES.index(lid_face)] = tuple(float(v) for v in lid_velocity)
    if two_d:
        bc[4] = bc[5] = "empty"
    return tuple(bc), tuple(ref)


def config1_cavity2d(n: int = 64, iters: int = 500) -> tuple[np.ndarray, CaseSpec, int]:
    """2-D lid-driven cavity, Re=100, steady SIMPLE, upwind, 0.7/0.3 relaxation."""
    nodes = cartesian_nodes((n, n, 1), (1.0, 1.0, 1.0 / n))
    bc, ref = lid_cavity_bcs("north", two_d=True)
    spec = CaseSpec(kind="simple", bc=bc, ref_vec=ref, rho=1.0, mu=0.01, time_accurate=False,
                    omega_u=0.7, omega_p=0.3, convection="upwind", mom_method="bicgstab_jacobi",
                    p_method="bicgstab_jacobi", mom_rtol=1e-8, p_rtol=1e-8, dt=1.0)
    return nodes, spec, iters


def config2_cavity3d(n: int = 128, steps: int = 200) -> tuple[np.ndarray, CaseSpec, int]:
    """3-D lid-driven cavity, Re=400, PISO (1 inner, 2 correctors), central, Jacobi-PCG p'."""
    nodes = cartesian_nodes((n, n, n), (1.0, 1.0, 1.0))
    bc, ref = lid_cavity_bcs("north")
    spec = CaseSpec(kind="piso", bc=bc, ref_vec=ref, rho=1.0, mu=0.0025, time_accurate=True,
                    omega_u=1.0, omega_p=1.0, n_inner=1, n_pcorr=2, convection="central",
                    mom_method="bicgstab_jacobi", p_method="cg_jacobi", mom_rtol=1e-8, p_rtol=1e-8,
                    dt=1e-3)
    return nodes, spec, steps


def config3_skewed(n: int = 128, steps: int = 200, seed: int = 0, p_form: str = "mixed"):
    """Sheared (30 deg) and jittered cavity, non-orthogonal correction on, Re=400 PISO."""
    nodes = skewed_nodes((n, n, n), (1.0, 1.0, 1.0), 30.0, 0.1, seed)
    bc, ref = lid_cavity_bcs("north")
    spec = CaseSpec(kind="piso", bc=bc, ref_vec=ref, rho=1.0, mu=0.0025, time_accurate=True,
                    omega_u=1.0, omega_p=1.0, n_inner=1, n_pcorr=2, convection="central", nonorth=True,
                    mom_method="bicgstab_jacobi", p_method="cg_jacobi", mom_rtol=1e-8, p_rtol=1e-8,
                    dt=5e-4, p_form=p_form)
    return nodes, spec, steps


def channel_bcs(u_in: float = 1.0):
    bc = ("outlet", "inlet", "wall", "wall", "wall", "wall")
    ref = ((0.0, 0.0, 0.0), (u_in, 0.0, 0.0)) + ((0.0, 0.0, 0.0),) * 4
    return bc, ref


def config4_channel_sphere(dims=(256, 128, 128), seed: int = 0, steps: int = 50):
    """Channel 4x1x1 with an immersed sphere R=0.1 at (1, 0.5, 0.5); Re ~ U[100, 300] from
    the seed, mu = rho U (2R) / Re (diameter-based Reynolds number).  Solver settings follow
    the reference's immersed-boundary example cases (ExampleCases/*IbSphere/case/case.info):
    upwind convection (the reference's momentum scheme), the field started at the inlet
    velocity, under-relaxation and inner iterations; without them (relaxation 1, one inner
    iteration) the IB-PISO scheme diverges within a few dozen steps."""
    rng = np.random.default_rng(seed)
    re = float(rng.uniform(100.0, 300.0))
    nodes = cartesian_nodes(dims, (4.0, 1.0, 1.0))
    bc, ref = channel_bcs(1.0)
    spec = CaseSpec(kind="ibpiso", bc=bc, ref_vec=ref, rho=1.0, mu=1.0 * 0.2 / re, time_accurate=True,
                    omega_u=0.7, omega_p=0.3, n_inner=2, n_pcorr=2, convection="upwind",
                    mom_method="bicgstab_jacobi", p_method="bicgstab_jacobi", mom_rtol=1e-8, p_rtol=1e-8,
                    dt=2e-3, ib_radius=0.1, ib_center=(1.0, 0.5, 0.5), u_init=(1.0, 0.0, 0.0))
    return nodes, spec, steps


def config5_sphere(dims=(384, 256, 256), steps: int = 500, p_form: str = "learned_mixed", re: float = 300.0):
    """Flow over an immersed sphere R=0.25 at (2,2,2) in an 8x4x4 box, Re=300 (diameter-based;
    `re` changes it), PISO with 3 correctors, dt=2e-3; the same stabilising settings as the
    channel case."""
    nodes = cartesian_nodes(dims, (8.0, 4.0, 4.0))
    bc, ref = channel_bcs(1.0)
    spec = CaseSpec(kind="ibpiso", bc=bc, ref_vec=ref, rho=1.0, mu=0.5 / float(re), time_accurate=True,
                    omega_u=0.7, omega_p=0.3, n_inner=2, n_pcorr=3, convection="upwind",
                    mom_method="bicgstab_jacobi", p_method="bicgstab_jacobi", mom_rtol=1e-8, p_rtol=1e-8,
                    dt=2e-3, ib_radius=0.25, ib_center=(2.0, 2.0, 2.0), p_form=p_form, u_init=(1.0, 0.0, 0.0))
    return nodes, spec, steps
