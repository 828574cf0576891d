"""Lock-step comparison of the oracle's Coupled and Diffusion restatements with the reference's
own solver code (src/Solvers/Coupled.cpp, src/Solvers/Diffusion.cpp, compiled into
oracle/_ref/libref_solver.so by oracle/Makefile).

The oracle takes a step phase by phase and keeps every linear system it assembles and every
solution its Krylov solver returns.  The reference then takes the same step with its KSPSolve
handing back the oracle's solutions in the same order, so both continue from identical numbers
and everything outside the Krylov solves -- the block rows with Rhie-Chow coupling, the boundary
folding, the diffusion rows on a skewed mesh, the post-solve fields, gradients and face values --
is compared bit for bit.
"""
from __future__ import annotations

import numpy as np
import pytest

from caffe_old_b200 import cases as C
from oracle import oracle as O
from oracle import ref_solver as R

needs_reference = pytest.mark.skipif(not R.available(), reason="the reference's sources are not compiled here")

RTOL = 1e-12


def _rows_from_oracle_csr(o):
    cnt, col, val = o.system()
    return [{int(col[r, p]): float(val[r, p]) for p in range(cnt[r])} for r in range(len(cnt))]


def _rows_from_csr(ptr, col, val):
    return [{int(col[p]): float(val[p]) for p in range(ptr[r], ptr[r + 1])} for r in range(len(ptr) - 1)]


def _nonzero(rows):
    # PETSc keeps explicit zeros of a row's structure after MatZeroEntries; compare the values
    return [{c: v for c, v in r.items() if v != 0.0} for r in rows]


def _coupled_cavity2d():
    nodes = C.cartesian_nodes((10, 8, 1), (1.0, 1.0, 1.0 / 8))
    bc, ref = C.lid_cavity_bcs("north", lid_velocity=(1.0, 0.0, 0.0), two_d=True)
    spec = C.CaseSpec(kind="simple", bc=bc, ref_vec=ref, rho=1.0, mu=0.01, time_accurate=False, omega_u=0.7, omega_p=0.3,
                      mom_method="bicgstab_jacobi", p_method="bicgstab_jacobi", mom_rtol=RTOL, p_rtol=RTOL, maxit=20000, dt=1.0)
    return nodes, spec


def _coupled_skewed3d():
    nodes = C.skewed_nodes((7, 6, 5), (1.0, 1.0, 1.0), 30.0, 0.1, 5)
    bc, ref = C.lid_cavity_bcs("north")
    spec = C.CaseSpec(kind="simple", bc=bc, ref_vec=ref, rho=1.3, mu=0.02, time_accurate=True, n_inner=2, omega_u=0.8,
                      omega_p=0.3, mom_method="bicgstab_jacobi", p_method="bicgstab_jacobi", mom_rtol=RTOL, p_rtol=RTOL,
                      maxit=20000, dt=0.05)
    return nodes, spec


def _coupled_channel():
    nodes = C.cartesian_nodes((12, 6, 5), (3.0, 1.0, 1.0))
    bc, ref = C.channel_bcs(1.0)
    spec = C.CaseSpec(kind="simple", bc=bc, ref_vec=ref, ref_val=(0.25, 0, 0, 0, 0, 0), rho=1.0, mu=0.05,
                      time_accurate=False, omega_u=0.7, omega_p=0.3, mom_method="bicgstab_jacobi",
                      p_method="bicgstab_jacobi", mom_rtol=RTOL, p_rtol=RTOL, maxit=20000, dt=1.0)
    return nodes, spec


COUPLED_CASES = {"cavity2d": _coupled_cavity2d, "skewed3d": _coupled_skewed3d, "channel": _coupled_channel}
COUPLED_FIELDS = ("u", "p", "gradP", "h", "d", "massFlowI", "massFlowJ", "massFlowK")


@needs_reference
@pytest.mark.parametrize("name", COUPLED_CASES)
def test_coupled_lockstep_bit_exact_with_reference_code(name):
    nodes, spec = COUPLED_CASES[name]()
    o = O.OracleCoupled(nodes, spec)
    r = R.RefSolver(nodes, spec, record=True, kind="coupled")
    inner = spec.n_inner if spec.time_accurate else 1
    try:
        for step in range(3):
            o.phase("save_u0")
            systems, sols = [], []
            for _ in range(inner):
                o.phase("assemble")
                systems.append((_nonzero(_rows_from_oracle_csr(o)), o.get("b")))
                o.phase("solve")
                sols.append(o.get("x"))
                o.phase("post")
            R.clear_injected()
            R.lib().refsolver_record(1)
            for x in sols:
                R.inject(x)
            r.solve(spec.dt)
            assert R.injected_left() == 0, (name, step)
            rec = R.recorded_systems()
            assert len(rec) == inner, (name, step, len(rec))
            for s, ((ptr, col, val, b, _), (rows, ob)) in enumerate(zip(rec, systems)):
                assert _nonzero(_rows_from_csr(ptr, col, val)) == rows, (name, step, s)
                assert np.array_equal(b, ob), (name, step, s)
            for nm in COUPLED_FIELDS:
                assert np.array_equal(r.get(nm), o.get(nm)), (name, step, nm)
    finally:
        r.close()
        o.close()


DIFFUSION_TYPES = ["fixed", "zeroGradient", "fixed", "zeroGradient", "empty", "zeroGradient"]
DIFFUSION_VALUES = [2.0, 0.0, -1.0, 0.0, 0.0, 0.0]


def _diffusion_rows(A, shape):
    """The oracle's (cells x 7) coefficients (self, east, west, north, south, top, bottom) as
    rows {column: value} of the global matrix."""
    nI, nJ, nK = shape
    A = A.reshape(-1, 7)
    rows = []
    for c in range(A.shape[0]):
        i, j, k = c % nI, (c // nI) % nJ, c // (nI * nJ)
        nb = [c, c + 1 if i < nI - 1 else None, c - 1 if i > 0 else None, c + nI if j < nJ - 1 else None,
              c - nI if j > 0 else None, c + nI * nJ if k < nK - 1 else None, c - nI * nJ if k > 0 else None]
        rows.append({nb[q]: float(A[c, q]) for q in range(7) if nb[q] is not None and A[c, q] != 0.0})
    return rows


@needs_reference
@pytest.mark.parametrize("skewed,time_accurate", [(False, False), (True, True), (True, False)])
def test_diffusion_lockstep_bit_exact_with_reference_code(skewed, time_accurate):
    nodes = (C.skewed_nodes((9, 7, 6), (1.0, 1.0, 1.0), 30.0, 0.1, 4) if skewed
             else C.cartesian_nodes((9, 7, 6), (1.0, 1.0, 0.5)))
    phi0 = 0.7 if time_accurate else 0.0
    o = O.OracleDiffusion(nodes, DIFFUSION_TYPES, DIFFUSION_VALUES, time_accurate=time_accurate, phi0=phi0,
                          method="bicgstab_jacobi", rtol=1e-13, maxit=20000)
    r = R.RefSolver(nodes, None, record=True, kind="diffusion",
                    diffusion=(DIFFUSION_TYPES, DIFFUSION_VALUES, time_accurate, phi0))
    try:
        for step in range(3 if time_accurate else 1):
            o.solve(0.05)
            R.clear_injected()
            R.lib().refsolver_record(1)
            R.inject(o.get("phi"))
            r.solve(0.05)
            rec = R.recorded_systems()
            assert len(rec) == 1
            ptr, col, val, b, _ = rec[0]
            assert _nonzero(_rows_from_csr(ptr, col, val)) == _diffusion_rows(o.get("A"), o.shape), step
            assert np.array_equal(b, o.get("b")), step
            for nm in ("phi", "gradPhi", "phiFaceI", "phiFaceJ", "phiFaceK"):
                assert np.array_equal(r.get(nm), o.get(nm)), (step, nm)
    finally:
        r.close()
        o.close()
