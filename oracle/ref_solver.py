"""ctypes driver of the reference's own solver code, compiled here against stand-in PETSc / MPI /
LAPACKE / Boost headers (oracle/Makefile target ``refsolver`` -> oracle/_ref/libref_solver.so).

Test infrastructure: it pins the oracle's restatement of Simple / Piso / IbPiso
(src/Solvers/Simple.cpp:78-449, Piso.cpp:12-29, IbPiso.cpp:43-190), Coupled
(src/Solvers/Coupled.cpp:5-339) and Diffusion (src/Solvers/Diffusion.cpp:35-131) to the
reference's own arithmetic.  The library exists only where the reference's sources do (it is built from them
where they lie); tests skip when it is absent and fall back to the committed golden vectors.

A case is written as the reference's case/case.info and case/initialConditions.info, the way
its module mains read them (Modules/caffeSimple.cpp:13-30).  The reference has no switch for
convection scheme, non-orthogonal correction or Krylov method: only upwind, orthogonal-only
cases map onto it.  Its KSPSolve is the stand-in's tight solve (restarted GMRES with ILU(0) to
``rtol`` on the true residual, singular all-Neumann systems projected), and every system the
reference assembles is recorded in assembly order.
"""
from __future__ import annotations

import ctypes
import os
import tempfile

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libref_solver.so")
_lib = None

FACES = ("east", "west", "north", "south", "top", "bottom")
KINDS = {"simple": 0, "piso": 1, "ibpiso": 2, "coupled": 3, "diffusion": 4}


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        L = ctypes.CDLL(LIB_PATH)
        vp, ci, cd = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
        L.refsolver_last_error.restype = ctypes.c_char_p
        L.refsolver_set_tolerance.argtypes = [cd, ci]
        L.refsolver_record.argtypes = [ci]
        L.refsolver_nsystems.restype = ci
        L.refsolver_system_size.argtypes = [ci, ctypes.POINTER(ci), ctypes.POINTER(ci)]
        L.refsolver_system.argtypes = [ci, vp, vp, vp, vp, vp]
        L.refsolver_create.restype = vp
        L.refsolver_create.argtypes = [ctypes.c_char_p, vp, ci, ci, ci, ci]
        L.refsolver_destroy.argtypes = [vp]
        L.refsolver_solve.restype = cd
        L.refsolver_solve.argtypes = [vp, cd]
        L.refsolver_field.restype = ctypes.c_long
        L.refsolver_field.argtypes = [vp, ctypes.c_char_p, vp, ctypes.c_long]
        L.refsolver_trilinear.argtypes = [vp, vp, vp]
        L.refsolver_inject.argtypes = [vp, ci]
        L.refsolver_zero_pressure_patch.argtypes = [vp, ci]
        L.refsolver_injected_left.restype = ci
        _lib = L
    return _lib


def _vec(v) -> str:
    return "(" + ",".join(repr(float(x)) for x in v) + ")"


def case_files(spec, directory: str) -> None:
    """case/case.info and case/initialConditions.info for a CaseSpec that the reference can run."""
    if spec.convection != "upwind" or spec.nonorth:
        raise ValueError("the reference has upwind convection and no non-orthogonal correction only")
    os.makedirs(os.path.join(directory, "case"), exist_ok=True)
    lines = ["Solver", "{",
             f"  timeAccurate {'ON' if spec.time_accurate else 'OFF'}",
             f"  relaxationFactorMomentum {spec.omega_u!r}",
             f"  relaxationFactorPCorr {spec.omega_p!r}",
             f"  rho {spec.rho!r}",
             f"  mu {spec.mu!r}",
             f"  numberOfInnerIterations {int(spec.n_inner)}",
             f"  numberOfPressureCorrections {int(spec.n_pcorr)}",
             "}", "Boundaries", "{"]
    for f, name in enumerate(FACES):
        lines += [f"  {name}", "  {", f"    type {spec.bc[f]}", f"    refVector {_vec(spec.ref_vec[f])}",
                  f"    refValue {float(spec.ref_val[f])!r}", "  }"]
    lines.append("}")
    if spec.kind == "ibpiso":
        lines += ["ImmersedBoundaries", "{", "  Sphere", "  {", f"    radius {float(spec.ib_radius)!r}",
                  f"    center {_vec(spec.ib_center)}", "  }", "}"]
    with open(os.path.join(directory, "case", "case.info"), "w") as fh:
        fh.write("\n".join(lines) + "\n")
    ic = ["u", "{", "  type uniform", f"  value {_vec(spec.u_init)}", "}",
          "p", "{", "  type uniform", f"  value {float(spec.p_init)!r}", "}"]
    with open(os.path.join(directory, "case", "initialConditions.info"), "w") as fh:
        fh.write("\n".join(ic) + "\n")


def diffusion_case_files(types, refs, time_accurate: bool, phi0: float, directory: str) -> None:
    """case/case.info and case/initialConditions.info of the reference's Diffusion solver: face
    types fixed / zeroGradient / empty with their reference values, a uniform phi."""
    os.makedirs(os.path.join(directory, "case"), exist_ok=True)
    lines = ["Solver", "{", f"  timeAccurate {'ON' if time_accurate else 'OFF'}", "}", "Boundaries", "{"]
    for f, name in enumerate(FACES):
        lines += [f"  {name}", "  {", f"    type {types[f]}", f"    refValue {float(refs[f])!r}", "  }"]
    lines.append("}")
    with open(os.path.join(directory, "case", "case.info"), "w") as fh:
        fh.write("\n".join(lines) + "\n")
    with open(os.path.join(directory, "case", "initialConditions.info"), "w") as fh:
        fh.write("\n".join(["phi", "{", "  type uniform", f"  value {float(phi0)!r}", "}"]) + "\n")


class RefSolver:
    """The reference's Simple / Piso / IbPiso (the spec's kind), Coupled (kind="coupled") or
    Diffusion (kind="diffusion", with `diffusion` = (types, refs, time_accurate, phi0)) on a
    node array (nK+1, nJ+1, nI+1, 3)."""

    def __init__(self, nodes: np.ndarray, spec, rtol: float = 1e-13, maxit: int = 200000, record: bool = False,
                 kind: str | None = None, diffusion=None):
        L = lib()
        L.refsolver_set_tolerance(float(rtol), int(maxit))
        L.refsolver_record(1 if record else 0)
        self.spec = spec
        self.kind = kind or spec.kind
        self.nodes = np.ascontiguousarray(nodes, dtype=np.float64)
        self.shape = (self.nodes.shape[2] - 1, self.nodes.shape[1] - 1, self.nodes.shape[0] - 1)
        self._dir = tempfile.TemporaryDirectory(prefix="caffe_ref_case_")
        if self.kind == "diffusion":
            diffusion_case_files(*diffusion, self._dir.name)
        else:
            case_files(spec, self._dir.name)
        self._h = L.refsolver_create(self._dir.name.encode(), self.nodes.ctypes.data_as(ctypes.c_void_p),
                                     self.nodes.shape[2], self.nodes.shape[1], self.nodes.shape[0], KINDS[self.kind])
        if not self._h:
            raise RuntimeError("reference solver set-up failed: " + L.refsolver_last_error().decode())
        # faces without a fixed pressure start from the zero that zero-initialised memory gives in
        # place of the reference's uninitialised refValues_ (see refsolver_zero_pressure_patch)
        if self.kind != "diffusion" and any(t == "outlet" for t in spec.bc):
            for f, t in enumerate(spec.bc):
                if t != "outlet":
                    L.refsolver_zero_pressure_patch(self._h, f)

    def close(self):
        if self._h:
            lib().refsolver_destroy(self._h)
            self._h = None
        self._dir.cleanup()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def solve(self, dt: float | None = None) -> float:
        v = lib().refsolver_solve(self._h, float(self.spec.dt if (dt is None and self.spec is not None) else (dt or 1.0)))
        if not np.isfinite(v) and lib().refsolver_last_error():
            raise RuntimeError("reference solve failed: " + lib().refsolver_last_error().decode())
        return float(v)

    def get(self, name: str) -> np.ndarray:
        L = lib()
        n = L.refsolver_field(self._h, name.encode(), None, 0)
        if n < 0:
            raise KeyError(name)
        out = np.empty(n, dtype=np.float64)
        L.refsolver_field(self._h, name.encode(), out.ctypes.data_as(ctypes.c_void_p), n)
        return out


def inject(x: np.ndarray) -> None:
    """Queue a solution: the next KSPSolve the reference's code makes returns it instead of solving."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    lib().refsolver_inject(x.ctypes.data_as(ctypes.c_void_p), int(x.size))


def clear_injected() -> None:
    lib().refsolver_clear_injected()


def injected_left() -> int:
    return int(lib().refsolver_injected_left())


def recorded_systems():
    """Every system KSPSolve received since the last RefSolver was created (or recording was
    switched on): list of (csr_ptr, csr_col, csr_val, b, x)."""
    L = lib()
    out = []
    for k in range(L.refsolver_nsystems()):
        n, nnz = ctypes.c_int(0), ctypes.c_int(0)
        L.refsolver_system_size(k, ctypes.byref(n), ctypes.byref(nnz))
        ptr = np.empty(n.value + 1, dtype=np.int32)
        col = np.empty(nnz.value, dtype=np.int32)
        val = np.empty(nnz.value, dtype=np.float64)
        b = np.empty(n.value, dtype=np.float64)
        x = np.empty(n.value, dtype=np.float64)
        L.refsolver_system(k, *(a.ctypes.data_as(ctypes.c_void_p) for a in (ptr, col, val, b, x)))
        out.append((ptr, col, val, b, x))
    return out


def trilinear(p8: np.ndarray, ip) -> np.ndarray:
    """Interpolation::computeTrilinearCoeffs (src/Math/Interpolation.cpp:135-180)."""
    p = np.ascontiguousarray(p8, dtype=np.float64).reshape(8, 3)
    q = np.ascontiguousarray(ip, dtype=np.float64).reshape(3)
    beta = np.empty(8, dtype=np.float64)
    if lib().refsolver_trilinear(p.ctypes.data_as(ctypes.c_void_p), q.ctypes.data_as(ctypes.c_void_p),
                                 beta.ctypes.data_as(ctypes.c_void_p)):
        raise RuntimeError(lib().refsolver_last_error().decode())
    return beta
