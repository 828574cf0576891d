"""TEST INFRASTRUCTURE ONLY -- ctypes binding of the CPU oracle (oracle.cpp).

The oracle restates CAFFE's SIMPLE / PISO / IB-PISO hot path on the CPU; it is the
checker of the CUDA library and the timed CPU baseline, never part of the product.
Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference legs
use this module.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None


def build() -> str:
    subprocess.run(["make", "-C", _HERE, "-s"], check=True)
    return _LIB_PATH


class OracleCase(ctypes.Structure):
    _fields_ = [
        ("kind", ctypes.c_int),
        ("bc_type", ctypes.c_int * 6),
        ("ref_vec", (ctypes.c_double * 3) * 6),
        ("ref_val", ctypes.c_double * 6),
        ("rho", ctypes.c_double), ("mu", ctypes.c_double),
        ("time_accurate", ctypes.c_int),
        ("omega_u", ctypes.c_double), ("omega_p", ctypes.c_double),
        ("n_inner", ctypes.c_int), ("n_pcorr", ctypes.c_int),
        ("convection", ctypes.c_int), ("nonorth", ctypes.c_int),
        ("mom_method", ctypes.c_int), ("p_method", ctypes.c_int),
        ("mom_rtol", ctypes.c_double), ("p_rtol", ctypes.c_double),
        ("maxit", ctypes.c_int),
        ("ib_radius", ctypes.c_double), ("ib_center", ctypes.c_double * 3),
        ("u_init", ctypes.c_double * 3), ("p_init", ctypes.c_double),
        ("mom_atol", ctypes.c_double), ("p_atol", ctypes.c_double),
    ]


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        L.oracle_create.restype = ctypes.c_void_p
        L.oracle_create.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(OracleCase)]
        L.oracle_destroy.argtypes = [ctypes.c_void_p]
        L.oracle_solve.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.POINTER(ctypes.c_double)]
        L.oracle_phase.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_double]
        L.oracle_stats.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.oracle_array.restype = ctypes.c_long
        L.oracle_array.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_void_p, ctypes.c_long, ctypes.c_int]
        L.oracle_last_error.restype = ctypes.c_char_p
        L.oracle_ksp7.argtypes = [ctypes.c_int] * 3 + [ctypes.c_void_p] * 3 + [ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                                                              ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double),
                                                                              ctypes.c_double]
        L.oracle_system.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int] + [ctypes.c_void_p] * 5
        L.oracle_hex_volume.restype = ctypes.c_double
        L.oracle_hex_volume.argtypes = [ctypes.c_void_p]
        L.oracle_quad_area.restype = ctypes.c_double
        L.oracle_quad_area.argtypes = [ctypes.c_void_p]
        L.oracle_hex_centroid.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.oracle_inside_hex.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.oracle_trilinear.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.oracle_nearest_intersect.argtypes = [ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.oracle_coupled_create.restype = ctypes.c_void_p
        L.oracle_coupled_create.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(OracleCase)]
        L.oracle_coupled_destroy.argtypes = [ctypes.c_void_p]
        L.oracle_coupled_solve.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.POINTER(ctypes.c_double)]
        L.oracle_coupled_stats.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.oracle_coupled_array.restype = ctypes.c_long
        L.oracle_coupled_array.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_void_p, ctypes.c_long, ctypes.c_int]
        L.oracle_coupled_phase.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_double]
        L.oracle_coupled_system.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.oracle_diffusion_create.restype = ctypes.c_void_p
        L.oracle_diffusion_create.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                              ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_double,
                                              ctypes.c_int]
        L.oracle_diffusion_destroy.argtypes = [ctypes.c_void_p]
        L.oracle_diffusion_solve.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.POINTER(ctypes.c_double)]
        L.oracle_diffusion_stats.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.oracle_diffusion_array.restype = ctypes.c_long
        L.oracle_diffusion_array.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_void_p, ctypes.c_long, ctypes.c_int]
        L.oracle_set_threads.argtypes = [ctypes.c_int]
        L.oracle_get_threads.restype = ctypes.c_int
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def make_case(spec) -> OracleCase:
    from caffe_old_b200 import cases as C
    spec.validate()
    oc = OracleCase()
    oc.kind = C.SOLVER_KINDS[spec.kind]
    for f in range(6):
        oc.bc_type[f] = C.FLOW_TYPES[spec.bc[f]]
        for q in range(3):
            oc.ref_vec[f][q] = float(spec.ref_vec[f][q])
        oc.ref_val[f] = float(spec.ref_val[f])
    oc.rho, oc.mu = float(spec.rho), float(spec.mu)
    oc.time_accurate = 1 if spec.time_accurate else 0
    oc.omega_u, oc.omega_p = float(spec.omega_u), float(spec.omega_p)
    oc.n_inner, oc.n_pcorr = int(spec.n_inner), int(spec.n_pcorr)
    oc.convection = C.CONVECTION[spec.convection]
    oc.nonorth = 1 if spec.nonorth else 0
    oc.mom_method = C.KSP_METHODS[spec.mom_method]
    oc.p_method = C.KSP_METHODS[spec.p_method]
    oc.mom_rtol, oc.p_rtol = float(spec.mom_rtol), float(spec.p_rtol)
    oc.maxit = int(spec.maxit)
    oc.ib_radius = float(spec.ib_radius)
    for q in range(3):
        oc.ib_center[q] = float(spec.ib_center[q])
        oc.u_init[q] = float(spec.u_init[q])
    oc.p_init = float(spec.p_init)
    oc.mom_atol, oc.p_atol = float(spec.mom_atol), float(spec.p_atol)
    return oc


def set_threads(n: int) -> None:
    lib().oracle_set_threads(int(n))


def get_threads() -> int:
    return int(lib().oracle_get_threads())


class OracleSolver:
    """CPU restatement of Simple / Piso / IbPiso (src/Solvers/*.cpp) on one block."""

    def __init__(self, nodes: np.ndarray, spec):
        L = lib()
        nodes = np.ascontiguousarray(nodes, dtype=np.float64)
        nK1, nJ1, nI1, _ = nodes.shape
        self.shape = (nI1 - 1, nJ1 - 1, nK1 - 1)
        self.ncells = self.shape[0] * self.shape[1] * self.shape[2]
        self._case = make_case(spec)
        self.spec = spec
        h = L.oracle_create(_ptr(nodes), nI1, nJ1, nK1, ctypes.byref(self._case))
        if not h:
            raise RuntimeError("oracle_create failed: " + L.oracle_last_error().decode())
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().oracle_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def solve(self, dt: float | None = None) -> float:
        out = ctypes.c_double(0.0)
        rc = lib().oracle_solve(self._h, float(self.spec.dt if dt is None else dt), ctypes.byref(out))
        if rc != 0:
            raise RuntimeError("oracle_solve: " + lib().oracle_last_error().decode())
        return out.value

    def phase(self, name: str, dt: float | None = None) -> None:
        rc = lib().oracle_phase(self._h, name.encode(), float(self.spec.dt if dt is None else dt))
        if rc != 0:
            raise RuntimeError(f"oracle phase {name}: " + lib().oracle_last_error().decode())

    def stats(self) -> dict:
        out = np.zeros(10)
        lib().oracle_stats(self._h, _ptr(out))
        keys = ("continuity", "courant", "mom_iters", "p_iters_last", "p_iters_total", "p_solves",
                "p_res_max", "mom_res_max", "ghosts", "rows")
        return dict(zip(keys, out.tolist()))

    def get(self, name: str) -> np.ndarray:
        L = lib()
        n = L.oracle_array(self._h, name.encode(), None, 0, 0)
        if n < 0:
            raise KeyError(name)
        out = np.zeros(n, dtype=np.float64)
        L.oracle_array(self._h, name.encode(), _ptr(out), n, 0)
        return out

    def set(self, name: str, values: np.ndarray) -> None:
        L = lib()
        n = L.oracle_array(self._h, name.encode(), None, 0, 0)
        if n < 0:
            raise KeyError(name)
        v = np.ascontiguousarray(values, dtype=np.float64).ravel()
        if v.size != n:
            raise ValueError(f"{name}: expected {n} values, got {v.size}")
        L.oracle_array(self._h, name.encode(), _ptr(v), n, 1)

    def system(self, which: int, comp: int = 0):
        """Assembled system `which` (0 momentum, 1 p') as {row: {col: value}} and right-hand side
        `comp`, in IndexMap row numbering; read right after the matching assemble phase."""
        L = lib()
        width = ctypes.c_int(0)
        n = L.oracle_system(self._h, which, comp, ctypes.byref(width), None, None, None, None)
        if n < 0:
            raise ValueError("invalid system")
        w = width.value
        cnt = np.zeros(n, dtype=np.int32)
        col = np.zeros(n * w, dtype=np.int32)
        val = np.zeros(n * w, dtype=np.float64)
        b = np.zeros(n, dtype=np.float64)
        L.oracle_system(self._h, which, comp, None, _ptr(cnt), _ptr(col), _ptr(val), _ptr(b))
        rows = []
        for r in range(n):
            rows.append({int(col[r * w + p]): float(val[r * w + p]) for p in range(cnt[r])})
        return rows, b


class OracleCoupled:
    """CPU restatement of the reference's Coupled solver (src/Solvers/Coupled.cpp): momentum
    and continuity in one linear system of 4 N unknowns.  The case record's boundary types,
    rho, mu, timeAccurate, relaxationFactorMomentum, numberOfInnerIterations and the momentum
    Krylov settings (method, tolerance, maxit) are used.  ``solve(dt)`` returns the maximum
    continuity error."""

    def __init__(self, nodes: np.ndarray, spec):
        L = lib()
        nodes = np.ascontiguousarray(nodes, dtype=np.float64)
        nK1, nJ1, nI1, _ = nodes.shape
        self.shape = (nI1 - 1, nJ1 - 1, nK1 - 1)
        self.ncells = self.shape[0] * self.shape[1] * self.shape[2]
        self.spec = spec
        self._case = make_case(spec)
        h = L.oracle_coupled_create(_ptr(nodes), nI1, nJ1, nK1, ctypes.byref(self._case))
        if not h:
            raise RuntimeError("oracle_coupled_create failed: " + L.oracle_last_error().decode())
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().oracle_coupled_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def solve(self, dt: float | None = None) -> float:
        out = ctypes.c_double(0.0)
        if lib().oracle_coupled_solve(self._h, float(self.spec.dt if dt is None else dt), ctypes.byref(out)) != 0:
            raise RuntimeError("oracle_coupled_solve: " + lib().oracle_last_error().decode())
        return out.value

    def stats(self) -> dict:
        out = np.zeros(3)
        lib().oracle_coupled_stats(self._h, _ptr(out))
        return {"iters": int(out[0]), "rel_res": float(out[1]), "status": int(out[2])}

    def get(self, name: str) -> np.ndarray:
        L = lib()
        n = L.oracle_coupled_array(self._h, name.encode(), None, 0, 0)
        if n < 0:
            raise KeyError(name)
        out = np.zeros(n, dtype=np.float64)
        L.oracle_coupled_array(self._h, name.encode(), _ptr(out), n, 0)
        return out

    def set(self, name: str, values: np.ndarray) -> None:
        v = np.ascontiguousarray(values, dtype=np.float64).ravel()
        n = lib().oracle_coupled_array(self._h, name.encode(), None, 0, 0)
        if n != v.size:
            raise ValueError(f"{name}: expected {n} values, got {v.size}")
        lib().oracle_coupled_array(self._h, name.encode(), _ptr(v), n, 1)

    def phase(self, name: str, dt: float | None = None) -> None:
        """One part of Coupled::computeMomentumAndPressure: save_u0, assemble, solve, post."""
        if lib().oracle_coupled_phase(self._h, name.encode(), float(self.spec.dt if dt is None else dt)) != 0:
            raise RuntimeError("oracle_coupled_phase: " + lib().oracle_last_error().decode())

    def system(self):
        """The assembled block system: per row its entries in insertion order, as
        (counts, columns, values) with columns -1 past each row's count, and the width."""
        L = lib()
        n = L.oracle_coupled_system(self._h, None, None, None, None)
        w = ctypes.c_int(0)
        L.oracle_coupled_system(self._h, ctypes.byref(w), None, None, None)
        cnt = np.zeros(n, dtype=np.int32)
        col = np.zeros(n * w.value, dtype=np.int32)
        val = np.zeros(n * w.value, dtype=np.float64)
        L.oracle_coupled_system(self._h, None, _ptr(cnt), _ptr(col), _ptr(val))
        return cnt, col.reshape(n, w.value), val.reshape(n, w.value)


DIFFUSION_BC = {"fixed": 0, "zeroGradient": 1, "empty": 2}


class OracleDiffusion:
    """CPU restatement of the reference's Diffusion solver (src/Solvers/Diffusion.cpp) on one
    block: unit diffusivity, boundary types fixed / zeroGradient / empty per face (east, west,
    north, south, top, bottom) with their reference values, a uniform initial phi.
    ``solve(dt)`` assembles and solves one linear system and returns ||A x - b||_inf."""

    def __init__(self, nodes: np.ndarray, bc_types, bc_values, time_accurate: bool = False, phi0: float = 0.0,
                 method: str = "bicgstab_sgs", rtol: float = 1e-8, maxit: int = 10000):
        from caffe_old_b200 import cases as C
        L = lib()
        nodes = np.ascontiguousarray(nodes, dtype=np.float64)
        nK1, nJ1, nI1, _ = nodes.shape
        self.shape = (nI1 - 1, nJ1 - 1, nK1 - 1)
        self.ncells = self.shape[0] * self.shape[1] * self.shape[2]
        types = np.array([DIFFUSION_BC[t] for t in bc_types], dtype=np.int32)
        refs = np.ascontiguousarray(bc_values, dtype=np.float64)
        if types.size != 6 or refs.size != 6:
            raise ValueError("six boundary types and values (east, west, north, south, top, bottom)")
        h = L.oracle_diffusion_create(_ptr(nodes), nI1, nJ1, nK1, _ptr(types), _ptr(refs), 1 if time_accurate else 0,
                                      float(phi0), C.KSP_METHODS[method], float(rtol), int(maxit))
        if not h:
            raise RuntimeError("oracle_diffusion_create failed: " + L.oracle_last_error().decode())
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().oracle_diffusion_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def solve(self, dt: float = 1.0) -> float:
        out = ctypes.c_double(0.0)
        if lib().oracle_diffusion_solve(self._h, float(dt), ctypes.byref(out)) != 0:
            raise RuntimeError("oracle_diffusion_solve: " + lib().oracle_last_error().decode())
        return out.value

    def stats(self) -> dict:
        out = np.zeros(2)
        lib().oracle_diffusion_stats(self._h, _ptr(out))
        return {"iters": int(out[0]), "rel_res": float(out[1])}

    def get(self, name: str) -> np.ndarray:
        L = lib()
        n = L.oracle_diffusion_array(self._h, name.encode(), None, 0, 0)
        if n < 0:
            raise KeyError(name)
        out = np.zeros(n, dtype=np.float64)
        L.oracle_diffusion_array(self._h, name.encode(), _ptr(out), n, 0)
        return out

    def set(self, name: str, values: np.ndarray) -> None:
        L = lib()
        n = L.oracle_diffusion_array(self._h, name.encode(), None, 0, 0)
        if n < 0:
            raise KeyError(name)
        v = np.ascontiguousarray(values, dtype=np.float64).ravel()
        if v.size != n:
            raise ValueError(f"{name}: expected {n} values, got {v.size}")
        L.oracle_diffusion_array(self._h, name.encode(), _ptr(v), n, 1)


def ksp7(shape, coef7: np.ndarray, b: np.ndarray, method: str, rtol: float, maxit: int, atol: float = 0.0):
    from caffe_old_b200 import cases as C
    nI, nJ, nK = shape
    coef7 = np.ascontiguousarray(coef7, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    x = np.zeros_like(b)
    it = ctypes.c_int(0)
    rr = ctypes.c_double(0.0)
    st = lib().oracle_ksp7(nI, nJ, nK, _ptr(coef7), _ptr(b), _ptr(x), C.KSP_METHODS[method], float(rtol), int(maxit),
                           ctypes.byref(it), ctypes.byref(rr), ctypes.c_double(float(atol)))
    return x, it.value, rr.value, st


def hex_volume(p8: np.ndarray) -> float:
    p = np.ascontiguousarray(p8, dtype=np.float64)
    return lib().oracle_hex_volume(_ptr(p))


def hex_centroid(p8: np.ndarray) -> np.ndarray:
    p = np.ascontiguousarray(p8, dtype=np.float64)
    out = np.zeros(3)
    lib().oracle_hex_centroid(_ptr(p), _ptr(out))
    return out


def quad_area(p4: np.ndarray) -> float:
    p = np.ascontiguousarray(p4, dtype=np.float64)
    return lib().oracle_quad_area(_ptr(p))


def inside_hex(pt, p8) -> bool:
    a = np.ascontiguousarray(pt, dtype=np.float64)
    p = np.ascontiguousarray(p8, dtype=np.float64)
    return bool(lib().oracle_inside_hex(_ptr(a), _ptr(p)))


def trilinear(p8, ip) -> np.ndarray:
    p = np.ascontiguousarray(p8, dtype=np.float64)
    a = np.ascontiguousarray(ip, dtype=np.float64)
    out = np.zeros(8)
    lib().oracle_trilinear(_ptr(p), _ptr(a), _ptr(out))
    return out


def nearest_intersect(radius, center, pt) -> np.ndarray:
    c = np.ascontiguousarray(center, dtype=np.float64)
    a = np.ascontiguousarray(pt, dtype=np.float64)
    out = np.zeros(3)
    lib().oracle_nearest_intersect(float(radius), _ptr(c), _ptr(a), _ptr(out))
    return out
