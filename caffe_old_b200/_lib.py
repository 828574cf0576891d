"""ctypes binding of the device library (include/caffe_b200.h).

The library is built in-tree (caffe_old_b200/_build/libcaffe_b200.so, see
caffe_old_b200/build.py).  There is no CPU fallback: if the library is missing or
cannot be loaded, every entry point raises.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import cases as C

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_build", "libcaffe_b200.so")
HEADER_PATH = os.path.join(os.path.dirname(_HERE), "include", "caffe_b200.h")
_lib = None


class CaffeError(RuntimeError):
    pass


class CaffeCase(ctypes.Structure):
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
        ("p_form", ctypes.c_int),
        ("mom_atol", ctypes.c_double), ("p_atol", ctypes.c_double),
    ]


class StepStats(ctypes.Structure):
    _fields_ = [
        ("continuity", ctypes.c_double), ("courant", ctypes.c_double),
        ("mom_iters", ctypes.c_int * 3),
        ("p_iters_last", ctypes.c_int), ("p_iters_total", ctypes.c_int), ("p_solves", ctypes.c_int),
        ("p_res_max", ctypes.c_double), ("mom_res_max", ctypes.c_double),
        ("status", ctypes.c_int), ("fallbacks", ctypes.c_int), ("n_ghost", ctypes.c_int), ("n_rows", ctypes.c_int),
        ("p_ms", ctypes.c_double), ("mom_ms", ctypes.c_double), ("step_ms", ctypes.c_double),
        ("cascades", ctypes.c_int), ("net_iters", ctypes.c_int),
    ]

    def as_dict(self) -> dict:
        out = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            out[name] = list(v) if name == "mom_iters" else v
        return out


EXPORTS = (
    "caffe_last_error", "caffe_dev_create", "caffe_dev_destroy", "caffe_dev_solve", "caffe_dev_phase",
    "caffe_dev_array", "caffe_dev_stats", "caffe_dev_stream", "caffe_dev_synchronize", "caffe_dev_set_stream",
    "caffe_slab_set_owned", "caffe_slab_halo", "caffe_slab_ksp", "caffe_slab_phase", "caffe_slab_reduce",
    "caffe_ksp7_solve", "caffe_ksp7_solve_device", "caffe_ksp7_solve_device_noalloc", "caffe_csr_solve", "caffe_csr_matvec",
    "caffe_diffusion_create", "caffe_diffusion_destroy", "caffe_diffusion_solve", "caffe_diffusion_phase", "caffe_diffusion_array",
    "caffe_coupled_create", "caffe_coupled_destroy", "caffe_coupled_solve", "caffe_coupled_phase", "caffe_coupled_stats",
    "caffe_coupled_system", "caffe_coupled_array",
    "caffe_precond_param_count", "caffe_precond_net_apply", "caffe_precond_net_grad",
    "caffe_dev_set_precond", "caffe_dev_get_precond", "caffe_dev_set_precond_mode", "caffe_dev_set_precond_options",
    "caffe_dev_set_precond_net_levels",
    "caffe_dev_record_pairs", "caffe_dev_pair_count", "caffe_dev_add_pairs", "caffe_dev_add_random_pairs", "caffe_dev_copy_pairs", "caffe_dev_train_precond",
    "caffe_dev_eval_precond", "caffe_launch_count",
)


def lib():
    """Load the device library; raise CaffeError when it is missing (no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise CaffeError(f"device library not built: {LIB_PATH} (run caffe_old_b200.build.build())")
    L = ctypes.CDLL(LIB_PATH)
    vp, ci, cd = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    L.caffe_last_error.restype = ctypes.c_char_p
    L.caffe_dev_create.argtypes = [vp, ci, ci, ci, ctypes.POINTER(CaffeCase), ci, ctypes.POINTER(vp)]
    L.caffe_dev_destroy.argtypes = [vp]
    L.caffe_dev_solve.argtypes = [vp, cd, ctypes.POINTER(StepStats)]
    L.caffe_dev_phase.argtypes = [vp, ctypes.c_char_p, cd]
    L.caffe_dev_array.restype = ctypes.c_long
    L.caffe_dev_array.argtypes = [vp, ctypes.c_char_p, vp, ctypes.c_long, ci]
    L.caffe_dev_stats.argtypes = [vp, ctypes.POINTER(StepStats)]
    L.caffe_dev_stream.restype = vp
    L.caffe_dev_stream.argtypes = [vp]
    L.caffe_dev_synchronize.argtypes = [vp]
    L.caffe_dev_set_stream.argtypes = [vp, vp]
    L.caffe_slab_set_owned.argtypes = [vp, ci, ci]
    L.caffe_slab_halo.restype = ctypes.c_long
    L.caffe_slab_halo.argtypes = [vp, ctypes.c_char_p, ci, ci, ci, vp]
    L.caffe_slab_ksp.argtypes = [vp, ci, ci, vp, vp]
    L.caffe_slab_phase.argtypes = [vp, ctypes.c_char_p, cd]
    L.caffe_slab_reduce.argtypes = [vp, ctypes.c_char_p, cd, vp]
    L.caffe_ksp7_solve.argtypes = [ci, ci, ci, vp, vp, vp, ci, cd, ci, ctypes.POINTER(ci), ctypes.POINTER(cd)]
    L.caffe_ksp7_solve_device.argtypes = [ci, ci, ci, vp, vp, vp, ci, cd, ci, vp, ctypes.POINTER(ci), ctypes.POINTER(cd)]
    L.caffe_ksp7_solve_device_noalloc.argtypes = [ci, ci, ci, vp, vp, vp, ci, cd, ci, vp, ctypes.POINTER(ci),
                                                  ctypes.POINTER(cd)]
    L.caffe_csr_solve.argtypes = [ci, vp, vp, vp, vp, vp, ci, cd, cd, ci, ctypes.POINTER(ci), ctypes.POINTER(cd)]
    L.caffe_csr_matvec.argtypes = [ci, ci, vp, vp, vp, vp, vp]
    L.caffe_diffusion_create.argtypes = [vp, ci, ci, ci, vp, vp, ci, cd, ci, cd, ci, ci, ctypes.POINTER(vp)]
    L.caffe_diffusion_destroy.argtypes = [vp]
    L.caffe_diffusion_solve.argtypes = [vp, cd, ctypes.POINTER(cd), ctypes.POINTER(ci), ctypes.POINTER(cd)]
    L.caffe_diffusion_phase.argtypes = [vp, ctypes.c_char_p, cd]
    L.caffe_diffusion_array.restype = ctypes.c_long
    L.caffe_diffusion_array.argtypes = [vp, ctypes.c_char_p, vp, ctypes.c_long, ci]
    L.caffe_coupled_create.argtypes = [vp, ci, ci, ci, ctypes.POINTER(CaffeCase), ci, ctypes.POINTER(vp)]
    L.caffe_coupled_destroy.argtypes = [vp]
    L.caffe_coupled_solve.argtypes = [vp, cd, ctypes.POINTER(cd)]
    L.caffe_coupled_phase.argtypes = [vp, ctypes.c_char_p, cd]
    L.caffe_coupled_stats.argtypes = [vp, ctypes.POINTER(ci), ctypes.POINTER(cd), ctypes.POINTER(ci)]
    L.caffe_coupled_system.restype = ctypes.c_longlong
    L.caffe_coupled_system.argtypes = [vp, vp, vp, vp]
    L.caffe_coupled_array.restype = ctypes.c_long
    L.caffe_coupled_array.argtypes = [vp, ctypes.c_char_p, vp, ctypes.c_long, ci]
    L.caffe_precond_param_count.restype = ci
    L.caffe_precond_net_apply.argtypes = [ci, ci, ci, vp, vp, vp]
    L.caffe_precond_net_grad.argtypes = [ci, ci, ci, vp, vp, vp, vp, vp]
    L.caffe_dev_set_precond.argtypes = [vp, vp]
    L.caffe_dev_get_precond.argtypes = [vp, vp]
    L.caffe_dev_set_precond_mode.argtypes = [vp, ci]
    L.caffe_dev_set_precond_options.argtypes = [vp, ci, ci, ci]
    L.caffe_dev_set_precond_net_levels.argtypes = [vp, ci, ci]
    L.caffe_dev_record_pairs.argtypes = [vp, ci, ci]
    L.caffe_dev_pair_count.argtypes = [vp]
    L.caffe_dev_add_pairs.argtypes = [vp, vp, vp, ci]
    L.caffe_dev_copy_pairs.argtypes = [vp, vp]
    L.caffe_dev_add_random_pairs.argtypes = [vp, ci, ctypes.c_uint]
    L.caffe_dev_train_precond.argtypes = [vp, ci, ci, ctypes.c_float, ctypes.c_uint, vp, vp]
    L.caffe_dev_eval_precond.argtypes = [vp, ci, vp]
    L.caffe_launch_count.restype = ctypes.c_longlong
    L.caffe_launch_count.argtypes = []
    _lib = L
    return L


def last_error() -> str:
    return lib().caffe_last_error().decode()


def make_case(spec: C.CaseSpec) -> CaffeCase:
    spec.validate()
    c = CaffeCase()
    c.kind = C.SOLVER_KINDS[spec.kind]
    for f in range(6):
        c.bc_type[f] = C.FLOW_TYPES[spec.bc[f]]
        for q in range(3):
            c.ref_vec[f][q] = float(spec.ref_vec[f][q])
        c.ref_val[f] = float(spec.ref_val[f])
    c.rho, c.mu = float(spec.rho), float(spec.mu)
    c.time_accurate = 1 if spec.time_accurate else 0
    c.omega_u, c.omega_p = float(spec.omega_u), float(spec.omega_p)
    c.n_inner, c.n_pcorr = int(spec.n_inner), int(spec.n_pcorr)
    c.convection = C.CONVECTION[spec.convection]
    c.nonorth = 1 if spec.nonorth else 0
    c.mom_method = C.KSP_METHODS[spec.mom_method]
    c.p_method = C.KSP_METHODS[spec.p_method]
    c.mom_rtol, c.p_rtol = float(spec.mom_rtol), float(spec.p_rtol)
    c.maxit = int(spec.maxit)
    c.ib_radius = float(spec.ib_radius)
    for q in range(3):
        c.ib_center[q] = float(spec.ib_center[q])
        c.u_init[q] = float(spec.u_init[q])
    c.p_init = float(spec.p_init)
    c.p_form = C.P_FORMS[spec.p_form]
    c.mom_atol, c.p_atol = float(spec.mom_atol), float(spec.p_atol)
    return c


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def ksp7_solve(shape, coef7: np.ndarray, b: np.ndarray, method: str = "bicgstab_jacobi", rtol: float = 1e-8,
               maxit: int = 20000):
    """SparseMatrix::solve on the device for a 7-point system given as 7 host arrays."""
    nI, nJ, nK = (int(v) for v in shape)
    coef7 = np.ascontiguousarray(coef7, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    x = np.zeros_like(b)
    it = ctypes.c_int(0)
    rr = ctypes.c_double(0.0)
    st = lib().caffe_ksp7_solve(nI, nJ, nK, _ptr(coef7), _ptr(b), _ptr(x), C.KSP_METHODS[method], float(rtol), int(maxit),
                                ctypes.byref(it), ctypes.byref(rr))
    if st == 1:
        raise CaffeError("caffe_ksp7_solve: " + last_error())
    return x, it.value, rr.value, st


def csr_solve(row_ptr, col, val, b, method: str = "bicgstab_jacobi", rtol: float = 1e-8, atol: float = 0.0,
              maxit: int = 20000):
    """SparseMatrix::solve for a general compressed-row system on the device; returns (x, iters,
    relative residual, status)."""
    row_ptr = np.ascontiguousarray(row_ptr, dtype=np.int32)
    col = np.ascontiguousarray(col, dtype=np.int32)
    val = np.ascontiguousarray(val, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    x = np.zeros_like(b)
    it, rr = ctypes.c_int(0), ctypes.c_double(0.0)
    st = lib().caffe_csr_solve(int(b.size), _ptr(row_ptr), _ptr(col), _ptr(val), _ptr(b), _ptr(x), C.KSP_METHODS[method],
                               float(rtol), float(atol), int(maxit), ctypes.byref(it), ctypes.byref(rr))
    if st == 1:
        raise CaffeError("caffe_csr_solve: " + last_error())
    return x, it.value, rr.value, st
