"""caffe_ksp7_solve_device_noalloc: the Krylov solve for callers that cannot allocate device
memory (a program whose own allocator owns the GPU's memory, or a loop that cannot take the
synchronisation cudaFree implies).  Its workspace is a fixed array inside the library, so it
must give the same answer as the allocating entry point, on consecutive calls of different
sizes (the array keeps the previous call's data), and refuse lattices beyond its limit.

This file is collected last on purpose: it also runs correctly on its own in a fresh process."""
import ctypes

import numpy as np
import pytest

from caffe_old_b200 import _lib
from caffe_old_b200 import cases as C

pytestmark = pytest.mark.gpu

RTOL_SOLVE = 1e-12
TOL = 1e-9   # relative L2 between solutions, as in the other Krylov parity tests


def seven_point_system(shape, seed, symmetric):
    rng = np.random.default_rng(seed)
    nI, nJ, nK = shape
    N = nI * nJ * nK
    idx = np.arange(N)
    i, j, k = idx % nI, (idx // nI) % nJ, idx // (nI * nJ)
    aE = rng.uniform(0.5, 1.5, N); aN = rng.uniform(0.5, 1.5, N); aT = rng.uniform(0.5, 1.5, N)
    aE[i == nI - 1] = 0; aN[j == nJ - 1] = 0; aT[k == nK - 1] = 0
    aW = np.zeros(N); aW[1:] = aE[:-1]; aW[i == 0] = 0
    aS = np.zeros(N); aS[nI:] = aN[:-nI]; aS[j == 0] = 0
    aB = np.zeros(N); aB[nI * nJ:] = aT[:-nI * nJ]; aB[k == 0] = 0
    aP = -(aE + aW + aN + aS + aT + aB) - rng.uniform(0.01, 0.1, N)
    if not symmetric:
        aE = aE * rng.uniform(0.7, 1.3, N)
        aE[i == nI - 1] = 0
    return np.stack([aP, aE, aW, aN, aS, aT, aB]), rng.standard_normal(N)


def seven_point_residual(shape, coef, x, b):
    nI, nJ, _ = shape
    y = coef[0] * x
    for q, off in ((1, 1), (3, nI), (5, nI * nJ)):
        y[:-off] += coef[q][:-off] * x[off:]
        y[off:] += coef[q + 1][off:] * x[:-off]
    return float(np.linalg.norm(b - y) / np.linalg.norm(b))


def solve_with(entry, shape, coef, b, method):
    import torch
    dc = torch.from_numpy(np.ascontiguousarray(coef)).cuda()
    db = torch.from_numpy(np.ascontiguousarray(b)).cuda()
    dx = torch.zeros_like(db)
    it, rr = ctypes.c_int(0), ctypes.c_double(0.0)
    stream = torch.cuda.current_stream().cuda_stream
    rc = entry(*shape, dc.data_ptr(), db.data_ptr(), dx.data_ptr(), C.KSP_METHODS[method], RTOL_SOLVE, 20000,
               ctypes.c_void_p(stream), ctypes.byref(it), ctypes.byref(rr))
    torch.cuda.synchronize()
    return rc, dx.cpu().numpy(), it.value, rr.value


def test_no_alloc_matches_allocating_solver_on_consecutive_calls():
    L = _lib.lib()
    cases = [((24, 20, 16), 11, "cg_jacobi"), ((13, 11, 7), 12, "bicgstab_jacobi")]
    for shape, seed, method in cases:   # two calls in a row, the second on a smaller lattice
        coef, b = seven_point_system(shape, seed, symmetric=method == "cg_jacobi")
        rc0, x0, it0, rr0 = solve_with(L.caffe_ksp7_solve_device, shape, coef, b, method)
        rc1, x1, it1, rr1 = solve_with(L.caffe_ksp7_solve_device_noalloc, shape, coef, b, method)
        assert rc0 == 0 and rc1 == 0, _lib.last_error()
        assert rr1 <= RTOL_SOLVE
        # the returned x itself solves the system: ||b - A x|| / ||b|| from NumPy, independent of
        # the residual the device reports (a small margin over the tolerance for the recomputation)
        assert seven_point_residual(shape, coef, x1, b) <= 10 * RTOL_SOLVE
        assert np.linalg.norm(x1 - x0) / np.linalg.norm(x0) < TOL
        assert abs(it1 - it0) <= 1


def test_no_alloc_rejects_lattices_beyond_its_workspace():
    import torch
    L = _lib.lib()
    tiny = torch.zeros(8, dtype=torch.float64, device="cuda")
    it, rr = ctypes.c_int(0), ctypes.c_double(0.0)
    rc = L.caffe_ksp7_solve_device_noalloc(200, 200, 200, tiny.data_ptr(), tiny.data_ptr(), tiny.data_ptr(),
                                           C.KSP_METHODS["cg_jacobi"], 1e-8, 100, None, ctypes.byref(it),
                                           ctypes.byref(rr))
    assert rc != 0
    assert "no-allocation" in _lib.last_error()
