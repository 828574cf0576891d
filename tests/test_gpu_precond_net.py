"""Tensor-core network kernels (forward, backward data and weight gradient) against the CPU FP64 restatement with
bf16 rounding at the same points.  Tolerances: 2e-2 relative L2 on the output and on each
layer's gradient block (bf16 has an 8-bit mantissa; FP32 vs FP64 accumulation can flip a
rounding)."""
import ctypes

import numpy as np
import pytest

from caffe_old_b200 import _lib

import cnn_reference as R

pytestmark = pytest.mark.gpu
TOL = 2e-2


def _call_apply(shape, params, x2):
    L = _lib.lib()
    n = shape[0] * shape[1] * shape[2]
    y = np.zeros(n, dtype=np.float32)
    p = np.ascontiguousarray(params, dtype=np.float32)
    x = np.ascontiguousarray(x2, dtype=np.float32)
    rc = L.caffe_precond_net_apply(*shape, p.ctypes.data_as(ctypes.c_void_p), x.ctypes.data_as(ctypes.c_void_p),
                                   y.ctypes.data_as(ctypes.c_void_p))
    assert rc == 0, _lib.last_error()
    return y


@pytest.mark.parametrize("shape", [(8, 16, 3), (20, 18, 12), (37, 5, 21)])
def test_forward_matches_fp64_reference(shape):
    assert _lib.lib().caffe_precond_param_count() == 4 * R.LAYER
    rng = np.random.default_rng(3)
    params = R.random_params(1)
    x2 = rng.standard_normal((np.prod(shape), 2)).astype(np.float32)
    y = _call_apply(shape, params, x2)
    yr, _ = R.forward(params.astype(np.float64), x2.astype(np.float64), shape)
    err = np.linalg.norm(y - yr) / np.linalg.norm(yr)
    assert err < TOL, err


@pytest.mark.parametrize("shape", [(20, 18, 12), (37, 5, 21)])
def test_gradients_match_fp64_reference(shape):
    """Backward data (tcgen05) and the weight gradient (tcgen05 implicit GEMM over the cells,
    including rows whose last 16-cell chunk is partly outside the lattice)."""
    n = int(np.prod(shape))
    rng = np.random.default_rng(4)
    params = R.random_params(2)
    x2 = rng.standard_normal((n, 2)).astype(np.float32)
    dy = rng.standard_normal(n).astype(np.float32)
    L = _lib.lib()
    y = np.zeros(n, dtype=np.float32)
    g = np.zeros(4 * R.LAYER, dtype=np.float32)
    rc = L.caffe_precond_net_grad(*shape, params.ctypes.data_as(ctypes.c_void_p), x2.ctypes.data_as(ctypes.c_void_p),
                                  dy.ctypes.data_as(ctypes.c_void_p), y.ctypes.data_as(ctypes.c_void_p),
                                  g.ctypes.data_as(ctypes.c_void_p))
    assert rc == 0, _lib.last_error()
    _, gr = R.grad(params.astype(np.float64), x2.astype(np.float64), dy.astype(np.float64), shape)
    for l in range(4):
        blk = slice(l * R.LAYER, (l + 1) * R.LAYER)
        ref = gr[blk]
        if l == 0:   # only input channels 0 and 1 carry data
            ref = ref.copy()
        err = np.linalg.norm(g[blk] - ref) / max(np.linalg.norm(ref), 1e-30)
        assert err < TOL, (l, err)
