"""Learned preconditioner of the pressure-correction solve: parameters, training pairs and
training on the device, through the C ABI.

The network (4 layers of 3x3x3 convolutions, 16 channels, BF16 weights, FP32 accumulation)
runs on a pyramid of coarsened lattices inside an FP32 flexible Krylov solve that sits in an
FP64 refinement loop; see ``csrc/learned.cu``.  Parameter layout, per layer l = 0..3:
``W_l[27 taps][16 out][16 in]`` then ``b_l[16]``; tap ``t = 9 (dk+1) + 3 (dj+1) + (di+1)``.
Input channels: 0 = restricted Jacobi-scaled residual / its RMS, 1 = fraction of active
cells, 2 = level / 8.  Output: channel 0 of the last layer.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from ._lib import CaffeError, last_error, lib

LAYERS = 4
CHANNELS = 16
TAPS = 27
CENTER = 13
LAYER_PARAMS = TAPS * CHANNELS * CHANNELS + CHANNELS
PARAMS = LAYERS * LAYER_PARAMS

MODES = {"jacobi": 0, "network": 1, "levels": 2}
INNER = {"auto": 0, "fcg": 1, "bicgstab": 2, "fgmres": 3}

DEFAULT_WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "precond_params.npy")


def weight_view(params: np.ndarray, layer: int) -> tuple[np.ndarray, np.ndarray]:
    """(W[27][16 out][16 in], b[16]) views of one layer."""
    off = layer * LAYER_PARAMS
    W = params[off:off + TAPS * CHANNELS * CHANNELS].reshape(TAPS, CHANNELS, CHANNELS)
    b = params[off + TAPS * CHANNELS * CHANNELS:off + LAYER_PARAMS]
    return W, b


def identity_params(seed: int = 0, noise: float = 0.02) -> np.ndarray:
    """Parameters whose network is the identity on input channel 0 (y = relu(x) - relu(-x)
    carried through two channels), plus small seeded noise on every other weight so that the
    remaining channels can learn.  With them the learned preconditioner starts as the plain
    level pyramid and training moves it from there."""
    rng = np.random.default_rng(seed)
    p = (noise * rng.standard_normal(PARAMS) / np.sqrt(TAPS * CHANNELS)).astype(np.float32)
    for l in range(LAYERS):
        W, b = weight_view(p, l)
        b[:] = 0.0
        W[:, 0, :] = 0.0           # output channels 0 and 1 carry the identity path only
        W[:, 1, :] = 0.0
        if l == 0:
            W[CENTER, 0, 0] = 1.0      # relu(x)
            W[CENTER, 1, 0] = -1.0     # relu(-x)
        elif l < LAYERS - 1:
            W[CENTER, 0, 0] = 1.0
            W[CENTER, 1, 1] = 1.0
        else:
            W[CENTER, 0, 0] = 1.0      # y = relu(x) - relu(-x) = x
            W[CENTER, 0, 1] = -1.0
    return p


def load_default() -> np.ndarray | None:
    """The trained parameters shipped with the package, or None."""
    if os.path.exists(DEFAULT_WEIGHTS):
        p = np.load(DEFAULT_WEIGHTS).astype(np.float32)
        if p.size == PARAMS:
            return p
    return None


def default_info() -> dict:
    """How the shipped parameters were trained (first network level, pairs, losses), or {}."""
    path = os.path.splitext(DEFAULT_WEIGHTS)[0] + ".json"
    if os.path.exists(path):
        import json
        with open(path) as f:
            return json.load(f)
    return {}


def pyramid_dims(dims) -> list:
    """The lattices of the learned preconditioner's level pyramid for a cell lattice `dims`
    (the rule of the device's learned_alloc: halve every direction longer than one cell until
    at most 64 cells remain, at most 12 levels)."""
    out = [[int(v) for v in dims]]
    while len(out) < 12:
        f = out[-1]
        if f[0] * f[1] * f[2] <= 64 or f == [1, 1, 1]:
            break
        out.append([(v + 1) // 2 if v > 1 else 1 for v in f])
    return out


def trained_last_level() -> int | None:
    """The last pyramid level that runs the network with the shipped parameters: the measured
    choice recorded with them, else the coarsest level they were trained on (the network has
    never seen the level channel of a coarser one), or None when unknown."""
    info = default_info()
    if "net_to_run" in info:
        return int(info["net_to_run"])
    if "net_to" in info:
        return int(info["net_to"])
    if "dims" in info:
        return len(pyramid_dims(info["dims"])) - 1
    return None


def _check(rc: int, what: str) -> None:
    if rc != 0:
        raise CaffeError(f"{what}: " + last_error())


def set_params(solver, params: np.ndarray | None) -> None:
    if params is None:
        _check(lib().caffe_dev_set_precond(solver._h, None), "set_precond")
        return
    p = np.ascontiguousarray(params, dtype=np.float32)
    if p.size != PARAMS:
        raise ValueError(f"expected {PARAMS} parameters, got {p.size}")
    _check(lib().caffe_dev_set_precond(solver._h, p.ctypes.data_as(ctypes.c_void_p)), "set_precond")


def get_params(solver) -> np.ndarray:
    p = np.zeros(PARAMS, dtype=np.float32)
    _check(lib().caffe_dev_get_precond(solver._h, p.ctypes.data_as(ctypes.c_void_p)), "get_precond")
    return p


def set_mode(solver, mode: str) -> None:
    _check(lib().caffe_dev_set_precond_mode(solver._h, MODES[mode]), "set_precond_mode")


def set_options(solver, inner: str = "auto", net_from_level: int = 1, restart: int = 40) -> None:
    """Inner Krylov method of the learned solve, the first pyramid level that runs the
    network (finer levels use the identity) and the FGMRES cycle length."""
    _check(lib().caffe_dev_set_precond_options(solver._h, INNER[inner], int(net_from_level), int(restart)),
           "set_precond_options")


def set_net_levels(solver, first_level: int = 1, last_level: int | None = None) -> None:
    """The pyramid levels that run the network (first_level .. last_level; None: down to the
    coarsest); the others use the identity."""
    _check(lib().caffe_dev_set_precond_net_levels(solver._h, int(first_level), -1 if last_level is None else int(last_level)),
           "set_precond_net_levels")


def record_pairs(solver, capacity: int, snapshots: int = 0) -> None:
    """Record (b, x) of every following p' solve, plus `snapshots` residual/correction pairs of
    truncated plain re-solves (8, 32, 128, ... iterations), until `capacity` pairs are held."""
    _check(lib().caffe_dev_record_pairs(solver._h, int(capacity), int(snapshots)), "record_pairs")


def pair_count(solver) -> int:
    n = lib().caffe_dev_pair_count(solver._h)
    if n < 0:
        raise CaffeError("pair_count: " + last_error())
    return int(n)


def add_pairs(solver, b: np.ndarray, x: np.ndarray) -> None:
    b = np.ascontiguousarray(b, dtype=np.float32).reshape(-1, solver.ncells)
    x = np.ascontiguousarray(x, dtype=np.float32).reshape(-1, solver.ncells)
    if b.shape != x.shape:
        raise ValueError("b and x must have the same shape")
    _check(lib().caffe_dev_add_pairs(solver._h, b.ctypes.data_as(ctypes.c_void_p), x.ctypes.data_as(ctypes.c_void_p), b.shape[0]),
           "add_pairs")


def add_random_pairs(solver, n: int, seed: int = 0) -> None:
    """Append n synthetic multi-scale pairs (A e, e) built with the solver's current p' matrix."""
    _check(lib().caffe_dev_add_random_pairs(solver._h, int(n), int(seed) & 0xFFFFFFFF), "add_random_pairs")


def copy_pairs(dst, src) -> None:
    _check(lib().caffe_dev_copy_pairs(dst._h, src._h), "copy_pairs")


def train(solver, params: np.ndarray, steps: int, batch: int = 4, lr: float = 1e-3, seed: int = 0) -> tuple[np.ndarray, np.ndarray]:
    """Train on the solver's stored pairs; returns (trained parameters, loss per step)."""
    p = np.ascontiguousarray(params, dtype=np.float32).copy()
    hist = np.zeros(max(int(steps), 1), dtype=np.float32)
    _check(lib().caffe_dev_train_precond(solver._h, int(steps), int(batch), float(lr), int(seed) & 0xFFFFFFFF,
                                         p.ctypes.data_as(ctypes.c_void_p), hist.ctypes.data_as(ctypes.c_void_p)),
           "train_precond")
    return p, hist[:int(steps)]


def evaluate(solver, mode: str = "network") -> np.ndarray:
    """Energy-norm loss of one application M(b) against x for every stored pair."""
    n = pair_count(solver)
    out = np.zeros(max(n, 1), dtype=np.float32)
    _check(lib().caffe_dev_eval_precond(solver._h, MODES[mode], out.ctypes.data_as(ctypes.c_void_p)), "eval_precond")
    return out[:n]


__all__ = ["PARAMS", "MODES", "INNER", "identity_params", "load_default", "default_info", "set_params", "get_params", "set_mode", "set_options",
           "record_pairs", "pair_count", "add_pairs", "add_random_pairs", "copy_pairs", "train", "evaluate", "weight_view"]
