"""Host side of the k-slab decomposition (caffe_old_b200/slab.py) on the CPU.

* ``partition`` / ``extended``: contiguous slabs covering the lattice, halo planes only where a
  neighbour exists.
* The distributed Krylov loops, run over CPU stand-ins of the device slab phases
  (tests/slab_cpu.py): split into 1, 2 and 3 slabs they solve the same system as one slab, to
  the requested tolerance.
* Under gloo with two processes (``DistTransport``: point-to-point halo exchange, all-reduce of
  the sums) the solve is bit-identical to the same two slabs driven in one process
  (``LocalTransport``), for BiCGStab on three right-hand sides, CG, and CG on a singular
  system with the mean projection.
"""
import os
import socket
import sys
from datetime import timedelta

import numpy as np
import pytest
import torch.multiprocessing as mp

from caffe_old_b200 import slab as S

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)

SHAPE = (6, 5, 9)   # nI, nJ, nK


def test_partition_covers_the_lattice_in_order():
    for nK in (1, 2, 7, 64, 257):
        for n in range(1, min(nK, 9) + 1):
            parts = S.partition(nK, n)
            assert parts[0][0] == 0 and parts[-1][1] == nK
            assert all(a[1] == b[0] for a, b in zip(parts, parts[1:]))
            sizes = [k1 - k0 for k0, k1 in parts]
            assert max(sizes) - min(sizes) <= 1 and min(sizes) >= 1
            for r, (k0, k1) in enumerate(parts):
                e0, e1 = S.extended(k0, k1, nK)
                assert e0 == (k0 - 1 if r > 0 else 0) and e1 == (k1 + 1 if r < n - 1 else nK)
    with pytest.raises(ValueError):
        S.partition(4, 5)
    with pytest.raises(ValueError):
        S.partition(4, 0)


def _system(kind, seed=3):
    from slab_cpu import random_system
    if kind == "bicgstab":
        return random_system(SHAPE, 3, False, seed)
    a, b = random_system(SHAPE, 1, True, seed)
    if kind == "cg_singular":
        # pure Neumann: rows sum to zero, the constant vector spans the null space
        a[0] = -a[1:].sum(axis=0)
    return a, b


def _solve(slabs, transport, kind):
    if kind == "bicgstab":
        return S.bicgstab(slabs, transport, 0, 3, "x", 1e-11, 5000)
    ncells = SHAPE[0] * SHAPE[1] * SHAPE[2]
    if kind == "cg_singular":
        S.project_mean(slabs, transport, 1, "b", ncells)
    out = S.cg(slabs, transport, 1, "x", 1e-11, 5000)
    if kind == "cg_singular":
        S.project_mean(slabs, transport, 1, "x", ncells)
    return out


def _local(kind, nslabs):
    from slab_cpu import NumpySlab
    a, b = _system(kind)
    parts = S.partition(SHAPE[2], nslabs)
    slabs = [NumpySlab(a, b, parts, r) for r in range(nslabs)]
    out = _solve(slabs, S.LocalTransport(nslabs), kind)
    return np.concatenate([s.owned_x() for s in slabs], axis=1), out, a, b


@pytest.mark.parametrize("kind", ["bicgstab", "cg", "cg_singular"])
@pytest.mark.parametrize("nslabs", [1, 2, 3])
def test_local_slabs_solve_the_system(kind, nslabs):
    from slab_cpu import apply7
    x, out, a, b = _local(kind, nslabs)
    assert all(s == 0 for s in out["status"]), out
    if kind == "cg_singular":
        b = b - b.mean()
        assert abs(x.mean()) < 1e-12
    res = b - apply7(a, x)
    for q in range(b.shape[0]):
        assert np.linalg.norm(res[q]) <= 1.0001e-11 * np.linalg.norm(b[q])
    x1, out1, _, _ = _local(kind, 1)
    assert np.linalg.norm(x - x1) <= 1e-9 * np.linalg.norm(x1)
    assert all(abs(i - j) <= 2 for i, j in zip(out["iters"], out1["iters"]))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, kind, q):
    sys.path[:0] = [ROOT, HERE]
    import torch.distributed as dist
    from slab_cpu import NumpySlab
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=timedelta(seconds=60))
    try:
        a, b = _system(kind)
        parts = S.partition(SHAPE[2], world)
        slab = NumpySlab(a, b, parts, rank)
        out = _solve([slab], S.DistTransport(), kind)
        q.put((rank, slab.owned_x(), out))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("kind", ["bicgstab", "cg", "cg_singular"])
def test_gloo_two_ranks_match_two_local_slabs_bit_for_bit(kind):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, kind, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted((q.get(timeout=120) for _ in range(2)), key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    x_dist = np.concatenate([g[1] for g in got], axis=1)
    assert got[0][2] == got[1][2]          # every rank took the same decisions
    x_loc, out_loc, _, _ = _local(kind, 2)
    assert got[0][2]["iters"] == out_loc["iters"]
    assert np.array_equal(x_dist, x_loc)
