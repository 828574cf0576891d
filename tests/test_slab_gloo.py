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
* The whole step (``SlabSolver.solve`` over CPU stand-ins of the device slabs): it takes the
  phases and halo exchanges of the documented halo set, in order, for SIMPLE, PISO with two
  inner iterations and the non-orthogonal extension; under gloo two ranks take exactly the
  steps of the same two slabs in one process, with bit-identical solutions.
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


# ---------------------------------------------------------------- the whole step's orchestration
STEP_SHAPE = (5, 4, 8)


def _step_spec(kind, nonorth=False):
    from caffe_old_b200 import cases as C
    bc, ref = C.lid_cavity_bcs("north")
    return C.CaseSpec(kind=kind, bc=bc, ref_vec=ref, time_accurate=kind == "piso", n_inner=2 if kind == "piso" else 1,
                      n_pcorr=2, nonorth=nonorth, convection="central" if nonorth else "upwind", p_method="cg_jacobi",
                      mom_rtol=1e-10, p_rtol=1e-10, maxit=500, dt=0.01)


def _step_factory():
    from slab_cpu import StepSlab
    return lambda nodes, spec, parts, rank: StepSlab(STEP_SHAPE, parts, rank)


def _nodes():
    from caffe_old_b200 import cases as C
    return C.cartesian_nodes(STEP_SHAPE, (1.0, 1.0, 1.0))


def _outline(log):
    """Phases, reductions and exchanges in order, without the Krylov phases and their vector
    exchanges, and with repeated exchanges of a solve's solution merged."""
    out = []
    for ev in log:
        if ev[0] == "ksp" or (ev[0] == "exchange" and ev[1][0] in ("kspPh", "kspSh")):
            continue
        if out and ev[0] == "exchange" and out[-1] == ev:
            continue
        out.append(ev)
    return out


def _expected_outline(spec):
    """The halo set of the step: which arrays each phase leaves to be exchanged."""
    ev = [("phase", "save_u0")]
    n_inner = spec.n_inner if spec.time_accurate else 1
    n_pc = 1 if spec.kind == "simple" else spec.n_pcorr
    for _ in range(n_inner):
        ev += [("phase", "assemble_momentum"), ("exchange", ("d",)), ("exchange", ("u",)), ("phase", "momentum_post")]
        for _ in range(n_pc):
            ev += [("phase", "assemble_pcorr"), ("exchange", ("pCorr",)), ("phase", "correct"),
                   ("exchange", ("u", "p", "gradP", "gradPCorr"))]
            if spec.nonorth:
                ev += [("phase", "grad_u"), ("exchange", ("gradU",))]
    return ev + [("reduce", "courant"), ("reduce", "continuity")]


@pytest.mark.parametrize("kind,nonorth", [("simple", False), ("piso", False), ("piso", True)])
def test_step_takes_the_documented_phases_and_exchanges(kind, nonorth):
    spec = _step_spec(kind, nonorth)
    sol = S.SlabSolver(_nodes(), spec, 3, slab_factory=_step_factory())
    for s in sol.slabs:
        s.log.clear()
    cont = sol.solve()
    for s in sol.slabs:
        assert _outline(s.log) == _expected_outline(spec), s.k0
    assert cont == float(STEP_SHAPE[2])                   # the max of the slabs' values
    assert sol.last_stats["courant"] == 0.5 * sol.parts[-1][0]
    assert sol.last_stats["status"] == 0


def _step_worker(rank, world, port, q):
    sys.path[:0] = [ROOT, HERE]
    import torch.distributed as dist
    import test_slab_gloo as T
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=timedelta(seconds=60))
    try:
        spec = T._step_spec("piso", True)
        sol = S.SlabSolver(T._nodes(), spec, world, ranks=[rank], transport=S.DistTransport(), slab_factory=T._step_factory())
        conts = [sol.solve() for _ in range(2)]
        s = sol.slabs[0]
        q.put((rank, conts, s.log, s.mom.owned_x(), s.pc.owned_x()))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_gloo_two_ranks_take_the_same_steps_as_two_local_slabs():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_step_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted((q.get(timeout=120) for _ in range(2)), key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    spec = _step_spec("piso", True)
    loc = S.SlabSolver(_nodes(), spec, 2, slab_factory=_step_factory())
    conts = [loc.solve() for _ in range(2)]
    assert got[0][1] == got[1][1] == conts
    for (rank, _, log, xm, xp), s in zip(got, loc.slabs):
        assert log == s.log, rank              # the same phases, solves and exchanges, in order
        assert np.array_equal(xm, s.mom.owned_x()) and np.array_equal(xp, s.pc.owned_x())


def test_mean_projection_only_for_singular_pressure_systems():
    """All walls: the p' system is singular and each p' solve projects b and x (two sums and two
    shifts); with a fixed-pressure outlet there is no projection."""
    from caffe_old_b200 import cases as C
    proj = {S.SS_SUM_B, S.SS_SUB_B, S.SS_SUM_X, S.SS_SUB_X}
    for bc, singular in ((C.lid_cavity_bcs("north")[0], True), (("wall",) * 4 + ("outlet", "inlet"), False)):
        spec = _step_spec("simple").replace(bc=bc)
        sol = S.SlabSolver(_nodes(), spec, 2, slab_factory=_step_factory())
        assert sol.singular is singular
        for s in sol.slabs:
            s.log.clear()
        sol.solve()
        got = [ev[2] for ev in sol.slabs[0].log if ev[0] == "ksp" and ev[1] == 1 and ev[2] in proj]
        assert got == ([S.SS_SUM_B, S.SS_SUB_B, S.SS_SUM_X, S.SS_SUB_X] if singular else [])
