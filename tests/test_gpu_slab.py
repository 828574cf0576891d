"""The k-slab decomposition on the device (caffe_old_b200/slab.py over csrc/slab.cu), with 2 to
4 slabs driven in one process on one GPU (``LocalTransport``: the same phases, exchanges and
sums as ranks on separate GPUs, with copies in place of the point-to-point messages).

* Halo planes: after an exchange every slab's halo planes hold its neighbours' owned planes.
* Lock step with the whole-lattice device solver, handing both the same Krylov solutions:
  every owned row of the momentum and p' systems, every right-hand side, d, the face fluxes,
  u, p, grad p, grad p' (and grad u with the non-orthogonal extension) are bit-identical to the
  whole lattice's, step after step.  This is the check of which arrays each phase needs in
  the halo planes.
* Free running (distributed Krylov solves included, every solve to 1e-13): fields within
  1e-9 of the whole-lattice device solver and of the oracle over several steps, for SIMPLE,
  PISO with two correctors, central convection with the non-orthogonal term on a sheared
  mesh, and a channel with a fixed-pressure outlet; the continuity error is the max over the
  slabs of the reference's scan of each slab's cells (its Parallel::max).
* Slabs of one plane each (halo planes on both sides of every owned plane) match the whole
  lattice too.
* The NCCL form of the transport (``DistTransport`` over a one-rank process group: the sums
  all-reduced on device tensors on the slabs' stream) takes the same steps.
* The immersed boundary and the mixed / learned pressure solves are refused.
"""
import numpy as np
import pytest

from caffe_old_b200 import cases as C
from caffe_old_b200 import slab as S
from caffe_old_b200._lib import CaffeError
from caffe_old_b200.solver import make_solver
from oracle import oracle as O

from helpers import KSP_RTOL, demean, rel_l2

pytestmark = pytest.mark.gpu

SLAB_RTOL = 1e-9


def _cavity3d(n=(7, 6, 9), kind="simple", central=False, cg=False):
    nodes = C.cartesian_nodes(n, (1.0, 1.0, 1.0))
    bc, ref = C.lid_cavity_bcs("north")
    spec = C.CaseSpec(kind=kind, bc=bc, ref_vec=ref, rho=1.0, mu=0.01, time_accurate=kind == "piso", omega_u=0.7 if kind == "simple" else 1.0,
                      omega_p=0.3 if kind == "simple" else 1.0, n_inner=1, n_pcorr=2, convection="central" if central else "upwind",
                      mom_method="bicgstab_jacobi", p_method="cg_jacobi" if cg else "bicgstab_jacobi", mom_rtol=KSP_RTOL,
                      p_rtol=KSP_RTOL, maxit=5000, dt=1.0 if kind == "simple" else 1e-2)
    return nodes, spec


def _skewed(n=(7, 6, 8)):
    nodes = C.skewed_nodes(n, (1.0, 1.0, 1.0), 30.0, 0.1, 3)
    bc, ref = C.lid_cavity_bcs("north")
    spec = C.CaseSpec(kind="piso", bc=bc, ref_vec=ref, rho=1.0, mu=0.0025, time_accurate=True, omega_u=1.0, omega_p=1.0,
                      n_inner=2, n_pcorr=2, convection="central", nonorth=True, mom_method="bicgstab_jacobi",
                      p_method="cg_jacobi", mom_rtol=KSP_RTOL, p_rtol=KSP_RTOL, maxit=5000, dt=5e-3)
    return nodes, spec


def _channel(n=(6, 5, 12)):
    # flow along k, so the outlet (a fixed-pressure face) lies on the last slab
    nodes = C.cartesian_nodes(n, (1.0, 1.0, 3.0))
    bc = ("wall", "wall", "wall", "wall", "outlet", "inlet")
    ref = ((0., 0., 0.),) * 5 + ((0., 0., 1.0),)
    spec = C.CaseSpec(kind="simple", bc=bc, ref_vec=ref, ref_val=(0., 0., 0., 0., 0.25, 0.), rho=1.0, mu=0.05,
                      time_accurate=False, omega_u=0.7, omega_p=0.3, mom_method="bicgstab_jacobi",
                      p_method="bicgstab_jacobi", mom_rtol=KSP_RTOL, p_rtol=KSP_RTOL, maxit=5000, dt=1.0, u_init=(0., 0., 1.0))
    return nodes, spec


CASES = {"simple_cavity": lambda: _cavity3d(), "piso_central_cg": lambda: _cavity3d(kind="piso", central=True, cg=True),
         "skewed_nonorth": _skewed, "channel_outlet": _channel}


def _faces(arr, shape, name):
    nI, nJ, nK = shape
    if name == "massFlowI":
        return arr.reshape(nK, nJ, nI + 1)
    if name == "massFlowJ":
        return arr.reshape(nK, nJ + 1, nI)
    return arr.reshape(nK + 1, nJ, nI)


class Pair:
    """The whole-lattice device solver and the slabs, side by side."""

    def __init__(self, nodes, spec, nslabs):
        self.g = make_solver(nodes, spec)
        self.S = S.SlabSolver(nodes, spec, nslabs)
        self.shape = self.g.shape
        self.nIJ = self.shape[0] * self.shape[1]
        self.spec = spec

    def close(self):
        self.S.close()
        self.g.close()

    def put(self, name):
        """The whole lattice's cell array `name` into every slab (halo planes included)."""
        v = self.g.field(name)
        comps = v.size // self.g.ncells
        v = v.reshape(self.g.ncells, comps)
        for s in self.S.slabs:
            s.solver.set_field(name, v[s.e0 * self.nIJ:s.e1 * self.nIJ])

    def same_cells(self, name, what):
        v = self.g.field(name)
        comps = v.size // self.g.ncells
        v = v.reshape(self.g.ncells, comps)
        for s in self.S.slabs:
            got = s.owned(name)
            want = v[s.k0 * self.nIJ:s.k1 * self.nIJ]
            assert np.array_equal(got, want), (what, name, s.rank, float(np.max(np.abs(got - want))))

    def same_faces(self, name, what):
        gv = _faces(self.g.field(name), self.shape, name)
        for s in self.S.slabs:
            sv = _faces(s.solver.field(name), s.solver.shape, name)
            lo, hi = s.k0 - s.e0, s.k1 - s.e0
            if name == "massFlowK":
                got, want = sv[lo:hi + 1], gv[s.k0:s.k1 + 1]
            else:
                got, want = sv[lo:hi], gv[s.k0:s.k1]
            assert np.array_equal(got, want), (what, name, s.rank)


def test_halo_exchange_fills_the_neighbours_planes():
    nodes, spec = _cavity3d(n=(5, 4, 10))
    sol = S.SlabSolver(nodes, spec, 4)
    try:
        nIJ = 20
        rng = np.random.default_rng(0)
        glob = rng.normal(size=(200, 3))
        for s in sol.slabs:
            v = glob[s.e0 * nIJ:s.e1 * nIJ].copy()
            lo, hi = (s.k0 - s.e0) * nIJ, (s.k1 - s.e0) * nIJ
            v[:lo] = -7.0      # halo planes poisoned; only the exchange can restore them
            v[hi:] = -7.0
            s.solver.set_field("u", v)
        S.exchange(sol.slabs, sol.transport, [("u", 3)])
        for s in sol.slabs:
            assert np.array_equal(s.solver.field("u").reshape(-1, 3), glob[s.e0 * nIJ:s.e1 * nIJ]), s.rank
    finally:
        sol.close()


@pytest.mark.parametrize("name,nslabs", [("simple_cavity", 3), ("piso_central_cg", 2), ("skewed_nonorth", 4),
                                         ("channel_outlet", 3)])
def test_lockstep_phases_bit_exact_with_the_whole_lattice(name, nslabs):
    nodes, spec = CASES[name]()
    P = Pair(nodes, spec, nslabs)
    g, sl = P.g, P.S
    dt = spec.dt
    n_inner = spec.n_inner if spec.time_accurate else 1
    n_pc = 1 if spec.kind == "simple" else spec.n_pcorr
    try:
        for step in range(3):
            g.phase("save_u0", dt)
            sl._phase("save_u0", dt)
            for it in range(n_inner):
                what = (step, it)
                g.phase("assemble_momentum", dt)
                sl._phase("assemble_momentum", dt)
                S.exchange(sl.slabs, sl.transport, [("d", 1)])
                for nm in ("momA", "momB", "d"):
                    P.same_cells(nm, what)
                g.phase("solve_momentum", dt)
                P.put("u")
                g.phase("momentum_post", dt)
                sl._phase("momentum_post", dt)
                for nm in ("massFlowI", "massFlowJ", "massFlowK"):
                    P.same_faces(nm, what)
                for q in range(n_pc):
                    what = (step, it, q)
                    g.phase("assemble_pcorr", dt)
                    sl._phase("assemble_pcorr", dt)
                    P.same_cells("pcA", what)
                    P.same_cells("pcB", what)
                    g.phase("solve_pcorr", dt)
                    P.put("pCorr")
                    g.phase("correct", dt)
                    sl._phase("correct", dt)
                    S.exchange(sl.slabs, sl.transport, [("u", 3), ("p", 1), ("gradP", 3), ("gradPCorr", 3)])
                    if spec.nonorth:
                        sl._phase("grad_u", dt)
                        S.exchange(sl.slabs, sl.transport, [("gradU", 9)])
                        P.same_cells("gradU", what)
                    for nm in ("u", "p", "gradP", "gradPCorr", "massFlow"):
                        P.same_cells(nm, what)
                    for nm in ("massFlowI", "massFlowJ", "massFlowK"):
                        P.same_faces(nm, what)
    finally:
        P.close()


def _scan(m, vol):
    """Simple::computeContinuityError's scan (Simple.cpp:358-380) over cells in order."""
    s = 0.0
    for mv, v in zip(m, vol):
        if abs(mv) > s:
            s = abs(mv) / v
    return s


@pytest.mark.parametrize("name,nslabs,steps", [("simple_cavity", 3, 6), ("piso_central_cg", 2, 4), ("skewed_nonorth", 4, 3),
                                               ("channel_outlet", 3, 6)])
def test_free_running_slabs_match_whole_lattice_and_oracle(name, nslabs, steps):
    nodes, spec = CASES[name]()
    P = Pair(nodes, spec, nslabs)
    o = O.OracleSolver(nodes, spec)
    try:
        for _ in range(steps):
            cont = P.S.solve()
            P.g.solve()
            o.solve()
            st = P.S.last_stats
            assert st["status"] == 0 and st["p_res_max"] <= 1.0001e-13 and st["mom_res_max"] <= 1.0001e-13, st
            # the reference's Parallel::max of every slab's own scan
            m, vol = P.S.field("massFlow"), P.S.field("vol")
            nIJ = P.nIJ
            want = max(_scan(m[s.k0 * nIJ:s.k1 * nIJ], vol[s.k0 * nIJ:s.k1 * nIJ]) for s in P.S.slabs)
            assert cont == want
        vol = P.g.field("vol")
        singular = P.S.singular
        for nm in ("u", "p", "gradP", "massFlow"):
            got = P.S.field(nm)
            for ref in (P.g.field(nm), o.get(nm)):
                if nm == "p" and singular:
                    assert rel_l2(demean(got, vol), demean(ref, vol)) < SLAB_RTOL, nm
                elif nm == "massFlow":
                    assert np.max(np.abs(got - ref)) < 1e-12, nm
                else:
                    assert rel_l2(got, ref) < SLAB_RTOL, nm
    finally:
        P.close()
        o.close()


def test_unsupported_forms_are_refused():
    nodes, spec = _cavity3d()
    with pytest.raises(ValueError):
        S.SlabSolver(nodes, spec.replace(kind="ibpiso", ib_radius=0.2, ib_center=(0.5, 0.5, 0.5)), 2)
    with pytest.raises(CaffeError):
        S.SlabSolver(nodes, spec.replace(p_form="mixed"), 2)
    sol = S.SlabSolver(nodes, spec, 2)
    try:
        with pytest.raises(CaffeError):
            sol.slabs[0].solver.solve()      # a slab's step runs through the slab phases only
    finally:
        sol.close()


def test_one_plane_slabs_match_the_whole_lattice():
    """Every slab owns a single plane, so every interior slab has halo planes on both sides of it."""
    nodes, spec = _cavity3d(n=(6, 5, 6))
    P = Pair(nodes, spec, 6)
    try:
        for _ in range(3):
            P.S.solve()
            P.g.solve()
        vol = P.g.field("vol")
        assert rel_l2(P.S.field("u"), P.g.field("u")) < SLAB_RTOL
        assert rel_l2(demean(P.S.field("p"), vol), demean(P.g.field("p"), vol)) < SLAB_RTOL
    finally:
        P.close()


def _nccl_one_rank(q):
    from datetime import timedelta

    import torch
    import torch.distributed as dist
    port = q.get()
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1, timeout=timedelta(seconds=60))
    try:
        torch.cuda.set_device(0)
        nodes, spec = _cavity3d(n=(6, 5, 8))
        sol = S.SlabSolver(nodes, spec, 1, ranks=[0], transport=S.DistTransport(), device=0)
        ref = make_solver(nodes, spec)
        for _ in range(2):
            c1 = sol.solve()
            c2 = ref.solve()
        q.put((c1, c2, rel_l2(sol.field("u"), ref.field("u"))))
        sol.close()
        ref.close()
    finally:
        dist.destroy_process_group()


def test_dist_transport_over_nccl_single_rank():
    """The NCCL form of the transport (all-reduce of the slab sums on device tensors, on the
    slabs' stream) in a one-rank process group: the same step as the whole-lattice solver."""
    import socket

    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    q.put(port)
    p = ctx.Process(target=_nccl_one_rank, args=(q,))
    p.start()
    p.join(timeout=300)
    assert p.exitcode == 0
    c1, c2, du = q.get(timeout=10)
    # the continuity errors are round-off sized (a few 1e-15) after these steps: compared absolutely
    assert du < SLAB_RTOL and abs(c1 - c2) <= 1e-12
