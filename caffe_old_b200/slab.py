"""k-slab decomposition of the Simple / Piso step: one slab of k-planes per rank, one GPU per
rank.

This is the B200 form of the reference's MPI decomposition (ParallelHexaFvmMesh::
initializeSubDomains, src/Domains/HexaFvmMesh/ParallelHexaFvmMesh.cpp:119-307; the PARALLEL
patch exchange of PrimitiveBoundaryCondition::setBoundaries, src/Domains/Field/
PrimitiveBoundaryCondition.tpp:54-141; PETSc's distributed KSPSolve, src/Math/
SparseMatrix.cpp:86-106; Parallel::max of the continuity error, src/Solvers/Simple.cpp:377):

* **Partition.** The global lattice's cell planes are split into contiguous slabs along k
  (``partition``).  Slab r owns planes [k0, k1); its device handle holds those planes plus
  one halo plane on each side that has a neighbour (``extended``), built from the global
  node array with the global case unchanged.
* **Halo planes.** Every finite-volume phase runs unchanged on the slab's lattice; it
  computes the owned cells exactly as on the whole lattice once the halo planes hold the
  neighbours' values of what the phase reads.  After each phase the arrays it wrote are
  exchanged: one nI x nJ plane per array and side, packed into one buffer per side, sent to
  the neighbour by the transport (``DistTransport``: ``torch.distributed`` point-to-point,
  NCCL over NVLink between GPUs, gloo between CPU processes).
* **Reductions.** The linear solves are the device's Jacobi BiCGStab and Chronopoulos-Gear
  CG split at every reduction (``bicgstab``, ``cg``): a phase sweeps the owned cells and
  leaves the slab's sums in an 8-double device buffer, which the transport sums over the
  ranks (an all-reduce) before the host takes the next decision.  Every rank receives the
  same sums and so takes the same decisions.  The continuity error is each slab's scan of
  its own cells, combined by max as the reference's Parallel::max does; the Courant number
  is the max over all cells.

``LocalTransport`` runs all slabs in one process (on one device): the same phases,
exchanges and sums, with copies in place of the point-to-point messages.
"""
from __future__ import annotations

import contextlib
import ctypes

import numpy as np

from . import cases as C

# Krylov phases of caffe_slab_ksp (include/caffe_b200.h)
SB_INIT, SB_P, SB_V, SB_S, SB_T, SB_X, SB_TRUE = 0, 1, 2, 3, 4, 5, 6
SC_INIT, SC_W, SC_UPD, SC_TRUE, SC_RESTART = 10, 11, 12, 13, 14
SS_SUM_B, SS_SUB_B, SS_SUM_X, SS_SUB_X = 20, 21, 22, 23
SF_RUN, SF_FRESH, SF_TRUE = 1, 2, 4

SUM, MAX = "sum", "max"


def partition(nK: int, nslabs: int) -> list[tuple[int, int]]:
    """Owned cell planes [k0, k1) of each slab: contiguous, in rank order, sizes differing by
    at most one (the first nK % nslabs slabs take the extra plane)."""
    if nslabs < 1 or nslabs > nK:
        raise ValueError(f"cannot split {nK} cell planes into {nslabs} slabs")
    base, extra = divmod(nK, nslabs)
    out, k = [], 0
    for r in range(nslabs):
        n = base + (1 if r < extra else 0)
        out.append((k, k + n))
        k += n
    return out


def extended(k0: int, k1: int, nK: int) -> tuple[int, int]:
    """Cell planes a slab's handle holds: the owned ones plus one halo plane on each side that
    has a neighbour."""
    return max(k0 - 1, 0), min(k1 + 1, nK)


def _div(a, b):
    """IEEE double division (inf / nan instead of an exception), as on the device."""
    with np.errstate(all="ignore"):
        return np.float64(a) / np.float64(b)


# ---------------------------------------------------------------------------- transports
class LocalTransport:
    """All slabs in this process: exchanges are copies between the slabs' buffers and a sum
    is taken in rank order."""

    def __init__(self, nslabs: int):
        self.nslabs = nslabs

    def exchange(self, bufs):
        """bufs[r] = (send, recv) for slab r, each a dict side -> tensor (side 0 below, 1 above)."""
        for r in range(len(bufs) - 1):
            lo_send, lo_recv = bufs[r]
            hi_send, hi_recv = bufs[r + 1]
            hi_recv[0].copy_(lo_send[1])
            lo_recv[1].copy_(hi_send[0])

    def allreduce(self, tensors, op):
        total = tensors[0].clone()
        for t in tensors[1:]:
            if op == SUM:
                total += t
            else:
                total = total.maximum(t)
        for t in tensors:
            t.copy_(total)


class DistTransport:
    """One slab per process over ``torch.distributed`` (NCCL for device tensors, gloo for CPU
    tensors): slab r is the process of rank r in ``group``."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.nslabs = dist.get_world_size(group)

    def exchange(self, bufs):
        dist = self.dist
        (send, recv), = bufs
        ops = []
        for side, peer in ((0, self.rank - 1), (1, self.rank + 1)):
            if side in send:
                g = peer if self.group is None else dist.get_global_rank(self.group, peer)
                ops.append(dist.P2POp(dist.isend, send[side], g, self.group))
                ops.append(dist.P2POp(dist.irecv, recv[side], g, self.group))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()

    def allreduce(self, tensors, op):
        dist = self.dist
        (t,) = tensors
        dist.all_reduce(t, op=dist.ReduceOp.SUM if op == SUM else dist.ReduceOp.MAX, group=self.group)


# ---------------------------------------------------------------------------- distributed phases
def _stream(slabs):
    """The stream the slabs' kernels run on, as the current stream of the transport's work."""
    f = getattr(slabs[0], "stream_context", None)
    return f() if f is not None else contextlib.nullcontext()


def _run(slabs, transport, sys: int, phase: int, scal=None) -> np.ndarray:
    """One Krylov phase on every local slab; the sums of the ranks, summed over the ranks."""
    K = 0
    for s in slabs:
        K = s.ksp(sys, phase, scal)
    if K == 0:
        return np.zeros(0)
    with _stream(slabs):
        transport.allreduce([s.red for s in slabs], SUM)
        return slabs[0].red[:K].cpu().numpy().astype(np.float64)


def allreduce_first(slabs, transport, op) -> float:
    """red[0] combined over the ranks (sum or max)."""
    with _stream(slabs):
        transport.allreduce([s.red[:1] for s in slabs], op)
        return float(slabs[0].red[0].cpu())


def exchange(slabs, transport, arrays) -> None:
    """Copy the owned boundary planes of `arrays` ((name, planes) pairs) into the neighbours'
    halo planes: one buffer per slab and side."""
    with _stream(slabs):
        bufs = []
        for s in slabs:
            send, recv = {}, {}
            for side in s.sides:
                send[side], recv[side] = s.buffers(arrays, side)
                off = 0
                for name, planes in arrays:
                    off += s.halo(name, planes, side, 0, send[side], off)
            bufs.append((send, recv))
        transport.exchange(bufs)
        for s, (send, recv) in zip(slabs, bufs):
            for side in s.sides:
                off = 0
                for name, planes in arrays:
                    off += s.halo(name, planes, side, 1, recv[side], off)


def _scal(alpha=(0., 0., 0.), beta=(0., 0., 0.), omega=(0., 0., 0.), flags=(0, 0, 0)) -> np.ndarray:
    v = np.zeros(12)
    for q in range(3):
        v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3] = alpha[q], beta[q], omega[q], flags[q]
    return v


def bicgstab(slabs, transport, sys: int, nr: int, xname: str, rtol: float, maxit: int, atol: float = 0.0) -> dict:
    """Right-preconditioned Jacobi BiCGStab (van der Vorst 1992) over the slabs from x = 0, in the
    device solver's control flow: restart from the true residual whenever the recursive one
    meets the tolerance, omega vanishes or maxit is reached; converged when
    ||b - A x|| <= max(rtol ||b||, atol).  Returns iterations, relative residuals and status
    (0 converged, 1 maxit, 2 breakdown, 3 non-finite) per right-hand side."""
    bb = _run(slabs, transport, sys, SB_INIT)
    tol2 = [max(rtol * rtol * bb[q], atol * atol) for q in range(nr)]
    rho = [np.float64(bb[q]) for q in range(nr)]
    rho_old = [np.float64(1.)] * nr
    alpha = [np.float64(1.)] * nr
    omega = [np.float64(1.)] * nr
    it = [0] * nr
    fresh = [True] * nr
    needT = [False] * nr
    relres = [0.] * nr
    done = [not (bb[q] > 0.) or bb[q] <= tol2[q] for q in range(nr)]
    status = [3 if bb[q] != bb[q] else 0 for q in range(nr)]
    for q in range(nr):
        if bb[q] > 0. and done[q]:
            relres[q] = 1.
    pad = lambda v, z=0.: list(v) + [z] * (3 - nr)
    while True:
        run = [not done[q] for q in range(nr)]
        if not any(run):
            break
        beta = [np.float64(0.) if fresh[q] else _div(rho[q], rho_old[q]) * _div(alpha[q], omega[q]) for q in range(nr)]
        flags = [(SF_RUN if run[q] else 0) | (SF_FRESH if fresh[q] else 0) for q in range(nr)]
        _run(slabs, transport, sys, SB_P, _scal(beta=pad(beta), omega=pad(omega), flags=pad(flags, 0)))
        exchange(slabs, transport, [("kspPh", nr)])
        rv = _run(slabs, transport, sys, SB_V, _scal(flags=pad(flags, 0)))
        for q in range(nr):
            if not run[q]:
                continue
            if rv[q] == 0. or rv[q] != rv[q]:
                needT[q] = True
                run[q] = False
            else:
                alpha[q] = _div(rho[q], rv[q])
        flags = [SF_RUN if run[q] else 0 for q in range(nr)]
        _run(slabs, transport, sys, SB_S, _scal(alpha=pad(alpha), flags=pad(flags, 0)))
        exchange(slabs, transport, [("kspSh", nr)])
        tot = _run(slabs, transport, sys, SB_T, _scal(alpha=pad(alpha), flags=pad(flags, 0)))
        for q in range(nr):
            if run[q]:
                omega[q] = np.float64(0.) if tot[2 * q + 1] == 0. else _div(tot[2 * q], tot[2 * q + 1])
        tot = _run(slabs, transport, sys, SB_X, _scal(alpha=pad(alpha), omega=pad(omega), flags=pad(flags, 0)))
        for q in range(nr):
            if run[q]:
                it[q] += 1
                fresh[q] = False
                rho_old[q] = rho[q]
                rho[q] = np.float64(tot[2 * q])
                rr = tot[2 * q + 1]
                if rr <= tol2[q] or omega[q] == 0. or it[q] >= maxit or rr != rr:
                    needT[q] = True
        if any(needT):
            exchange(slabs, transport, [(xname, nr)])
            flags = [SF_TRUE if needT[q] else 0 for q in range(nr)]
            rrT = _run(slabs, transport, sys, SB_TRUE, _scal(flags=pad(flags, 0)))
            for q in range(nr):
                if not needT[q]:
                    continue
                needT[q] = False
                relres[q] = float(np.sqrt(_div(rrT[q], bb[q])))
                if rrT[q] <= tol2[q]:
                    done[q], status[q] = True, 0
                elif rrT[q] != rrT[q]:
                    done[q], status[q] = True, 3
                elif it[q] >= maxit:
                    done[q], status[q] = True, 1
                else:
                    fresh[q] = True
                    rho[q], rho_old[q], alpha[q], omega[q] = np.float64(rrT[q]), np.float64(1.), np.float64(1.), np.float64(1.)
    exchange(slabs, transport, [(xname, nr)])
    return {"iters": it, "relres": relres, "status": status}


def cg(slabs, transport, sys: int, xname: str, rtol: float, maxit: int, atol: float = 0.0) -> dict:
    """Jacobi CG in the Chronopoulos-Gear single-reduction form over the slabs from x = 0, in
    the device solver's control flow (true-residual check and restart when the recursive
    residual meets the tolerance or a denominator vanishes)."""
    _run(slabs, transport, sys, SC_INIT)
    exchange(slabs, transport, [("kspPh", 1)])
    tot = _run(slabs, transport, sys, SC_W)
    gamma, bb = np.float64(tot[0]), np.float64(tot[2])
    tol2 = max(rtol * rtol * bb, atol * atol)
    alpha = _div(gamma, tot[1]) if tot[1] != 0. else np.float64(0.)
    beta = np.float64(0.)
    it, status, relres = 0, 0, 0.
    done = not (bb > 0.) or bb <= tol2
    if bb > 0. and done:
        relres = 1.
    if bb != bb:
        status = 3
    while not done:
        _run(slabs, transport, sys, SC_UPD, _scal(alpha=(alpha, 0., 0.), beta=(beta, 0., 0.)))
        exchange(slabs, transport, [("kspPh", 1)])
        tot = _run(slabs, transport, sys, SC_W)
        it += 1
        gn, dn, rr = np.float64(tot[0]), np.float64(tot[1]), np.float64(tot[2])
        check = rr <= tol2 or it >= maxit or rr != rr
        bn = _div(gn, gamma)
        den = dn - bn * _div(gn, alpha)
        if den == 0. or den != den or gamma == 0.:
            check = True
        beta, alpha, gamma = bn, _div(gn, den), gn
        if check:
            exchange(slabs, transport, [(xname, 1)])
            t1 = _run(slabs, transport, sys, SC_TRUE)[0]
            relres = float(np.sqrt(_div(t1, bb)))
            if t1 <= tol2:
                done, status = True, 0
            elif t1 != t1:
                done, status = True, 3
            elif it >= maxit:
                done, status = True, 1
            else:
                _run(slabs, transport, sys, SC_RESTART)
                exchange(slabs, transport, [("kspPh", 1)])
                t2 = _run(slabs, transport, sys, SC_W)
                gamma = np.float64(t2[0])
                alpha = _div(gamma, t2[1]) if t2[1] != 0. else np.float64(0.)
                beta = np.float64(0.)
                if gamma == 0.:
                    done, status = True, 2
    exchange(slabs, transport, [(xname, 1)])
    return {"iters": [it], "relres": [relres], "status": [status]}


def project_mean(slabs, transport, sys: int, which: str, ncells: int) -> None:
    """Remove the global mean of b ("b") or of the solution ("x") of a singular system."""
    s_phase, sub_phase = (SS_SUM_B, SS_SUB_B) if which == "b" else (SS_SUM_X, SS_SUB_X)
    tot = _run(slabs, transport, sys, s_phase)
    mean = _div(tot[0], float(ncells))
    _run(slabs, transport, sys, sub_phase, _scal(alpha=(mean, 0., 0.)))


# ---------------------------------------------------------------------------- device slabs
class DeviceSlab:
    """Slab `rank` of a partition on one device: a handle over the slab's extended lattice,
    the owned range declared, the handle's work on the caller's (torch's current) stream."""

    def __init__(self, nodes: np.ndarray, spec: C.CaseSpec, parts, rank: int, device: int = 0, stream=None):
        import torch
        from ._lib import CaffeError, last_error, lib
        from .solver import make_solver
        self._torch, self._lib, self._err, self._last_error = torch, lib(), CaffeError, last_error
        nK = nodes.shape[0] - 1
        self.rank, self.nslabs = rank, len(parts)
        self.k0, self.k1 = parts[rank]
        self.e0, self.e1 = extended(self.k0, self.k1, nK)
        self.solver = make_solver(np.ascontiguousarray(nodes[self.e0:self.e1 + 1]), spec, device)
        self.h = self.solver._h
        self.device = torch.device("cuda", device)
        self.stream = stream if stream is not None else torch.cuda.Stream(self.device)
        if self._lib.caffe_dev_set_stream(self.h, ctypes.c_void_p(self.stream.cuda_stream)) != 0:
            raise CaffeError("caffe_dev_set_stream: " + last_error())
        if self._lib.caffe_slab_set_owned(self.h, self.k0 - self.e0, self.k1 - self.e0) != 0:
            raise CaffeError("caffe_slab_set_owned: " + last_error())
        self.sides = [side for side, ok in ((0, self.k0 > 0), (1, self.k1 < nK)) if ok]
        self.nIJ = self.solver.shape[0] * self.solver.shape[1]
        with self.stream_context():
            self.red = torch.zeros(8, dtype=torch.float64, device=self.device)
        self._bufs: dict = {}

    def stream_context(self):
        return self._torch.cuda.stream(self.stream)

    def close(self):
        self.stream.synchronize()
        self.solver.close()

    def ksp(self, sys: int, phase: int, scal=None) -> int:
        sp = None if scal is None else np.ascontiguousarray(scal, dtype=np.float64)
        n = self._lib.caffe_slab_ksp(self.h, int(sys), int(phase), None if sp is None else sp.ctypes.data_as(ctypes.c_void_p),
                                     ctypes.c_void_p(self.red.data_ptr()))
        if n < 0:
            raise self._err(f"caffe_slab_ksp(phase {phase}): " + self._last_error())
        return n

    def buffers(self, arrays, side: int):
        key = (tuple(arrays), side)
        if key not in self._bufs:
            n = sum(planes for _, planes in arrays) * self.nIJ
            t = self._torch
            self._bufs[key] = (t.empty(n, dtype=t.float64, device=self.device), t.empty(n, dtype=t.float64, device=self.device))
        return self._bufs[key]

    def halo(self, name: str, planes: int, side: int, dir: int, buf, offset: int) -> int:
        n = self._lib.caffe_slab_halo(self.h, name.encode(), int(planes), int(side), int(dir),
                                      ctypes.c_void_p(buf.data_ptr() + 8 * offset))
        if n < 0:
            raise self._err(f"caffe_slab_halo({name}): " + self._last_error())
        return int(n)

    def phase(self, name: str, dt: float) -> None:
        if self._lib.caffe_slab_phase(self.h, name.encode(), float(dt)) != 0:
            raise self._err(f"caffe_slab_phase({name}): " + self._last_error())

    def reduce(self, what: str, dt: float) -> None:
        if self._lib.caffe_slab_reduce(self.h, what.encode(), float(dt), ctypes.c_void_p(self.red.data_ptr())) != 0:
            raise self._err(f"caffe_slab_reduce({what}): " + self._last_error())

    # -- fields on the owned planes, in the global lattice's cell order
    def owned(self, name: str) -> np.ndarray:
        v = self.solver.field(name)
        comps = v.size // self.solver.ncells
        lo, hi = (self.k0 - self.e0) * self.nIJ, (self.k1 - self.e0) * self.nIJ
        return v.reshape(self.solver.ncells, comps)[lo:hi]


class SlabSolver:
    """Simple or Piso (the spec's kind) on a k-slab decomposition of the lattice `nodes`.

    ``nslabs`` slabs in all; this process drives the slabs ``ranks`` (all of them, with the
    default ``LocalTransport``; its own one, ``[dist.get_rank()]``, with ``DistTransport``).
    ``solve(dt)`` takes one step, as Solver::solve does, and returns the continuity error."""

    FIELD_ARRAYS = (("u", 3), ("p", 1), ("pCorr", 1), ("d", 1), ("gradP", 3), ("gradPCorr", 3))

    def __init__(self, nodes: np.ndarray, spec: C.CaseSpec, nslabs: int, ranks=None, transport=None, device: int = 0,
                 slab_factory=None):
        """slab_factory(nodes, spec, parts, rank) builds a slab with DeviceSlab's interface in
        place of a device slab (the host-side tests use CPU stand-ins)."""
        if spec.kind not in ("simple", "piso"):
            raise ValueError("the slab decomposition runs Simple and Piso")
        nodes = np.ascontiguousarray(nodes, dtype=np.float64)
        self.spec = spec
        self.nK = nodes.shape[0] - 1
        self.ncells = (nodes.shape[2] - 1) * (nodes.shape[1] - 1) * self.nK
        self.parts = partition(self.nK, nslabs)
        self.ranks = list(range(nslabs)) if ranks is None else list(ranks)
        self.transport = transport if transport is not None else LocalTransport(nslabs)
        if slab_factory is None:
            import torch
            self.stream = torch.cuda.Stream(torch.device("cuda", device))   # shared by this process's slabs
            self.slabs = [DeviceSlab(nodes, spec, self.parts, r, device, self.stream) for r in self.ranks]
        else:
            self.stream = None
            self.slabs = [slab_factory(nodes, spec, self.parts, r) for r in self.ranks]
        self.singular = not any(t == "outlet" for t in spec.bc)
        self.last_stats: dict = {}
        self.sync_halos()

    def close(self):
        for s in self.slabs:
            s.close()

    def sync_halos(self) -> None:
        arrays = list(self.FIELD_ARRAYS) + ([("gradU", 9)] if self.spec.nonorth else [])
        exchange(self.slabs, self.transport, arrays)

    def _phase(self, name: str, dt: float) -> None:
        for s in self.slabs:
            s.phase(name, dt)

    def _p_solve(self) -> dict:
        sp = self.spec
        if self.singular:
            project_mean(self.slabs, self.transport, 1, "b", self.ncells)
        if sp.p_method == "cg_jacobi":
            out = cg(self.slabs, self.transport, 1, "pCorr", sp.p_rtol, sp.maxit, sp.p_atol)
        else:
            out = bicgstab(self.slabs, self.transport, 1, 1, "pCorr", sp.p_rtol, sp.maxit, sp.p_atol)
        if self.singular:
            project_mean(self.slabs, self.transport, 1, "x", self.ncells)
        return out

    def solve(self, time_step: float | None = None) -> float:
        sp = self.spec
        dt = float(sp.dt if time_step is None else time_step)
        n_inner = sp.n_inner if sp.time_accurate else 1
        n_pc = 1 if sp.kind == "simple" else sp.n_pcorr
        mom, pres = [], []
        self._phase("save_u0", dt)
        for _ in range(n_inner):
            self._phase("assemble_momentum", dt)
            exchange(self.slabs, self.transport, [("d", 1)])
            mom.append(bicgstab(self.slabs, self.transport, 0, 3, "u", sp.mom_rtol, sp.maxit, sp.mom_atol))
            self._phase("momentum_post", dt)
            for _ in range(n_pc):
                self._phase("assemble_pcorr", dt)
                pres.append(self._p_solve())
                self._phase("correct", dt)
                exchange(self.slabs, self.transport, [("u", 3), ("p", 1), ("gradP", 3), ("gradPCorr", 3)])
                if sp.nonorth:
                    self._phase("grad_u", dt)
                    exchange(self.slabs, self.transport, [("gradU", 9)])
        for s in self.slabs:
            s.reduce("courant", dt)
        courant = allreduce_first(self.slabs, self.transport, MAX)
        for s in self.slabs:
            s.reduce("continuity", dt)
        continuity = allreduce_first(self.slabs, self.transport, MAX)
        statuses = [st for r in mom + pres for st in r["status"]]
        self.last_stats = {
            "continuity": continuity, "courant": courant,
            "mom_iters": mom[-1]["iters"], "p_iters_last": pres[-1]["iters"][0],
            "p_iters_total": sum(r["iters"][0] for r in pres), "p_solves": len(pres),
            "p_res_max": max(r["relres"][0] for r in pres), "mom_res_max": max(max(r["relres"]) for r in mom),
            "status": max(statuses) if statuses else 0,
        }
        return continuity

    def field(self, name: str) -> np.ndarray:
        """A cell field on this process's slabs, in the global lattice's cell order (all of
        it with ``LocalTransport``)."""
        return np.concatenate([s.owned(name) for s in self.slabs], axis=0).ravel()


def main(argv=None) -> None:
    """Times the lid-driven cavity (PISO, Re 400, n^3 cells) on the whole lattice and as `slabs`
    slabs driven from this process on one GPU, from the same state, and prints one JSON line:
    seconds per step, Krylov iterations and the largest field difference."""
    import argparse
    import json
    import time

    import torch

    from .solver import make_solver
    ap = argparse.ArgumentParser(description=main.__doc__)
    ap.add_argument("--size", type=int, default=128)
    ap.add_argument("--slabs", type=int, default=2)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=1)
    a = ap.parse_args(argv)
    nodes, spec, _ = C.config2_cavity3d(n=a.size)
    whole = make_solver(nodes, spec)
    sl = SlabSolver(nodes, spec, a.slabs)
    out = {"workload": f"piso_lid_cavity3d_{a.size}^3_re400_cg_jacobi_fp64", "slabs": a.slabs, "transport": "in-process, one GPU"}
    try:
        for name, run in (("whole", lambda: whole.solve()), ("slabs", lambda: sl.solve())):
            for _ in range(a.warmup):
                run()
            torch.cuda.synchronize()
            iters = []
            t0 = time.perf_counter()
            for _ in range(a.steps):
                run()
                st = whole.last_stats if name == "whole" else sl.last_stats
                iters.append(st["p_iters_total"])
            torch.cuda.synchronize()
            out[f"{name}_s_per_step"] = (time.perf_counter() - t0) / a.steps
            out[f"{name}_p_iters"] = iters
        out["slab_over_whole"] = out["slabs_s_per_step"] / out["whole_s_per_step"]
        out["max_abs_du"] = float(np.max(np.abs(sl.field("u") - whole.field("u"))))
    finally:
        sl.close()
        whole.close()
    print(json.dumps(out))


if __name__ == "__main__":
    main()
