"""A CPU stand-in for one device slab's Krylov phases (caffe_old_b200/csrc/slab.cu), so the
host side of the k-slab decomposition -- the distributed BiCGStab / CG control flow, the
halo-plane exchanges and the all-reduces of caffe_old_b200/slab.py -- runs under gloo on CPU
processes.  It holds one 7-point system of the global lattice restricted to the slab's
extended planes and applies the same phase definitions as the device (test infrastructure
only)."""
from __future__ import annotations

import numpy as np
import torch

from caffe_old_b200 import slab as S


def random_system(shape, nr: int, symmetric: bool, seed: int):
    """A diagonally dominant 7-point system on an (nI, nJ, nK) lattice: coefficients
    (7, nK, nJ, nI) in the order P, E, W, N, S, T, B with zero columns outside the lattice,
    and nr right-hand sides."""
    nI, nJ, nK = shape
    rng = np.random.default_rng(seed)
    a = np.zeros((7, nK, nJ, nI))
    if symmetric:
        up = -rng.uniform(0.5, 1.5, (3, nK, nJ, nI))
        up[0][:, :, -1] = 0.
        up[1][:, -1, :] = 0.
        up[2][-1, :, :] = 0.
        a[1], a[3], a[5] = up[0], up[1], up[2]
        a[2][:, :, 1:] = up[0][:, :, :-1]
        a[4][:, 1:, :] = up[1][:, :-1, :]
        a[6][1:, :, :] = up[2][:-1, :, :]
    else:
        a[1:] = -rng.uniform(0.2, 1.5, (6, nK, nJ, nI))
        a[1][:, :, -1] = 0.
        a[2][:, :, 0] = 0.
        a[3][:, -1, :] = 0.
        a[4][:, 0, :] = 0.
        a[5][-1, :, :] = 0.
        a[6][0, :, :] = 0.
    a[0] = -a[1:].sum(axis=0) + rng.uniform(0.05, 0.3, (nK, nJ, nI))
    b = rng.normal(size=(nr, nK, nJ, nI))
    return a, b


def apply7(a, x):
    """y = A x for coefficients a (7, K, J, I) and vectors x (nr, K, J, I); neighbours outside
    the arrays count as zero."""
    y = a[0] * x
    y[..., :-1] += a[1][..., :-1] * x[..., 1:]
    y[..., 1:] += a[2][..., 1:] * x[..., :-1]
    y[..., :-1, :] += a[3][..., :-1, :] * x[..., 1:, :]
    y[..., 1:, :] += a[4][..., 1:, :] * x[..., :-1, :]
    y[..., :-1, :, :] += a[5][:-1] * x[..., 1:, :, :]
    y[..., 1:, :, :] += a[6][1:] * x[..., :-1, :, :]
    return y


class NumpySlab:
    """Slab `rank` of `parts` holding the global system (a, b) on its extended planes."""

    def __init__(self, a, b, parts, rank: int):
        nK = a.shape[1]
        self.k0, self.k1 = parts[rank]
        self.e0, self.e1 = S.extended(self.k0, self.k1, nK)
        self.lo, self.hi = self.k0 - self.e0, self.k1 - self.e0
        self.a = a[:, self.e0:self.e1].copy()
        self.b = b[:, self.e0:self.e1].copy()
        self.nr = b.shape[0]
        self.nIJ = a.shape[2] * a.shape[3]
        z = lambda: np.zeros_like(self.b)
        self.x, self.r, self.rp, self.p, self.v, self.t, self.ph, self.sh = (z() for _ in range(8))
        self.invD = np.ones_like(self.a[0])
        self.sides = [side for side, ok in ((0, self.k0 > 0), (1, self.k1 < nK)) if ok]
        self.red = torch.zeros(8, dtype=torch.float64)

    def _own(self, v):
        return v[..., self.lo:self.hi, :, :]

    def _A(self, v):
        return self._own(apply7(self.a, v))

    def ksp(self, sys: int, phase: int, scal=None) -> int:
        o = self._own
        s = np.zeros(12) if scal is None else np.asarray(scal)
        al, be, om, fl = s[0::4], s[1::4], s[2::4], s[3::4].astype(int)
        sums = []
        if phase in (S.SB_INIT, S.SC_INIT):
            d = o(self.a[0])
            o(self.invD)[...] = np.where(d != 0., 1. / np.where(d != 0., d, 1.), 1.)
            o(self.x)[...] = 0.
            o(self.r)[...] = o(self.b)
            if phase == S.SB_INIT:
                o(self.rp)[...] = o(self.b)
                sums = [float(np.sum(o(self.b)[q] ** 2)) for q in range(self.nr)]
            else:
                o(self.ph)[...] = o(self.invD) * o(self.b)
                o(self.p)[...] = 0.
                o(self.t)[...] = 0.
        elif phase == S.SB_P:
            for q in range(self.nr):
                if not fl[q] & S.SF_RUN:
                    continue
                if fl[q] & S.SF_FRESH:
                    o(self.p)[q] = o(self.r)[q]
                    o(self.rp)[q] = o(self.r)[q]
                else:
                    o(self.p)[q] = o(self.r)[q] + be[q] * (o(self.p)[q] - om[q] * o(self.v)[q])
                o(self.ph)[q] = o(self.invD) * o(self.p)[q]
        elif phase == S.SB_V:
            y = self._A(self.ph)
            for q in range(self.nr):
                if fl[q] & S.SF_RUN:
                    o(self.v)[q] = y[q]
            sums = [float(np.sum(o(self.rp)[q] * y[q])) if fl[q] & S.SF_RUN else 0. for q in range(self.nr)]
        elif phase == S.SB_S:
            for q in range(self.nr):
                if fl[q] & S.SF_RUN:
                    o(self.sh)[q] = o(self.invD) * (o(self.r)[q] - al[q] * o(self.v)[q])
        elif phase == S.SB_T:
            y = self._A(self.sh)
            for q in range(self.nr):
                if fl[q] & S.SF_RUN:
                    sv = o(self.r)[q] - al[q] * o(self.v)[q]
                    o(self.t)[q] = y[q]
                    sums += [float(np.sum(y[q] * sv)), float(np.sum(y[q] * y[q]))]
                else:
                    sums += [0., 0.]
        elif phase == S.SB_X:
            for q in range(self.nr):
                if fl[q] & S.SF_RUN:
                    sv = o(self.r)[q] - al[q] * o(self.v)[q]
                    o(self.x)[q] = o(self.x)[q] + (al[q] * o(self.ph)[q] + om[q] * o(self.sh)[q])
                    rn = sv - om[q] * o(self.t)[q]
                    o(self.r)[q] = rn
                    sums += [float(np.sum(rn * o(self.rp)[q])), float(np.sum(rn * rn))]
                else:
                    sums += [0., 0.]
        elif phase in (S.SB_TRUE, S.SC_TRUE):
            y = self._A(self.x)
            for q in range(self.nr):
                if phase == S.SB_TRUE and not fl[q] & S.SF_TRUE:
                    sums.append(0.)
                    continue
                o(self.r)[q] = o(self.b)[q] - y[q]
                sums.append(float(np.sum(o(self.r)[q] ** 2)))
        elif phase == S.SC_W:
            y = self._A(self.ph)[0]
            o(self.v)[0] = y
            u, r = o(self.ph)[0], o(self.r)[0]
            sums = [float(np.sum(r * u)), float(np.sum(y * u)), float(np.sum(r * r))]
        elif phase == S.SC_UPD:
            si = o(self.v)[0] + be[0] * o(self.p)[0]
            pi = o(self.ph)[0] + be[0] * o(self.t)[0]
            o(self.x)[0] = o(self.x)[0] + al[0] * pi
            o(self.r)[0] = o(self.r)[0] - al[0] * si
            o(self.p)[0] = si
            o(self.t)[0] = pi
            o(self.ph)[0] = o(self.invD) * o(self.r)[0]
        elif phase == S.SC_RESTART:
            o(self.ph)[0] = o(self.invD) * o(self.r)[0]
            o(self.p)[0] = 0.
            o(self.t)[0] = 0.
        elif phase == S.SS_SUM_B:
            sums = [float(np.sum(o(self.b)[0]))]
        elif phase == S.SS_SUB_B:
            o(self.b)[0] -= al[0]
        elif phase == S.SS_SUM_X:
            sums = [float(np.sum(o(self.x)[0]))]
        elif phase == S.SS_SUB_X:
            self.x[0] -= al[0]
        else:
            raise ValueError(phase)
        for q, v in enumerate(sums):
            self.red[q] = v
        return len(sums)

    def buffers(self, arrays, side: int):
        n = sum(planes for _, planes in arrays) * self.nIJ
        return torch.zeros(n, dtype=torch.float64), torch.zeros(n, dtype=torch.float64)

    def halo(self, name: str, planes: int, side: int, dir: int, buf, offset: int) -> int:
        arr = {"kspPh": self.ph, "kspSh": self.sh, "x": self.x}[name]
        plane = (self.lo if side == 0 else self.hi - 1) if dir == 0 else (self.lo - 1 if side == 0 else self.hi)
        n = planes * self.nIJ
        view = buf[offset:offset + n].numpy().reshape(planes, -1)
        if dir == 0:
            view[...] = arr[:planes, plane].reshape(planes, -1)
        else:
            arr[:planes, plane] = view.reshape(arr[:planes, plane].shape)
        return n

    def owned_x(self):
        return self._own(self.x).copy()


class StepSlab:
    """A CPU stand-in for a whole device slab of SlabSolver: the momentum system (three
    right-hand sides) and the p' system are random 7-point systems solved by NumpySlab engines;
    the finite-volume phases only record their names; every cell array the step exchanges is a
    plain array whose owned boundary planes are exchanged for real.  `log` receives
    ("phase", name), ("ksp", sys, phase) and ("exchange", names) in call order."""

    CELL_ARRAYS = {"u": 3, "p": 1, "d": 1, "gradP": 3, "gradPCorr": 3, "gradU": 9}

    def __init__(self, shape, parts, rank: int, seed: int = 5):
        am, bm = random_system(shape, 3, False, seed)
        ap, bp = random_system(shape, 1, True, seed + 1)
        self.mom = NumpySlab(am, bm, parts, rank)
        self.pc = NumpySlab(ap, bp, parts, rank)
        self.sides = self.mom.sides
        self.nIJ = self.mom.nIJ
        self.k0, self.k1 = self.mom.k0, self.mom.k1
        nKe = self.mom.a.shape[1]
        rng = np.random.default_rng(seed + 10 + rank)
        self.cells = {n: rng.normal(size=(c, nKe) + self.mom.a.shape[2:]) for n, c in self.CELL_ARRAYS.items()}
        self.red = torch.zeros(8, dtype=torch.float64)
        self.log = []
        self._cur = self.mom

    def close(self):
        pass

    def phase(self, name: str, dt: float) -> None:
        self.log.append(("phase", name))

    def ksp(self, sys: int, phase: int, scal=None) -> int:
        self.log.append(("ksp", sys, phase))
        self._cur = self.mom if sys == 0 else self.pc
        n = self._cur.ksp(sys, phase, scal)
        self.red.copy_(self._cur.red)
        return n

    def reduce(self, what: str, dt: float) -> None:
        self.log.append(("reduce", what))
        self.red[0] = float(self.k1) if what == "continuity" else 0.5 * float(self.k0)

    def buffers(self, arrays, side: int):
        if side == self.sides[0]:
            self.log.append(("exchange", tuple(name for name, _ in arrays)))
        return self.mom.buffers(arrays, side)

    def halo(self, name: str, planes: int, side: int, dir: int, buf, offset: int) -> int:
        if name in ("kspPh", "kspSh"):
            return self._cur.halo(name, planes, side, dir, buf, offset)
        # u and p' are the solutions of the two systems; the rest are plain arrays
        arr = self.mom.x if name == "u" else (self.pc.x if name == "pCorr" else self.cells[name])
        lo, hi = self.mom.lo, self.mom.hi
        plane = (lo if side == 0 else hi - 1) if dir == 0 else (lo - 1 if side == 0 else hi)
        n = planes * self.nIJ
        view = buf[offset:offset + n].numpy().reshape(planes, -1)
        if dir == 0:
            view[...] = arr[:planes, plane].reshape(planes, -1)
        else:
            arr[:planes, plane] = view.reshape(arr[:planes, plane].shape)
        return n
