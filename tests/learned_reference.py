"""NumPy restatement of the learned preconditioner's level pyramid (csrc/learned.cu), used as
the checker of the device kernels: cell-centred trilinear prolongation P, restriction
R = P^T scaled to a cell average, and the preconditioner
    M(r) = D^-1 r + P_1 w_1,   w_l = gain_l s y_l + P_(l+1) w_(l+1)
with y_l = u_l / s (the LEVELS form) or the odd network term (net(x) - net(-x)) / 2 of
cnn_reference (the NETWORK form).
Arrays are indexed [k, j, i]."""
from __future__ import annotations

import numpy as np

import cnn_reference as R


def _weights_1d(nf: int, nc: int) -> np.ndarray:
    """P along one direction as a dense (nf, nc) matrix."""
    P = np.zeros((nf, nc))
    for f in range(nf):
        I = f >> 1
        J = (I + 1) if (f & 1) else (I - 1)
        J = min(max(J, 0), nc - 1)
        P[f, I] += 0.75
        P[f, J] += 0.25
    return P


def coarse_dims(d):
    return tuple(n if n == 1 else (n + 1) // 2 for n in d)


def pyramid(dims_kji):
    """Level dimensions [k, j, i] from the cell lattice down to about 64 cells."""
    levels = [tuple(dims_kji)]
    while len(levels) < 12:
        f = levels[-1]
        if np.prod(f) <= 64 or all(n == 1 for n in f):
            break
        levels.append(coarse_dims(f))
    return levels


def prolong(w: np.ndarray, fine) -> np.ndarray:
    out = w
    for ax in range(3):
        P = _weights_1d(fine[ax], w.shape[ax])
        out = np.moveaxis(np.tensordot(P, np.moveaxis(out, ax, 0), axes=(1, 0)), 0, ax)
    return out


def prolong_T(v: np.ndarray, coarse) -> np.ndarray:
    out = v
    for ax in range(3):
        P = _weights_1d(v.shape[ax], coarse[ax])
        out = np.moveaxis(np.tensordot(P.T, np.moveaxis(out, ax, 0), axes=(1, 0)), 0, ax)
    return out


def rscale(fine) -> float:
    return 1.0 / 2 ** sum(1 for n in fine if n > 1)


def apply_M(r: np.ndarray, invD: np.ndarray, active: np.ndarray, mode: str = "levels", params=None, bf: bool = False):
    """M(r) on a [k, j, i] lattice; active: boolean mask (all True without an immersed body);
    bf: round the network's input, weights and activations to bfloat16 as the device does."""
    dims = r.shape
    levels = pyramid(dims)
    u0 = np.where(active, invD * r, 0.0)
    z = np.where(active, invD * r, 0.0)
    if mode == "jacobi" or len(levels) < 2:
        return z
    s = np.sqrt(np.sum(u0[active] ** 2) / max(active.sum(), 1)) if active.any() else 1.0
    s = s if s > 0 else 1.0
    us, masks = [None], [None]
    m = active.astype(np.float64)
    u = u0
    for l in range(1, len(levels)):
        u = rscale(levels[l - 1]) * prolong_T(u, levels[l])
        m = rscale(levels[l - 1]) * prolong_T(m, levels[l])
        us.append(u)
        masks.append(m)
    w = None
    for l in range(len(levels) - 1, 0, -1):
        gain = 4.0 ** l
        if mode == "levels":
            y = us[l] / s
        else:
            # the network term is odd: (net(x) - net(-x)) / 2
            shape = (levels[l][2], levels[l][1], levels[l][0])
            xp = np.stack([us[l].ravel() / s, masks[l].ravel()], axis=1)
            xn = np.stack([-us[l].ravel() / s, masks[l].ravel()], axis=1)
            yp, _ = R.forward(params.astype(np.float64), xp, shape, bf=bf, extra_const=l / 8.0)
            yn, _ = R.forward(params.astype(np.float64), xn, shape, bf=bf, extra_const=l / 8.0)
            y = (0.5 * (yp - yn)).reshape(us[l].shape)
        v = gain * s * y
        if w is not None:
            v = v + prolong(w, levels[l])
        w = v
    return z + np.where(active, prolong(w, dims), 0.0)


def poisson7(dims_kji):
    """Negative-definite 7-point operator with unit spacing (Neumann faces closed, one
    Dirichlet face at i = n-1), as a function plus its diagonal."""
    nk, nj, ni = dims_kji
    cE = np.ones((nk, nj, ni))
    cN = np.ones((nk, nj, ni))
    cT = np.ones((nk, nj, ni))
    cE[:, :, -1] = 0.0
    cN[:, -1, :] = 0.0
    cT[-1, :, :] = 0.0
    diag = -(cE + np.roll(cE, 1, axis=2) * (np.arange(ni) > 0) + cN + np.roll(cN, 1, axis=1) * (np.arange(nj)[:, None] > 0)
             + cT + np.roll(cT, 1, axis=0) * (np.arange(nk)[:, None, None] > 0))
    diag[:, :, -1] -= 2.0   # Dirichlet face

    def A(x):
        y = diag * x
        y[:, :, :-1] += cE[:, :, :-1] * x[:, :, 1:]
        y[:, :, 1:] += cE[:, :, :-1] * x[:, :, :-1]
        y[:, :-1, :] += cN[:, :-1, :] * x[:, 1:, :]
        y[:, 1:, :] += cN[:, :-1, :] * x[:, :-1, :]
        y[:-1, :, :] += cT[:-1, :, :] * x[1:, :, :]
        y[1:, :, :] += cT[:-1, :, :] * x[:-1, :, :]
        return y

    return A, diag


def fcg(A, b, M, rtol=1e-8, maxit=5000):
    """Flexible CG truncated to one direction (the device's inner iteration), FP64."""
    x = np.zeros_like(b)
    r = b.copy()
    bn = np.linalg.norm(b)
    p_old = q_old = None
    pq_old = 1.0
    for it in range(1, maxit + 1):
        z = M(r)
        if p_old is None:
            p = z
        else:
            beta = np.vdot(z, q_old) / pq_old
            p = z - beta * p_old
        q = A(p)
        pq = np.vdot(p, q)
        alpha = np.vdot(p, r) / pq
        x += alpha * p
        r -= alpha * q
        if np.linalg.norm(r) <= rtol * bn:
            return x, it
        p_old, q_old, pq_old = p, q, pq
    return x, maxit


def fgmres(A, b, M, m=40, rtol=1e-5, maxit=2000):
    """Restarted right-preconditioned FGMRES (Saad 1993), FP64, modified Gram-Schmidt."""
    x = np.zeros_like(b)
    bn = np.linalg.norm(b)
    tot = 0
    while tot < maxit:
        r = b - A(x)
        beta = np.linalg.norm(r)
        if beta <= rtol * bn:
            return x, tot
        V, Z = [r / beta], []
        H = np.zeros((m + 1, m))
        y = np.zeros(0)
        for j in range(m):
            z = M(V[j])
            w = A(z)
            Z.append(z)
            for i in range(j + 1):
                H[i, j] = np.vdot(w, V[i])
                w = w - H[i, j] * V[i]
            H[j + 1, j] = np.linalg.norm(w)
            tot += 1
            e1 = np.zeros(j + 2)
            e1[0] = beta
            y, *_ = np.linalg.lstsq(H[:j + 2, :j + 1], e1, rcond=None)
            if np.linalg.norm(H[:j + 2, :j + 1] @ y - e1) <= rtol * bn or H[j + 1, j] == 0.0 or tot >= maxit:
                break
            V.append(w / H[j + 1, j])
        x = x + sum(yi * zi for yi, zi in zip(y, Z))
    return x, tot
