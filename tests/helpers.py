"""Shared helpers for the parity tests: small seeded cases and oracle -> device state copies."""
from __future__ import annotations

import numpy as np

from caffe_old_b200 import cases as C

# Tolerances written here, used by every parity test:
#  * kernels outside the Krylov solves: bit-exact (np.array_equal);
#  * fields after whole steps solved to KSP_RTOL on both sides: FIELD_RTOL relative L2
#    (pressure compared after removing its volume-weighted mean, because the all-Neumann
#    cavity pressure is defined up to a constant).
KSP_RTOL = 1e-13
# the immersed-boundary pressure system (non-symmetric ghost rows) has a round-off floor
# just above 1e-13 for its round-off sized second-corrector right-hand side
KSP_RTOL_IB = 1e-12
FIELD_RTOL = 1e-10


# Configuration 1 exactly (64 x 64 x 1 SIMPLE cavity, Re = 100, upwind, 0.7 / 0.3, 500 outer
# iterations) with every solve taken to KSP_RTOL; the p' solves also stop at the absolute floor
# C1_P_ATOL = 1e-13 x the first iteration's ||b|| (9.1e-5).  Without it the relative 1e-13 is
# below this p' system's round-off floor (condition number ~4e3) once SIMPLE has converged a few
# decades, and Jacobi-BiCGStab diverges there (iteration ~375) instead of stagnating.
C1_P_ATOL = 1e-17


def c1_parity():
    nodes, spec, iters = C.config1_cavity2d(n=64)
    return nodes, spec.replace(mom_rtol=KSP_RTOL, p_rtol=KSP_RTOL, p_atol=C1_P_ATOL), iters


def small_cavity2d(n=12, m=10):
    nodes = C.cartesian_nodes((n, m, 1), (1.0, 1.0, 1.0 / n))
    bc, ref = C.lid_cavity_bcs("north", two_d=True)
    spec = C.CaseSpec(kind="simple", bc=bc, ref_vec=ref, rho=1.0, mu=0.01, time_accurate=False, omega_u=0.7,
                      omega_p=0.3, convection="upwind", mom_method="bicgstab_jacobi", p_method="bicgstab_jacobi",
                      mom_rtol=KSP_RTOL, p_rtol=KSP_RTOL, maxit=5000, dt=1.0)
    return nodes, spec


def small_cavity3d(n=(8, 6, 5), central=True, cg=True):
    nodes = C.cartesian_nodes(n, (1.0, 1.0, 1.0))
    bc, ref = C.lid_cavity_bcs("north")
    spec = C.CaseSpec(kind="piso", bc=bc, ref_vec=ref, rho=1.0, mu=0.0025, time_accurate=True, omega_u=1.0, omega_p=1.0,
                      n_inner=1, n_pcorr=2, convection="central" if central else "upwind",
                      mom_method="bicgstab_jacobi", p_method="cg_jacobi" if cg else "bicgstab_jacobi",
                      mom_rtol=KSP_RTOL, p_rtol=KSP_RTOL, maxit=5000, dt=1e-2)
    return nodes, spec


def small_skewed(n=(9, 7, 6), seed=3, nonorth=True):
    nodes = C.skewed_nodes(n, (1.0, 1.0, 1.0), 30.0, 0.1, seed)
    bc, ref = C.lid_cavity_bcs("north")
    spec = C.CaseSpec(kind="piso", bc=bc, ref_vec=ref, rho=1.0, mu=0.0025, time_accurate=True, omega_u=1.0, omega_p=1.0,
                      n_inner=1, n_pcorr=2, convection="central", nonorth=nonorth, mom_method="bicgstab_jacobi",
                      p_method="cg_jacobi", mom_rtol=KSP_RTOL, p_rtol=KSP_RTOL, maxit=5000, dt=5e-3)
    return nodes, spec


def small_channel_sphere(n=(32, 12, 12), seed=0):
    nodes = C.cartesian_nodes(n, (4.0, 1.0, 1.0))
    bc, ref = C.channel_bcs(1.0)
    rng = np.random.default_rng(seed)
    re = float(rng.uniform(100.0, 300.0))
    spec = C.CaseSpec(kind="ibpiso", bc=bc, ref_vec=ref, rho=1.0, mu=0.4 / re, time_accurate=True, omega_u=1.0, omega_p=1.0,
                      n_inner=1, n_pcorr=2, convection="upwind", mom_method="bicgstab_jacobi",
                      p_method="bicgstab_jacobi", mom_rtol=KSP_RTOL_IB, p_rtol=KSP_RTOL_IB, maxit=5000, dt=1e-2,
                      ib_radius=0.2, ib_center=(1.0, 0.5, 0.5))
    return nodes, spec


STATE_NAMES = ("u", "p", "gradP", "d", "massFlowI", "massFlowJ", "massFlowK", "massFlow") + tuple(
    f"pPatch{f}" for f in range(6))


def copy_state(oracle, dev, names=STATE_NAMES):
    for nm in names:
        dev.set_field(nm, oracle.get(nm))


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    den = np.linalg.norm(b)
    if den == 0.0:
        return float(np.linalg.norm(a - b))
    return float(np.linalg.norm(a - b) / den)


def demean(p, vol, mask=None):
    p = np.asarray(p, dtype=np.float64)
    if mask is None:
        mask = np.ones_like(p, dtype=bool)
    w = vol[mask]
    return p - np.sum(p[mask] * w) / np.sum(w)


def oracle_dmet_to_faces(oracle, shape):
    """Per-cell D of the reference (dE..dB) -> the per-face arrays the device keeps."""
    nI, nJ, nK = shape
    out = {}
    d = [oracle.get(f"dmet{f}").reshape(nK, nJ, nI) for f in range(6)]
    DI = np.empty((nK, nJ, nI + 1)); DI[:, :, 1:] = d[0]; DI[:, :, 0] = d[1][:, :, 0]
    DJ = np.empty((nK, nJ + 1, nI)); DJ[:, 1:, :] = d[2]; DJ[:, 0, :] = d[3][:, 0, :]
    DK = np.empty((nK + 1, nJ, nI)); DK[1:] = d[4]; DK[0] = d[5][0]
    out["DI"], out["DJ"], out["DK"] = DI.ravel(), DJ.ravel(), DK.ravel()
    # the west/south/bottom values of interior faces must be the same numbers
    out["W_check"] = np.array_equal(d[1][:, :, 1:], d[0][:, :, :-1]) and np.array_equal(d[3][:, 1:, :], d[2][:, :-1, :]) \
        and np.array_equal(d[5][1:], d[4][:-1])
    return out


def small_piso_inner(n=(8, 6, 5)):
    """PISO with two inner iterations and three correctors per step (Piso.cpp:12-29)."""
    nodes, spec = small_cavity3d(n, central=False, cg=True)
    return nodes, spec.replace(n_inner=2, n_pcorr=3)


def small_simple_transient(n=(7, 6, 5)):
    """Time-accurate SIMPLE: two inner iterations per step (Simple.cpp:78-91)."""
    nodes = C.cartesian_nodes(n, (1.0, 1.0, 1.0))
    bc, ref = C.lid_cavity_bcs("north")
    spec = C.CaseSpec(kind="simple", bc=bc, ref_vec=ref, rho=1.0, mu=0.01, time_accurate=True, n_inner=2, omega_u=0.7,
                      omega_p=0.3, convection="upwind", mom_method="bicgstab_jacobi", p_method="bicgstab_jacobi",
                      mom_rtol=KSP_RTOL, p_rtol=KSP_RTOL, maxit=5000, dt=0.05)
    return nodes, spec


def small_outlet_top(n=(6, 5, 10)):
    """SIMPLE channel along k: inlet at the bottom, fixed-pressure outlet at the top."""
    nodes = C.cartesian_nodes(n, (1.0, 1.0, 3.0))
    bc = ("wall", "wall", "wall", "wall", "outlet", "inlet")
    ref = ((0.0, 0.0, 0.0),) * 5 + ((0.0, 0.0, 1.0),)
    spec = C.CaseSpec(kind="simple", bc=bc, ref_vec=ref, ref_val=(0.0, 0.0, 0.0, 0.0, 0.25, 0.0), rho=1.0, mu=0.05,
                      time_accurate=False, omega_u=0.7, omega_p=0.3, convection="upwind", mom_method="bicgstab_jacobi",
                      p_method="bicgstab_jacobi", mom_rtol=KSP_RTOL, p_rtol=KSP_RTOL, maxit=5000, dt=1.0,
                      u_init=(0.0, 0.0, 1.0))
    return nodes, spec
