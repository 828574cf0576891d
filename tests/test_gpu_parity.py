"""Parity of the CUDA path (through the C ABI) with the CPU oracle.

Kernels outside the Krylov solves are compared bit for bit on identical inputs; whole
steps are compared field-wise after solving every system to a 1e-13 relative residual
on both sides (tolerance FIELD_RTOL = 1e-10 relative L2, pressure without its mean)."""
import os

import numpy as np
import pytest

from oracle.oracle import OracleSolver
from caffe_old_b200.solver import make_solver
from caffe_old_b200 import cases as C

from helpers import (FIELD_RTOL, STATE_NAMES, c1_parity, copy_state, demean, oracle_dmet_to_faces, rel_l2,
                     small_cavity2d, small_cavity3d, small_channel_sphere, small_outlet_top, small_piso_inner,
                     small_simple_transient, small_skewed)

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("maker", [small_cavity2d, small_cavity3d, small_skewed])
def test_metrics_bit_exact(maker):
    nodes, spec = maker()
    o = OracleSolver(nodes, spec)
    d = make_solver(nodes, spec)
    for nm in ("vol", "cc", "SI", "SJ", "SK", "fcI", "fcJ", "fcK"):
        a, b = d.field(nm), o.get(nm)
        assert np.array_equal(a, b), nm
    faces = oracle_dmet_to_faces(o, d.shape)
    assert faces["W_check"]
    for nm in ("DI", "DJ", "DK"):
        assert np.array_equal(d.field(nm), faces[nm]), nm


def _advance_oracle(o, steps):
    for _ in range(steps):
        o.solve()


@pytest.mark.parametrize("maker,steps", [(small_cavity2d, 3), (small_cavity3d, 2), (small_skewed, 2),
                                         (small_channel_sphere, 3), (small_piso_inner, 2), (small_simple_transient, 2),
                                         (small_outlet_top, 3)])
def test_phases_bit_exact(maker, steps):
    """Every phase outside the Krylov solves, from the same state: bit for bit.  The skewed mesh
    runs with the non-orthogonal correction (its cell velocity gradient is part of the state);
    the immersed-boundary channel compares the rows of active cells here (ghost rows: below)."""
    nodes, spec = maker()
    o = OracleSolver(nodes, spec)
    _advance_oracle(o, steps)
    d = make_solver(nodes, spec)
    dt = spec.dt
    ib = spec.kind == "ibpiso"
    # momentum assembly
    copy_state(o, d, STATE_NAMES + (("gradU",) if spec.nonorth else ()))
    o.phase("save_u0", dt)
    d.phase("save_u0", dt)
    if ib:
        for nm in ("ib_field", "ib_coeffs"):
            o.phase(nm, dt)
            d.phase(nm, dt)
        assert np.array_equal(d.field("status"), o.get("status"))
    rows = o.get("status") == 0 if ib else slice(None)
    o.phase("assemble_momentum", dt)
    d.phase("assemble_momentum", dt)
    N = d.ncells
    oa, da = o.get("momA").reshape(N, 7), d.field("momA").reshape(N, 7)
    assert np.array_equal(oa[rows], da[rows])
    assert np.array_equal(o.get("momB").reshape(N, 3)[rows], d.field("momB").reshape(N, 3)[rows])
    assert np.array_equal(o.get("d")[rows], d.field("d")[rows])
    # Rhie-Chow after the (oracle's) momentum solution
    o.phase("solve_momentum", dt)
    d.set_field("u", o.get("u"))
    o.phase("momentum_post", dt)
    d.phase("momentum_post", dt)
    for nm in ("massFlowI", "massFlowJ", "massFlowK"):
        assert np.array_equal(o.get(nm), d.field(nm)), nm
    # pressure-correction assembly
    o.phase("assemble_pcorr", dt)
    d.phase("assemble_pcorr", dt)
    assert np.array_equal(o.get("pcA").reshape(N, 7)[rows], d.field("pcA").reshape(N, 7)[rows])
    assert np.array_equal(o.get("pcB")[rows], d.field("pcB")[rows])
    # correction after the (oracle's) p' solution
    o.phase("solve_pcorr", dt)
    d.set_field("pCorr", o.get("pCorr"))
    o.phase("correct", dt)
    d.phase("correct", dt)
    for nm in ("u", "p", "massFlow", "massFlowI", "massFlowJ", "massFlowK", "gradP", "gradPCorr") + tuple(
            f"pPatch{f}" for f in range(6)) + (("gradU",) if spec.nonorth else ()):
        assert np.array_equal(o.get(nm), d.field(nm)), nm
    # reductions
    o.phase("continuity", dt)
    d.phase("continuity", dt)
    assert d.stats()["continuity"] == o.stats()["continuity"]
    if not ib:   # IbPiso::solve computes no Courant number (IbPiso.cpp:43-61)
        o.phase("courant", dt)
        d.phase("courant", dt)
        assert d.stats()["courant"] == o.stats()["courant"]


@pytest.mark.parametrize("maker,steps", [(small_cavity2d, 12), (small_cavity3d, 4), (small_skewed, 3),
                                         (small_channel_sphere, 3), (small_piso_inner, 3), (small_simple_transient, 4),
                                         (small_outlet_top, 6)])
def test_steps_match_oracle(maker, steps):
    nodes, spec = maker()
    o = OracleSolver(nodes, spec)
    d = make_solver(nodes, spec)
    for _ in range(steps):
        co = o.solve()
        cd = d.solve()
        assert d.last_stats["status"] == 0, d.last_stats
    vol = o.get("vol")
    status = o.get("status")
    mask = status != 2
    uo, ud = o.get("u"), d.field("u")
    assert rel_l2(ud, uo) < FIELD_RTOL
    po, pd = o.get("p"), d.field("p")
    assert rel_l2(demean(pd, vol, mask), demean(po, vol, mask)) < FIELD_RTOL
    for nm in ("massFlowI", "massFlowJ", "massFlowK"):
        assert rel_l2(d.field(nm), o.get(nm)) < FIELD_RTOL, nm
    assert np.isfinite(cd) and np.isfinite(co)


def test_c1_exactly_matches_reference_code_after_500_iterations():
    """BASELINE configuration 1 as stated (64 x 64 x 1 unit-square cavity, Re = 100, SIMPLE,
    upwind, 0.7 / 0.3 relaxation, zero initial fields, 500 outer iterations) on the device,
    against the reference's own solver code run here (tests/golden/reference_solver.npz, written
    by tests/golden/make_reference_solver_golden.py) and against the oracle: u, v, p (p without
    its mean: the all-Neumann cavity fixes it up to a constant) within FIELD_RTOL = 1e-10."""
    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_solver.npz"))
    nodes, spec, iters = c1_parity()
    d = make_solver(nodes, spec)
    o = OracleSolver(nodes, spec)
    for _ in range(iters):
        d.solve()
        o.solve()
        assert d.last_stats["status"] == 0, d.last_stats
    vol = o.get("vol")
    ud, pd = d.field("u"), d.field("p")
    for ref_u, ref_p in ((g["c1_u"], g["c1_p"]), (o.get("u"), o.get("p"))):
        assert rel_l2(ud.reshape(-1, 3)[:, :2], ref_u.reshape(-1, 3)[:, :2]) < FIELD_RTOL
        assert rel_l2(demean(pd, vol), demean(ref_p, vol)) < FIELD_RTOL
    assert rel_l2(d.field("massFlowI"), g["c1_massFlowI"]) < FIELD_RTOL
    assert rel_l2(d.field("massFlowJ"), g["c1_massFlowJ"]) < FIELD_RTOL


def test_skewed_32_cubed_ten_steps_match_oracle():
    """Configuration 3's sheared (30 degrees) and jittered mesh at 32^3 with the non-orthogonal
    correction, 10 PISO steps."""
    nodes, spec = small_skewed(n=(32, 32, 32))
    o = OracleSolver(nodes, spec)
    d = make_solver(nodes, spec)
    for _ in range(10):
        o.solve()
        d.solve()
        assert d.last_stats["status"] == 0, d.last_stats
    vol = o.get("vol")
    assert rel_l2(d.field("u"), o.get("u")) < FIELD_RTOL
    assert rel_l2(demean(d.field("p"), vol), demean(o.get("p"), vol)) < FIELD_RTOL
    for nm in ("massFlowI", "massFlowJ", "massFlowK"):
        assert rel_l2(d.field(nm), o.get(nm)) < FIELD_RTOL, nm


def test_ib_stencils_bit_exact():
    """Ghost classification and image-point rows (IbPiso.cpp:65-190) equal the oracle's."""
    nodes, spec = small_channel_sphere()
    o = OracleSolver(nodes, spec)
    o.phase("ib_field")
    o.phase("ib_coeffs")
    d = make_solver(nodes, spec)
    status = o.get("status")
    assert np.array_equal(d.field("status"), status)
    cells = np.flatnonzero(status == 1)
    assert np.array_equal(d.field("ibCell"), cells)
    beta = o.get("ibBeta").reshape(-1, 8)
    sten = o.get("ibStencil").reshape(-1, 8).astype(int)
    col = d.field("ibCol").reshape(-1, 9).astype(int)
    vm = d.field("ibValMom").reshape(-1, 9)
    vp = d.field("ibValP").reshape(-1, 9)
    assert np.array_equal(col[:, 0], cells)
    for g, c in enumerate(cells):
        dm, dp = 1.0, -1.0
        for m in range(8):
            if sten[g, m] == c:
                dm += beta[g, m]
                dp = -1.0 + beta[g, m]
                assert col[g, m + 1] == -1
            else:
                dp = -1.0
                assert col[g, m + 1] == (-1 if status[sten[g, m]] == 2 else sten[g, m])
                assert vm[g, m + 1] == beta[g, m] and vp[g, m + 1] == beta[g, m]
        assert vm[g, 0] == dm and vp[g, 0] == dp
    d.solve()
    ost = o.stats()
    assert d.last_stats["n_ghost"] == int(ost["ghosts"]) == len(cells)


@pytest.mark.parametrize("method", ["cg_jacobi", "bicgstab_jacobi"])
def test_ksp7_matches_oracle(method):
    from oracle import oracle as O
    from caffe_old_b200._lib import ksp7_solve
    rng = np.random.default_rng(7)
    nI, nJ, nK = 17, 13, 11
    N = nI * nJ * nK
    # symmetric, negative definite 7-point operator like the p' system
    aE = rng.uniform(0.5, 1.5, N); aN = rng.uniform(0.5, 1.5, N); aT = rng.uniform(0.5, 1.5, N)
    idx = np.arange(N); i = idx % nI; j = (idx // nI) % nJ; k = idx // (nI * nJ)
    aE[i == nI - 1] = 0; aN[j == nJ - 1] = 0; aT[k == nK - 1] = 0
    aW = np.zeros(N); aW[1:] = aE[:-1]; aW[i == 0] = 0
    aS = np.zeros(N); aS[nI:] = aN[:-nI]; aS[j == 0] = 0
    aB = np.zeros(N); aB[nI * nJ:] = aT[:-nI * nJ]; aB[k == 0] = 0
    aP = -(aE + aW + aN + aS + aT + aB) - rng.uniform(0.01, 0.1, N)
    if method == "bicgstab_jacobi":
        aE = aE * rng.uniform(0.7, 1.3, N)
        aE[i == nI - 1] = 0
    coef = np.stack([aP, aE, aW, aN, aS, aT, aB])
    b = rng.standard_normal(N)
    xd, itd, rrd, std = ksp7_solve((nI, nJ, nK), coef, b, method, 1e-12, 10000)
    xo, ito, rro, sto = O.ksp7((nI, nJ, nK), coef, b, method, 1e-12, 10000)
    assert std == 0 and sto == 0
    assert rrd <= 1e-12
    assert rel_l2(xd, xo) < 1e-9
    assert abs(itd - ito) <= max(3, 0.1 * ito)
