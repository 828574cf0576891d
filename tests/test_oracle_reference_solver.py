"""The oracle pinned to the reference's own solver code.

The reference's Simple / Piso / IbPiso and everything they call (src/Solvers, src/Domains,
src/Schemes, src/Math, src/RunControl, src/Parallel) are compiled from its sources with
stand-in PETSc / MPI / LAPACKE / Boost headers (oracle/Makefile target ``refsolver``,
oracle/ref_solver.py).  Two kinds of check:

* lock step (needs the compiled reference): the reference takes each step with its KSPSolve
  returning the oracle's solutions, so everything outside the Krylov solves is compared bit for
  bit -- every assembled matrix row and right-hand side, the fields after every step and the
  continuity error.  The ghost rows' trilinear weights are the one exception: the reference
  inverts their 8 x 8 monomial matrix through LAPACK (src/Math/Matrix.cpp:149-154), replaced here
  by a textbook LU, so they agree to the round-off of that inverse (1e-9 relative);
* fixtures (always): tests/golden/reference_solver.npz holds the reference's outputs (written by
  tests/golden/make_reference_solver_golden.py); the oracle's own runs must reproduce them --
  bit for bit after the lock-step cases' steps, within 1e-10 relative L2 after the 500 SIMPLE
  iterations of the BASELINE's 64 x 64 cavity with both sides solving to 1e-13 (the oracle's
  p' solves also stop at the absolute floor helpers.C1_P_ATOL).
"""
import os

import numpy as np
import pytest

from oracle import ref_solver as R
from oracle.oracle import OracleSolver

import helpers as H
import ref_pin as P

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_solver.npz")
FIELDS = ("u", "p", "massFlowI", "massFlowJ", "massFlowK")
CASES = ("cavity2d", "cavity3d", "skewed", "channel", "piso_inner", "simple_transient", "outlet_top")


def _case(name):
    if name == "cavity2d":
        return H.small_cavity2d()
    if name == "cavity3d":
        return H.small_cavity3d(central=False)
    if name == "skewed":
        nodes, spec = H.small_skewed(nonorth=False)
        return nodes, spec.replace(convection="upwind")
    if name == "piso_inner":
        return H.small_piso_inner()
    if name == "simple_transient":
        return H.small_simple_transient()
    if name == "outlet_top":
        return H.small_outlet_top()
    return H.small_channel_sphere()


needs_reference = pytest.mark.skipif(not R.available(), reason="the reference's sources are not compiled here")


@needs_reference
@pytest.mark.parametrize("name", CASES)
def test_lockstep_bit_exact_with_reference_code(name):
    nodes, spec = _case(name)
    for k, rep in enumerate(P.lockstep(nodes, spec, 3)):
        for s, (plain, ghost, rhs) in enumerate(rep["systems"]):
            assert plain and ghost and rhs, (name, k, s, plain, ghost, rhs)
        assert all(rep["fields"].values()), (name, k, rep["max_field_diff"])
        assert rep["continuity"][0] == rep["continuity"][1]


@pytest.mark.parametrize("name", CASES)
def test_oracle_reproduces_reference_fixture_bit_for_bit(name):
    g = np.load(GOLDEN)
    nodes, spec = _case(name)
    o = OracleSolver(nodes, spec)
    cont = [o.solve() for _ in range(3)]
    for nm in FIELDS:
        assert np.array_equal(o.get(nm), g[f"ls_{name}_{nm}"]), (name, nm)
    assert cont == g[f"ls_{name}_continuity"].tolist()
    o.close()


def test_oracle_matches_reference_on_the_64x64_cavity_after_500_iterations():
    """BASELINE configuration 1 exactly, free running on both sides (1e-13 solves)."""
    g = np.load(GOLDEN)
    nodes, spec, iters = H.c1_parity()
    assert iters == 500 and nodes.shape == (2, 65, 65, 3)
    o = OracleSolver(nodes, spec)
    for _ in range(iters):
        o.solve()
    vol = o.get("vol")
    assert H.rel_l2(o.get("u"), g["c1_u"]) < H.FIELD_RTOL
    assert H.rel_l2(H.demean(o.get("p"), vol), H.demean(g["c1_p"], vol)) < H.FIELD_RTOL
    for nm in ("massFlowI", "massFlowJ"):
        assert H.rel_l2(o.get(nm), g[f"c1_{nm}"]) < H.FIELD_RTOL, nm
    o.close()


@needs_reference
def test_trilinear_weights_match_reference_code():
    """Interpolation::computeTrilinearCoeffs (Interpolation.cpp:135-180) vs the oracle's."""
    from oracle import oracle as O
    rng = np.random.default_rng(21)
    for _ in range(64):
        base = rng.uniform(0.0, 4.0, 3)
        h = rng.uniform(0.05, 0.3, 3)
        corners = np.array([[i, j, k] for k in (0, 1) for j in (0, 1) for i in (0, 1)], dtype=float)
        p8 = base + corners * h + rng.uniform(-0.05, 0.05, (8, 3)) * h
        ip = base + rng.uniform(0.2, 0.8, 3) * h
        b_ref = R.trilinear(p8, ip)
        b_orc = O.trilinear(p8, ip)
        assert np.max(np.abs(b_ref - b_orc)) <= 1e-9 * np.max(np.abs(b_ref))
        assert abs(b_ref.sum() - 1.0) < 1e-9
