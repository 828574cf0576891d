"""Lock-step comparison of the oracle's Coupled and Diffusion restatements with the reference's
own solver code (src/Solvers/Coupled.cpp, src/Solvers/Diffusion.cpp, compiled into
oracle/_ref/libref_solver.so by oracle/Makefile), and the fixture that keeps the pin where the
reference's sources are absent.

The oracle takes a step phase by phase and keeps every linear system it assembles and every
solution its Krylov solver returns.  The reference then takes the same step with its KSPSolve
handing back the oracle's solutions in the same order, so both continue from identical numbers
and everything outside the Krylov solves -- the block rows with Rhie-Chow coupling, the boundary
folding, the diffusion rows on a skewed mesh, the post-solve fields, gradients and face values --
is compared bit for bit.  tests/golden/reference_coupled.npz holds the reference's fields after
those steps (tests/golden/make_reference_coupled_golden.py); the oracle alone reproduces them.
"""
from __future__ import annotations

import os

import numpy as np
import pytest

import ref_pin as P
from oracle import oracle as O
from oracle import ref_solver as R

needs_reference = pytest.mark.skipif(not R.available(), reason="the reference's sources are not compiled here")

STEPS = 3
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_coupled.npz")


@needs_reference
@pytest.mark.parametrize("name", list(P.coupled_cases()))
def test_coupled_lockstep_bit_exact_with_reference_code(name):
    nodes, spec = P.coupled_cases()[name]
    for step, rep in enumerate(P.coupled_lockstep(nodes, spec, STEPS)):
        assert rep["left"] == 0 and rep["n_systems"] == rep["n_expected"], (name, step)
        for s, (rows, rhs) in enumerate(rep["systems"]):
            assert rows and rhs, (name, step, s)
        for nm in P.COUPLED_FIELDS:
            assert np.array_equal(rep["ref_fields"][nm], rep["oracle_fields"][nm]), (name, step, nm)


@needs_reference
@pytest.mark.parametrize("name", list(P.diffusion_cases()))
def test_diffusion_lockstep_bit_exact_with_reference_code(name):
    nodes, ta, phi0 = P.diffusion_cases()[name]
    for step, rep in enumerate(P.diffusion_lockstep(nodes, ta, phi0, STEPS if ta else 1)):
        assert rep["n_systems"] == 1 and rep["system"] and rep["rhs"], (name, step)
        for nm in P.DIFFUSION_FIELDS:
            assert np.array_equal(rep["ref_fields"][nm], rep["oracle_fields"][nm]), (name, step, nm)


@pytest.mark.parametrize("name", list(P.coupled_cases()))
def test_coupled_oracle_reproduces_reference_fixture_bit_for_bit(name):
    g = np.load(GOLDEN)
    nodes, spec = P.coupled_cases()[name]
    o = O.OracleCoupled(nodes, spec)
    try:
        for _ in range(STEPS):
            o.solve()
        for nm in P.COUPLED_FIELDS:
            assert np.array_equal(o.get(nm), g[f"coupled_{name}_{nm}"]), (name, nm)
    finally:
        o.close()


@pytest.mark.parametrize("name", list(P.diffusion_cases()))
def test_diffusion_oracle_reproduces_reference_fixture_bit_for_bit(name):
    g = np.load(GOLDEN)
    nodes, ta, phi0 = P.diffusion_cases()[name]
    o = O.OracleDiffusion(nodes, P.DIFFUSION_TYPES, P.DIFFUSION_VALUES, time_accurate=ta, phi0=phi0,
                          method="bicgstab_jacobi", rtol=1e-13, maxit=20000)
    try:
        for _ in range(STEPS if ta else 1):
            o.solve(P.DIFFUSION_DT)
        for nm in P.DIFFUSION_FIELDS:
            assert np.array_equal(o.get(nm), g[f"diffusion_{name}_{nm}"]), (name, nm)
    finally:
        o.close()
