"""The oracle against its committed fixtures (tests/golden/oracle_fields.npz, written by
tests/golden/make_oracle_golden.py): u and p of reduced-size versions of the four cases after
1, 5 and 50 steps (1 and 20 for the immersed-boundary channel) stay within the whole-step
parity bar (1e-10 relative L2; pressure after removing its volume-weighted mean).  OpenMP
thread counts change the order of the oracle's sums, so results agree to round-off, not
bit for bit."""
import importlib.util
import os

import numpy as np
import pytest

from oracle.oracle import OracleSolver

from helpers import FIELD_RTOL, demean, rel_l2

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden", "oracle_fields.npz")


def _generator():
    spec = importlib.util.spec_from_file_location("make_oracle_golden", os.path.join(HERE, "golden", "make_oracle_golden.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


GEN = _generator()
CASES = GEN.golden_cases()


@pytest.fixture(scope="module")
def golden():
    with np.load(GOLDEN) as z:
        return {k: z[k] for k in z.files}


@pytest.mark.parametrize("name", list(CASES))
def test_oracle_reproduces_its_fixture(golden, name):
    nodes, spec, steps = CASES[name]
    # the case generators still give the nodes the fixture was made on
    assert np.array_equal(golden[f"{name}/nodes"], nodes)
    o = OracleSolver(golden[f"{name}/nodes"], spec)
    vol, status = o.get("vol"), o.get("status")
    mask = status != 2
    prev = None
    for s in range(1, max(steps) + 1):
        o.solve()
        if s not in steps:
            continue
        u, p = o.get("u"), o.get("p")
        gu, gp = golden[f"{name}/u{s}"], golden[f"{name}/p{s}"]
        eu = rel_l2(u, gu)
        ep = rel_l2(demean(p, vol, mask), demean(gp, vol, mask))
        assert eu < FIELD_RTOL and ep < FIELD_RTOL, (name, s, eu, ep)
        # the fixture moves between its snapshots by far more than the tolerance
        if prev is not None:
            assert rel_l2(gu, prev) > 1e3 * FIELD_RTOL, (name, s)
        prev = gu
    o.close()
