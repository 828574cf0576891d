"""Precision form: FP32 inner solves inside FP64 iterative refinement for the pressure
correction.  Every p' solve must still reach the FP64 true-residual tolerance, and the fields
stay within 1e-6 relative L2 of the FP64 oracle (the bound for the combined learned +
mixed-precision form); the per-field error is printed."""
import numpy as np
import pytest

from oracle.oracle import OracleSolver
from caffe_old_b200.solver import make_solver

from helpers import demean, rel_l2, small_cavity3d, small_channel_sphere, small_skewed

pytestmark = pytest.mark.gpu

MIXED_FIELD_RTOL = 1e-6
P_RTOL = 1e-8


@pytest.mark.parametrize("maker,steps", [(small_cavity3d, 5), (small_skewed, 4), (small_channel_sphere, 4)])
def test_mixed_precision_fields_match_fp64_oracle(maker, steps):
    nodes, spec = maker()
    o = OracleSolver(nodes, spec)                       # FP64, tight tolerance
    d = make_solver(nodes, spec.replace(p_form="mixed", p_rtol=P_RTOL, mom_rtol=1e-10))
    for _ in range(steps):
        o.solve()
        d.solve()
        st = d.last_stats
        assert st["status"] == 0 and st["fallbacks"] == 0, st
        assert st["p_res_max"] <= P_RTOL, st
    vol, status = o.get("vol"), o.get("status")
    mask = status != 2
    errs = {"u": rel_l2(d.field("u"), o.get("u")),
            "p": rel_l2(demean(d.field("p"), vol, mask), demean(o.get("p"), vol, mask))}
    for nm in ("massFlowI", "massFlowJ", "massFlowK"):
        errs[nm] = rel_l2(d.field(nm), o.get(nm))
    print(maker.__name__, {k: f"{v:.2e}" for k, v in errs.items()})
    for k, v in errs.items():
        assert v < MIXED_FIELD_RTOL, (k, v)
