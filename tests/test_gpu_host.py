"""The C++ module executables on the GPU: hexaMesh + caffePiso / caffeIbPiso / caffeSimple
run a case directory in the reference's layout, and the fields they write after the last step
match the CPU oracle run on the same nodes and case (relative L2 1e-10, the whole-step bar;
pressure after removing its volume-weighted mean where the system is singular)."""
import os
import subprocess

import numpy as np
import pytest

from caffe_old_b200 import build as B, cases as C
from oracle.oracle import OracleSolver

from helpers import KSP_RTOL, KSP_RTOL_IB, demean, rel_l2
from host_cases import read_tec360_last_zone, write_case

pytestmark = pytest.mark.gpu
BIN = os.path.join(os.path.dirname(B.__file__), "_build", "bin")
FIELD_RTOL = 1e-10


def _nodes_from_dat(path):
    with open(path) as f:
        head, body = f.read().split("DATAPACKING = BLOCK\n", 1)
    import re
    ni, nj, nk = (int(re.search(rf"{a} = (\d+)", head).group(1)) for a in "IJK")
    vals = np.array([float(v) for v in body.split()]).reshape(3, nk, nj, ni)
    return np.ascontiguousarray(np.moveaxis(vals, 0, -1))


def _run(tmp_path, module, spec, lengths, nodes_ijk, steps):
    write_case(str(tmp_path), spec, lengths, nodes_ijk, steps=steps)
    subprocess.run([os.path.join(BIN, "hexaMesh")], cwd=tmp_path, check=True, capture_output=True)
    r = subprocess.run([os.path.join(BIN, module)], cwd=tmp_path, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    nodes = _nodes_from_dat(tmp_path / "mesh" / "structuredMesh.dat")
    n = int(np.prod([d - 1 for d in nodes.shape[:3]]))
    p, u = read_tec360_last_zone(str(tmp_path / "solution" / "testMesh.dat"), n)
    return nodes, np.array(p), np.array(u)


@pytest.mark.parametrize("module,kind", [("caffePiso", "piso"), ("caffeIbPiso", "ibpiso"), ("caffeSimple", "simple")])
def test_module_run_matches_oracle(tmp_path, module, kind):
    if kind == "piso":
        spec = C.config2_cavity3d(n=10)[1].replace(mom_rtol=KSP_RTOL, p_rtol=KSP_RTOL)
        lengths, res, steps = (1.0, 1.0, 1.0), (11, 9, 8), 3
    elif kind == "ibpiso":
        spec = C.config4_channel_sphere((32, 12, 12), seed=2)[1].replace(mom_rtol=KSP_RTOL_IB, p_rtol=KSP_RTOL_IB)
        lengths, res, steps = (4.0, 1.0, 1.0), (33, 13, 13), 3
    else:
        spec = C.config1_cavity2d(n=12)[1].replace(mom_rtol=KSP_RTOL, p_rtol=KSP_RTOL)
        lengths, res, steps = (1.0, 1.0, 1.0 / 12), (13, 13, 2), 5
    nodes, p, u = _run(tmp_path, module, spec, lengths, res, steps)
    o = OracleSolver(nodes, spec)
    for _ in range(steps):
        o.solve(spec.dt)
    vol, status = o.get("vol"), o.get("status")
    mask = status != 2
    eu = rel_l2(u.reshape(3, -1).T.ravel(), o.get("u"))     # the file holds u planes; the oracle u is N x 3
    ep = rel_l2(demean(p, vol, mask), demean(o.get("p"), vol, mask))
    print(module, "u", eu, "p", ep)
    assert eu < FIELD_RTOL and ep < FIELD_RTOL
