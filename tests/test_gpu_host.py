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
from host_cases import read_tec360_fields, read_tec360_last_zone, write_case

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
    mf = np.array(read_tec360_fields(str(tmp_path / "solution" / "testMesh.dat"), len(p))["massFlow"])
    assert rel_l2(mf, o.get("massFlow")) < FIELD_RTOL or np.linalg.norm(mf - o.get("massFlow")) < 1e-14


def test_piso_module_continued_from_restart_files(tmp_path):
    """caffePiso writes uRestart.rst / pRestart.rst (RunControl.writeRestart ON) after 3 steps; a
    second run of the module starts from them (initial conditions of type restart, the reader the
    reference declares in InitialConditions.h:69) and takes 2 more steps.  The oracle does the same:
    3 steps, then a fresh solver given those cell values, 2 steps.  The restart files hold the
    first run's fields exactly (17 digits), and the continued run matches the oracle at 1e-10."""
    from caffe_old_b200 import restart as RS
    spec = C.config2_cavity3d(n=10)[1].replace(mom_rtol=KSP_RTOL, p_rtol=KSP_RTOL)
    lengths, res = (1.0, 1.0, 1.0), (11, 9, 8)
    first, second = tmp_path / "first", tmp_path / "second"
    first.mkdir()
    second.mkdir()
    write_case(str(first), spec, lengths, res, steps=3, run_control_extra="\twriteRestart ON\n")
    subprocess.run([os.path.join(BIN, "hexaMesh")], cwd=first, check=True, capture_output=True)
    r = subprocess.run([os.path.join(BIN, "caffePiso")], cwd=first, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    nodes = _nodes_from_dat(first / "mesh" / "structuredMesh.dat")
    nI, nJ, nK = (int(d) - 1 for d in nodes.shape[2::-1])
    n = nI * nJ * nK
    o = OracleSolver(nodes, spec)
    for _ in range(3):
        o.solve(spec.dt)
    u_rst = RS.read_restart(str(first / "uRestart.rst"), (nI, nJ, nK), 3)     # N x 3
    p_rst = RS.read_restart(str(first / "pRestart.rst"), (nI, nJ, nK))
    assert np.array_equal(u_rst.ravel(), o.get("u").ravel()) or rel_l2(u_rst.ravel(), o.get("u")) < FIELD_RTOL
    ics = (f"u\n{{\n\ttype restart\n\tfile {first / 'uRestart.rst'}\n}}\n\n"
           f"p\n{{\n\ttype restart\n\tfile {first / 'pRestart.rst'}\n}}\n")
    write_case(str(second), spec, lengths, res, steps=2, initial_conditions=ics)
    subprocess.run([os.path.join(BIN, "hexaMesh")], cwd=second, check=True, capture_output=True)
    r = subprocess.run([os.path.join(BIN, "caffePiso")], cwd=second, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    p2, u2 = read_tec360_last_zone(str(second / "solution" / "testMesh.dat"), n)
    o2 = OracleSolver(nodes, spec)
    o2.set("u", u_rst.ravel())
    o2.set("p", p_rst)
    for _ in range(2):
        o2.solve(spec.dt)
    vol = o2.get("vol")
    assert rel_l2(np.array(u2).reshape(3, -1).T.ravel(), o2.get("u")) < FIELD_RTOL
    assert rel_l2(demean(np.array(p2), vol), demean(o2.get("p"), vol)) < FIELD_RTOL


def test_coupled_module_run_matches_oracle(tmp_path):
    """caffeCoupled (the reference's Modules/caffeCoupled.cpp flow) runs a 2-D lid-driven cavity
    case directory; u and p after the last iteration match the oracle's Coupled restatement on
    the same nodes (1e-8: the block solves stop at a 1e-12 relative residual on each side)."""
    from oracle.oracle import OracleCoupled
    spec = C.config1_cavity2d(n=10)[1].replace(mom_method="bicgstab_jacobi", mom_rtol=1e-12, p_rtol=1e-12, maxit=20000)
    steps = 6
    nodes, p, u = _run(tmp_path, "caffeCoupled", spec, (1.0, 1.0, 0.1), (11, 11, 2), steps)
    o = OracleCoupled(nodes, spec)
    for _ in range(steps):
        o.solve(spec.dt)
    eu = rel_l2(u.reshape(3, -1).T.ravel(), o.get("u"))
    po = o.get("p")
    ep = rel_l2(p - p.mean(), po - po.mean())
    print("caffeCoupled u", eu, "p", ep)
    assert eu < 1e-8 and ep < 1e-8
    o.close()


def test_diffusion_module_run_matches_oracle(tmp_path):
    """caffeDiffusion (the reference's Modules/caffeDiffusion.cpp flow) runs the layout of the
    reference's FlatPlateDiffusion2D example (fixed west 1, other sides 0, empty top and bottom)
    on a generated mesh; phi and its gradient after the last solve match the oracle's Diffusion
    restatement (1e-9: the solves stop at a 1e-12 relative residual on each side)."""
    from oracle.oracle import OracleDiffusion
    root = tmp_path
    spec = C.config1_cavity2d(n=4)[1]
    write_case(str(root), spec, (1.0, 1.0, 0.05), (17, 13, 2), steps=2)
    types = ("fixed", "fixed", "fixed", "fixed", "empty", "empty")
    refs = (0.0, 1.0, 0.0, 0.0, 0.0, 0.0)
    with open(root / "case" / "case.info", "w") as f:
        f.write("RunControl\n{\n\tterminationCondition iterations\n\tmaxNumberOfIterations 3\n\tfileWriteInterval 1000\n"
                "\ttimeStep 0.01\n\tmaxSimTime 48\n\tmaxRealTimeHours 48\n}\n\nSolver\n{\n\ttimeAccurate OFF\n}\n\n"
                "LinearSolvers\n{\n\ttolerance 1e-12\n\tmaxIterations 20000\n}\n\nBoundaries\n{\n")
        for face, t, v in zip(C.FACES, types, refs):
            f.write(f"\t{face}\n\t{{\n\t\ttype {t}\n\t\trefValue {v!r}\n\t}}\n")
        f.write("}\n")
    with open(root / "case" / "initialConditions.info", "w") as f:
        f.write("phi\n{\n\ttype uniform\n\tvalue 0\n}\n")
    subprocess.run([os.path.join(BIN, "hexaMesh")], cwd=root, check=True, capture_output=True)
    r = subprocess.run([os.path.join(BIN, "caffeDiffusion")], cwd=root, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    nodes = _nodes_from_dat(root / "mesh" / "structuredMesh.dat")
    n = int(np.prod([d - 1 for d in nodes.shape[:3]]))
    fields = read_tec360_fields(str(root / "solution" / "testMesh.dat"), n)
    o = OracleDiffusion(nodes, types, refs, time_accurate=False, phi0=0.0, method="bicgstab_jacobi", rtol=1e-12, maxit=20000)
    for _ in range(2):
        o.solve(0.01)
    ephi = rel_l2(np.array(fields["phi"]), o.get("phi"))
    grad = np.stack([fields["gradPhi_x"], fields["gradPhi_y"], fields["gradPhi_z"]], axis=1).ravel()
    eg = rel_l2(grad, o.get("gradPhi"))
    print("caffeDiffusion phi", ephi, "gradPhi", eg)
    assert ephi < 1e-9 and eg < 1e-9
    o.close()
