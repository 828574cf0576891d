"""C++ host layer (caffe_old_b200/host): the reference's Input / RunControl / HexaFvmMesh /
Solver interface over the device library.  CPU checks: the INFO-file parse maps every key
to the same case record as the Python host; hexaMesh writes the same nodes; the reference's
own module mains compile unchanged against these headers, and its shipped example cases and
meshes parse (when its sources are present)."""
import json
import os
import subprocess

import numpy as np
import pytest

from caffe_old_b200 import build as B, cases as C
from caffe_old_b200._lib import make_case

from host_cases import write_case

BIN = os.path.join(os.path.dirname(B.__file__), "_build", "bin")
REF_ROOT = B.reference_root()
REF_MODULES = os.path.join(REF_ROOT, "Modules")


@pytest.fixture(scope="module")
def host_bins():
    B.build_device()
    B.build_host()
    return BIN


def _cases():
    nodes2, spec2, _ = C.config2_cavity3d(n=8)
    _, spec4, _ = C.config4_channel_sphere((16, 8, 8), seed=3)
    spec4 = spec4.replace(p_form="learned_mixed")
    _, spec1, _ = C.config1_cavity2d(n=6)
    return [("piso", spec2), ("ibpiso", spec4), ("simple", spec1)]


@pytest.mark.parametrize("kind,spec", _cases())
def test_case_info_parse_matches_python_case(tmp_path, host_bins, kind, spec):
    write_case(str(tmp_path), spec, (1.0, 1.0, 1.0), (9, 9, 9), steps=3)
    out = subprocess.run([os.path.join(host_bins, "caffeCaseInfo"), kind], cwd=tmp_path, capture_output=True, text=True, check=True)
    got = json.loads(out.stdout)
    ref = make_case(spec)
    for key in ("kind", "rho", "mu", "time_accurate", "omega_u", "omega_p", "n_pcorr", "convection", "nonorth",
                "mom_method", "p_method", "p_rtol", "maxit", "ib_radius", "p_init", "p_form"):
        want = getattr(ref, key)
        if key == "n_pcorr" and kind == "simple":
            want = 1
        assert got[key] == want, (key, got[key], want)
    assert got["n_inner"] == (ref.n_inner if ref.time_accurate else 1)
    assert got["bc_type"] == [ref.bc_type[f] for f in range(6)]
    assert got["ref_vec"] == [[ref.ref_vec[f][q] for q in range(3)] for f in range(6)]
    assert got["ref_val"] == [ref.ref_val[f] for f in range(6)]
    assert got["u_init"] == [ref.u_init[q] for q in range(3)]
    if kind == "ibpiso":
        assert got["ib_center"] == [ref.ib_center[q] for q in range(3)]


def test_hexamesh_writes_the_box_nodes(tmp_path, host_bins):
    spec = C.config2_cavity3d(n=4)[1]
    write_case(str(tmp_path), spec, (2.0, 1.0, 0.5), (7, 5, 4), steps=1)
    subprocess.run([os.path.join(host_bins, "hexaMesh")], cwd=tmp_path, capture_output=True, check=True)
    with open(tmp_path / "mesh" / "structuredMesh.dat") as f:
        lines = f.read().split("DATAPACKING = BLOCK\n", 1)[1]
    vals = np.array([float(v) for v in lines.split()])
    got = vals.reshape(3, 4, 5, 7)                    # (xyz, k, j, i)
    want = C.cartesian_nodes((6, 4, 3), (2.0, 1.0, 0.5))   # (k, j, i, xyz)
    assert np.allclose(np.moveaxis(got, 0, -1), want, rtol=0, atol=1e-15)


def test_info_parser_errors_are_reported(tmp_path, host_bins):
    spec = C.config2_cavity3d(n=4)[1]
    write_case(str(tmp_path), spec, (1.0, 1.0, 1.0), (5, 5, 5), steps=1)
    case = tmp_path / "case" / "case.info"
    case.write_text(case.read_text().replace("relaxationFactorPCorr", "relaxationFactorPressure"))
    out = subprocess.run([os.path.join(host_bins, "caffeCaseInfo"), "piso"], cwd=tmp_path, capture_output=True, text=True)
    assert out.returncode != 0 and "relaxationFactorPCorr" in out.stderr


@pytest.mark.skipif(not os.path.isdir(REF_MODULES), reason="reference sources not present")
@pytest.mark.parametrize("module", ["caffeSimple.cpp", "caffePiso.cpp", "caffeIbPiso.cpp", "caffeMultiphasePiso.cpp", "caffeCoupled.cpp",
                                    "caffeDiffusion.cpp", "hexaMesh.cpp"])
def test_reference_module_mains_compile_unchanged(tmp_path, host_bins, module):
    """The reference's module mains, read where they lie, compile and link against the host
    layer's headers with no change (the drop-in property of the host interface)."""
    host = os.path.join(os.path.dirname(B.__file__), "host")
    build = os.path.join(os.path.dirname(B.__file__), "_build")
    exe = tmp_path / module.replace(".cpp", "")
    cmd = ["g++", "-std=c++17", "-O0", "-I", os.path.join(host, "include"), "-I", os.path.join(os.path.dirname(build), "..", "include"),
           os.path.join(REF_MODULES, module), "-o", str(exe), os.path.join(build, "libcaffe_host.a"), "-L", build, "-lcaffe_b200"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]


REF_EXAMPLES = os.path.join(REF_ROOT, "ExampleCases")


def _example_cases():
    if not os.path.isdir(REF_EXAMPLES):
        return []
    out = []
    for name in sorted(os.listdir(REF_EXAMPLES)):
        case = os.path.join(REF_EXAMPLES, name, "case", "case.info")
        if not os.path.isfile(case):
            continue
        text = open(case).read()
        if "relaxationFactorMomentum" not in text:
            continue                      # the diffusion example has no flow solver keys
        kind = "ibpiso" if "ImmersedBoundaries" in text else ("piso" if "timeAccurate ON" in text else "simple")
        out.append((name, kind))
    return out


def _info_value(text, block, key):
    """The value of `key` inside `block { ... }` of an INFO file (plain text scan)."""
    import re
    body = text[text.index(block):]
    return re.search(rf"^\s*{key}\s+(\S+)", body, flags=re.M).group(1)


@pytest.mark.skipif(not os.path.isdir(REF_EXAMPLES), reason="reference example cases not present")
@pytest.mark.parametrize("name,kind", _example_cases())
def test_reference_example_cases_parse(tmp_path, host_bins, name, kind):
    """Every flow example case the reference ships (ExampleCases/*/case), read where it lies,
    parses with the host layer's INFO reader into the device library's case record, with
    the values the files give.  An example without Boundaries.<face>.refValue is refused
    with the missing key named: FlowBoundaryConditions.cpp reads refValue for every face
    with no default, so the reference's own lookup throws on that file too."""
    import shutil
    shutil.copytree(os.path.join(REF_EXAMPLES, name, "case"), tmp_path / "case")
    out = subprocess.run([os.path.join(host_bins, "caffeCaseInfo"), kind], cwd=tmp_path, capture_output=True, text=True)
    text = (tmp_path / "case" / "case.info").read_text()
    if text[text.index("Boundaries"):].count("refValue") < 6:
        assert out.returncode == 1 and "refValue" in out.stderr, out.stderr
        return
    assert out.returncode == 0, out.stderr
    got = json.loads(out.stdout)
    assert got["rho"] == float(_info_value(text, "Solver", "rho"))
    assert got["mu"] == float(_info_value(text, "Solver", "mu"))
    assert got["omega_u"] == float(_info_value(text, "Solver", "relaxationFactorMomentum"))
    assert got["omega_p"] == float(_info_value(text, "Solver", "relaxationFactorPCorr"))
    assert got["time_accurate"] == (1 if _info_value(text, "Solver", "timeAccurate") == "ON" else 0)
    faces = ["east", "west", "north", "south", "top", "bottom"]
    types = {"inlet": 0, "outlet": 1, "wall": 2, "empty": 3, "zeroGradient": 4}
    for f, face in enumerate(faces):
        block = text[text.index("Boundaries"):]
        assert got["bc_type"][f] == types[_info_value(block, face, "type")], face
    if kind == "ibpiso":
        assert got["ib_radius"] == float(_info_value(text, "ImmersedBoundaries", "radius"))


def _example_meshes():
    if not os.path.isdir(REF_EXAMPLES):
        return []
    return [n for n in sorted(os.listdir(REF_EXAMPLES)) if os.path.isfile(os.path.join(REF_EXAMPLES, n, "mesh", "structuredMesh.info"))]


@pytest.mark.skipif(not os.path.isdir(REF_EXAMPLES), reason="reference example cases not present")
@pytest.mark.parametrize("name", _example_meshes())
def test_reference_example_meshes_generate(tmp_path, host_bins, name):
    """hexaMesh reads every mesh/structuredMesh.info the reference ships (with its resolution
    reduced to 6 x 5 x 4 nodes to keep the file small): the corner nodes are the file's
    vertices times its MetricConversion."""
    import re
    src = open(os.path.join(REF_EXAMPLES, name, "mesh", "structuredMesh.info")).read()
    small = re.sub(r"^(\s*Resolution\s+)\([^)]*\)", r"\1(6,5,4)", src, flags=re.M)
    assert small != src
    (tmp_path / "mesh").mkdir()
    (tmp_path / "mesh" / "structuredMesh.info").write_text(small)
    r = subprocess.run([os.path.join(host_bins, "hexaMesh")], cwd=tmp_path, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    with open(tmp_path / "mesh" / "structuredMesh.dat") as f:
        body = f.read().split("DATAPACKING = BLOCK\n", 1)[1]
    nodes = np.moveaxis(np.array([float(v) for v in body.split()]).reshape(3, 4, 5, 6), 0, -1)   # (k, j, i, xyz)
    scale = float(re.search(r"^\s*MetricConversion\s*=?\s*(\S+)", src, flags=re.M).group(1))
    verts = [np.array([float(x) for x in re.search(rf"^\s*v{q}\s+\(([^)]*)\)", src, flags=re.M).group(1).split(",")])
             for q in range(1, 9)]
    corners = [nodes[0, 0, 0], nodes[0, 0, -1], nodes[0, -1, -1], nodes[0, -1, 0],
               nodes[-1, 0, 0], nodes[-1, 0, -1], nodes[-1, -1, -1], nodes[-1, -1, 0]]
    for q in range(8):
        assert np.allclose(corners[q], scale * verts[q], rtol=0, atol=1e-14), (name, q, corners[q], verts[q])
