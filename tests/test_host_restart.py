"""Restart files of the C++ host layer (CPU): InitialConditions writes fields in the layout of
the reference's writeRestart (src/Domains/Field/InitialConditions.cpp:77-119; i fastest, one
line per j row, an empty line after each k plane, vector components side by side) and reads
them back as the `restart` initial-condition type, bit for bit.  Files in the reference's own
6-digit form read the same way, and a file with the wrong number of values is refused."""
import os
import subprocess

import numpy as np
import pytest

from caffe_old_b200 import build as B

BUILD = os.path.join(os.path.dirname(B.__file__), "_build")
HOST = os.path.join(os.path.dirname(B.__file__), "host")
INCLUDE = os.path.join(os.path.dirname(os.path.dirname(B.__file__)), "include")

PROGRAM = r"""
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <vector>
#include "InitialConditions.h"

// write <raw> <rst> <components> nI nJ nK : raw float64 planes -> restart file
// read <ic.info> <field> <components> <nCells> <raw> : restart initial condition -> raw planes
int main(int argc, char** argv) {
    try {
        if (argc == 8 && std::strcmp(argv[1], "write") == 0) {
            int c = std::atoi(argv[4]), nI = std::atoi(argv[5]), nJ = std::atoi(argv[6]), nK = std::atoi(argv[7]);
            std::vector<double> v((size_t)c * nI * nJ * nK);
            std::FILE* f = std::fopen(argv[2], "rb");
            if (!f || std::fread(v.data(), 8, v.size(), f) != v.size()) return 3;
            std::fclose(f);
            InitialConditions::writeRestartFile(argv[3], v, c, nI, nJ, nK);
            return 0;
        }
        if (argc == 7 && std::strcmp(argv[1], "read") == 0) {
            Input input("case.info", argv[2]);
            InitialConditions ics(input);
            int c = std::atoi(argv[4]);
            size_t n = (size_t)std::atol(argv[5]);
            std::vector<double> cc(3 * n, 0.);
            std::vector<double> v = ics.values(argv[3], c, cc);
            std::FILE* f = std::fopen(argv[6], "wb");
            if (!f || std::fwrite(v.data(), 8, v.size(), f) != v.size()) return 3;
            std::fclose(f);
            return 0;
        }
    } catch (const char* e) {
        std::cerr << "Error: " << e << std::endl;
        return 1;
    }
    return 2;
}
"""

DIMS = (5, 4, 3)
N = DIMS[0] * DIMS[1] * DIMS[2]


@pytest.fixture(scope="module")
def restart_tool(tmp_path_factory):
    B.build_device()
    B.build_host()
    d = tmp_path_factory.mktemp("restart_tool")
    src = d / "restart_tool.cpp"
    src.write_text(PROGRAM)
    exe = d / "restart_tool"
    cmd = ["g++", "-std=c++17", "-O1", "-I", os.path.join(HOST, "include"), "-I", INCLUDE, str(src), "-o", str(exe),
           os.path.join(BUILD, "libcaffe_host.a"), "-L", BUILD, "-lcaffe_b200", "-Wl,-rpath," + BUILD]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    return str(exe)


def _planes(components, seed):
    rng = np.random.default_rng(seed)
    v = rng.standard_normal((components, N)) * 10.0 ** rng.integers(-300, 300, (components, N))
    v[0, 0] = 1.0 / 3.0
    v[0, 1] = -0.0
    v[-1, -1] = 5e-324
    return v


def _reference_layout(planes, fmt):
    """The text the reference's writeRestart produces for these planes (with number format fmt)."""
    nI, nJ, nK = DIMS
    comp = planes.shape[0]
    out = []
    c = 0
    for _k in range(nK):
        for _j in range(nJ):
            row = ""
            for _i in range(nI):
                for q in range(comp):
                    row += fmt(planes[q, c]) + " "
                c += 1
            out.append(row + "\n")
        out.append("\n")
    return "".join(out)


def _read(tool, tmp_path, field, components, rst_name, with_file_key=True):
    (tmp_path / "case.info").write_text("; empty case\n")
    key = f"\tfile {rst_name}\n" if with_file_key else ""
    (tmp_path / "ic.info").write_text(f"{field}\n{{\n\ttype restart\n{key}}}\n")
    r = subprocess.run([tool, "read", "ic.info", field, str(components), str(N), "out.raw"], cwd=tmp_path, capture_output=True, text=True)
    return r, (np.fromfile(tmp_path / "out.raw", dtype=np.float64).reshape(components, N) if r.returncode == 0 else None)


@pytest.mark.parametrize("components,field", [(1, "p"), (3, "u")])
def test_restart_file_round_trip_is_bit_exact(restart_tool, tmp_path, components, field):
    planes = _planes(components, seed=components)
    planes.tofile(tmp_path / "in.raw")
    r = subprocess.run([restart_tool, "write", "in.raw", f"{field}Restart.rst", str(components), *map(str, DIMS)], cwd=tmp_path,
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    text = (tmp_path / f"{field}Restart.rst").read_text()
    # the reference's layout: nJ lines per plane, then an empty line; nI * components values a line
    want = _reference_layout(planes, lambda x: "X")
    got_shape = ["X " * len(line.split()) + "\n" if line.strip() else "\n" for line in text.splitlines()]
    assert "".join(got_shape) == want
    # default file name <field>Restart.rst (no file key), read back bit for bit
    r, back = _read(restart_tool, tmp_path, field, components, None, with_file_key=False)
    assert r.returncode == 0, r.stderr
    assert np.array_equal(back.view(np.uint64), planes.view(np.uint64))


def test_restart_reads_the_references_six_digit_files(restart_tool, tmp_path):
    planes = _planes(3, seed=7)
    (tmp_path / "ref_u.rst").write_text(_reference_layout(planes, lambda x: "%g" % x))
    r, back = _read(restart_tool, tmp_path, "u", 3, "ref_u.rst")
    assert r.returncode == 0, r.stderr
    want = np.array([[float("%g" % x) for x in row] for row in planes])
    assert np.array_equal(back, want)


def test_restart_file_with_wrong_size_is_refused(restart_tool, tmp_path):
    planes = _planes(1, seed=9)
    text = _reference_layout(planes, lambda x: repr(float(x)))
    (tmp_path / "short.rst").write_text(text.rsplit(" ", 2)[0] + "\n")
    r, _ = _read(restart_tool, tmp_path, "p", 1, "short.rst")
    assert r.returncode == 1 and "were expected" in r.stderr
    (tmp_path / "bad.rst").write_text(text.replace(repr(float(planes[0, 3])), "abc", 1))
    r, _ = _read(restart_tool, tmp_path, "p", 1, "bad.rst")
    assert r.returncode == 1 and "not a number" in r.stderr
    r, _ = _read(restart_tool, tmp_path, "p", 1, "missing.rst")
    assert r.returncode == 1 and "cannot open" in r.stderr


def test_python_and_cpp_restart_files_are_interchangeable(restart_tool, tmp_path):
    """caffe_old_b200.restart writes what the C++ host layer reads and reads what it writes,
    bit for bit, for a scalar and a vector field."""
    from caffe_old_b200.restart import read_restart, write_restart
    for components, field in [(1, "p"), (3, "u")]:
        planes = _planes(components, seed=20 + components)
        cells = planes.T if components == 3 else planes[0]
        write_restart(str(tmp_path / f"py_{field}.rst"), cells, DIMS)
        r, back = _read(restart_tool, tmp_path, field, components, f"py_{field}.rst")
        assert r.returncode == 0, r.stderr
        assert np.array_equal(back.view(np.uint64), planes.view(np.uint64))
        planes.tofile(tmp_path / "in.raw")
        r = subprocess.run([restart_tool, "write", "in.raw", f"cpp_{field}.rst", str(components), *map(str, DIMS)], cwd=tmp_path,
                           capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        got = read_restart(str(tmp_path / f"cpp_{field}.rst"), DIMS, components)
        assert np.array_equal(np.asarray(got).view(np.uint64), np.ascontiguousarray(cells).view(np.uint64))
    with pytest.raises(ValueError, match="were expected"):
        read_restart(str(tmp_path / "py_p.rst"), DIMS, 3)
