"""The host layer's SparseMatrix / SparseVector (the reference's linear-algebra interface,
src/Math/SparseMatrix.h:34-81, SparseVector.h:8-43) and the compressed-row device solve behind
them (caffe_csr_solve).  CPU: assembly semantics -- INSERT, negative indices ignored, zeroEntries
keeps the structure -- norms and products, and a solve that fails loudly without a GPU.  GPU: the
class solves non-symmetric (BiCGStab) and symmetric (CG) systems to a 1e-10 true residual, and
caffe_csr_solve agrees with a direct solve."""
import os
import subprocess

import numpy as np
import pytest

from caffe_old_b200 import build as B
from caffe_old_b200 import _lib

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def sparse_check(tmp_path_factory):
    B.build_device()
    B.build_host()
    build = os.path.join(os.path.dirname(B.__file__), "_build")
    host = os.path.join(os.path.dirname(B.__file__), "host")
    exe = str(tmp_path_factory.mktemp("sparse") / "sparse_check")
    cmd = ["g++", "-std=c++17", "-O1", "-I", os.path.join(host, "include"), "-I", os.path.join(os.path.dirname(HERE), "include"),
           os.path.join(HERE, "cpp", "sparse_check.cpp"), "-o", exe, os.path.join(build, "libcaffe_host.a"), "-L", build,
           "-lcaffe_b200", "-Wl,-rpath," + build]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    return exe


def test_assembly_semantics(sparse_check):
    r = subprocess.run([sparse_check, "semantics"], capture_output=True, text=True)
    assert r.returncode == 0 and "OK semantics" in r.stdout, r.stdout


def test_solve_without_gpu_raises(sparse_check):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    r = subprocess.run([sparse_check, "solve", "8"], capture_output=True, text=True)
    assert r.returncode == 2 and "no CUDA device available" in r.stdout, r.stdout


def test_csr_entry_rejects_invalid_input_before_device_calls():
    L = _lib.lib()
    ptr = np.array([0, 1, 3], dtype=np.int32)
    col = np.array([0, 0, 2], dtype=np.int32)   # column 2 of a 2 x 2 matrix
    val = np.ones(3)
    b = np.ones(2)
    x = np.zeros(2)
    with pytest.raises(_lib.CaffeError, match="out of range"):
        _lib.csr_solve(ptr, col, val, b)
    with pytest.raises(_lib.CaffeError, match="symmetric Gauss-Seidel"):
        _lib.csr_solve(ptr, np.array([0, 0, 1], dtype=np.int32), val, b, method="bicgstab_sgs")
    del L, x


@pytest.mark.gpu
def test_sparse_matrix_class_solves_on_device(sparse_check):
    r = subprocess.run([sparse_check, "solve", "48"], capture_output=True, text=True)
    assert r.returncode == 0 and "OK solve" in r.stdout, r.stdout


@pytest.mark.gpu
@pytest.mark.parametrize("method", ["bicgstab_jacobi", "cg_jacobi"])
def test_csr_solve_matches_direct_solve(method):
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla
    rng = np.random.default_rng(3)
    n = 3000
    # random sparse rows, diagonally dominant (symmetric for CG)
    M = sp.random(n, n, density=4.0 / n, random_state=rng, format="csr")
    M.data = -np.abs(M.data)
    if method == "cg_jacobi":
        M = (M + M.T) * 0.5
    M = M + sp.diags(np.asarray(abs(M).sum(axis=1)).ravel() + rng.uniform(0.5, 1.0, n))
    M = sp.csr_matrix(M)
    M.sort_indices()
    b = rng.standard_normal(n)
    x, it, rr, st = _lib.csr_solve(M.indptr, M.indices, M.data, b, method=method, rtol=1e-12, maxit=10000)
    assert st == 0 and rr <= 1e-12
    xd = spla.spsolve(M.tocsc(), b)
    assert np.linalg.norm(x - xd) / np.linalg.norm(xd) < 1e-9
