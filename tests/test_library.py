"""The C-ABI library loads on a CPU-only host and exports every symbol include/caffe_b200.h
declares; the case translation rejects invalid input (no GPU calls)."""
import ctypes
import os
import re

import numpy as np
import pytest

from caffe_old_b200 import _lib
from caffe_old_b200 import build as B
from caffe_old_b200 import cases as C


@pytest.fixture(scope="module")
def built():
    B.build_device()
    return _lib.LIB_PATH


def header_functions():
    src = open(_lib.HEADER_PATH).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?(?:long\s+)?\w+\s*\*?\s*(caffe_\w+)\s*\(", src, flags=re.M)))


def test_header_lists_entry_points():
    names = header_functions()
    assert set(_lib.EXPORTS) == set(names)


def test_library_exports_every_declared_symbol(built):
    L = ctypes.CDLL(built)
    for name in header_functions():
        assert hasattr(L, name), name


def test_case_struct_matches_header(built):
    # caffe_case in the header and CaffeCase in the binding have the same field order
    src = open(_lib.HEADER_PATH).read()
    body = src[src.index("typedef struct caffe_case {"):src.index("} caffe_case;")]
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    fields = []
    for decl in body.split(";"):
        decl = decl.strip()
        if not decl or decl.startswith("typedef"):
            decl = decl.split("{")[-1].strip()
            if not decl:
                continue
        toks = decl.replace(",", " ").split()
        fields += [re.sub(r"\[.*", "", t) for t in toks[1:]]
    assert fields == [f for f, _ in _lib.CaffeCase._fields_]


def test_invalid_cases_rejected():
    with pytest.raises(ValueError):
        C.CaseSpec(kind="coupled").validate()
    with pytest.raises(ValueError):
        C.CaseSpec(bc=("wall",) * 5).validate()
    with pytest.raises(ValueError):
        C.CaseSpec(kind="ibpiso", ib_radius=0.0).validate()
    with pytest.raises(ValueError):
        C.CaseSpec(p_method="gmres").validate()


def test_make_case_roundtrip():
    nodes, spec, _ = C.config2_cavity3d(n=8, steps=1)
    c = _lib.make_case(spec)
    assert c.kind == 1 and c.p_method == C.KSP_METHODS["cg_jacobi"]
    assert c.ref_vec[2][0] == 1.0 and c.bc_type[2] == C.FLOW_TYPES["wall"]
    assert c.convection == 1 and c.n_pcorr == 2


def test_create_without_gpu_fails_loudly(built):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from caffe_old_b200.solver import Piso
    nodes, spec, _ = C.config2_cavity3d(n=4, steps=1)
    with pytest.raises(_lib.CaffeError):
        Piso(nodes, spec)


def test_c_abi_rejects_invalid_arguments_before_any_device_call(built):
    """caffe_dev_create checks its arguments and the case record before it looks for a GPU,
    and reports each problem through caffe_last_error (runs the same with or without a GPU)."""
    L = _lib.lib()
    nodes, spec, _ = C.config2_cavity3d(n=4, steps=1)
    nodes = np.ascontiguousarray(nodes, dtype=np.float64)
    ptr = nodes.ctypes.data_as(ctypes.c_void_p)
    h = ctypes.c_void_p()

    def create(case, n=(5, 5, 5), p=ptr, out=ctypes.byref(h)):
        rc = L.caffe_dev_create(p, n[0], n[1], n[2], ctypes.byref(case) if case is not None else None, 0, out)
        return rc, _lib.last_error()

    good = _lib.make_case(spec)
    assert create(good, p=None) == (1, "nodes is NULL")
    assert create(good, out=None) == (1, "out is NULL")
    assert create(good, n=(1, 5, 5)) == (1, "a mesh needs at least 2 nodes per direction")
    assert create(None) == (1, "case is NULL")
    bad = [("kind", 7, "invalid solver kind"), ("omega_p", 0.0, "relaxation factors must be positive"),
           ("n_pcorr", 0, "numberOfPressureCorrections must be >= 1"), ("maxit", 0, "maxit must be >= 1"),
           ("mom_method", C.KSP_METHODS["cg_jacobi"], "the momentum matrix is not symmetric: CG cannot solve it"),
           ("p_form", 9, "invalid pressure-solve form"),
           ("p_atol", -1.0, "absolute tolerances must be >= 0")]
    for field, value, msg in bad:
        c = _lib.make_case(spec)
        setattr(c, field, value)
        assert create(c) == (1, msg), field
    assert not h.value
    # the reference's own preconditioner (PETSc's sequential SOR sweep) is refused, not replaced
    for field in ("mom_method", "p_method"):
        c = _lib.make_case(spec)
        setattr(c, field, C.KSP_METHODS["bicgstab_sgs"])
        rc, msg = create(c)
        assert rc == 1 and "symmetric Gauss-Seidel" in msg and "not implemented on the device" in msg
