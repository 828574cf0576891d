"""Pins the oracle's geometry against the reference's own code: src/Math/Geometry.cpp,
Sphere.cpp, Vector3D.cpp and Tensor3D.cpp compiled where they lie (`make -C oracle ref`,
oracle/_ref/libref_geometry.so).  On seeded jittered and sheared hexahedra, the oracle's
volume, centroid, face area and centroid, point-in-cell test and sphere intersection must be
bit-identical to the reference's: both are FP64 with every product and sum rounded separately
in the same order.  The same library holds the reference's Array3D container, which pins the
oracle's cell storage order.  Skipped where the reference sources are absent (the library is
not part of the repository); the committed golden fixture covers that case."""
import ctypes
import os

import numpy as np
import pytest

from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(os.path.dirname(HERE), "oracle", "_ref", "libref_geometry.so")


@pytest.fixture(scope="module")
def libs():
    from caffe_old_b200 import build as B
    if not B.build_oracle_ref():
        pytest.skip("reference geometry sources not present")
    ref = ctypes.CDLL(REF_LIB)
    O.lib()                                    # builds the oracle if needed
    ora = ctypes.CDLL(O._LIB_PATH)             # own handle: the argument types below stay local
    dp = ctypes.POINTER(ctypes.c_double)
    for L, pre in ((ref, "ref_"), (ora, "oracle_")):
        getattr(L, pre + "hex_volume").restype = ctypes.c_double
        getattr(L, pre + "hex_volume").argtypes = [dp]
        getattr(L, pre + "hex_centroid").argtypes = [dp, dp]
        getattr(L, pre + "quad_area").restype = ctypes.c_double
        getattr(L, pre + "quad_area").argtypes = [dp]
        getattr(L, pre + "inside_hex").argtypes = [dp, dp]
        getattr(L, pre + "nearest_intersect").argtypes = [ctypes.c_double, dp, dp, dp]
    ref.ref_quad_centroid.argtypes = [dp, dp]
    return ref, ora


def _p(a):
    return np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _hexes(n, seed):
    """Unit-ish hexahedra in HexaFvmMesh vertex order, sheared and jittered."""
    rng = np.random.default_rng(seed)
    base = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]], float)
    out = []
    for _ in range(n):
        h = base * rng.uniform(0.5, 2.0, 3) + rng.uniform(-3, 3, 3)
        h[:, 0] += np.tan(np.radians(30.0)) * h[:, 2]
        h += rng.uniform(-0.1, 0.1, h.shape)
        out.append(h)
    return out


def test_hexahedron_volume_and_centroid_are_the_references(libs):
    ref, ora = libs
    for h in _hexes(200, 1):
        assert ref.ref_hex_volume(_p(h)) == ora.oracle_hex_volume(_p(h))
        cr, co = np.zeros(3), np.zeros(3)
        ref.ref_hex_centroid(_p(h), _p(cr))
        ora.oracle_hex_centroid(_p(h), _p(co))
        assert np.array_equal(cr, co), (cr, co)


def test_face_area_and_centroid_are_the_references(libs):
    ref, ora = libs
    for h in _hexes(100, 2):
        for face in ([1, 2, 6, 5], [0, 4, 7, 3], [3, 7, 6, 2], [0, 1, 5, 4]):
            q = h[face]
            assert ref.ref_quad_area(_p(q)) == ora.oracle_quad_area(_p(q))


def test_point_in_cell_and_sphere_intersection_are_the_references(libs):
    ref, ora = libs
    rng = np.random.default_rng(3)
    for h in _hexes(60, 4):
        lo, hi = h.min(0), h.max(0)
        for _ in range(20):
            pt = rng.uniform(lo - 0.2, hi + 0.2)
            assert ref.ref_inside_hex(_p(pt), _p(h)) == ora.oracle_inside_hex(_p(pt), _p(h))
    for _ in range(200):
        c, pt, r = rng.uniform(-2, 2, 3), rng.uniform(-3, 3, 3), float(rng.uniform(0.05, 1.0))
        a, b = np.zeros(3), np.zeros(3)
        ref.ref_nearest_intersect(r, _p(c), _p(pt), _p(a))
        ora.oracle_nearest_intersect(r, _p(c), _p(pt), _p(b))
        assert np.array_equal(a, b), (a, b)


def _ref_offsets(ref, dims, cells):
    ref.ref_array3d_offset.restype = ctypes.c_long
    ref.ref_array3d_offset.argtypes = [ctypes.c_int] * 6
    return np.array([ref.ref_array3d_offset(*dims, *c) for c in cells])


def _oracle_cell_index(dims):
    """Where the oracle stores each cell (i, j, k) of a Cartesian mesh: the index of the
    centroid it reports for that cell."""
    from caffe_old_b200 import cases as C
    nI, nJ, nK = dims
    s = O.OracleSolver(C.cartesian_nodes(dims, (nI, nJ, nK)), C.CaseSpec(kind="simple"))
    cc = s.get("cc").reshape(-1, 3)
    s.close()
    ijk = np.floor(cc).astype(int)                     # unit cells: centroid (i+.5, j+.5, k+.5)
    index = np.empty((nI, nJ, nK), dtype=int)
    index[ijk[:, 0], ijk[:, 1], ijk[:, 2]] = np.arange(len(cc))
    return index


def test_cell_storage_order_is_the_references_array3d(libs):
    """The oracle stores cell (i, j, k) at the element the reference's Array3D gives it
    (Array3D.tpp:41-59, i fastest), and the reference's bounds-checked access refuses indices
    outside the array."""
    ref, _ = libs
    dims = (7, 5, 3)
    index = _oracle_cell_index(dims)
    cells = [(i, j, k) for k in range(dims[2]) for j in range(dims[1]) for i in range(dims[0])]
    assert np.array_equal(_ref_offsets(ref, dims, cells), [index[c] for c in cells])
    assert list(_ref_offsets(ref, dims, [(-1, 0, 0), (0, 5, 0), (0, 0, 3), (7, 4, 2)])) == [-1, -1, -1, -1]


def test_oracle_matches_the_reference_golden_geometry():
    """The committed outputs of the reference's geometry code (tests/golden/, written by
    tests/golden/make_geometry_golden.py) against the oracle, bit for bit; needs no reference
    sources."""
    g = np.load(os.path.join(HERE, "golden", "reference_geometry.npz"))
    ora = ctypes.CDLL(O.lib()._name)
    dp = ctypes.POINTER(ctypes.c_double)
    ora.oracle_hex_volume.restype = ctypes.c_double
    ora.oracle_hex_volume.argtypes = [dp]
    ora.oracle_hex_centroid.argtypes = [dp, dp]
    ora.oracle_quad_area.restype = ctypes.c_double
    ora.oracle_quad_area.argtypes = [dp]
    ora.oracle_nearest_intersect.argtypes = [ctypes.c_double, dp, dp, dp]
    for q, h in enumerate(g["hexes"]):
        assert ora.oracle_hex_volume(_p(h)) == g["volume"][q]
        c = np.zeros(3)
        ora.oracle_hex_centroid(_p(h), _p(c))
        assert np.array_equal(c, g["centroid"][q])
        for f, face in enumerate(g["faces"]):
            assert ora.oracle_quad_area(_p(h[face])) == g["face_area"][q, f]
    for q, row in enumerate(g["sphere"]):
        o = np.zeros(3)
        ora.oracle_nearest_intersect(float(row[0]), _p(row[1:4]), _p(row[4:7]), _p(o))
        assert np.array_equal(o, g["nearest"][q])
    # cell storage order: the reference Array3D's offsets of every cell of a 7 x 5 x 3 array
    dims = tuple(int(v) for v in g["array3d_dims"])
    index = _oracle_cell_index(dims)
    assert np.array_equal(g["array3d_offsets"], [index[tuple(c)] for c in g["array3d_cells"]])
    # metric arrays of the sheared, jittered mesh
    from caffe_old_b200 import cases as C
    s = O.OracleSolver(g["mesh_nodes"], C.CaseSpec(kind="piso"))
    assert np.array_equal(s.get("vol"), g["mesh_vol"])
    assert np.array_equal(s.get("cc").reshape(-1, 3), g["mesh_cc"])
    for d in "IJK":
        assert np.array_equal(s.get("fc" + d).reshape(-1, 3), g["mesh_fc" + d]), d
        assert np.array_equal(s.get("S" + d).reshape(-1, 3), g["mesh_S" + d]), d
    dc = g["mesh_d_and_c"].reshape(6, -1, 4)
    for f in range(6):
        assert np.array_equal(s.get(f"dmet{f}"), dc[f, :, 0]), f
        assert np.array_equal(s.get(f"cvec{f}").reshape(-1, 3), dc[f, :, 1:]), f
    s.close()
    # immersed-boundary geometry of the channel with a sphere
    nodes, radius, center = _geometry_generator().ib_case()
    status, stencil = _oracle_ib(nodes, radius, center)
    assert np.array_equal(g["ib_solid"].ravel(), status != 0)
    assert np.array_equal(g["ib_ghosts"], np.flatnonzero(status == 1))
    assert np.array_equal(g["ib_stencils"], stencil)
    # velocity-gradient tensors after one step of the sheared, jittered cavity
    import sys
    sys.path.insert(0, HERE)
    from helpers import small_skewed
    nodes, spec = small_skewed()
    s = O.OracleSolver(nodes, spec)
    s.solve()
    assert np.array_equal(s.get("gradU").reshape(g["skewed_step1_gradU"].shape), g["skewed_step1_gradU"])
    s.close()


def test_mesh_metric_arrays_are_the_references(libs):
    """The oracle's metric arrays of a sheared, jittered mesh -- cell volumes and centroids
    (HexaFvmMesh::initializeCells, HexaFvmMesh.cpp:626-655) and face centroids and face vectors
    (initializeFaces, :699-789) -- equal, bit for bit, the reference's Geometry and Vector3D
    routines applied to the same nodes in the mesh set-up's vertex orders."""
    from caffe_old_b200 import cases as C
    ref, _ = libs
    dp = ctypes.POINTER(ctypes.c_double)
    ref.ref_face_vector.argtypes = [dp, dp]
    nI, nJ, nK = 6, 5, 4
    nodes = C.skewed_nodes((nI, nJ, nK), (1.0, 1.0, 1.0), 30.0, 0.1, 5)     # (k, j, i, xyz)
    s = O.OracleSolver(nodes, C.CaseSpec(kind="piso"))
    vol, cc = s.get("vol"), s.get("cc").reshape(-1, 3)
    fc = {d: s.get("fc" + d).reshape(-1, 3) for d in "IJK"}
    sv = {d: s.get("S" + d).reshape(-1, 3) for d in "IJK"}
    s.close()
    X = lambda i, j, k: nodes[k, j, i]
    for k in range(nK):
        for j in range(nJ):
            for i in range(nI):
                h = np.array([X(i, j, k), X(i + 1, j, k), X(i + 1, j + 1, k), X(i, j + 1, k),
                              X(i, j, k + 1), X(i + 1, j, k + 1), X(i + 1, j + 1, k + 1), X(i, j + 1, k + 1)])
                c = (k * nJ + j) * nI + i
                assert ref.ref_hex_volume(_p(h)) == vol[c]
                o = np.zeros(3)
                ref.ref_hex_centroid(_p(h), _p(o))
                assert np.array_equal(o, cc[c])
    quads = {   # face arrays: I (nI+1) x nJ x nK, J nI x (nJ+1) x nK, K nI x nJ x (nK+1), i fastest
        "I": (nI + 1, nJ, nK, lambda i, j, k: [X(i, j, k), X(i, j + 1, k), X(i, j + 1, k + 1), X(i, j, k + 1)]),
        "J": (nI, nJ + 1, nK, lambda i, j, k: [X(i, j, k), X(i, j, k + 1), X(i + 1, j, k + 1), X(i + 1, j, k)]),
        "K": (nI, nJ, nK + 1, lambda i, j, k: [X(i, j, k), X(i + 1, j, k), X(i + 1, j + 1, k), X(i, j + 1, k)]),
    }
    for d, (fI, fJ, fK, quad) in quads.items():
        for k in range(fK):
            for j in range(fJ):
                for i in range(fI):
                    q = np.array(quad(i, j, k))
                    f = (k * fJ + j) * fI + i
                    o = np.zeros(3)
                    ref.ref_quad_centroid(_p(q), _p(o))
                    assert np.array_equal(o, fc[d][f]), (d, i, j, k)
                    ref.ref_face_vector(_p(q), _p(o))
                    assert np.array_equal(o, sv[d][f]), (d, i, j, k)


def test_diffusion_metrics_are_the_references(libs):
    """D_f = |S|^2 / (S . r) and c_f = S - r |S|^2 / (S . r) of every face of every cell
    (HexaFvmMesh::computeMeshMetrics, HexaFvmMesh.cpp:872-884): the oracle's values equal the
    reference's Vector3D arithmetic on the same face vector S (outward: fAreaNorm*,
    HexaFvmMesh.h:79-84) and cell-to-cell vector r (cell-to-face on the boundary: rCell*,
    HexaFvmMesh.cpp:218-294), bit for bit, on a sheared, jittered mesh."""
    from caffe_old_b200 import cases as C
    ref, _ = libs
    dp = ctypes.POINTER(ctypes.c_double)
    ref.ref_d_and_c.argtypes = [dp, dp, dp]
    nI, nJ, nK = 6, 5, 4
    nodes = C.skewed_nodes((nI, nJ, nK), (1.0, 1.0, 1.0), 30.0, 0.1, 5)
    s = O.OracleSolver(nodes, C.CaseSpec(kind="piso"))
    cc = s.get("cc").reshape(nK, nJ, nI, 3)
    fcI, fcJ, fcK = (s.get("fc" + d).reshape(*shp, 3) for d, shp in
                     (("I", (nK, nJ, nI + 1)), ("J", (nK, nJ + 1, nI)), ("K", (nK + 1, nJ, nI))))
    SI, SJ, SK = (s.get("S" + d).reshape(*shp, 3) for d, shp in
                  (("I", (nK, nJ, nI + 1)), ("J", (nK, nJ + 1, nI)), ("K", (nK + 1, nJ, nI))))
    dmet = [s.get(f"dmet{f}").reshape(nK, nJ, nI) for f in range(6)]
    cvec = [s.get(f"cvec{f}").reshape(nK, nJ, nI, 3) for f in range(6)]
    s.close()
    for k in range(nK):
        for j in range(nJ):
            for i in range(nI):
                c = cc[k, j, i]
                faces = [  # (S outward, r) for east, west, north, south, top, bottom
                    (SI[k, j, i + 1], cc[k, j, i + 1] - c if i < nI - 1 else fcI[k, j, i + 1] - c),
                    (-SI[k, j, i], cc[k, j, i - 1] - c if i > 0 else fcI[k, j, i] - c),
                    (SJ[k, j + 1, i], cc[k, j + 1, i] - c if j < nJ - 1 else fcJ[k, j + 1, i] - c),
                    (-SJ[k, j, i], cc[k, j - 1, i] - c if j > 0 else fcJ[k, j, i] - c),
                    (SK[k + 1, j, i], cc[k + 1, j, i] - c if k < nK - 1 else fcK[k + 1, j, i] - c),
                    (-SK[k, j, i], cc[k - 1, j, i] - c if k > 0 else fcK[k, j, i] - c),
                ]
                for f, (sv, r) in enumerate(faces):
                    out = np.zeros(4)
                    ref.ref_d_and_c(_p(sv), _p(r), _p(out))
                    assert out[0] == dmet[f][k, j, i], (f, i, j, k)
                    assert np.array_equal(out[1:], cvec[f][k, j, i]), (f, i, j, k)


def _geometry_generator():
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_geometry_golden", os.path.join(HERE, "golden", "make_geometry_golden.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _oracle_ib(nodes, radius, center):
    from caffe_old_b200 import cases as C
    bc, refv = C.channel_bcs(1.0)
    spec = C.CaseSpec(kind="ibpiso", bc=bc, ref_vec=refv, ib_radius=radius, ib_center=tuple(center))
    o = O.OracleSolver(nodes, spec)
    o.phase("ib_field")
    o.phase("ib_coeffs")
    status = o.get("status")
    stencil = o.get("ibStencil").reshape(-1, 8).astype(np.int64)
    o.close()
    return status, stencil


def test_immersed_boundary_geometry_is_the_references(libs):
    """Ghost-cell geometry of IbPiso (IbPiso.cpp:65-140) on the channel with a sphere: the
    oracle's solid cells are the cells whose centroid the reference's Sphere::isInside accepts,
    and each ghost cell's 8-cell interpolation stencil is the one the reference's cell search
    finds for the image point 2 BP - x_G computed by its own Vector3D arithmetic
    (tests/golden/make_geometry_golden.py: ib_reference)."""
    ref, _ = libs
    gen = _geometry_generator()
    nodes, radius, center = gen.ib_case()
    solid, ghosts, stencils = gen.ib_reference(ref, nodes, radius, center)
    status, stencil = _oracle_ib(nodes, radius, center)
    assert np.array_equal(solid.ravel(), status != 0)
    assert np.array_equal(np.flatnonzero(status == 1), ghosts) and len(ghosts) > 0
    assert np.array_equal(stencil, stencils)


def test_velocity_gradient_tensor_is_the_references(libs):
    """The cell velocity gradient of the non-orthogonal correction, sum_f u_f (x) S_f / V
    (FvVectorScheme.cpp:64-69), from the oracle's face velocities after a step on a sheared,
    jittered cavity, equals the reference's Vector3D / Tensor3D arithmetic bit for bit."""
    import sys
    sys.path.insert(0, HERE)
    from helpers import small_skewed
    ref, _ = libs
    dp = ctypes.POINTER(ctypes.c_double)
    ref.ref_grad_tensor.argtypes = [dp, dp, ctypes.c_double, dp]
    nodes, spec = small_skewed()
    assert spec.nonorth
    s = O.OracleSolver(nodes, spec)
    s.solve()
    nK, nJ, nI = (d - 1 for d in nodes.shape[:3])
    gU = s.get("gradU").reshape(nK, nJ, nI, 9)
    uI = s.get("uFaceI").reshape(nK, nJ, nI + 1, 3)
    uJ = s.get("uFaceJ").reshape(nK, nJ + 1, nI, 3)
    uK = s.get("uFaceK").reshape(nK + 1, nJ, nI, 3)
    SI = s.get("SI").reshape(nK, nJ, nI + 1, 3)
    SJ = s.get("SJ").reshape(nK, nJ + 1, nI, 3)
    SK = s.get("SK").reshape(nK + 1, nJ, nI, 3)
    vol = s.get("vol").reshape(nK, nJ, nI)
    s.close()
    assert np.abs(gU).max() > 0
    for k in range(nK):
        for j in range(nJ):
            for i in range(nI):
                uf = np.array([uI[k, j, i + 1], uI[k, j, i], uJ[k, j + 1, i], uJ[k, j, i], uK[k + 1, j, i], uK[k, j, i]])
                sf = np.array([SI[k, j, i + 1], -SI[k, j, i], SJ[k, j + 1, i], -SJ[k, j, i], SK[k + 1, j, i], -SK[k, j, i]])
                out = np.zeros(9)
                ref.ref_grad_tensor(_p(uf), _p(sf), float(vol[k, j, i]), _p(out))
                assert np.array_equal(out, gU[k, j, i]), (i, j, k)
