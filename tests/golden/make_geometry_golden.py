"""Writes tests/golden/reference_geometry.npz: outputs of the reference's own geometry code
(src/Math/Geometry.cpp and Sphere.cpp, compiled where they lie into
oracle/_ref/libref_geometry.so by `make -C oracle ref`) on seeded sheared and jittered
hexahedra, its Array3D container's element offsets, and the metric arrays (cell volumes and
centroids, face centroids and face vectors, D_f and c_f) of a sheared, jittered mesh built
from those routines, the immersed-boundary geometry of the channel with a sphere (solid
cells, ghost cells and their 8-cell stencils), and the velocity-gradient tensors of one step
of the sheared cavity, so that the oracle stays pinned to them where the reference sources
are absent.

  python tests/golden/make_geometry_golden.py
"""
import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)


def hexes(n, seed):
    rng = np.random.default_rng(seed)
    base = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]], float)
    out = []
    for _ in range(n):
        h = base * rng.uniform(0.5, 2.0, 3) + rng.uniform(-3, 3, 3)
        h[:, 0] += np.tan(np.radians(30.0)) * h[:, 2]
        h += rng.uniform(-0.1, 0.1, h.shape)
        out.append(h)
    return np.array(out)


def ib_reference(ref, nodes, radius, center):
    """Solid cells and ghost-cell stencils of one sphere on these nodes, from the reference's
    own routines: cell centroids (Geometry::computeHexahedronCentroid), Sphere::isInside, the
    image point 2 BP - x_G (Sphere::nearestIntersect, Vector3D arithmetic) and the search of
    HexaFvmMesh::locateCell / locateEnclosingCells (HexaFvmMesh.cpp:345-418: the first node
    hexahedron in k-j-i order that contains the point, then the first cell-centre hexahedron of
    the 2 x 2 x 2 window below it, both by Geometry::isInsideHexahedron).  Ghost cells are solid
    cells with a fluid 6-neighbour, a neighbour outside the domain counting as fluid
    (IbPiso.cpp:65-117).  Returns (solid[k, j, i], ghost cell ids, stencils[ghost][8])."""
    dp = ctypes.POINTER(ctypes.c_double)
    p = lambda a: np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(dp)
    ref.ref_hex_centroid.argtypes = [dp, dp]
    ref.ref_sphere_is_inside.argtypes = [ctypes.c_double, dp, dp]
    ref.ref_image_point.argtypes = [ctypes.c_double, dp, dp, dp]
    ref.ref_inside_hex.argtypes = [dp, dp]
    nK, nJ, nI = (d - 1 for d in nodes.shape[:3])
    X = lambda i, j, k: nodes[k, j, i]

    def hex_of(pt_of, i, j, k):
        return np.array([pt_of(i, j, k), pt_of(i + 1, j, k), pt_of(i + 1, j + 1, k), pt_of(i, j + 1, k),
                         pt_of(i, j, k + 1), pt_of(i + 1, j, k + 1), pt_of(i + 1, j + 1, k + 1), pt_of(i, j + 1, k + 1)])

    cc = np.zeros((nK, nJ, nI, 3))
    for k in range(nK):
        for j in range(nJ):
            for i in range(nI):
                ref.ref_hex_centroid(p(hex_of(X, i, j, k)), p(cc[k, j, i]))
    ctr = np.asarray(center, dtype=np.float64)
    solid = np.array([[[bool(ref.ref_sphere_is_inside(radius, p(ctr), p(cc[k, j, i]))) for i in range(nI)] for j in range(nJ)]
                      for k in range(nK)])
    S = lambda i, j, k: 0 <= i < nI and 0 <= j < nJ and 0 <= k < nK and solid[k, j, i]
    C = lambda i, j, k: cc[k, j, i]
    ghosts, stencils = [], []
    for k in range(nK):
        for j in range(nJ):
            for i in range(nI):
                if not solid[k, j, i] or all(S(*n) for n in ((i + 1, j, k), (i - 1, j, k), (i, j + 1, k), (i, j - 1, k),
                                                             (i, j, k + 1), (i, j, k - 1))):
                    continue
                ip = np.zeros(3)
                ref.ref_image_point(radius, p(ctr), p(cc[k, j, i]), p(ip))
                cell = next((a, b, c) for c in range(nK) for b in range(nJ) for a in range(nI)
                            if ref.ref_inside_hex(p(ip), p(hex_of(X, a, b, c))))
                found = None
                for c in (cell[2] - 1, cell[2]):
                    for b in (cell[1] - 1, cell[1]):
                        for a in (cell[0] - 1, cell[0]):
                            if found is not None:
                                continue
                            # the reference's bounds-checked Array3D throws beyond the cell-centre lattice
                            if not (0 <= a < nI - 1 and 0 <= b < nJ - 1 and 0 <= c < nK - 1):
                                raise ValueError("image point outside the cell-centre lattice")
                            if ref.ref_inside_hex(p(ip), p(hex_of(C, a, b, c))):
                                found = (a, b, c)
                a, b, c = found
                ghosts.append((k * nJ + j) * nI + i)
                stencils.append([((c + dk) * nJ + (b + dj)) * nI + (a + di) for di, dj, dk in
                                 ((0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1))])
    return solid, np.array(ghosts, dtype=np.int64), np.array(stencils, dtype=np.int64)


def ib_case():
    """Nodes and sphere of the immersed-boundary fixture: the 32 x 12 x 12 channel of the
    parity tests."""
    sys.path.insert(0, os.path.dirname(HERE))
    from helpers import small_channel_sphere
    nodes, spec = small_channel_sphere()
    return nodes, float(spec.ib_radius), np.array(spec.ib_center, dtype=float)


def main():
    from caffe_old_b200 import build as B
    if not B.build_oracle_ref():
        raise SystemExit("reference sources not present")
    ref = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libref_geometry.so"))
    dp = ctypes.POINTER(ctypes.c_double)
    ref.ref_hex_volume.restype = ctypes.c_double
    ref.ref_hex_volume.argtypes = [dp]
    ref.ref_hex_centroid.argtypes = [dp, dp]
    ref.ref_quad_area.restype = ctypes.c_double
    ref.ref_quad_area.argtypes = [dp]
    ref.ref_nearest_intersect.argtypes = [ctypes.c_double, dp, dp, dp]
    p = lambda a: np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(dp)
    H = hexes(64, 11)
    vol = np.array([ref.ref_hex_volume(p(h)) for h in H])
    cen = np.zeros((len(H), 3))
    for q, h in enumerate(H):
        c = np.zeros(3)
        ref.ref_hex_centroid(p(h), p(c))
        cen[q] = c
    faces = np.array([[1, 2, 6, 5], [0, 4, 7, 3], [3, 7, 6, 2], [0, 1, 5, 4], [4, 5, 6, 7], [0, 3, 2, 1]])
    area = np.array([[ref.ref_quad_area(p(h[f])) for f in faces] for h in H])
    rng = np.random.default_rng(12)
    sph = rng.uniform(-2, 2, (64, 7))
    sph[:, 0] = np.abs(sph[:, 0]) * 0.5 + 0.05
    near = np.zeros((64, 3))
    for q, row in enumerate(sph):
        o = np.zeros(3)
        ref.ref_nearest_intersect(float(row[0]), p(row[1:4]), p(row[4:7]), p(o))
        near[q] = o
    ref.ref_array3d_offset.restype = ctypes.c_long
    ref.ref_array3d_offset.argtypes = [ctypes.c_int] * 6
    dims = (7, 5, 3)
    cells = np.array([(i, j, k) for k in range(dims[2]) for j in range(dims[1]) for i in range(dims[0])])
    offs = np.array([ref.ref_array3d_offset(*dims, *map(int, c)) for c in cells])
    # metric arrays of a sheared, jittered 6 x 5 x 4 mesh, built the way the mesh set-up does
    # (HexaFvmMesh.cpp:626-655, 699-789) from the reference's routines
    from caffe_old_b200 import cases as C
    ref.ref_face_vector.argtypes = [ctypes.POINTER(ctypes.c_double)] * 2
    nI, nJ, nK = 6, 5, 4
    nodes = C.skewed_nodes((nI, nJ, nK), (1.0, 1.0, 1.0), 30.0, 0.1, 5)
    X = lambda i, j, k: nodes[k, j, i]
    mvol, mcc = [], []
    for k in range(nK):
        for j in range(nJ):
            for i in range(nI):
                h = np.array([X(i, j, k), X(i + 1, j, k), X(i + 1, j + 1, k), X(i, j + 1, k),
                              X(i, j, k + 1), X(i + 1, j, k + 1), X(i + 1, j + 1, k + 1), X(i, j + 1, k + 1)])
                mvol.append(ref.ref_hex_volume(p(h)))
                c = np.zeros(3)
                ref.ref_hex_centroid(p(h), p(c))
                mcc.append(c)
    quads = {"I": (nI + 1, nJ, nK, lambda i, j, k: [X(i, j, k), X(i, j + 1, k), X(i, j + 1, k + 1), X(i, j, k + 1)]),
             "J": (nI, nJ + 1, nK, lambda i, j, k: [X(i, j, k), X(i, j, k + 1), X(i + 1, j, k + 1), X(i + 1, j, k)]),
             "K": (nI, nJ, nK + 1, lambda i, j, k: [X(i, j, k), X(i + 1, j, k), X(i + 1, j + 1, k), X(i, j + 1, k)])}
    mesh = {"mesh_nodes": nodes, "mesh_vol": np.array(mvol), "mesh_cc": np.array(mcc)}
    for d, (fI, fJ, fK, quad) in quads.items():
        fcs, svs = [], []
        for k in range(fK):
            for j in range(fJ):
                for i in range(fI):
                    q = np.array(quad(i, j, k))
                    a, b = np.zeros(3), np.zeros(3)
                    ref.ref_quad_centroid(p(q), p(a))
                    ref.ref_face_vector(p(q), p(b))
                    fcs.append(a)
                    svs.append(b)
        mesh["mesh_fc" + d], mesh["mesh_S" + d] = np.array(fcs), np.array(svs)
    # D_f and c_f of every face of every cell (HexaFvmMesh.cpp:872-884) from those arrays
    ref.ref_d_and_c.argtypes = [ctypes.POINTER(ctypes.c_double)] * 3
    cc = mesh["mesh_cc"].reshape(nK, nJ, nI, 3)
    FI, FJ, FK = (mesh["mesh_fc" + d].reshape(*shp, 3) for d, shp in
                  (("I", (nK, nJ, nI + 1)), ("J", (nK, nJ + 1, nI)), ("K", (nK + 1, nJ, nI))))
    SI, SJ, SK = (mesh["mesh_S" + d].reshape(*shp, 3) for d, shp in
                  (("I", (nK, nJ, nI + 1)), ("J", (nK, nJ + 1, nI)), ("K", (nK + 1, nJ, nI))))
    dc = np.zeros((6, nK, nJ, nI, 4))
    for k in range(nK):
        for j in range(nJ):
            for i in range(nI):
                c = cc[k, j, i]
                sides = [(SI[k, j, i + 1], cc[k, j, i + 1] - c if i < nI - 1 else FI[k, j, i + 1] - c),
                         (-SI[k, j, i], cc[k, j, i - 1] - c if i > 0 else FI[k, j, i] - c),
                         (SJ[k, j + 1, i], cc[k, j + 1, i] - c if j < nJ - 1 else FJ[k, j + 1, i] - c),
                         (-SJ[k, j, i], cc[k, j - 1, i] - c if j > 0 else FJ[k, j, i] - c),
                         (SK[k + 1, j, i], cc[k + 1, j, i] - c if k < nK - 1 else FK[k + 1, j, i] - c),
                         (-SK[k, j, i], cc[k - 1, j, i] - c if k > 0 else FK[k, j, i] - c)]
                for f, (sv, r) in enumerate(sides):
                    out = np.zeros(4)
                    ref.ref_d_and_c(p(np.ascontiguousarray(sv)), p(np.ascontiguousarray(r)), p(out))
                    dc[f, k, j, i] = out
    mesh["mesh_d_and_c"] = dc
    # velocity-gradient tensors of the non-orthogonal correction (FvVectorScheme.cpp:64-69) by
    # the reference's Tensor3D arithmetic, from the face velocities and face vectors of one
    # oracle step on the sheared, jittered cavity of the parity tests (the inputs only)
    sys.path.insert(0, os.path.dirname(HERE))
    from helpers import small_skewed
    from oracle.oracle import OracleSolver
    ref.ref_grad_tensor.argtypes = [dp, dp, ctypes.c_double, dp]
    gnodes, gspec = small_skewed()
    o = OracleSolver(gnodes, gspec)
    o.solve()
    gK, gJ, gI = (d - 1 for d in gnodes.shape[:3])
    uI = o.get("uFaceI").reshape(gK, gJ, gI + 1, 3)
    uJ = o.get("uFaceJ").reshape(gK, gJ + 1, gI, 3)
    uK = o.get("uFaceK").reshape(gK + 1, gJ, gI, 3)
    SI = o.get("SI").reshape(gK, gJ, gI + 1, 3)
    SJ = o.get("SJ").reshape(gK, gJ + 1, gI, 3)
    SK = o.get("SK").reshape(gK + 1, gJ, gI, 3)
    gvol = o.get("vol").reshape(gK, gJ, gI)
    o.close()
    gradU = np.zeros((gK, gJ, gI, 9))
    for k in range(gK):
        for j in range(gJ):
            for i in range(gI):
                uf = np.array([uI[k, j, i + 1], uI[k, j, i], uJ[k, j + 1, i], uJ[k, j, i], uK[k + 1, j, i], uK[k, j, i]])
                sf = np.array([SI[k, j, i + 1], -SI[k, j, i], SJ[k, j + 1, i], -SJ[k, j, i], SK[k + 1, j, i], -SK[k, j, i]])
                ref.ref_grad_tensor(p(uf), p(sf), float(gvol[k, j, i]), p(gradU[k, j, i]))
    ib_nodes, ib_r, ib_c = ib_case()
    solid, ghosts, stencils = ib_reference(ref, ib_nodes, ib_r, ib_c)
    ib = {"ib_solid": solid, "ib_ghosts": ghosts, "ib_stencils": stencils, "skewed_step1_gradU": gradU}
    np.savez(os.path.join(HERE, "reference_geometry.npz"), hexes=H, volume=vol, centroid=cen, faces=faces, face_area=area,
             sphere=sph, nearest=near, array3d_dims=np.array(dims), array3d_cells=cells, array3d_offsets=offs, **mesh, **ib)
    print("wrote", os.path.join(HERE, "reference_geometry.npz"))


if __name__ == "__main__":
    main()
