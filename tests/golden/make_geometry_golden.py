"""Writes tests/golden/reference_geometry.npz: outputs of the reference's own geometry code
(src/Math/Geometry.cpp and Sphere.cpp, compiled where they lie into
oracle/_ref/libref_geometry.so by `make -C oracle ref`) on seeded sheared and jittered
hexahedra, its Array3D container's element offsets, and the metric arrays (cell volumes and
centroids, face centroids and face vectors, D_f and c_f) of a sheared, jittered mesh built
from those routines, so that the oracle stays pinned to them where the reference sources are
absent.

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
    np.savez(os.path.join(HERE, "reference_geometry.npz"), hexes=H, volume=vol, centroid=cen, faces=faces, face_area=area,
             sphere=sph, nearest=near, array3d_dims=np.array(dims), array3d_cells=cells, array3d_offsets=offs, **mesh)
    print("wrote", os.path.join(HERE, "reference_geometry.npz"))


if __name__ == "__main__":
    main()
