"""Writes tests/golden/reference_geometry.npz: outputs of the reference's own geometry code
(src/Math/Geometry.cpp and Sphere.cpp, compiled where they lie into
oracle/_ref/libref_geometry.so by `make -C oracle ref`) on seeded sheared and jittered
hexahedra, and its Array3D container's element offsets, so that the oracle stays pinned to
them where the reference sources are absent.

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
    np.savez(os.path.join(HERE, "reference_geometry.npz"), hexes=H, volume=vol, centroid=cen, faces=faces, face_area=area,
             sphere=sph, nearest=near, array3d_dims=np.array(dims), array3d_cells=cells, array3d_offsets=offs)
    print("wrote", os.path.join(HERE, "reference_geometry.npz"))


if __name__ == "__main__":
    main()
