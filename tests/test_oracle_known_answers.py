"""The oracle against the reference's own unit-test assertions (re-expressed, CPU only).

Sources of the known answers (reference test files):
  * test/GeometryTest.cpp:24-28, 54-56 -- unit cube volume 1, face area 1, (0.8,0.5,0.5) inside
  * test/MatrixTest.cpp:23-36 -- dense inverse / solve to 1e-11 relative
  * test/IndexMapTest.cpp:30-39 -- row of cell (i,j,k) is k*nJ*nI + j*nI + i on one block
  * test/FieldTest.cpp:108-213 -- FIXED patches and zero-gradient refresh of boundary patches
  * test/Array3DTest.cpp:54-92 -- i-fastest storage order
"""
import numpy as np
import pytest

from oracle import oracle as O
from caffe_old_b200 import cases as C

UNIT_CUBE = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]], dtype=float)


def test_unit_cube_volume_area_centroid():
    assert O.hex_volume(UNIT_CUBE) == 1.0
    assert O.quad_area(UNIT_CUBE[:4]) == 1.0
    assert np.allclose(O.hex_centroid(UNIT_CUBE), [0.5, 0.5, 0.5], rtol=0, atol=1e-15)


def test_point_in_hexahedron():
    assert O.inside_hex([0.8, 0.5, 0.5], UNIT_CUBE)
    assert not O.inside_hex([1.2, 0.5, 0.5], UNIT_CUBE)
    assert O.inside_hex([1.0, 0.5, 0.5], UNIT_CUBE)   # faces count as inside (dot < 0 rejects)


def test_sphere_nearest_intersect():
    pt = np.array([1.2, 1.1, 1.1])
    out = O.nearest_intersect(1.0, [0.0, 0.0, 0.0], pt)
    assert np.allclose(out, pt / np.linalg.norm(pt), rtol=0, atol=1e-15)


def test_trilinear_weights_reproduce_trilinear_functions():
    rng = np.random.default_rng(1)
    for _ in range(20):
        base = rng.uniform(0.5, 3.0, 3)
        h = rng.uniform(0.01, 0.2, 3)
        pts = np.array([base + h * np.array(o) for o in
                        [(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)]])
        pts += rng.uniform(-0.05, 0.05, pts.shape) * h
        ip = base + h * rng.uniform(0.1, 0.9, 3)
        beta = O.trilinear(pts, ip)
        # exact for 1, x, y, z, xy, yz, xz, xyz (Interpolation.cpp:135-180)
        def mono(p):
            x, y, z = p
            return np.array([1, x * y * z, x * y, y * z, x * z, x, y, z])
        M = np.array([mono(p) for p in pts])
        ref = np.linalg.solve(M.T, mono(ip))
        assert np.allclose(beta, ref, rtol=1e-8, atol=1e-9)
        assert abs(beta.sum() - 1.0) < 1e-9


def test_row_numbering_and_storage_order():
    nodes = C.cartesian_nodes((5, 4, 3), (1, 1, 1))
    spec = C.CaseSpec(kind="simple")
    s = O.OracleSolver(nodes, spec)
    st = s.get("status")
    assert st.shape == (60,) and np.all(st == 0)
    assert s.stats()["rows"] == 60
    cc = s.get("cc").reshape(3, 4, 5, 3)    # (k, j, i, xyz): i fastest
    assert np.allclose(cc[1, 2, 3], [(3 + 0.5) / 5, (2 + 0.5) / 4, (1 + 0.5) / 3], atol=1e-15)


def test_fixed_and_zero_gradient_patches():
    """FieldTest test4/test5: a FIXED face keeps its reference value on the patch;
    a zero-gradient face copies the boundary cell after the refresh."""
    nodes = C.cartesian_nodes((6, 5, 4), (1, 1, 1))
    bc = ("outlet", "inlet", "wall", "wall", "wall", "wall")
    ref_val = (2.5, 0.0, 0.0, 0.0, 0.0, 0.0)
    spec = C.CaseSpec(kind="piso", bc=bc, ref_vec=((0, 0, 0), (1, 0, 0)) + ((0, 0, 0),) * 4, ref_val=ref_val,
                      time_accurate=True, omega_u=1.0, omega_p=1.0, n_pcorr=1, dt=0.1, mu=0.1,
                      p_method="bicgstab_jacobi", mom_rtol=1e-12, p_rtol=1e-12)
    s = O.OracleSolver(nodes, spec)
    assert np.all(s.get("pPatch0") == 2.5)          # east: outlet -> p FIXED at refValue
    s.solve()
    p = s.get("p").reshape(4, 5, 6)
    assert np.all(s.get("pPatch0") == 2.5)
    assert np.array_equal(s.get("pPatch1").reshape(4, 5), p[:, :, 0])   # west: zero gradient
    assert np.array_equal(s.get("pPatch2").reshape(4, 6), p[:, -1, :])  # north
    assert np.array_equal(s.get("pPatch5").reshape(5, 6), p[0, :, :])   # bottom


def test_dense_solve_accuracy_like_matrix_test():
    # 8x8 systems from random trilinear stencils solve to 1e-11 relative (MatrixTest.cpp:23-36)
    rng = np.random.default_rng(5)
    pts = rng.uniform(0.0, 1.0, (8, 3))
    ip = rng.uniform(0.2, 0.8, 3)
    beta = O.trilinear(pts, ip)
    x, y, z = pts.T
    M = np.stack([np.ones(8), x * y * z, x * y, y * z, x * z, x, y, z], axis=1)
    X, Y, Z = ip
    rhs = np.array([1, X * Y * Z, X * Y, Y * Z, X * Z, X, Y, Z])
    assert np.allclose(M.T @ beta, rhs, rtol=1e-11, atol=1e-11)


def test_cavity_mass_conservation_and_symmetry():
    nodes, spec, _ = C.config1_cavity2d(n=16, iters=1)
    spec = spec.replace(mom_rtol=1e-12, p_rtol=1e-12)
    s = O.OracleSolver(nodes, spec)
    for _ in range(30):
        s.solve()
    # closed cavity: no flux through the walls
    FI = s.get("massFlowI").reshape(1, 16, 17)
    FJ = s.get("massFlowJ").reshape(1, 17, 16)
    assert np.abs(FI[:, :, 0]).max() == 0.0 and np.abs(FI[:, :, -1]).max() == 0.0
    assert np.abs(FJ[:, 0, :]).max() == 0.0
    u = s.get("u").reshape(16, 16, 3)
    assert np.all(u[:, :, 2] == 0.0)           # 2-D: no z velocity
    assert u[-1, :, 0].mean() > 0.2            # lid drags the top row
    assert u[4, :, 0].mean() < 0.0             # return flow below


def test_sphere_crossing_the_boundary():
    """Edge case of IbPiso::computeIbField (IbPiso.cpp:65-117): a neighbour outside the domain
    is read from the ib field's boundary patch, which stays 0 = FLUID, so every solid cell on
    the boundary is a ghost cell even when all its in-domain neighbours are solid.  Image
    points that fall between the boundary and the first cell centres have no enclosing cells:
    the reference raises there (HexaFvmMesh::locateEnclosingCells, HexaFvmMesh.cpp:378-418),
    and so does the oracle (the device library refuses such a case at creation)."""
    from helpers import small_channel_sphere
    nodes, spec = small_channel_sphere()
    o = O.OracleSolver(nodes, spec.replace(ib_center=(0.0, 0.5, 0.5), ib_radius=0.4))
    o.phase("ib_field")
    st = o.get("status").reshape(12, 12, 32)
    solid = st != 0
    assert solid[:, :, 0].any()
    assert np.all(st[:, :, 0][solid[:, :, 0]] == 1)
    # some of them have only solid neighbours inside the domain
    inner = solid[1:-1, 1:-1, 0] & solid[1:-1, 1:-1, 1] & solid[2:, 1:-1, 0] & solid[:-2, 1:-1, 0] \
        & solid[1:-1, 2:, 0] & solid[1:-1, :-2, 0]
    assert inner.any()
    # away from the boundary the ordinary rule holds: solid cells with only solid neighbours are inactive
    assert (st[:, :, 1:] == 2).any()
    with pytest.raises(RuntimeError, match="outside the cell-centre lattice"):
        o.phase("ib_coeffs")
    o.close()


def _neumann_laplacian(shape, seed=5):
    """7-point p'-like operator with zero row sums (all-Neumann: singular, constant null space)."""
    rng = np.random.default_rng(seed)
    nI, nJ, nK = shape
    N = nI * nJ * nK
    idx = np.arange(N)
    i, j, k = idx % nI, (idx // nI) % nJ, idx // (nI * nJ)
    aE = rng.uniform(0.5, 1.5, N); aN = rng.uniform(0.5, 1.5, N); aT = rng.uniform(0.5, 1.5, N)
    aE[i == nI - 1] = 0; aN[j == nJ - 1] = 0; aT[k == nK - 1] = 0
    aW = np.zeros(N); aW[1:] = aE[:-1]; aW[i == 0] = 0
    aS = np.zeros(N); aS[nI:] = aN[:-nI]; aS[j == 0] = 0
    aB = np.zeros(N); aB[nI * nJ:] = aT[:-nI * nJ]; aB[k == 0] = 0
    aP = -(aE + aW + aN + aS + aT + aB)
    return np.stack([aP, aE, aW, aN, aS, aT, aB])


@pytest.mark.parametrize("method", ["cg_jacobi", "bicgstab_jacobi"])
def test_absolute_floor_accepts_round_off_right_hand_side(method):
    """A second PISO corrector's right-hand side is round-off (||b|| ~ 1e-19 here), partly along
    the null space of the singular all-Neumann operator, so no Krylov method can reduce it by a
    relative 1e-13.  With the absolute floor atol (PETSc's ||r|| <= max(rtol ||b||, atol)) at
    the round-off level the solve is converged at once (status 0, x = 0); without it, it can
    only run to maxit."""
    shape = (9, 7, 5)
    coef = _neumann_laplacian(shape)
    rng = np.random.default_rng(11)
    b = 1e-19 * rng.standard_normal(int(np.prod(shape)))   # mean not removed: inconsistent
    floor = 1e-16
    x, it, rr, st = O.ksp7(shape, coef, b, method, 1e-13, 200, atol=floor)
    assert st == 0 and it == 0 and not np.any(x)
    x, it, rr, st = O.ksp7(shape, coef, b, method, 1e-13, 200)
    assert st == 1 and it == 200
    # a consistent right-hand side far above the floor is still solved to the relative tolerance
    b = rng.standard_normal(b.size)
    b -= b.mean()
    x, it, rr, st = O.ksp7(shape, coef, b, method, 1e-10, 5000, atol=floor)
    assert st == 0 and rr <= 1e-10 and it > 0
