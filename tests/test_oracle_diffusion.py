"""The oracle's restatement of the reference's Diffusion solver (src/Solvers/Diffusion.cpp),
on the CPU: known answers of the discrete equations it assembles and solves.

* Steady, fixed values on two opposite faces and zero gradient elsewhere: the cell values
  are the linear profile between them, and the gradient (divergence theorem over the
  extrapolated and limited faces, FvScalarScheme.cpp:70-156) is the constant slope.
* The assembled rows are the reference's as written (Diffusion.cpp:73-85): a_nb = +D_f,
  a_P = -sum D_f + V/dt, b = (V/dt) phi0; a fixed face moves -a_f * value to the right-hand
  side and a zero-gradient face folds a_f into a_P (PrimitiveBoundaryCondition.tpp:145-255).
* The returned value is ||A x - b||_inf (Diffusion.cpp:127-130).
"""
import numpy as np
import pytest

from oracle import oracle as O
from caffe_old_b200 import cases as C


def _box(n=(10, 6, 4), lengths=(2.0, 1.0, 0.5)):
    return C.cartesian_nodes(n, lengths), n, lengths


@pytest.mark.parametrize("axis", [0, 1, 2])
def test_steady_linear_profile_and_gradient(axis):
    nodes, n, lengths = _box()
    types = ["zeroGradient"] * 6
    values = [0.0] * 6
    hi, lo = 2 * axis, 2 * axis + 1                 # east/west, north/south, top/bottom
    types[hi], types[lo] = "fixed", "fixed"
    values[hi], values[lo] = -1.0, 3.0
    d = O.OracleDiffusion(nodes, types, values, method="bicgstab_jacobi", rtol=1e-13, maxit=5000)
    r = d.solve()
    L = lengths[axis]
    cc_axis = (np.indices(n[::-1])[2 - axis].ravel() + 0.5) * L / n[axis]
    want = 3.0 + (-1.0 - 3.0) * cc_axis / L
    phi = d.get("phi")
    assert np.abs(phi - want).max() < 1e-11
    assert r < 1e-11
    g = d.get("gradPhi").reshape(-1, 3)
    slope = np.zeros(3)
    slope[axis] = -4.0 / L
    assert np.abs(g - slope).max() < 1e-9
    d.close()


def test_assembled_rows_keep_the_references_coefficients():
    nodes, n, lengths = _box((6, 5, 4), (1.0, 1.0, 1.0))
    types = ["fixed", "zeroGradient", "fixed", "zeroGradient", "empty", "zeroGradient"]
    values = [2.0, 0.0, -1.0, 0.0, 0.0, 0.0]
    dt, phi0 = 0.25, 0.7
    d = O.OracleDiffusion(nodes, types, values, time_accurate=True, phi0=phi0, method="bicgstab_jacobi", rtol=1e-12)
    d.solve(dt)
    A = d.get("A").reshape(-1, 7)
    b = d.get("b")
    nI, nJ, nK = n
    h = (1.0 / nI, 1.0 / nJ, 1.0 / nK)
    V = h[0] * h[1] * h[2]
    D = [h[1] * h[2] / h[0]] * 2 + [h[0] * h[2] / h[1]] * 2 + [h[0] * h[1] / h[2]] * 2
    # boundary faces: D = |S|^2 / (S . r) with r the half cell to the face
    Db = [2.0 * x for x in D]
    for c in range(nI * nJ * nK):
        i, j, k = c % nI, (c // nI) % nJ, c // (nI * nJ)
        at = [i == nI - 1, i == 0, j == nJ - 1, j == 0, k == nK - 1, k == 0]
        aP = V / dt
        rhs = V / dt * phi0
        want = np.zeros(7)
        for f in range(6):
            Df = Db[f] if at[f] else D[f]
            aP -= Df
            if not at[f]:
                want[f + 1] = Df
            elif types[f] == "fixed":
                rhs -= Df * values[f]
            else:
                aP += Df
        want[0] = aP
        assert np.allclose(A[c], want, rtol=1e-12, atol=1e-12), (i, j, k, A[c], want)
        assert abs(b[c] - rhs) <= 1e-12 * max(1.0, abs(rhs)), (i, j, k)
    d.close()


def test_residual_and_repeated_solves():
    """Each call re-assembles from the current phi and returns ||A x - b||_inf; a steady
    case is at its solution after the first call and stays there."""
    nodes, n, _ = _box((8, 8, 3), (1.0, 1.0, 0.25))
    types = ["fixed", "fixed", "zeroGradient", "zeroGradient", "empty", "empty"]
    d = O.OracleDiffusion(nodes, types, [0.0, 1.0, 0, 0, 0, 0], method="bicgstab_sgs", rtol=1e-12, maxit=5000)
    r1 = d.solve()
    p1 = d.get("phi")
    r2 = d.solve()
    p2 = d.get("phi")
    assert r1 < 1e-10 and r2 < 1e-10
    assert np.abs(p1 - p2).max() < 1e-10
    st = d.stats()
    assert st["iters"] > 0 and st["rel_res"] < 1e-10
    d.close()


def test_all_zero_gradient_steady_case_gives_zero():
    """With every face zero-gradient and no time term the right-hand side is zero, and the
    solve from a zero guess leaves phi = 0 whatever it started at (the system is singular and
    the reference's Krylov solve returns its initial guess)."""
    nodes, n, _ = _box((5, 4, 3), (1.0, 1.0, 1.0))
    d = O.OracleDiffusion(nodes, ["zeroGradient"] * 6, [0.0] * 6, phi0=3.0, method="bicgstab_jacobi")
    r = d.solve()
    assert r == 0.0 and np.all(d.get("phi") == 0.0)
    d.close()


def test_invalid_boundary_type_is_refused():
    nodes, n, _ = _box((3, 3, 3), (1.0, 1.0, 1.0))
    with pytest.raises(KeyError):
        O.OracleDiffusion(nodes, ["wall"] + ["fixed"] * 5, [0.0] * 6)


def _plate_exact(X, Y, terms=399):
    """Steady temperature of the unit plate with T = 1 on x = 0 and T = 0 on the other three
    sides (the reference's FlatPlateDiffusion2D example): the Fourier series
    sum over odd m of 4/(m pi) sin(m pi y) sinh(m pi (1 - x)) / sinh(m pi)."""
    T = np.zeros_like(X)
    for m in range(1, terms + 1, 2):
        r = np.exp(-m * np.pi * X) * (1 - np.exp(-2 * m * np.pi * (1 - X))) / (1 - np.exp(-2 * m * np.pi))
        T += 4 / (m * np.pi) * np.sin(m * np.pi * Y) * r
    return T


def test_flat_plate_converges_to_the_analytical_solution():
    """The reference's FlatPlateDiffusion2D set-up (fixed 1 on the west face, fixed 0 on the
    east, north and south faces, empty top and bottom) on 20^2 and 40^2 cells: the relative
    L2 error against the series solution is below 1e-2 and halves with the cell size (first
    order, from the discontinuous corners)."""
    errs = []
    for n in (20, 40):
        nodes = C.cartesian_nodes((n, n, 1), (1.0, 1.0, 1.0))
        d = O.OracleDiffusion(nodes, ["fixed", "fixed", "fixed", "fixed", "empty", "empty"], [0.0, 1.0, 0.0, 0.0, 0.0, 0.0],
                              method="bicgstab_jacobi", rtol=1e-12, maxit=20000)
        d.solve()
        phi = d.get("phi").reshape(n, n)
        x = (np.arange(n) + 0.5) / n
        X, Y = np.meshgrid(x, x)
        T = _plate_exact(X, Y)
        errs.append(np.linalg.norm(phi - T) / np.linalg.norm(T))
        d.close()
    assert errs[0] < 1e-2 and errs[1] < 1e-2
    assert 1.8 < errs[0] / errs[1] < 2.2, errs
