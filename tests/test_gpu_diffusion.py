"""Device path of the reference's Diffusion solver (src/Solvers/Diffusion.cpp:35-131) against the
oracle's restatement of it:

* the assembled rows and right-hand side are bit-exact (same coefficients, boundary folding and
  operand order);
* from the same linear-solve result x, everything after the solve -- phi, the zero-gradient
  patches, the interior faces interpolated then re-extrapolated from both cells' gradients and
  clamped, the cell gradients and ||A x - b||_inf -- is bit-exact;
* whole solves (steady, and unsteady steps on a sheared, jittered mesh) agree within 1e-10
  relative L2 with both sides solving to 1e-13."""
import numpy as np
import pytest

from caffe_old_b200 import cases as C
from caffe_old_b200.solver import Diffusion
from oracle import oracle as O

from helpers import rel_l2

pytestmark = pytest.mark.gpu

TYPES = ["fixed", "zeroGradient", "fixed", "zeroGradient", "empty", "zeroGradient"]
VALUES = [2.0, 0.0, -1.0, 0.0, 0.0, 0.0]


def _pair(nodes, time_accurate, phi0, method="bicgstab_jacobi", rtol=1e-13):
    o = O.OracleDiffusion(nodes, TYPES, VALUES, time_accurate=time_accurate, phi0=phi0, method=method, rtol=rtol, maxit=20000)
    d = Diffusion(nodes, TYPES, VALUES, time_accurate=time_accurate, phi0=phi0, method=method, rtol=rtol, maxit=20000)
    return o, d


@pytest.mark.parametrize("skewed", [False, True])
def test_phases_bit_exact(skewed):
    nodes = C.skewed_nodes((9, 7, 6), (1.0, 1.0, 1.0), 30.0, 0.1, 4) if skewed else C.cartesian_nodes((9, 7, 6), (1.0, 1.0, 0.5))
    o, d = _pair(nodes, True, 0.7)
    dt = 0.05
    for step in range(2):
        o.solve(dt)                 # the oracle's whole step
        d.phase("assemble", dt)
        assert np.array_equal(d.get("A").reshape(-1, 7), o.get("A").reshape(-1, 7)), step
        assert np.array_equal(d.get("b"), o.get("b")), step
        d.set("x", o.get("phi"))    # the oracle's solution: the rest must follow bit for bit
        d.phase("post", dt)
        assert np.array_equal(d.get("phi"), o.get("phi"))
        for nm in ("phiFaceI", "phiFaceJ", "phiFaceK", "gradPhi") + tuple(f"phiPatch{f}" for f in range(6)):
            assert np.array_equal(d.get(nm), o.get(nm)), (step, nm)
    o.close()
    d.close()


@pytest.mark.parametrize("method", ["bicgstab_jacobi", "cg_jacobi"])
def test_steady_solve_matches_oracle(method):
    nodes = C.cartesian_nodes((24, 16, 12), (2.0, 1.0, 0.5))
    o, d = _pair(nodes, False, 0.0, method=method)
    ro, rd = o.solve(), d.solve()
    assert rel_l2(d.get("phi"), o.get("phi")) < 1e-10
    assert rel_l2(d.get("gradPhi"), o.get("gradPhi")) < 1e-9
    assert d.rel_res <= 1e-13 and rd < 1e-10 and ro < 1e-10


def test_unsteady_steps_on_skewed_mesh_match_oracle():
    nodes = C.skewed_nodes((20, 16, 12), (1.0, 1.0, 1.0), 30.0, 0.1, 7)
    o, d = _pair(nodes, True, 0.3)
    for _ in range(5):
        o.solve(0.02)
        d.solve(0.02)
    assert rel_l2(d.get("phi"), o.get("phi")) < 1e-10
    for nm in ("phiFaceI", "phiFaceJ", "phiFaceK"):
        assert rel_l2(d.get(nm), o.get(nm)) < 1e-10, nm
