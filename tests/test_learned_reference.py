"""CPU checks of the level-pyramid restatement that serves as the checker of the learned
preconditioner's device kernels."""
import numpy as np

import learned_reference as LR
from caffe_old_b200 import precond as P

import cnn_reference as R


def test_restriction_is_the_adjoint_of_prolongation():
    rng = np.random.default_rng(0)
    for f in [(7, 10, 13), (1, 6, 9), (2, 2, 3)]:
        c = LR.coarse_dims(f)
        w = rng.standard_normal(c)
        v = rng.standard_normal(f)
        assert abs(np.vdot(LR.prolong(w, f), v) - np.vdot(w, LR.prolong_T(v, c))) < 1e-12 * np.abs(v).sum() * np.abs(w).sum()


def test_restriction_averages_constants():
    # even directions: every coarse cell averages (with the clamped edges folded in)
    for f in [(8, 6, 10), (1, 6, 8), (4, 4, 4)]:
        c = LR.coarse_dims(f)
        avg = LR.rscale(f) * LR.prolong_T(np.ones(f), c)
        assert np.allclose(avg, 1.0)
        assert np.allclose(LR.prolong(np.ones(c), f), 1.0)


def test_pyramid_of_the_25m_cell_lattice():
    dims = LR.pyramid((256, 256, 384))
    assert dims[1] == (128, 128, 192)
    assert dims[-1] == (2, 2, 3)
    assert len(dims) == 8


def test_identity_parameters_make_the_network_an_identity():
    p = P.identity_params(3)
    shape = (6, 5, 4)
    n = int(np.prod(shape))
    x2 = np.random.default_rng(1).standard_normal((n, 2))
    y, _ = R.forward(p.astype(np.float64), x2, shape, bf=False, extra_const=0.25)
    assert np.abs(y - x2[:, 0]).max() < 1e-12


def test_level_pyramid_cuts_flexible_cg_iterations():
    """The pyramid with an identity in place of the network already needs several times
    fewer flexible-CG iterations than Jacobi on a 7-point Poisson problem; the network form
    with identity parameters gives the same iterations."""
    rng = np.random.default_rng(2)
    dims = (16, 24, 24)
    A, diag = LR.poisson7(dims)
    b = rng.standard_normal(dims)
    invD = 1.0 / diag
    act = np.ones(dims, bool)
    its = {}
    for mode in ["jacobi", "levels"]:
        x, its[mode] = LR.fcg(A, b, lambda r: LR.apply_M(r, invD, act, mode), 1e-8, 3000)
        assert np.linalg.norm(b - A(x)) <= 1.01e-8 * np.linalg.norm(b)
    assert its["levels"] * 2.5 < its["jacobi"], its
    params = P.identity_params(0)
    _, it_net = LR.fcg(A, b, lambda r: LR.apply_M(r, invD, act, "network", params), 1e-8, 3000)
    assert abs(it_net - its["levels"]) <= 1, (it_net, its)


def test_odd_network_form_keeps_fgmres_convergent():
    """A network with biases and constant input channels has an input-independent part; the
    odd form (net(x) - net(-x)) / 2 the device applies removes it exactly (the output of a
    zero residual is zero, and M(-r) = -M(r)), and FGMRES with it converges like the pyramid."""
    rng = np.random.default_rng(4)
    dims = (12, 16, 16)
    A, diag = LR.poisson7(dims)
    b = rng.standard_normal(dims)
    invD = 1.0 / diag
    act = np.ones(dims, bool)
    params = P.identity_params(1, noise=0.3)
    for l in range(P.LAYERS):
        _, bias = P.weight_view(params, l)
        bias[:] = 0.05 * rng.standard_normal(bias.shape)
    r = rng.standard_normal(dims)
    zp = LR.apply_M(r, invD, act, "network", params)
    zn = LR.apply_M(-r, invD, act, "network", params)
    assert np.allclose(zp, -zn, atol=1e-12 * np.abs(zp).max())
    assert np.abs(LR.apply_M(np.zeros(dims), invD, act, "network", params)).max() == 0.0
    _, it_lev = LR.fgmres(A, b, lambda v: LR.apply_M(v, invD, act, "levels"), 40, 1e-6, 400)
    x, it_net = LR.fgmres(A, b, lambda v: LR.apply_M(v, invD, act, "network", params), 40, 1e-6, 400)
    assert np.linalg.norm(b - A(x)) <= 1.01e-6 * np.linalg.norm(b)
    assert it_net < 3 * it_lev, (it_net, it_lev)
