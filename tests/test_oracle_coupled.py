"""The oracle's restatement of the reference's Coupled solver (src/Solvers/Coupled.cpp), on
the CPU: momentum and continuity assembled into one system of 4 N unknowns and solved
together, then the Rhie-Chow face fluxes.  Known properties of the reference's formulation:

* every coupled linear solve converges and the lid-driven cavity reaches a steady state;
* a cavity with every wall at rest stays at rest;
* the face mass flux carries no density (Coupled.cpp:282-314) while every continuity row is
  proportional to it, so a steady solution does not depend on rho;
* the reported continuity error is the largest face-flux imbalance per volume
  (Coupled.cpp:316-339).

The reference never interpolates p to interior faces before its divergence-theorem gradient
(Coupled.cpp:257-258), so those faces keep their initial zero; the restatement keeps that,
which holds its steady cavity about 10% away from SIMPLE's on the same mesh (with the
interpolation added, the two agree within 0.3%).
"""
import numpy as np

from oracle import oracle as O
from oracle.oracle import OracleSolver
from caffe_old_b200 import cases as C

from helpers import rel_l2


def _cavity(rho=1.0, lid=1.0, method="bicgstab_sgs"):
    nodes = C.cartesian_nodes((8, 8, 1), (1.0, 1.0, 1.0 / 8))
    bc, ref = C.lid_cavity_bcs("north", lid_velocity=(lid, 0.0, 0.0), two_d=True)
    spec = C.CaseSpec(kind="simple", bc=bc, ref_vec=ref, rho=rho, mu=0.01, time_accurate=False, omega_u=0.7, omega_p=0.3,
                      mom_method=method, p_method="bicgstab_jacobi", mom_rtol=1e-11, p_rtol=1e-11, maxit=20000, dt=1.0)
    return nodes, spec


def _run(nodes, spec, iters):
    s = O.OracleCoupled(nodes, spec)
    cont = None
    for _ in range(iters):
        cont = s.solve()
        st = s.stats()
        assert st["status"] == 0 and st["rel_res"] <= 1e-10, st
    return s, cont


def test_coupled_solves_converge_to_a_steady_cavity():
    nodes, spec = _cavity()
    s, _ = _run(nodes, spec, 200)
    u1 = s.get("u")
    s.solve()
    assert rel_l2(s.get("u"), u1) < 1e-8
    assert 0.3 < np.abs(u1).max() < 1.0
    s.close()


def test_cavity_at_rest_stays_at_rest():
    nodes, spec = _cavity(lid=0.0)
    s, cont = _run(nodes, spec, 3)
    assert np.abs(s.get("u")).max() == 0.0 and np.abs(s.get("p")).max() == 0.0 and cont == 0.0
    s.close()


def test_steady_solution_does_not_depend_on_rho():
    a, _ = _run(*_cavity(rho=1.0), 40)
    b, _ = _run(*_cavity(rho=2.5), 40)
    assert rel_l2(b.get("u"), a.get("u")) < 1e-9
    pa, pb = a.get("p"), b.get("p")
    assert rel_l2(pb - pb.mean(), pa - pa.mean()) < 1e-8
    a.close()
    b.close()


def test_continuity_error_is_the_largest_face_flux_imbalance():
    nodes, spec = _cavity()
    s, cont = _run(nodes, spec, 5)
    nI, nJ, nK = s.shape
    FI = s.get("massFlowI").reshape(nK, nJ, nI + 1)
    FJ = s.get("massFlowJ").reshape(nK, nJ + 1, nI)
    FK = s.get("massFlowK").reshape(nK + 1, nJ, nI)
    imbalance = (FI[:, :, 1:] - FI[:, :, :-1]) + (FJ[:, 1:, :] - FJ[:, :-1, :]) + (FK[1:] - FK[:-1])
    vol = 1.0 / (nI * nJ) * (1.0 / 8)
    assert abs(np.abs(imbalance).max() / vol - cont) <= 1e-12 * cont
    s.close()


def test_steady_cavity_near_simple():
    nodes, spec = _cavity(method="bicgstab_jacobi")
    o = OracleSolver(nodes, spec)
    for _ in range(400):
        o.solve()
    s, _ = _run(nodes, spec, 60)
    assert rel_l2(s.get("u"), o.get("u")) < 0.2
    s.close()
    o.close()
