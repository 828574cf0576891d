"""Lock-step comparison of the oracle with the reference's own solver code (oracle/ref_solver.py).

The oracle is driven phase by phase; every linear system it assembles and every solution its
Krylov solver returns is collected.  The reference's Simple / Piso / IbPiso then takes the same
step with its KSPSolve handing back the oracle's solutions in the same order, so both sides
continue from identical numbers and everything outside the Krylov solves -- assembly with the
boundary folding, the immersed-boundary rows, Rhie-Chow, the corrections, the gradients and the
continuity error -- can be compared bit for bit.  The same is done for the reference's Coupled
and Diffusion solvers.
"""
from __future__ import annotations

import numpy as np

from caffe_old_b200 import cases as _C
from oracle import oracle as _O
from oracle import ref_solver as R
from oracle.oracle import OracleSolver

FIELDS = ("u", "p", "gradP", "massFlowI", "massFlowJ", "massFlowK")


def _csr_to_rows(ptr, col, val):
    rows = []
    for r in range(len(ptr) - 1):
        rows.append({int(col[p]): float(val[p]) for p in range(ptr[r], ptr[r + 1])})
    return rows


def _nonzero(rows):
    # PETSc keeps explicit zeros of a row's structure after MatZeroEntries; compare the values
    return [{c: v for c, v in r.items() if v != 0.0} for r in rows]


def oracle_step(o, spec):
    """One oracle step, phase by phase: (systems in KSPSolve order, solutions in that order,
    continuity error).  A system is (rows, b)."""
    dt = spec.dt
    systems, sols = [], []
    status = o.get("status") if spec.kind == "ibpiso" else None
    keep = (status != 2) if status is not None else slice(None)
    o.phase("save_u0", dt)
    if spec.kind == "ibpiso":
        o.phase("ib_field", dt)
    n_in = spec.n_inner if spec.time_accurate else 1
    n_pc = 1 if spec.kind == "simple" else spec.n_pcorr
    for _ in range(n_in):
        if spec.kind == "ibpiso":
            o.phase("ib_coeffs", dt)
            status = o.get("status")
            keep = status != 2
        o.phase("assemble_momentum", dt)
        for comp in range(3):
            systems.append(o.system(0, comp))
        o.phase("solve_momentum", dt)
        u = o.get("u").reshape(-1, 3)
        for comp in range(3):
            sols.append(u[keep, comp].copy())
        o.phase("momentum_post", dt)
        for _ in range(n_pc):
            o.phase("assemble_pcorr", dt)
            systems.append(o.system(1, 0))
            o.phase("solve_pcorr", dt)
            sols.append(o.get("pCorr")[keep].copy())
            o.phase("correct", dt)
    o.phase("continuity", dt)
    if spec.kind != "ibpiso":
        o.phase("courant", dt)
    return systems, sols, o.stats()["continuity"]


def _ghost_rows_close(rrows, orows, ghost_rows, tol):
    """Ghost rows: the same columns, values within `tol` relative.  Their trilinear weights come
    from an 8 x 8 inverse that the reference takes through LAPACK (Matrix.cpp:149-154), replaced
    here by a textbook LU, so they agree to round-off of that ill-conditioned inverse only."""
    for g in ghost_rows:
        a, b = rrows[g], orows[g]
        if set(a) != set(b):
            return False
        scale = max(abs(v) for v in b.values())
        if any(abs(a[c] - b[c]) > tol * scale for c in b):
            return False
    return True


def lockstep(nodes, spec, steps, keep_fields=False, ghost_tol=1e-9):
    """Run both for `steps` steps; returns a list of per-step reports:
    {"systems": [(non-ghost rows equal, ghost rows close, b equal)], "fields": {name: equal},
    "continuity": (ref, oracle)}."""
    o = OracleSolver(nodes, spec)
    r = R.RefSolver(nodes, spec, record=True)
    reports = []
    try:
        for _ in range(steps):
            o_sys, sols, cont_o = oracle_step(o, spec)
            R.clear_injected()
            R.lib().refsolver_record(1)
            for x in sols:
                R.inject(x)
            cont_r = r.solve()
            assert R.injected_left() == 0, "the reference made fewer linear solves than the oracle"
            rec = R.recorded_systems()
            assert len(rec) == len(o_sys), (len(rec), len(o_sys))
            status = o.get("status") if spec.kind == "ibpiso" else np.zeros(o.get("vol").size)
            rows_of = np.flatnonzero(status != 2)
            ghost = set(int(q) for q in np.flatnonzero(status[rows_of] == 1))
            sys_eq = []
            for (ptr, col, val, b, _x), (orow, ob) in zip(rec, o_sys):
                rrows = _nonzero(_csr_to_rows(ptr, col, val))
                orows = _nonzero(orow)
                plain = all(rrows[q] == orows[q] for q in range(len(orows)) if q not in ghost) and len(rrows) == len(orows)
                sys_eq.append((plain, _ghost_rows_close(rrows, orows, ghost, ghost_tol), np.array_equal(b, ob)))
            fields = {nm: np.array_equal(r.get(nm), o.get(nm)) for nm in FIELDS}
            rep = {"systems": sys_eq, "fields": fields, "continuity": (cont_r, cont_o),
                   "max_field_diff": {nm: float(np.max(np.abs(r.get(nm) - o.get(nm)))) for nm in FIELDS}}
            if keep_fields:
                rep["ref_fields"] = {nm: r.get(nm) for nm in FIELDS + ("massFlow",)}
            reports.append(rep)
    finally:
        R.clear_injected()
        r.close()
        o.close()
    return reports


# ---------------------------------------------------------------- Coupled and Diffusion
# src/Solvers/Coupled.cpp and src/Solvers/Diffusion.cpp, driven like the flow solvers above: the
# oracle takes each step phase by phase, the reference's KSPSolve returns the oracle's solutions.

COUPLED_RTOL = 1e-12
COUPLED_FIELDS = ("u", "p", "gradP", "h", "d", "massFlowI", "massFlowJ", "massFlowK")
DIFFUSION_FIELDS = ("phi", "gradPhi", "phiFaceI", "phiFaceJ", "phiFaceK")
DIFFUSION_TYPES = ["fixed", "zeroGradient", "fixed", "zeroGradient", "empty", "zeroGradient"]
DIFFUSION_VALUES = [2.0, 0.0, -1.0, 0.0, 0.0, 0.0]
DIFFUSION_DT = 0.05


def coupled_cases():
    C, RT = _C, COUPLED_RTOL
    nodes = C.cartesian_nodes((10, 8, 1), (1.0, 1.0, 1.0 / 8))
    bc, ref = C.lid_cavity_bcs("north", lid_velocity=(1.0, 0.0, 0.0), two_d=True)
    cav = (nodes, C.CaseSpec(kind="simple", bc=bc, ref_vec=ref, rho=1.0, mu=0.01, time_accurate=False, omega_u=0.7,
                             omega_p=0.3, mom_method="bicgstab_jacobi", p_method="bicgstab_jacobi", mom_rtol=RT, p_rtol=RT,
                             maxit=20000, dt=1.0))
    nodes = C.skewed_nodes((7, 6, 5), (1.0, 1.0, 1.0), 30.0, 0.1, 5)
    bc, ref = C.lid_cavity_bcs("north")
    skw = (nodes, C.CaseSpec(kind="simple", bc=bc, ref_vec=ref, rho=1.3, mu=0.02, time_accurate=True, n_inner=2, omega_u=0.8,
                             omega_p=0.3, mom_method="bicgstab_jacobi", p_method="bicgstab_jacobi", mom_rtol=RT, p_rtol=RT,
                             maxit=20000, dt=0.05))
    nodes = C.cartesian_nodes((12, 6, 5), (3.0, 1.0, 1.0))
    bc, ref = C.channel_bcs(1.0)
    chn = (nodes, C.CaseSpec(kind="simple", bc=bc, ref_vec=ref, ref_val=(0.25, 0, 0, 0, 0, 0), rho=1.0, mu=0.05,
                             time_accurate=False, omega_u=0.7, omega_p=0.3, mom_method="bicgstab_jacobi",
                             p_method="bicgstab_jacobi", mom_rtol=RT, p_rtol=RT, maxit=20000, dt=1.0))
    return {"cavity2d": cav, "skewed3d": skw, "channel": chn}


def diffusion_cases():
    """(nodes, time_accurate, phi0) per case."""
    C = _C
    skewed = C.skewed_nodes((9, 7, 6), (1.0, 1.0, 1.0), 30.0, 0.1, 4)
    return {"cartesian_steady": (C.cartesian_nodes((9, 7, 6), (1.0, 1.0, 0.5)), False, 0.0),
            "skewed_unsteady": (skewed, True, 0.7),
            "skewed_steady": (skewed, False, 0.0)}


def _oracle_rows(o):
    cnt, col, val = o.system()
    return [{int(col[r, p]): float(val[r, p]) for p in range(cnt[r])} for r in range(len(cnt))]


def diffusion_rows(A, shape):
    """The oracle's (cells x 7) coefficients (self, east, west, north, south, top, bottom) as
    rows {column: value} of the global matrix, nonzero entries only."""
    nI, nJ, nK = shape
    A = A.reshape(-1, 7)
    rows = []
    for c in range(A.shape[0]):
        i, j, k = c % nI, (c // nI) % nJ, c // (nI * nJ)
        nb = [c, c + 1 if i < nI - 1 else None, c - 1 if i > 0 else None, c + nI if j < nJ - 1 else None,
              c - nI if j > 0 else None, c + nI * nJ if k < nK - 1 else None, c - nI * nJ if k > 0 else None]
        rows.append({nb[q]: float(A[c, q]) for q in range(7) if nb[q] is not None and A[c, q] != 0.0})
    return rows


def coupled_lockstep(nodes, spec, steps):
    """Per step: (systems equal, right-hand sides equal) per inner iteration, the reference's and
    the oracle's fields."""
    o = _O.OracleCoupled(nodes, spec)
    r = R.RefSolver(nodes, spec, record=True, kind="coupled")
    inner = spec.n_inner if spec.time_accurate else 1
    out = []
    try:
        for _ in range(steps):
            o.phase("save_u0")
            systems, sols = [], []
            for _ in range(inner):
                o.phase("assemble")
                systems.append((_nonzero(_oracle_rows(o)), o.get("b")))
                o.phase("solve")
                sols.append(o.get("x"))
                o.phase("post")
            R.clear_injected()
            R.lib().refsolver_record(1)
            for x in sols:
                R.inject(x)
            r.solve(spec.dt)
            rec = R.recorded_systems()
            checks = [(_nonzero(_csr_to_rows(p_, c_, v_)) == rows, bool(np.array_equal(b_, ob)))
                      for (p_, c_, v_, b_, _), (rows, ob) in zip(rec, systems)]
            out.append({"systems": checks, "n_systems": len(rec), "n_expected": inner, "left": R.injected_left(),
                        "ref_fields": {nm: r.get(nm) for nm in COUPLED_FIELDS},
                        "oracle_fields": {nm: o.get(nm) for nm in COUPLED_FIELDS}})
    finally:
        r.close()
        o.close()
    return out


def diffusion_lockstep(nodes, time_accurate, phi0, steps):
    o = _O.OracleDiffusion(nodes, DIFFUSION_TYPES, DIFFUSION_VALUES, time_accurate=time_accurate, phi0=phi0,
                           method="bicgstab_jacobi", rtol=1e-13, maxit=20000)
    r = R.RefSolver(nodes, None, record=True, kind="diffusion",
                    diffusion=(DIFFUSION_TYPES, DIFFUSION_VALUES, time_accurate, phi0))
    out = []
    try:
        for _ in range(steps):
            o.solve(DIFFUSION_DT)
            R.clear_injected()
            R.lib().refsolver_record(1)
            R.inject(o.get("phi"))
            r.solve(DIFFUSION_DT)
            rec = R.recorded_systems()
            p_, c_, v_, b_, _ = rec[0]
            out.append({"n_systems": len(rec),
                        "system": _nonzero(_csr_to_rows(p_, c_, v_)) == diffusion_rows(o.get("A"), o.shape),
                        "rhs": bool(np.array_equal(b_, o.get("b"))),
                        "ref_fields": {nm: r.get(nm) for nm in DIFFUSION_FIELDS},
                        "oracle_fields": {nm: o.get(nm) for nm in DIFFUSION_FIELDS}})
    finally:
        r.close()
        o.close()
    return out
