"""Lock-step comparison of the oracle with the reference's own solver code (oracle/ref_solver.py).

The oracle is driven phase by phase; every linear system it assembles and every solution its
Krylov solver returns is collected.  The reference's Simple / Piso / IbPiso then takes the same
step with its KSPSolve handing back the oracle's solutions in the same order, so both sides
continue from identical numbers and everything outside the Krylov solves -- assembly with the
boundary folding, the immersed-boundary rows, Rhie-Chow, the corrections, the gradients and the
continuity error -- can be compared bit for bit.
"""
from __future__ import annotations

import numpy as np

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
