"""Writes tests/golden/reference_solver.npz: outputs of the reference's own solver code.

The reference's Simple / Piso / IbPiso (src/Solvers/*.cpp with the mesh, field, scheme and math
sources they use) are compiled from its sources with stand-in PETSc / MPI / LAPACKE / Boost
headers (``make -C oracle refsolver``, oracle/ref_solver.py) and run here.  Stored:

* ``c1_*``: the BASELINE's first configuration exactly -- SIMPLE, 2-D lid-driven cavity on the
  unit square with 64 x 64 x 1 cells, Re = 100, upwind, relaxation 0.7 / 0.3, zero initial
  fields, 500 outer iterations -- with every linear system solved to a 1e-13 true relative
  residual (the stand-in KSPSolve): u (N x 3), p, the face mass fluxes and the continuity error
  of every iteration.
* ``ls_<case>_*``: small cases run in lock step with the oracle (the reference's KSPSolve
  returns the oracle's solutions, so both continue from identical numbers): the reference's
  fields.  These equal the oracle's bit for bit; with the fixture the oracle
  stays pinned where the reference's sources are absent.

Run from the repository root after ``make -C oracle refsolver``:
    python tests/golden/make_reference_solver_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

_ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, _ROOT)
sys.path.insert(0, os.path.join(_ROOT, "tests"))

from caffe_old_b200 import cases as C  # noqa: E402
from oracle import ref_solver as R  # noqa: E402
import helpers as H  # noqa: E402
import ref_pin as P  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_solver.npz")
FIELDS = ("u", "p", "massFlowI", "massFlowJ", "massFlowK")
C1_ITERATIONS = 500
LOCKSTEP_STEPS = 3


def lockstep_cases():
    """Small cases the reference can run (upwind convection, no non-orthogonal correction)."""
    skewed_nodes, skewed_spec = H.small_skewed(nonorth=False)
    return {
        "cavity2d": H.small_cavity2d(),
        "cavity3d": H.small_cavity3d(central=False),
        "skewed": (skewed_nodes, skewed_spec.replace(convection="upwind")),
        "channel": H.small_channel_sphere(),
        "piso_inner": H.small_piso_inner(),
        "simple_transient": H.small_simple_transient(),
        "outlet_top": H.small_outlet_top(),
    }


def main():
    out = {}
    nodes, spec, _ = C.config1_cavity2d(n=64)
    spec = spec.replace(mom_rtol=1e-13, p_rtol=1e-13)
    r = R.RefSolver(nodes, spec, rtol=1e-13)
    cont = [r.solve() for _ in range(C1_ITERATIONS)]
    for nm in FIELDS:
        out[f"c1_{nm}"] = r.get(nm)
    out["c1_continuity"] = np.array(cont)
    r.close()
    for name, (nodes, spec) in lockstep_cases().items():
        reports = P.lockstep(nodes, spec, LOCKSTEP_STEPS, keep_fields=True)
        for nm in FIELDS:
            out[f"ls_{name}_{nm}"] = reports[-1]["ref_fields"][nm]
        out[f"ls_{name}_continuity"] = np.array([rep["continuity"][0] for rep in reports])
    np.savez_compressed(OUT, **out)
    print("wrote", OUT, sum(v.nbytes for v in out.values()), "bytes uncompressed")


if __name__ == "__main__":
    main()
