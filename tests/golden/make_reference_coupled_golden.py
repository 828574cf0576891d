"""Writes tests/golden/reference_coupled.npz: fields of the reference's own Coupled and Diffusion
solvers (src/Solvers/Coupled.cpp, src/Solvers/Diffusion.cpp, compiled from its sources with
stand-in PETSc / MPI / LAPACKE / Boost headers by ``make -C oracle refsolver``), run here in lock
step with the oracle (the reference's KSPSolve returns the oracle's solutions).

Stored per case (tests/ref_pin.py ``coupled_cases``, ``diffusion_cases``): the reference's
fields after the lock-step steps, ``coupled_<case>_<field>`` and ``diffusion_<case>_<field>``.
The oracle reproduces them bit for bit, so the fixture keeps the pin where the reference's
sources are absent.

Run from the repository root after ``make -C oracle refsolver``:
    python tests/golden/make_reference_coupled_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

_ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, _ROOT)
sys.path.insert(0, os.path.join(_ROOT, "tests"))

import ref_pin as P  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_coupled.npz")
STEPS = 3


def main():
    out = {}
    for name, (nodes, spec) in P.coupled_cases().items():
        reps = P.coupled_lockstep(nodes, spec, STEPS)
        for nm in P.COUPLED_FIELDS:
            out[f"coupled_{name}_{nm}"] = reps[-1]["ref_fields"][nm]
    for name, (nodes, ta, phi0) in P.diffusion_cases().items():
        reps = P.diffusion_lockstep(nodes, ta, phi0, STEPS if ta else 1)
        for nm in P.DIFFUSION_FIELDS:
            out[f"diffusion_{name}_{nm}"] = reps[-1]["ref_fields"][nm]
    np.savez_compressed(OUT, **out)
    print("wrote", OUT, sum(v.nbytes for v in out.values()), "bytes uncompressed")


if __name__ == "__main__":
    main()
