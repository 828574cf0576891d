"""Writes tests/golden/oracle_fields.npz: the oracle's u and p after 1, 5 and 50 outer
iterations / time steps (1 and 20 for the immersed-boundary channel) of reduced-size
versions of the four cases:
  * the 2-D lid-driven cavity (steady SIMPLE, upwind);
  * the 3-D cavity (PISO, central convection, Jacobi-PCG);
  * the sheared and jittered cavity (non-orthogonal correction on);
  * the channel with an immersed sphere (IB-PISO).

Every linear solve runs to a 1e-13 true relative residual (1e-12 with the sphere's ghost
rows), as in the parity tests.  The fixtures lock the oracle's results: a change to the
oracle that moves them shows up in tests/test_oracle_golden.py on any machine.  The nodes are
stored with the fields, so the fixtures do not depend on the mesh generators.

  python tests/golden/make_oracle_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

OUT = os.path.join(HERE, "oracle_fields.npz")
KSP_RTOL = 1e-13
KSP_RTOL_IB = 1e-12


def golden_cases():
    """name -> (nodes, spec, steps at which u and p are stored)."""
    from caffe_old_b200 import cases as C
    n1, s1, _ = C.config1_cavity2d(n=16)
    n2, s2, _ = C.config2_cavity3d(n=8)
    n3, s3, _ = C.config3_skewed(n=8, seed=0, p_form="fp64")
    n4, s4, _ = C.config4_channel_sphere((32, 12, 12), seed=2)
    return {
        "cavity2d_16": (n1, s1.replace(mom_rtol=KSP_RTOL, p_rtol=KSP_RTOL), (1, 5, 50)),
        "cavity3d_8": (n2, s2.replace(mom_rtol=KSP_RTOL, p_rtol=KSP_RTOL), (1, 5, 50)),
        "skewed_8": (n3, s3.replace(mom_rtol=KSP_RTOL, p_rtol=KSP_RTOL), (1, 5, 50)),
        "channel_sphere_32x12x12": (n4, s4.replace(mom_rtol=KSP_RTOL_IB, p_rtol=KSP_RTOL_IB), (1, 20)),
    }


def run_case(nodes, spec, steps):
    """{step: (u, p)} of the oracle run on these nodes."""
    from oracle.oracle import OracleSolver
    o = OracleSolver(nodes, spec)
    out = {}
    for s in range(1, max(steps) + 1):
        o.solve()
        if s in steps:
            out[s] = (o.get("u").copy(), o.get("p").copy())
    o.close()
    return out


def main():
    arrays = {}
    for name, (nodes, spec, steps) in golden_cases().items():
        res = run_case(nodes, spec, steps)
        arrays[f"{name}/nodes"] = nodes
        for s, (u, p) in res.items():
            arrays[f"{name}/u{s}"] = u
            arrays[f"{name}/p{s}"] = p
        print(name, "steps", steps)
    np.savez_compressed(OUT, **arrays)
    print("wrote", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    main()
