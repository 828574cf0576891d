"""Restart files of one cell field, in the layout of the reference's
InitialConditions::writeRestart (src/Domains/Field/InitialConditions.cpp:77-119): cells in
i-fastest order, one text line per j row, an empty line after each k plane, and for a vector
field the three components of a cell side by side.  Values are written with 17 significant
digits, so reading a file back gives the same doubles; files the reference wrote (6 digits)
read the same way.  The C++ host layer reads and writes the same files
(InitialConditions::writeRestartFile / readRestartFile, and the `restart` initial-condition
type of case/initialConditions.info).
"""
from __future__ import annotations

import numpy as np


def write_restart(path: str, values: np.ndarray, shape: tuple[int, int, int]) -> None:
    """values: one value per cell (N,) or per cell and component (N, C), cells i-fastest."""
    nI, nJ, nK = shape
    n = nI * nJ * nK
    v = np.asarray(values, dtype=np.float64).reshape(n, -1)
    rows = v.reshape(nK, nJ, nI * v.shape[1])
    with open(path, "w") as f:
        for plane in rows:
            for row in plane:
                f.write("".join("%.17g " % x for x in row) + "\n")
            f.write("\n")


def read_restart(path: str, shape: tuple[int, int, int], components: int = 1) -> np.ndarray:
    """(N,) for one component, (N, components) otherwise; raises ValueError on a file that does
    not hold exactly N x components numbers."""
    nI, nJ, nK = shape
    n = nI * nJ * nK
    with open(path) as f:
        tokens = f.read().split()
    if len(tokens) != n * components:
        raise ValueError(f"{path} holds {len(tokens)} values; {n * components} ({components} per cell) were expected")
    try:
        v = np.array([float(t) for t in tokens], dtype=np.float64)
    except ValueError as e:
        raise ValueError(f"{path} holds a value that is not a number: {e}") from None
    return v if components == 1 else v.reshape(n, components)
