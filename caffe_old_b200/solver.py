"""Host-side mirror of the reference's solver interface, over the C ABI.

``Simple``, ``Piso`` and ``IbPiso`` keep the reference's names and call pattern: the
constructor takes the mesh (node array) and the case, and ``solve(time_step)``
advances one outer iteration / time step and returns the maximum continuity error,
as Solver::solve does (src/Solvers/Solver.h:20, Simple.cpp:78-91, Piso.cpp:12-29,
IbPiso.cpp:43-61).  Fields stay in HBM; ``field(name)`` copies one out.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import cases as C
from ._lib import CaffeError, StepStats, _ptr, last_error, lib, make_case


class DeviceSolver:
    """One device handle: mesh metrics, fields, linear systems, Krylov workspace."""

    kind = None

    def __init__(self, nodes: np.ndarray, spec: C.CaseSpec, device: int = 0):
        if self.kind is not None and spec.kind != self.kind:
            spec = spec.replace(kind=self.kind)
        L = lib()
        nodes = np.ascontiguousarray(nodes, dtype=np.float64)
        if nodes.ndim != 4 or nodes.shape[-1] != 3:
            raise ValueError("nodes must have shape (nK+1, nJ+1, nI+1, 3)")
        nK1, nJ1, nI1, _ = nodes.shape
        self.shape = (nI1 - 1, nJ1 - 1, nK1 - 1)
        self.ncells = self.shape[0] * self.shape[1] * self.shape[2]
        self.spec = spec
        self._case = make_case(spec)
        h = ctypes.c_void_p()
        rc = L.caffe_dev_create(_ptr(nodes), nI1, nJ1, nK1, ctypes.byref(self._case), int(device), ctypes.byref(h))
        if rc != 0 or not h.value:
            raise CaffeError("caffe_dev_create: " + last_error())
        self._h = h
        self.last_stats: dict = {}

    # -- lifecycle
    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().caffe_dev_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- the reference's interface
    def solve(self, time_step: float | None = None, stats: bool = True) -> float:
        dt = float(self.spec.dt if time_step is None else time_step)
        st = StepStats()
        rc = lib().caffe_dev_solve(self._h, dt, ctypes.byref(st) if stats else None)
        if rc != 0:
            raise CaffeError(f"caffe_dev_solve (status {rc}): " + last_error())
        if stats:
            self.last_stats = st.as_dict()
            return st.continuity
        return float("nan")

    def stats(self) -> dict:
        st = StepStats()
        if lib().caffe_dev_stats(self._h, ctypes.byref(st)) != 0:
            raise CaffeError("caffe_dev_stats: " + last_error())
        self.last_stats = st.as_dict()
        return self.last_stats

    def phase(self, name: str, time_step: float | None = None) -> None:
        dt = float(self.spec.dt if time_step is None else time_step)
        rc = lib().caffe_dev_phase(self._h, name.encode(), dt)
        if rc != 0:
            raise CaffeError(f"caffe_dev_phase({name}): " + last_error())

    def synchronize(self) -> None:
        if lib().caffe_dev_synchronize(self._h) != 0:
            raise CaffeError("synchronize: " + last_error())

    @property
    def stream(self) -> int:
        return int(lib().caffe_dev_stream(self._h) or 0)

    # -- field access
    def size_of(self, name: str) -> int:
        n = lib().caffe_dev_array(self._h, name.encode(), None, 0, 0)
        if n < 0:
            raise KeyError(name)
        return int(n)

    def field(self, name: str, planar: bool = False) -> np.ndarray:
        n = self.size_of(name)
        out = np.empty(n, dtype=np.float64)
        self.get_into(name, out, planar)
        return out

    def get_into(self, name: str, out: np.ndarray, planar: bool = False) -> None:
        n = lib().caffe_dev_array(self._h, name.encode(), out.ctypes.data_as(ctypes.c_void_p), out.size, 2 if planar else 0)
        if n < 0:
            raise CaffeError(f"get {name}: " + last_error())

    def set_field(self, name: str, values: np.ndarray, planar: bool = False) -> None:
        v = np.ascontiguousarray(values, dtype=np.float64).ravel()
        n = lib().caffe_dev_array(self._h, name.encode(), v.ctypes.data_as(ctypes.c_void_p), v.size, 3 if planar else 1)
        if n < 0:
            raise CaffeError(f"set {name}: " + last_error())

    def set_from_ptr(self, name: str, ptr: int, count: int, planar: bool = True) -> None:
        """Upload from a raw host pointer (e.g. a pinned buffer)."""
        n = lib().caffe_dev_array(self._h, name.encode(), ctypes.c_void_p(ptr), int(count), 3 if planar else 1)
        if n < 0:
            raise CaffeError(f"set {name}: " + last_error())

    def get_to_ptr(self, name: str, ptr: int, count: int, planar: bool = True) -> None:
        n = lib().caffe_dev_array(self._h, name.encode(), ctypes.c_void_p(ptr), int(count), 2 if planar else 0)
        if n < 0:
            raise CaffeError(f"get {name}: " + last_error())

    # -- restart files (the reference's writeRestart layout; see restart.py)
    def write_restart(self, name: str, path: str | None = None) -> str:
        """Writes cell field ``name`` ("u" or "p") to ``path`` (default <name>Restart.rst)."""
        from .restart import write_restart
        path = path or f"{name}Restart.rst"
        write_restart(path, self.field(name).reshape(self.ncells, -1), self.shape)
        return path

    def read_restart(self, name: str, path: str | None = None) -> None:
        """Sets cell field ``name`` from a restart file (default <name>Restart.rst)."""
        from .restart import read_restart
        comps = self.size_of(name) // self.ncells
        self.set_field(name, read_restart(path or f"{name}Restart.rst", self.shape, comps))


class Simple(DeviceSolver):
    """SIMPLE (src/Solvers/Simple.h:33)."""
    kind = "simple"


class Piso(DeviceSolver):
    """PISO (src/Solvers/Piso.h:6)."""
    kind = "piso"


class IbPiso(DeviceSolver):
    """Ghost-cell immersed-boundary PISO with one sphere (src/Solvers/IbPiso.h:33)."""
    kind = "ibpiso"


def make_solver(nodes: np.ndarray, spec: C.CaseSpec, device: int = 0) -> DeviceSolver:
    return {"simple": Simple, "piso": Piso, "ibpiso": IbPiso}[spec.kind](nodes, spec, device)
