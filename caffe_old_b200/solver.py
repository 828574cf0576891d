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


DIFFUSION_BC = {"fixed": 0, "zeroGradient": 1, "empty": 2}


class Diffusion:
    """The reference's Diffusion solver (src/Solvers/Diffusion.cpp) on the device: unit
    diffusivity, boundary types fixed / zeroGradient / empty per face (east, west, north, south,
    top, bottom) with their reference values, a uniform initial phi.  ``solve(dt)`` assembles and
    solves one linear system and returns ||A x - b||_inf, as Diffusion::solve does."""

    def __init__(self, nodes: np.ndarray, bc_types, bc_values, time_accurate: bool = False, phi0: float = 0.0,
                 method: str = "bicgstab_jacobi", rtol: float = 1e-8, maxit: int = 10000, device: int = 0):
        from . import _lib
        L = _lib.lib()
        nodes = np.ascontiguousarray(nodes, dtype=np.float64)
        nK1, nJ1, nI1, _ = nodes.shape
        self.shape = (nI1 - 1, nJ1 - 1, nK1 - 1)
        self.ncells = int(np.prod(self.shape))
        types = np.array([DIFFUSION_BC[t] for t in bc_types], dtype=np.int32)
        refs = np.ascontiguousarray(bc_values, dtype=np.float64)
        if types.size != 6 or refs.size != 6:
            raise ValueError("six boundary types and values (east, west, north, south, top, bottom)")
        h = ctypes.c_void_p()
        rc = L.caffe_diffusion_create(nodes.ctypes.data_as(ctypes.c_void_p), nI1, nJ1, nK1, types.ctypes.data_as(ctypes.c_void_p),
                                      refs.ctypes.data_as(ctypes.c_void_p), 1 if time_accurate else 0, float(phi0),
                                      C.KSP_METHODS[method], float(rtol), int(maxit), int(device), ctypes.byref(h))
        if rc != 0:
            raise _lib.CaffeError("caffe_diffusion_create: " + _lib.last_error())
        self._h = h.value
        self.iters, self.rel_res = 0, 0.0

    def close(self):
        from . import _lib
        if getattr(self, "_h", None):
            _lib.lib().caffe_diffusion_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def solve(self, dt: float = 1.0) -> float:
        from . import _lib
        r, it, rr = ctypes.c_double(0.0), ctypes.c_int(0), ctypes.c_double(0.0)
        if _lib.lib().caffe_diffusion_solve(self._h, float(dt), ctypes.byref(r), ctypes.byref(it), ctypes.byref(rr)) != 0:
            raise _lib.CaffeError("caffe_diffusion_solve: " + _lib.last_error())
        self.iters, self.rel_res = it.value, rr.value
        return r.value

    def phase(self, name: str, dt: float = 1.0) -> None:
        from . import _lib
        if _lib.lib().caffe_diffusion_phase(self._h, name.encode(), float(dt)) != 0:
            raise _lib.CaffeError(f"caffe_diffusion_phase {name}: " + _lib.last_error())

    def get(self, name: str) -> np.ndarray:
        from . import _lib
        L = _lib.lib()
        n = L.caffe_diffusion_array(self._h, name.encode(), None, 0, 0)
        if n < 0:
            raise KeyError(name)
        out = np.zeros(n, dtype=np.float64)
        if L.caffe_diffusion_array(self._h, name.encode(), out.ctypes.data_as(ctypes.c_void_p), n, 0) < 0:
            raise _lib.CaffeError(_lib.last_error())
        return out

    def set(self, name: str, values: np.ndarray) -> None:
        from . import _lib
        v = np.ascontiguousarray(values, dtype=np.float64).ravel()
        if _lib.lib().caffe_diffusion_array(self._h, name.encode(), v.ctypes.data_as(ctypes.c_void_p), v.size, 1) < 0:
            raise _lib.CaffeError(_lib.last_error())


class Coupled:
    """The reference's Coupled solver (src/Solvers/Coupled.cpp) on the device: momentum and
    continuity assembled into one block system of 4 N unknowns (u_x, u_y, u_z, p) and solved
    together, then the Rhie-Chow face fluxes.  The case is a CaseSpec (boundary conditions, rho,
    mu, omega_u, time_accurate / n_inner, mom_method / mom_rtol / mom_atol / maxit).
    ``solve(dt)`` is Coupled::solve and returns the continuity error."""

    def __init__(self, nodes: np.ndarray, spec: C.CaseSpec, device: int = 0):
        from . import _lib
        L = _lib.lib()
        nodes = np.ascontiguousarray(nodes, dtype=np.float64)
        nK1, nJ1, nI1, _ = nodes.shape
        self.shape = (nI1 - 1, nJ1 - 1, nK1 - 1)
        self.ncells = int(np.prod(self.shape))
        self.spec = spec
        self._case = _lib.make_case(spec)
        h = ctypes.c_void_p()
        if L.caffe_coupled_create(nodes.ctypes.data_as(ctypes.c_void_p), nI1, nJ1, nK1, ctypes.byref(self._case), int(device),
                                  ctypes.byref(h)) != 0:
            raise _lib.CaffeError("caffe_coupled_create: " + _lib.last_error())
        self._h = h.value

    def close(self):
        from . import _lib
        if getattr(self, "_h", None):
            _lib.lib().caffe_coupled_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def solve(self, dt: float | None = None) -> float:
        from . import _lib
        r = ctypes.c_double(0.0)
        if _lib.lib().caffe_coupled_solve(self._h, float(self.spec.dt if dt is None else dt), ctypes.byref(r)) != 0:
            raise _lib.CaffeError("caffe_coupled_solve: " + _lib.last_error())
        return r.value

    def phase(self, name: str, dt: float | None = None) -> None:
        from . import _lib
        if _lib.lib().caffe_coupled_phase(self._h, name.encode(), float(self.spec.dt if dt is None else dt)) != 0:
            raise _lib.CaffeError(f"caffe_coupled_phase {name}: " + _lib.last_error())

    def stats(self) -> dict:
        from . import _lib
        it, rr, st = ctypes.c_int(0), ctypes.c_double(0.0), ctypes.c_int(0)
        _lib.lib().caffe_coupled_stats(self._h, ctypes.byref(it), ctypes.byref(rr), ctypes.byref(st))
        return {"iters": it.value, "rel_res": rr.value, "status": st.value}

    def system(self):
        """The block matrix in compressed rows: (row_ptr, col, val)."""
        from . import _lib
        L = _lib.lib()
        nnz = L.caffe_coupled_system(self._h, None, None, None)
        ptr = np.zeros(4 * self.ncells + 1, dtype=np.int32)
        col = np.zeros(nnz, dtype=np.int32)
        val = np.zeros(nnz, dtype=np.float64)
        if L.caffe_coupled_system(self._h, ptr.ctypes.data_as(ctypes.c_void_p), col.ctypes.data_as(ctypes.c_void_p),
                                  val.ctypes.data_as(ctypes.c_void_p)) < 0:
            raise _lib.CaffeError(_lib.last_error())
        return ptr, col, val

    def get(self, name: str) -> np.ndarray:
        from . import _lib
        L = _lib.lib()
        n = L.caffe_coupled_array(self._h, name.encode(), None, 0, 0)
        if n < 0:
            raise KeyError(name)
        out = np.zeros(n, dtype=np.float64)
        if L.caffe_coupled_array(self._h, name.encode(), out.ctypes.data_as(ctypes.c_void_p), n, 0) < 0:
            raise _lib.CaffeError(_lib.last_error())
        return out

    def set(self, name: str, values: np.ndarray) -> None:
        from . import _lib
        v = np.ascontiguousarray(values, dtype=np.float64).ravel()
        if _lib.lib().caffe_coupled_array(self._h, name.encode(), v.ctypes.data_as(ctypes.c_void_p), v.size, 1) < 0:
            raise _lib.CaffeError(_lib.last_error())
