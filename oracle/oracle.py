"""ctypes wrapper of the oracle (test infrastructure only).

The oracle is a CPU restatement of zephyr's SmFluid step (``zoracle.cpp``);
tests, the smoke check and the bench's CPU-baseline leg use it as the checker.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from . import build as _build

_lib = None

BC_WALL, BC_ZOE, BC_PERIODIC = 1, 2, 3
FLUX_HLL, FLUX_HLLC = 2, 3
EOS_IDEAL, EOS_STIFFENED = 0, 1
SCHEME_REF, SCHEME_HEUN = 0, 1

_P = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int)


def lib():
    global _lib
    if _lib is None:
        path = _build.build()
        L = C.CDLL(str(path))
        L.zo_mesh_rect.restype = C.c_void_p
        L.zo_mesh_rect.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, _I]
        L.zo_mesh_free.argtypes = [C.c_void_p]
        L.zo_mesh_arrays.restype = C.c_void_p
        L.zo_mesh_arrays.argtypes = [C.c_int, _P, _P, _P, _P, _I, _I, _P, _P, _P, _P, _P]
        L.zo_mesh_ncells.argtypes = [C.c_void_p]
        L.zo_mesh_ncells.restype = C.c_int
        L.zo_mesh_geometry.argtypes = [C.c_void_p, _P, _P, _P, _I, _I, _P, _P, _P, _P, _P]
        L.zo_solver_create.restype = C.c_void_p
        L.zo_solver_create.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_double, C.c_double, C.c_int,
                                       C.c_int, C.c_int, C.c_int, C.c_double, C.c_int]
        L.zo_solver_free.argtypes = [C.c_void_p]
        L.zo_solver_set_max_dt.argtypes = [C.c_void_p, C.c_double]
        L.zo_solver_set_threads.argtypes = [C.c_void_p, C.c_int]
        L.zo_solver_set_state.argtypes = [C.c_void_p, _P, _P, _P, _P, _P]
        L.zo_solver_get_state.argtypes = [C.c_void_p, _P, _P, _P, _P, _P]
        L.zo_solver_get_wait.argtypes = [C.c_void_p, _I]
        L.zo_solver_set_wait.argtypes = [C.c_void_p, _I]
        L.zo_solver_grad.argtypes = [C.c_void_p, _P, _P]
        L.zo_solver_compute_dt.argtypes = [C.c_void_p]
        L.zo_solver_compute_dt.restype = C.c_double
        L.zo_solver_step.argtypes = [C.c_void_p]
        L.zo_solver_step.restype = C.c_double
        L.zo_solver_steps.argtypes = [C.c_void_p, C.c_int, _P]
        L.zo_solver_steps.restype = C.c_double
        L.zo_solver_set_flags.argtypes = [C.c_void_p, _I]
        L.zo_flux.argtypes = [C.c_int, _P, _P, C.c_int, C.c_double, C.c_double, C.c_double, _P]
        L.zo_limiter.argtypes = [C.c_int, C.c_double, C.c_double]
        L.zo_limiter.restype = C.c_double
        L.zo_eos.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double, _P]
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(_P)


def _ip(a):
    return a.ctypes.data_as(_I)


class Mesh:
    """Restated AmrCells(Rectangle) (amr_cells_gen.cpp:128-281)."""

    def __init__(self, nx, ny, x_min=0.0, x_max=1.0, y_min=0.0, y_max=1.0, bounds=(BC_ZOE,) * 4):
        b = np.ascontiguousarray(bounds, dtype=np.int32)
        self.h = lib().zo_mesh_rect(nx, ny, x_min, x_max, y_min, y_max, _ip(b))
        self.nx, self.ny, self.n = nx, ny, nx * ny

    @classmethod
    def from_arrays(cls, g):
        """Mesh given cell by cell: dict with cx, cy, vol, inc (n) and
        boundary, neib, nx, ny, fx, fy, area (8 n)."""
        self = cls.__new__(cls)
        keep = {k: np.ascontiguousarray(g[k], dtype=np.int32 if k in ("boundary", "neib") else np.float64)
                for k in ("cx", "cy", "vol", "inc", "boundary", "neib", "nx", "ny", "fx", "fy", "area")}
        self._keep = keep
        n = keep["cx"].size
        self.h = lib().zo_mesh_arrays(n, _dp(keep["cx"]), _dp(keep["cy"]), _dp(keep["vol"]), _dp(keep["inc"]),
                                      _ip(keep["boundary"]), _ip(keep["neib"]), _dp(keep["nx"]), _dp(keep["ny"]),
                                      _dp(keep["fx"]), _dp(keep["fy"]), _dp(keep["area"]))
        self.nx, self.ny, self.n = 0, 0, n
        return self

    def geometry(self):
        n = self.n
        cx, cy, vol = np.empty(n), np.empty(n), np.empty(n)
        bnd, adj = np.empty(8 * n, np.int32), np.empty(8 * n, np.int32)
        nx, ny, fx, fy, area = (np.empty(8 * n) for _ in range(5))
        lib().zo_mesh_geometry(self.h, _dp(cx), _dp(cy), _dp(vol), _ip(bnd), _ip(adj), _dp(nx), _dp(ny),
                               _dp(fx), _dp(fy), _dp(area))
        return dict(cx=cx, cy=cy, vol=vol, boundary=bnd, adj=adj, nx=nx, ny=ny, fx=fx, fy=fy, area=area)

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.zo_mesh_free(self.h)
            self.h = None


class Solver:
    """Restated SmFluid (sm_fluid.cpp); state as five float64 arrays."""

    def __init__(self, mesh, eos_kind=EOS_IDEAL, gamma=1.4, P0=0.0, e0=0.0, flux=FLUX_HLLC, limiter=3,
                 accuracy=1, scheme=SCHEME_REF, CFL=0.5, threads=1):
        self.mesh = mesh
        self.h = lib().zo_solver_create(mesh.h, eos_kind, gamma, P0, e0, flux, limiter, accuracy, scheme,
                                        CFL, threads)

    def set_max_dt(self, dt):
        lib().zo_solver_set_max_dt(self.h, dt)

    def set_threads(self, n):
        lib().zo_solver_set_threads(self.h, n)

    def set_state(self, rho, u, v, p, e):
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (rho, u, v, p, e)]
        lib().zo_solver_set_state(self.h, *map(_dp, arrs))

    def state(self):
        out = [np.empty(self.mesh.n) for _ in range(5)]
        lib().zo_solver_get_state(self.h, *map(_dp, out))
        return out

    def wait(self):
        w = np.empty(self.mesh.n, np.int32)
        lib().zo_solver_get_wait(self.h, _ip(w))
        return w

    def set_wait(self, w):
        w = np.ascontiguousarray(w, dtype=np.int32)
        lib().zo_solver_set_wait(self.h, _ip(w))

    def grad(self):
        n = self.mesh.n
        gx, gy = np.empty(5 * n), np.empty(5 * n)
        lib().zo_solver_grad(self.h, _dp(gx), _dp(gy))
        return gx.reshape(5, n), gy.reshape(5, n)

    def compute_dt(self):
        return lib().zo_solver_compute_dt(self.h)

    def step(self):
        return lib().zo_solver_step(self.h)

    def steps(self, n):
        dts = np.empty(max(n, 1))
        lib().zo_solver_steps(self.h, n, _dp(dts))
        return dts[:n]

    def set_flags(self):
        f = np.empty(self.mesh.n, np.int32)
        lib().zo_solver_set_flags(self.h, _ip(f))
        return f

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.zo_solver_free(self.h)
            self.h = None


def flux(kind, zL, zR, eos_kind=EOS_IDEAL, gamma=1.4, P0=0.0, e0=0.0):
    zL = np.ascontiguousarray(zL, dtype=np.float64)
    zR = np.ascontiguousarray(zR, dtype=np.float64)
    out = np.empty(5)
    lib().zo_flux(kind, _dp(zL), _dp(zR), eos_kind, gamma, P0, e0, _dp(out))
    return out


def limiter(kind, a, b):
    return lib().zo_limiter(kind, a, b)


def eos(eos_kind, gamma, P0, e0, rho, x):
    out = np.empty(3)
    lib().zo_eos(eos_kind, gamma, P0, e0, rho, x, _dp(out))
    return out
