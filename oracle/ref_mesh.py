"""ctypes wrapper of the real-mesh checker ``oracle/_ref/libzref_mesh.so``
(TEST INFRASTRUCTURE ONLY): zephyr's own EuMesh, AMR (refine) and SmFluid
compiled from the reference sources."""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB = Path(__file__).resolve().parent / "_ref" / "libzref_mesh.so"
_P = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int)
_lib = None


def available() -> bool:
    return LIB.exists()


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(str(LIB))
        L.zm_create.restype = C.c_void_p
        L.zm_create.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, _I, C.c_int,
                                C.c_double, C.c_double, C.c_double, C.c_int, C.c_char_p, C.c_int, C.c_double,
                                C.c_int, C.c_char_p]
        L.zm_create_ax.restype = C.c_void_p
        L.zm_create_ax.argtypes = L.zm_create.argtypes + [C.c_int]
        L.zm_axial_geometry.argtypes = [C.c_void_p, _P, _P]
        L.zm_axial_geometry.restype = C.c_int
        L.zm_free.argtypes = [C.c_void_p]
        L.zm_threads.argtypes = [C.c_int]
        L.zm_n_cells.argtypes = [C.c_void_p]
        L.zm_n_cells.restype = C.c_int
        L.zm_cells.argtypes = [C.c_void_p, _P, _P, _P, _P, _I, _I, _I, _I]
        L.zm_faces.argtypes = [C.c_void_p, _I, _I, _P, _P, _P, _P, _P]
        L.zm_faces.restype = C.c_int
        L.zm_verts.argtypes = [C.c_void_p, _P, _P]
        L.zm_set_state.argtypes = [C.c_void_p, _P, _P, _P, _P, _P]
        L.zm_get_state.argtypes = [C.c_void_p, _P, _P, _P, _P, _P]
        L.zm_set_wait.argtypes = [C.c_void_p, _I]
        L.zm_get_wait.argtypes = [C.c_void_p, _I]
        L.zm_set_max_dt.argtypes = [C.c_void_p, C.c_double]
        L.zm_step.argtypes = [C.c_void_p]
        L.zm_step.restype = C.c_double
        L.zm_solver_flags.argtypes = [C.c_void_p, _I]
        L.zm_put_flags.argtypes = [C.c_void_p, _I]
        L.zm_grad.argtypes = [C.c_void_p, _P, _P]
        L.zm_refine.argtypes = [C.c_void_p]
        L.zm_refine.restype = C.c_int
        L.zm_check.argtypes = [C.c_void_p]
        L.zm_check.restype = C.c_int
        L.zm_check_refined.argtypes = [C.c_void_p]
        L.zm_check_refined.restype = C.c_int
        L.zm_vtu.argtypes = [C.c_void_p, C.c_char_p, C.c_char_p, C.c_int]
        L.zm_pvd_open.restype = C.c_void_p
        L.zm_pvd_open.argtypes = [C.c_char_p, C.c_char_p]
        L.zm_pvd_save.argtypes = [C.c_void_p, C.c_void_p, C.c_double, C.c_char_p, C.c_int]
        L.zm_pvd_close.argtypes = [C.c_void_p]
        L.zm_threads(0)
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(_P)


def _ip(a):
    return a.ctypes.data_as(_I)


class RefEuMesh:
    """zephyr's EuMesh(Rectangle) with an SmFluid on it (the reference's code)."""

    def __init__(self, nx, ny, box=(0.0, 1.0, 0.0, 1.0), bounds=(2, 2, 2, 2), eos_kind=0, gamma=1.4, P0=0.0,
                 e0=0.0, flux=3, limiter="MC", accuracy=1, CFL=0.5, max_level=0, distributor="slope", axial=False):
        b = np.ascontiguousarray(bounds, dtype=np.int32)
        self.h = lib().zm_create_ax(nx, ny, *box, _ip(b), eos_kind, gamma, P0, e0, flux, limiter.encode(),
                                    accuracy, CFL, max_level, distributor.encode(), int(bool(axial)))

    def axial_geometry(self):
        """(volume_alt per cell, area_alt per face slot) of an axial mesh."""
        n = self.n
        vol = np.empty(n)
        area = np.empty(8 * n)
        if lib().zm_axial_geometry(self.h, _dp(vol), _dp(area)) != 0:
            raise RuntimeError("not a mesh of 8-slot cells")
        return vol, area

    @property
    def n(self):
        return lib().zm_n_cells(self.h)

    def cells(self):
        n = self.n
        cx, cy, vol, inc = (np.empty(n) for _ in range(4))
        level, flag, b_idx, z_idx = (np.empty(n, np.int32) for _ in range(4))
        lib().zm_cells(self.h, _dp(cx), _dp(cy), _dp(vol), _dp(inc), _ip(level), _ip(flag), _ip(b_idx),
                       _ip(z_idx))
        return dict(cx=cx, cy=cy, vol=vol, inc=inc, level=level, flag=flag, b_idx=b_idx, z_idx=z_idx)

    def faces(self):
        n = self.n
        boundary, neib = np.empty(8 * n, np.int32), np.empty(8 * n, np.int32)
        area, nx, ny, fx, fy = (np.empty(8 * n) for _ in range(5))
        rc = lib().zm_faces(self.h, _ip(boundary), _ip(neib), _dp(area), _dp(nx), _dp(ny), _dp(fx), _dp(fy))
        if rc != 0:
            raise RuntimeError("cells without 8 face slots")
        return dict(boundary=boundary, neib=neib, area=area, nx=nx, ny=ny, fx=fx, fy=fy)

    def verts(self):
        """The 9 map points of every cell (x, y), 9 n each."""
        n = self.n
        vx, vy = np.empty(9 * n), np.empty(9 * n)
        lib().zm_verts(self.h, _dp(vx), _dp(vy))
        return vx, vy

    def mesh_arrays(self):
        g = self.cells()
        g.update(self.faces())
        return g

    def set_state(self, rho, u, v, p, e):
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (rho, u, v, p, e)]
        lib().zm_set_state(self.h, *map(_dp, arrs))

    def state(self):
        out = [np.empty(self.n) for _ in range(5)]
        lib().zm_get_state(self.h, *map(_dp, out))
        return out

    def set_wait(self, w):
        w = np.ascontiguousarray(w, dtype=np.int32)
        lib().zm_set_wait(self.h, _ip(w))

    def wait(self):
        w = np.empty(self.n, np.int32)
        lib().zm_get_wait(self.h, _ip(w))
        return w

    def step(self):
        return lib().zm_step(self.h)

    def solver_flags(self):
        f = np.empty(self.n, np.int32)
        lib().zm_solver_flags(self.h, _ip(f))
        return f

    def put_flags(self, flags):
        f = np.ascontiguousarray(flags, dtype=np.int32)
        lib().zm_put_flags(self.h, _ip(f))

    def refine(self):
        return lib().zm_refine(self.h)

    def check(self):
        return lib().zm_check(self.h)

    def check_refined(self):
        return lib().zm_check_refined(self.h)

    def write_vtu(self, filename, names=("level",), with_state=True):
        """io::VtuFile::save with the named variables and the SmFluid state."""
        lib().zm_vtu(self.h, str(filename).encode(), ",".join(names).encode(), int(with_state))

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.zm_free(self.h)
            self.h = None


def grad_of(mesh: "RefEuMesh"):
    """d_dx, d_dy (density, vx, vy, pressure) as (4, n) arrays."""
    n = mesh.n
    gx, gy = np.empty(4 * n), np.empty(4 * n)
    lib().zm_grad(mesh.h, _dp(gx), _dp(gy))
    return gx.reshape(4, n), gy.reshape(4, n)


class RefPvd:
    """io::PvdFile(filename, directory) saving RefEuMesh instances."""

    def __init__(self, filename, directory):
        self.h = lib().zm_pvd_open(str(filename).encode(), str(directory).encode())

    def save(self, mesh: RefEuMesh, timestep, names=("level",), with_state=True):
        lib().zm_pvd_save(self.h, mesh.h, timestep, ",".join(names).encode(), int(with_state))

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.zm_pvd_close(self.h)
            self.h = None
