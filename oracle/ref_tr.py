"""ctypes wrapper of the reference's Transfer solver built from its sources
(``oracle/_ref/libzref_mesh.so``, driver ``ref_tr_driver.cpp``).  TEST
INFRASTRUCTURE ONLY: used to pin the oracle's VOF transport restatement and to
write golden fixtures; needs the reference tree at build time."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import ref_build

_P = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int)
_lib = None

# Transfer::Method (transfer.h:25-51)
METHODS = ["CRP_V3", "CRP_V5", "CRP_SE", "CRP_N1", "CRP_N2", "VOF", "VOF_CRP", "MUSCLd", "MUSCLn",
           "MUSCLd_CRP", "MUSCLn_CRP", "MUSCL_MC", "MUSCL_MC_CRP", "WENO", "WENO_CRP"]


def available() -> bool:
    return ref_build.LIB_MESH.exists()


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(str(ref_build.LIB_MESH))
        L.ztr_create.restype = C.c_void_p
        L.ztr_create.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, _I, C.c_int,
                                 C.c_double, C.c_int, _P]
        L.ztr_free.argtypes = [C.c_void_p]
        L.ztr_n_cells.argtypes = [C.c_void_p]
        L.ztr_n_cells.restype = C.c_int
        L.ztr_disk.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_double, _P]
        L.ztr_set_u.argtypes = [C.c_void_p, _P]
        L.ztr_update_interface.argtypes = [C.c_void_p, C.c_int]
        L.ztr_compute_dt.argtypes = [C.c_void_p]
        L.ztr_compute_dt.restype = C.c_double
        L.ztr_set_dt.argtypes = [C.c_void_p, C.c_double]
        L.ztr_update.argtypes = [C.c_void_p, C.c_int]
        L.ztr_get.argtypes = [C.c_void_p, _P, _P, _P]
        L.ztr_flags.argtypes = [C.c_void_p, _I]
        L.zm_threads(0)
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(_P)


class RefTransfer:
    """The reference's Transfer with the transfer problem's velocity field:
    ``vel=("translation", vx, vy)`` or ``vel=("rotation", cx, cy, omega)``."""

    def __init__(self, nx, ny, box=(0.0, 1.0, 0.0, 1.0), bounds=(2, 2, 2, 2), method="VOF", CFL=0.5,
                 vel=("translation", 0.7, -0.35)):
        b = np.ascontiguousarray(bounds, dtype=np.int32)
        kind = 0 if vel[0] == "translation" else 1
        v = np.ascontiguousarray(list(vel[1:]) + [0.0] * (3 - len(vel[1:])), dtype=np.float64)
        self.h = lib().ztr_create(nx, ny, *box, b.ctypes.data_as(_I), METHODS.index(method), CFL, kind, _dp(v))
        self.n = lib().ztr_n_cells(self.h)

    def __del__(self):
        if getattr(self, "h", None):
            lib().ztr_free(self.h)
            self.h = None

    def disk(self, cx, cy, R):
        u = np.empty(self.n)
        lib().ztr_disk(self.h, cx, cy, R, _dp(u))
        return u

    def set_u(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        lib().ztr_set_u(self.h, _dp(u))

    def update_interface(self, smoothing=3):
        lib().ztr_update_interface(self.h, smoothing)

    def compute_dt(self):
        return lib().ztr_compute_dt(self.h)

    def set_dt(self, dt):
        lib().ztr_set_dt(self.h, dt)

    def update(self, direction=0):
        lib().ztr_update(self.h, direction)

    def get(self):
        u = np.empty(self.n)
        nrm = np.empty((self.n, 2))
        pt = np.empty((self.n, 2))
        lib().ztr_get(self.h, _dp(u), _dp(nrm), _dp(pt))
        return u, nrm, pt

    def flags(self):
        f = np.empty(self.n, dtype=np.int32)
        lib().ztr_flags(self.h, f.ctypes.data_as(_I))
        return f
