"""ctypes wrapper of the reference-source checker ``oracle/_ref/libzref.so``
(TEST INFRASTRUCTURE ONLY): the reference's own SmFluid, fluxes, limiters and
EoS compiled from its sources, run on a stand-in mesh.  Used to pin the
oracle and to generate the golden fixtures under tests/golden.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB = Path(__file__).resolve().parent / "_ref" / "libzref.so"
_P = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int)
_lib = None


def available() -> bool:
    return LIB.exists()


def lib():
    global _lib
    if _lib is None:
        if not LIB.exists():
            from . import ref_build
            ref_build.build()
        L = C.CDLL(str(LIB))
        L.zr_create.restype = C.c_void_p
        L.zr_create.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, _I, C.c_int,
                                C.c_double, C.c_double, C.c_double, C.c_int, C.c_char_p, C.c_int, C.c_double]
        L.zr_free.argtypes = [C.c_void_p]
        L.zr_set_max_dt.argtypes = [C.c_void_p, C.c_double]
        L.zr_set_state.argtypes = [C.c_void_p, _P, _P, _P, _P, _P]
        L.zr_get_state.argtypes = [C.c_void_p, _P, _P, _P, _P, _P]
        L.zr_set_wait.argtypes = [C.c_void_p, _I]
        L.zr_get_wait.argtypes = [C.c_void_p, _I]
        L.zr_set_threads.argtypes = [C.c_void_p, C.c_int]
        L.zr_steps.argtypes = [C.c_void_p, C.c_int]
        L.zr_steps.restype = C.c_double
        L.zr_step.argtypes = [C.c_void_p]
        L.zr_step.restype = C.c_double
        L.zr_set_flags.argtypes = [C.c_void_p, _I]
        L.zr_grad.argtypes = [C.c_void_p, _P, _P]
        L.zr_flux.argtypes = [C.c_int, _P, _P, C.c_int, C.c_double, C.c_double, C.c_double, _P]
        L.zr_limiter.argtypes = [C.c_char_p, C.c_double, C.c_double]
        L.zr_limiter.restype = C.c_double
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(_P)


class RefSolver:
    """zephyr's SmFluid on a Rectangle(nx, ny) mesh (the reference's code)."""

    def __init__(self, nx, ny, box=(0.0, 1.0, 0.0, 1.0), bounds=(2, 2, 2, 2), eos_kind=0, gamma=1.4, P0=0.0,
                 e0=0.0, flux=3, limiter="MC", accuracy=1, CFL=0.5):
        b = np.ascontiguousarray(bounds, dtype=np.int32)
        self.n = nx * ny
        self.h = lib().zr_create(nx, ny, *box, b.ctypes.data_as(_I), eos_kind, gamma, P0, e0, flux,
                                 limiter.encode(), accuracy, CFL)

    def set_max_dt(self, dt):
        lib().zr_set_max_dt(self.h, dt)

    def set_state(self, rho, u, v, p, e):
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (rho, u, v, p, e)]
        lib().zr_set_state(self.h, *map(_dp, arrs))

    def state(self):
        out = [np.empty(self.n) for _ in range(5)]
        lib().zr_get_state(self.h, *map(_dp, out))
        return out

    def set_wait(self, w):
        w = np.ascontiguousarray(w, dtype=np.int32)
        lib().zr_set_wait(self.h, w.ctypes.data_as(_I))

    def wait(self):
        w = np.empty(self.n, np.int32)
        lib().zr_get_wait(self.h, w.ctypes.data_as(_I))
        return w

    def set_threads(self, n):
        """Worker threads of the mesh loops (the reference's threads::on(n))."""
        lib().zr_set_threads(self.h, n)

    def step(self):
        return lib().zr_step(self.h)

    def steps(self, n):
        return lib().zr_steps(self.h, n)

    def set_flags(self):
        f = np.empty(self.n, np.int32)
        lib().zr_set_flags(self.h, f.ctypes.data_as(_I))
        return f

    def grad(self):
        gx, gy = np.empty(5 * self.n), np.empty(5 * self.n)
        lib().zr_grad(self.h, _dp(gx), _dp(gy))
        return gx.reshape(5, self.n), gy.reshape(5, self.n)

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.zr_free(self.h)
            self.h = None


def flux(kind, zL, zR, eos_kind=0, gamma=1.4, P0=0.0, e0=0.0):
    zL = np.ascontiguousarray(zL, dtype=np.float64)
    zR = np.ascontiguousarray(zR, dtype=np.float64)
    out = np.empty(5)
    lib().zr_flux(kind, _dp(zL), _dp(zR), eos_kind, gamma, P0, e0, _dp(out))
    return out


def limiter(name, a, b):
    return lib().zr_limiter(name.encode(), a, b)
