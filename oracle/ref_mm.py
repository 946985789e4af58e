"""ctypes wrapper of the reference's MmFluid built from its sources
(``oracle/_ref/libzref_mesh.so``, driver ``ref_mm_driver.cpp``).  TEST
INFRASTRUCTURE ONLY: used to pin the oracle's multi-material restatement and
to write golden fixtures; needs the reference tree at build time."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import ref_build

_P = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int)
_lib = None

NSTATE = 14  # density, vx, vy, P, e, T, beta[4], rhos[4]


def available() -> bool:
    return ref_build.LIB_MESH.exists()


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(str(ref_build.LIB_MESH))
        L.zmm_create.restype = C.c_void_p
        L.zmm_create.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, _I, C.c_char_p,
                                 C.c_double, C.c_int, C.c_int]
        L.zmm_free.argtypes = [C.c_void_p]
        L.zmm_set_split.argtypes = [C.c_void_p, C.c_int]
        L.zmm_set_limiter.argtypes = [C.c_void_p, C.c_char_p]
        L.zm_threads.argtypes = [C.c_int]
        L.zmm_n_cells.argtypes = [C.c_void_p]
        L.zmm_n_cells.restype = C.c_int
        L.zmm_make_states.argtypes = [C.c_void_p, _P, _P, _P, _P, _P]
        L.zmm_set_states.argtypes = [C.c_void_p, _P]
        L.zmm_get_states.argtypes = [C.c_void_p, _P]
        L.zmm_step.argtypes = [C.c_void_p]
        L.zmm_step.restype = C.c_double
        L.zmm_compute_dt.argtypes = [C.c_void_p]
        L.zmm_compute_dt.restype = C.c_double
        L.zmm_interface.argtypes = [C.c_void_p, _P, _P]
        L.zmm_fractions_grad.argtypes = [C.c_void_p, _P]
        L.zmm_flags.argtypes = [C.c_void_p, _I]
        L.zmm_state_from_q.argtypes = [C.c_void_p, _P, _P, _P]
        L.zmm_sound_speed.argtypes = [C.c_void_p, _P]
        L.zmm_sound_speed.restype = C.c_double
        L.zmm_hllc.argtypes = [C.c_void_p, _P, _P, _P]
        L.zmm_crp_flux.argtypes = [C.c_void_p, _P, _P, C.c_double, C.c_double, C.c_int, C.c_double, C.c_double, _P]
        for name, nargs in (("zmm_face_fraction", 2), ("zmm_quad_find_section", 5),
                            ("zmm_quad_volume_fraction", 5), ("zmm_average_flux", 3)):
            fn = getattr(L, name)
            fn.argtypes = [C.c_double] * nargs
            fn.restype = C.c_double
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(_P)


class RefMmFluid:
    """The reference's MmFluid on Rectangle(box) with nx by ny cells.
    materials: e.g. "stiffened:Water,ideal:Air"; crp_mode: 0 plain HLLC,
    4 CRP with PLIC (the reference's CrpMode values)."""

    def __init__(self, nx, ny, box=(0.0, 1.0, 0.0, 1.0), bounds=(2, 2, 2, 2), materials="stiffened:Water,ideal:Air",
                 CFL=0.4, accuracy=1, crp_mode=4):
        b = np.ascontiguousarray(bounds, dtype=np.int32)
        self.h = lib().zmm_create(nx, ny, *box, b.ctypes.data_as(_I), materials.encode(), CFL, accuracy, crp_mode)
        self.n = lib().zmm_n_cells(self.h)
        self.nmat = materials.count(",") + 1

    def set_limiter(self, name):
        lib().zmm_set_limiter(self.h, name.encode())

    def set_splitting(self, split):
        """MmFluid::set_splitting: 0 NONE, 1 SIMPLE, 2 STRANG."""
        lib().zmm_set_split(self.h, int(split))

    def set_threads(self, n):
        """Worker threads of the reference's threads::for_each (0 or 1: off)."""
        lib().zm_threads(n)

    def make_states(self, rho, vx, vy, P, beta):
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (rho, vx, vy, P)]
        b = np.zeros((self.n, 4))
        b[:, :np.asarray(beta).shape[1]] = beta
        lib().zmm_make_states(self.h, *map(_dp, arrs), _dp(np.ascontiguousarray(b)))

    def set_states(self, s):
        s = np.ascontiguousarray(s, dtype=np.float64).reshape(self.n, NSTATE)
        lib().zmm_set_states(self.h, _dp(s))

    def states(self):
        s = np.empty((self.n, NSTATE))
        lib().zmm_get_states(self.h, _dp(s))
        return s

    def step(self):
        return lib().zmm_step(self.h)

    def compute_dt(self):
        return lib().zmm_compute_dt(self.h)

    def interface(self):
        nrm = np.empty((self.n, self.nmat, 2))
        off = np.empty((self.n, self.nmat))
        lib().zmm_interface(self.h, _dp(nrm), _dp(off))
        return nrm, off

    def fractions_grad(self):
        """MmFluid::fractions_grad of the current state: (n, nmat, 2)."""
        g = np.empty((self.n, self.nmat, 2))
        lib().zmm_fractions_grad(self.h, _dp(g))
        return g

    def flags(self):
        f = np.empty(self.n, np.int32)
        lib().zmm_flags(self.h, f.ctypes.data_as(_I))
        return f

    def state_from_q(self, q, guess):
        out = np.empty(NSTATE)
        lib().zmm_state_from_q(self.h, _dp(np.ascontiguousarray(q, float)), _dp(np.ascontiguousarray(guess, float)),
                               _dp(out))
        return out

    def sound_speed(self, s):
        return lib().zmm_sound_speed(self.h, _dp(np.ascontiguousarray(s, float)))

    def hllc(self, sl, sr):
        out = np.empty(8)
        lib().zmm_hllc(self.h, _dp(np.ascontiguousarray(sl, float)), _dp(np.ascontiguousarray(sr, float)), _dp(out))
        return out

    def crp_flux(self, sl, sr, hL, hR, iA, a_sig, dt):
        out = np.empty(8)
        lib().zmm_crp_flux(self.h, _dp(np.ascontiguousarray(sl, float)), _dp(np.ascontiguousarray(sr, float)), hL, hR,
                           iA, a_sig, dt, _dp(out))
        return out

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.zmm_free(self.h)
            self.h = None


def face_fraction(a1, a2):
    return lib().zmm_face_fraction(a1, a2)


def quad_find_section(alpha, nx, ny, A, B):
    return lib().zmm_quad_find_section(alpha, nx, ny, A, B)


def quad_volume_fraction(p, nx, ny, A, B):
    return lib().zmm_quad_volume_fraction(p, nx, ny, A, B)


def average_flux(alpha, cos, CFL):
    return lib().zmm_average_flux(alpha, cos, CFL)
