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
FLUX_HLLC_M, FLUX_HLLC_LM, FLUX_CIR1, FLUX_CIR2 = 4, 5, 6, 7
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
        L.zo_solver_cfl_min.argtypes = [C.c_void_p]
        L.zo_solver_cfl_min.restype = C.c_double
        L.zo_solver_step.argtypes = [C.c_void_p]
        L.zo_solver_step.restype = C.c_double
        L.zo_solver_steps.argtypes = [C.c_void_p, C.c_int, _P]
        L.zo_solver_steps.restype = C.c_double
        L.zo_solver_set_flags.argtypes = [C.c_void_p, _I]
        L.zo_flux.argtypes = [C.c_int, _P, _P, C.c_int, C.c_double, C.c_double, C.c_double, _P]
        L.zo_limiter.argtypes = [C.c_int, C.c_double, C.c_double]
        L.zo_limiter.restype = C.c_double
        L.zo_eos.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double, _P]
        L.zo_mm_material.argtypes = [C.c_char_p, C.c_char_p, _P]
        L.zo_mm_material.restype = C.c_int
        L.zo_mm_create.restype = C.c_void_p
        L.zo_mm_create.argtypes = [C.c_void_p, C.c_int, _P, C.c_double, C.c_int, C.c_int]
        for name in ("zo_mm_free",):
            getattr(L, name).argtypes = [C.c_void_p]
        L.zo_mm_set_max_dt.argtypes = [C.c_void_p, C.c_double]
        L.zo_mm_set_threads.argtypes = [C.c_void_p, C.c_int]
        L.zo_mm_set_split.argtypes = [C.c_void_p, C.c_int]
        L.zo_mm_set_accuracy.argtypes = [C.c_void_p, C.c_int, C.c_int]
        L.zo_mm_make_states.argtypes = [C.c_void_p, _P, _P, _P, _P, _P]
        L.zo_mm_set_states.argtypes = [C.c_void_p, _P]
        L.zo_mm_get_states.argtypes = [C.c_void_p, _P]
        L.zo_mm_step.argtypes = [C.c_void_p]
        L.zo_mm_step.restype = C.c_double
        L.zo_mm_steps.argtypes = [C.c_void_p, C.c_int, _P]
        L.zo_mm_steps.restype = C.c_double
        L.zo_mm_compute_dt.argtypes = [C.c_void_p]
        L.zo_mm_compute_dt.restype = C.c_double
        L.zo_mm_bad.argtypes = [C.c_void_p]
        L.zo_mm_bad.restype = C.c_int
        L.zo_mm_interface.argtypes = [C.c_void_p, _P, _P]
        L.zo_mm_flags.argtypes = [C.c_void_p, _I]
        L.zo_mm_state_from_q.argtypes = [C.c_void_p, _P, _P, _P]
        L.zo_mm_sound_speed.argtypes = [C.c_void_p, _P]
        L.zo_mm_sound_speed.restype = C.c_double
        L.zo_mm_hllc.argtypes = [C.c_void_p, _P, _P, _P]
        L.zo_mm_hllc.restype = C.c_int
        L.zo_mm_crp_flux.argtypes = [C.c_void_p, _P, _P, C.c_double, C.c_double, C.c_int, C.c_double, C.c_double, _P]
        L.zo_mm_crp_flux.restype = C.c_int
        for name, nargs in (("zo_mm_face_fraction", 2), ("zo_mm_quad_find_section", 5),
                            ("zo_mm_quad_volume_fraction", 5), ("zo_mm_average_flux", 3)):
            getattr(L, name).argtypes = [C.c_double] * nargs
            getattr(L, name).restype = C.c_double
        L.zo_tr_create.restype = C.c_void_p
        L.zo_tr_create.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_int, _P]
        L.zo_tr_free.argtypes = [C.c_void_p]
        L.zo_tr_set_u.argtypes = [C.c_void_p, _P]
        L.zo_tr_update_interface.argtypes = [C.c_void_p, C.c_int]
        L.zo_tr_compute_dt.argtypes = [C.c_void_p]
        L.zo_tr_compute_dt.restype = C.c_double
        L.zo_tr_set_dt.argtypes = [C.c_void_p, C.c_double]
        L.zo_tr_update.argtypes = [C.c_void_p, C.c_int]
        L.zo_tr_get.argtypes = [C.c_void_p, _P, _P, _P]
        L.zo_tr_flags.argtypes = [C.c_void_p, _I]
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

    def cfl_min(self):
        """min over cells of incircle / (|v| + c), before CFL and max_dt."""
        return lib().zo_solver_cfl_min(self.h)

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


# ---------------------------------------------------------------------------
# Multi-material step (zoracle_mm.inc): restated MmFluid, first order.
CRP_NONE, CRP_V3, CRP_V5, CRP_VS, CRP_PLIC = 0, 1, 2, 3, 4
MM_NSTATE = 14  # density, vx, vy, P, e, T, beta[4], rhos[4]


def mm_material(kind, name):
    """(stiffened, gamma, P0, e0, Cv, T0, rho_ref) of IdealGas(name) /
    StiffenedGas(name)."""
    out = np.empty(7)
    if lib().zo_mm_material(kind.encode(), name.encode(), _dp(out)) != 0:
        raise ValueError(f"unknown material {kind}:{name}")
    return out


class MmSolver:
    """Restated MmFluid (mm_fluid.cpp) on an oracle Mesh."""

    def __init__(self, mesh, materials=(("stiffened", "Water"), ("ideal", "Air")), CFL=0.4, crp_mode=CRP_PLIC,
                 threads=1):
        self.mesh = mesh
        self.nmat = len(materials)
        mats = np.concatenate([mm_material(k, n) for k, n in materials])
        self._mats = mats
        self.h = lib().zo_mm_create(mesh.h, self.nmat, _dp(mats), CFL, crp_mode, threads)

    def make_states(self, rho, vx, vy, p, beta):
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (rho, vx, vy, p)]
        b = np.zeros((self.mesh.n, 4))
        b[:, :np.asarray(beta).shape[1]] = beta
        lib().zo_mm_make_states(self.h, *map(_dp, arrs), _dp(np.ascontiguousarray(b)))

    def set_states(self, s):
        s = np.ascontiguousarray(s, dtype=np.float64).reshape(self.mesh.n, MM_NSTATE)
        lib().zo_mm_set_states(self.h, _dp(s))

    def states(self):
        s = np.empty((self.mesh.n, MM_NSTATE))
        lib().zo_mm_get_states(self.h, _dp(s))
        return s

    def set_max_dt(self, dt):
        lib().zo_mm_set_max_dt(self.h, dt)

    def set_threads(self, n):
        lib().zo_mm_set_threads(self.h, n)

    def set_accuracy(self, acc, limiter=3):
        """MmFluid::set_accuracy (mm_fluid.cpp:46-48) and the limiter (default MC)."""
        lib().zo_mm_set_accuracy(self.h, int(acc), int(limiter))

    def set_splitting(self, split):
        """DirSplit: 0 NONE, 1 SIMPLE, 2 STRANG (mm_fluid.cpp:112-137)."""
        lib().zo_mm_set_split(self.h, int(split))

    def step(self):
        return lib().zo_mm_step(self.h)

    def steps(self, n):
        dts = np.empty(max(n, 1))
        lib().zo_mm_steps(self.h, n, _dp(dts))
        return dts[:n]

    def compute_dt(self):
        return lib().zo_mm_compute_dt(self.h)

    def bad(self):
        return bool(lib().zo_mm_bad(self.h))

    def interface(self):
        nrm = np.empty((self.mesh.n, self.nmat, 2))
        off = np.empty((self.mesh.n, self.nmat))
        lib().zo_mm_interface(self.h, _dp(nrm), _dp(off))
        return nrm, off

    def flags(self):
        f = np.empty(self.mesh.n, np.int32)
        lib().zo_mm_flags(self.h, _ip(f))
        return f

    def state_from_q(self, q, guess):
        out = np.empty(MM_NSTATE)
        lib().zo_mm_state_from_q(self.h, _dp(np.ascontiguousarray(q, float)),
                                 _dp(np.ascontiguousarray(guess, float)), _dp(out))
        return out

    def sound_speed(self, s):
        return lib().zo_mm_sound_speed(self.h, _dp(np.ascontiguousarray(s, float)))

    def hllc(self, sl, sr):
        out = np.empty(8)
        lib().zo_mm_hllc(self.h, _dp(np.ascontiguousarray(sl, float)), _dp(np.ascontiguousarray(sr, float)), _dp(out))
        return out

    def crp_flux(self, sl, sr, hL, hR, iA, a_sig, dt):
        out = np.empty(8)
        lib().zo_mm_crp_flux(self.h, _dp(np.ascontiguousarray(sl, float)), _dp(np.ascontiguousarray(sr, float)),
                             hL, hR, iA, a_sig, dt, _dp(out))
        return out

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.zo_mm_free(self.h)
            self.h = None


def mm_face_fraction(a1, a2):
    return lib().zo_mm_face_fraction(a1, a2)


def mm_quad_find_section(alpha, nx, ny, A, B):
    return lib().zo_mm_quad_find_section(alpha, nx, ny, A, B)


def mm_quad_volume_fraction(p, nx, ny, A, B):
    return lib().zo_mm_quad_volume_fraction(p, nx, ny, A, B)


def mm_average_flux(alpha, cos, CFL):
    return lib().zo_mm_average_flux(alpha, cos, CFL)


# Transfer::Method values (transfer.h:25-51) that the restatement covers
TR_METHODS = {"CRP_V3": 0, "CRP_V5": 1, "CRP_SE": 2, "CRP_N1": 3, "CRP_N2": 4, "VOF": 5, "VOF_CRP": 6,
              "MUSCLd": 7, "MUSCLn": 8, "MUSCLd_CRP": 9, "MUSCLn_CRP": 10, "MUSCL_MC": 11, "MUSCL_MC_CRP": 12,
              "WENO": 13, "WENO_CRP": 14}


class TrSolver:
    """Restated Transfer (transfer.cpp) on an oracle Mesh; ``vel`` is
    ``("translation", vx, vy)`` or ``("rotation", cx, cy, omega)``."""

    def __init__(self, mesh, method="VOF", CFL=0.5, vel=("translation", 0.7, -0.35)):
        self.mesh = mesh
        kind = 0 if vel[0] == "translation" else 1
        v = np.ascontiguousarray(list(vel[1:]) + [0.0] * (3 - len(vel[1:])), dtype=np.float64)
        self.h = lib().zo_tr_create(mesh.h, TR_METHODS[method], CFL, kind, _dp(v))

    def set_u(self, u):
        lib().zo_tr_set_u(self.h, _dp(np.ascontiguousarray(u, dtype=np.float64)))

    def update_interface(self, smoothing=3):
        lib().zo_tr_update_interface(self.h, smoothing)

    def compute_dt(self):
        return lib().zo_tr_compute_dt(self.h)

    def set_dt(self, dt):
        lib().zo_tr_set_dt(self.h, dt)

    def update(self, direction=0):
        lib().zo_tr_update(self.h, direction)

    def get(self):
        n = self.mesh.n
        u, nrm, pt = np.empty(n), np.empty((n, 2)), np.empty((n, 2))
        lib().zo_tr_get(self.h, _dp(u), _dp(nrm), _dp(pt))
        return u, nrm, pt

    def flags(self):
        f = np.empty(self.mesh.n, np.int32)
        lib().zo_tr_flags(self.h, _ip(f))
        return f

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.zo_tr_free(self.h)
