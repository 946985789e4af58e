"""Python mirror of zephyr's scalar VOF transport solver Transfer
(math/solver/transfer.h:21-150) on top of the C ABI (``zg_tr_*``).

    solver = Transfer()                        # Transfer(): VOF, CFL 0.5
    solver.set_velocity_rotation(0.5, 0.5, math.pi)  # the Solver::velocity override
    solver.set_method(Method.VOF)
    solver.add_types(mesh)                     # mesh: smf.EuMesh of a non-periodic Rectangle
    solver.set_u1(mesh, u0)                    # cell[data.u1] = ...
    solver.update_interface(mesh)
    dt = solver.compute_dt(mesh); solver.set_dt(dt)
    solver.update(mesh, Direction.X); solver.update(mesh, Direction.Y)

The velocity field, which the reference sets by overriding the virtual
Transfer::velocity, is one of the transfer problem's fields
(problems/transfer.cpp:367-380): a translation or a rotation about z.
There is no CPU fallback: the calls go to the CUDA library.
"""
from __future__ import annotations

import ctypes as C
import enum

import numpy as np

from ._lib import TrParams, ZgError, check, load
from .smf import EuMesh

_P = C.POINTER(C.c_double)


class Method(enum.IntEnum):
    """Transfer::Method (transfer.h:25-51)."""
    CRP_V3 = 0
    CRP_V5 = 1
    CRP_SE = 2
    CRP_N1 = 3
    CRP_N2 = 4
    VOF = 5
    VOF_CRP = 6
    MUSCLd = 7
    MUSCLn = 8
    MUSCLd_CRP = 9
    MUSCLn_CRP = 10
    MUSCL_MC = 11
    MUSCL_MC_CRP = 12
    WENO = 13
    WENO_CRP = 14


class Direction(enum.IntEnum):
    """mesh::Direction (amr_faces.h:75-80)"""
    ANY = 0
    X = 1
    Y = 2


TRANSLATION, ROTATION = 0, 1


class Transfer:
    """Transfer() with its setters; u1, n and p live on the mesh's device
    context after add_types."""

    def __init__(self):
        self._lib = load()
        self.p = TrParams()
        self._lib.zg_tr_default_params(C.byref(self.p))  # transfer.cpp:44-49
        self.mesh = None

    def _push(self):
        if self.mesh is not None:
            check(self.mesh.ctx, self._lib.zg_tr_configure(self.mesh.ctx, C.byref(self.p)))

    def add_types(self, mesh: EuMesh):  # transfer.cpp:51-61
        self.mesh = mesh
        self._push()
        return self

    def CFL(self) -> float:
        return self.p.CFL

    def set_CFL(self, C_: float):  # transfer.cpp:65-67
        self.p.CFL = max(0.0, min(C_, 1.0))
        self._push()

    def method(self) -> Method:
        return Method(self.p.method)

    def set_method(self, method: Method):  # transfer.cpp:73-75
        self.p.method = int(method)
        self._push()

    def set_velocity_translation(self, vx: float, vy: float):
        self.p.velocity = TRANSLATION
        self.p.vel[:] = [vx, vy, 0.0]
        self._push()

    def set_velocity_rotation(self, cx: float, cy: float, omega: float):
        self.p.velocity = ROTATION
        self.p.vel[:] = [cx, cy, omega]
        self._push()

    def _require(self, mesh):
        if mesh is not self.mesh:
            raise ZgError(-3, "call add_types(mesh) first")

    def set_u1(self, mesh: EuMesh, u1):
        """u1 of every cell (u2 = 0)."""
        self._require(mesh)
        u = np.ascontiguousarray(u1, dtype=np.float64)
        if u.size != mesh.n_cells():
            raise ValueError("one value per cell")
        check(mesh.ctx, self._lib.zg_tr_upload(mesh.ctx, u.ctypes.data_as(_P)))

    def u1(self, mesh: EuMesh):
        self._require(mesh)
        u = np.empty(mesh.n_cells())
        check(mesh.ctx, self._lib.zg_tr_download(mesh.ctx, u.ctypes.data_as(_P), None, None))
        return u

    def interface(self, mesh: EuMesh):
        """(u1, n, p): the volume fraction, interface normals (n, 2) and base points (n, 2)."""
        self._require(mesh)
        m = mesh.n_cells()
        u, nrm, pt = np.empty(m), np.empty((m, 2)), np.empty((m, 2))
        check(mesh.ctx, self._lib.zg_tr_download(mesh.ctx, u.ctypes.data_as(_P), nrm.ctypes.data_as(_P),
                                                 pt.ctypes.data_as(_P)))
        return u, nrm, pt

    def get_dt(self) -> float:  # transfer.cpp:77-79
        d = C.c_double()
        check(self.mesh.ctx, self._lib.zg_tr_get_dt(self.mesh.ctx, C.byref(d)))
        return d.value

    def set_dt(self, dt: float):  # transfer.cpp:81-83
        check(self.mesh.ctx, self._lib.zg_tr_set_dt(self.mesh.ctx, dt))

    def compute_dt(self, mesh: EuMesh) -> float:  # transfer.cpp:98-105
        self._require(mesh)
        d = C.c_double()
        check(mesh.ctx, self._lib.zg_tr_compute_dt(mesh.ctx, C.byref(d)))
        return d.value

    def update(self, mesh: EuMesh, direction: Direction = Direction.ANY):  # transfer.cpp:471-485
        self._require(mesh)
        check(mesh.ctx, self._lib.zg_tr_update(mesh.ctx, int(direction)))

    def update_interface(self, mesh: EuMesh, smoothing: int = 3):  # transfer.cpp:656-658
        self._require(mesh)
        check(mesh.ctx, self._lib.zg_tr_update_interface(mesh.ctx, smoothing))

    def advance(self, mesh: EuMesh, steps: int, t: float, t_end: float, splitting: bool = True) -> float:
        """`steps` iterations of the transfer problem's time loop
        (problems/transfer.cpp:213-236) on the device; returns the new time."""
        self._require(mesh)
        tt = C.c_double(t)
        check(mesh.ctx, self._lib.zg_tr_advance(mesh.ctx, steps, 1 if splitting else 0, t_end, C.byref(tt)))
        return tt.value

    def set_flags(self, mesh: EuMesh):  # transfer.cpp:660-680
        self._require(mesh)
        f = np.empty(mesh.n_cells(), np.int32)
        check(mesh.ctx, self._lib.zg_tr_set_flags(mesh.ctx, f.ctypes.data_as(C.POINTER(C.c_int))))
        return f
