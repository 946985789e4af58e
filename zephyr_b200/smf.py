"""Host-side mirror of zephyr's single-material solver API on the B200 library.

The classes keep the reference's names and argument meaning so that a driver
such as problems/single-fluid/smf_test_2D.cpp:34-160 reads the same:

    gen = Rectangle(0.0, 1.0, 0.0, 1.0)          # geom/generator/rectangle.h
    gen.set_boundaries(Boundaries(ZOE, ZOE, ZOE, ZOE))
    gen.set_nx(256)                              # rectangle.cpp:105-118
    mesh = EuMesh(gen)                           # mesh/euler/eu_mesh.h
    solver = SmFluid(IdealGas(1.4))              # math/solver/sm_fluid.h:41
    solver.set_accuracy(2); solver.set_CFL(0.4)
    solver.set_limiter("van Albada"); solver.set_method(Fluxes.HLLC)
    part = solver.add_types(mesh)                # sm_fluid.cpp:25-35
    mesh.set_state(rho, vx, vy, p, e)            # the driver's init loop
    solver.update(mesh)                          # sm_fluid.cpp:81-102
    solver.dt()

Cell data cross the boundary as host arrays in the reference's numbering
(ic = i * ny + j).  Errors raise ZgError (the reference throws
std::runtime_error).
"""
from __future__ import annotations

import ctypes as C
import enum
import math
from dataclasses import dataclass

import numpy as np

from ._lib import SmfParams, ZgError, check, load


class Boundary(enum.IntEnum):
    """geom/boundary.h:9-16"""
    UNDEFINED = -1
    INNER = 0
    WALL = 1
    ZOE = 2
    PERIODIC = 3
    FUNCTION = 4


class Fluxes(enum.IntEnum):
    """math/cfd/flux/num_flux.h:11-21"""
    GODUNOV = 0
    RUSANOV = 1
    HLL = 2
    HLLC = 3
    HLLC_M = 4
    HLLC_LM = 5
    CIR1 = 6
    CIR2 = 7
    CRP = 8


class Scheme(enum.IntEnum):
    PREDICTOR_CORRECTOR = 0  # the reference scheme (sm_fluid.cpp:89-98)
    HEUN = 1                 # extension: Heun RK2 on the corrector's operator


class Precision(enum.IntEnum):
    FP64 = 0
    MIXED = 1


class Kernels(enum.IntEnum):
    PARITY = 0
    FAST = 1
    FAST_TWO_PASS = 2


@dataclass(frozen=True)
class IdealGas:
    """phys/matter/eos/ideal_gas.cpp: P = (gamma - 1) rho e."""
    gamma: float = 1.4
    kind = 0
    P0 = 0.0
    e0 = 0.0

    def energy_rP(self, rho, P):  # ideal_gas.cpp:50-57
        return P / ((self.gamma - 1.0) * rho)

    def pressure_re(self, rho, e):  # ideal_gas.cpp:32-39
        return (self.gamma - 1.0) * rho * e


@dataclass(frozen=True)
class StiffenedGas:
    """phys/matter/eos/stiffened_gas.cpp: P = (gamma - 1) rho (e - e0) - gamma P0."""
    gamma: float
    P0: float = 0.0
    e0: float = 0.0
    kind = 1

    def energy_rP(self, rho, P):  # stiffened_gas.cpp:121-128
        return self.e0 + (P + self.gamma * self.P0) / ((self.gamma - 1.0) * rho)

    def pressure_re(self, rho, e):  # stiffened_gas.cpp:103-110
        return (self.gamma - 1.0) * rho * (e - self.e0) - self.gamma * self.P0


@dataclass
class Boundaries:
    """geom/generator/rectangle.h Boundaries {left, right, bottom, top}."""
    left: int = Boundary.ZOE
    right: int = Boundary.ZOE
    bottom: int = Boundary.ZOE
    top: int = Boundary.ZOE


class Rectangle:
    """geom/generator/rectangle.{h,cpp} (the non-Voronoi generator)."""

    def __init__(self, x_min, x_max, y_min, y_max):
        self.x_min, self.x_max, self.y_min, self.y_max = map(float, (x_min, x_max, y_min, y_max))
        self.bounds = Boundaries()
        self.m_nx = self.m_ny = 1

    def set_boundaries(self, bounds: Boundaries):  # rectangle.cpp:182-189
        b = Boundaries(bounds.left, bounds.right, bounds.bottom, bounds.top)
        if Boundary.PERIODIC in (b.left, b.right):
            b.left = b.right = Boundary.PERIODIC
        if Boundary.PERIODIC in (b.bottom, b.top):
            b.bottom = b.top = Boundary.PERIODIC
        self.bounds = b

    def set_nx(self, nx: int):  # rectangle.cpp:105-118
        if nx < 1:
            raise ValueError("Rectangle: Nx < 1")
        self.m_nx = nx
        self.m_ny = max(int(_round_half_away(nx * (self.y_max - self.y_min) / (self.x_max - self.x_min))), 1)

    def set_ny(self, ny: int):  # rectangle.cpp:120-133
        if ny < 1:
            raise ValueError("Rectangle: Ny < 1")
        self.m_ny = ny
        self.m_nx = max(int(_round_half_away(ny * (self.x_max - self.x_min) / (self.y_max - self.y_min))), 1)

    def set_sizes(self, nx: int, ny: int):  # rectangle.cpp:135-162
        if nx < 1 or ny < 1:
            raise ValueError("Rectangle: Nx < 1 or Ny < 1")
        self.m_nx, self.m_ny = nx, ny

    def nx(self):
        return self.m_nx

    def ny(self):
        return self.m_ny


def _round_half_away(x):
    """std::round: halves away from zero."""
    return math.floor(x + 0.5) if x >= 0 else -math.floor(-x + 0.5)


class EuMesh:
    """mesh/euler/eu_mesh.h over one GPU context.  Owns the device data."""

    def __init__(self, gen: Rectangle, device: int = 0, stream=None):
        self._lib = load()
        self.ctx = C.c_void_p()
        check(None, self._lib.zg_create(C.byref(self.ctx), device))
        self.device = device
        if stream is not None:
            self.set_stream(stream)
        b = (C.c_int * 4)(int(gen.bounds.left), int(gen.bounds.right), int(gen.bounds.bottom),
                          int(gen.bounds.top))
        check(self.ctx, self._lib.zg_mesh_rectangle(self.ctx, gen.nx(), gen.ny(), gen.x_min, gen.x_max,
                                                    gen.y_min, gen.y_max, b))
        self.nx, self.ny = gen.nx(), gen.ny()
        self.gen = gen
        self.solver = None
        self._amr = False

    @classmethod
    def from_arrays(cls, g: dict, device: int = 0, stream=None):
        """A mesh given cell by cell (for example a refined zephyr mesh):
        dict with cx, cy, vol, inc (n cells) and boundary, neib, nx, ny, fx,
        fy, area (8 slots per cell), in zephyr's AmrCells order."""
        from ._lib import MeshView
        self = cls.__new__(cls)
        self._lib = load()
        self.ctx = C.c_void_p()
        check(None, self._lib.zg_create(C.byref(self.ctx), device))
        self.device = device
        if stream is not None:
            self.set_stream(stream)
        keep = {k: np.ascontiguousarray(g[k], dtype=np.int32 if k in ("boundary", "neib") else np.float64)
                for k in ("cx", "cy", "vol", "inc", "boundary", "neib", "nx", "ny", "fx", "fy", "area")}
        n = keep["cx"].size
        for k in ("boundary", "neib", "nx", "ny", "fx", "fy", "area"):
            if keep[k].size != 8 * n:
                raise ZgError(-1, f"{k} must have 8 entries per cell")
        dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
        ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int))
        view = MeshView(n, dp(keep["cx"]), dp(keep["cy"]), dp(keep["vol"]), dp(keep["inc"]),
                        ip(keep["boundary"]), ip(keep["neib"]), dp(keep["nx"]), dp(keep["ny"]),
                        dp(keep["fx"]), dp(keep["fy"]), dp(keep["area"]))
        check(self.ctx, self._lib.zg_mesh_upload(self.ctx, C.byref(view)))
        if "vol_alt" in g and "area_alt" in g:
            self.set_axial(g["vol_alt"], g["area_alt"])
        self.nx = self.ny = 0
        self.gen = None
        self.solver = None
        self._amr = False
        return self

    def set_axial(self, vol_alt, area_alt):
        """Axisymmetric geometry of a mesh given cell by cell (Rectangle /
        SmFluid set_axial): volume_alt per cell, area_alt per face slot."""
        v = np.ascontiguousarray(vol_alt, dtype=np.float64)
        a = np.ascontiguousarray(area_alt, dtype=np.float64)
        dp = lambda x: x.ctypes.data_as(C.POINTER(C.c_double))
        check(self.ctx, self._lib.zg_mesh_set_axial(self.ctx, dp(v), dp(a)))

    def set_stream(self, stream):
        """Queue all work on `stream` (a cudaStream_t handle as int, or None)."""
        handle = int(stream) if stream is not None else None
        check(self.ctx, self._lib.zg_set_stream(self.ctx, C.c_void_p(handle) if handle else None))

    def n_cells(self) -> int:
        n = C.c_int()
        check(self.ctx, self._lib.zg_mesh_n_cells(self.ctx, C.byref(n)))
        return n.value

    def centers(self):
        """Cell centres (x, y) in cell order, with the reference's formulas."""
        if self._amr:
            from ._lib import AmrCells
            n = self.n_cells()
            cx, cy = np.empty(n), np.empty(n)
            view = AmrCells(cx.ctypes.data_as(C.POINTER(C.c_double)), cy.ctypes.data_as(C.POINTER(C.c_double)))
            check(self.ctx, self._lib.zg_amr_download(self.ctx, C.byref(view)))
            return cx, cy
        g = self.gen
        X = g.x_min + ((g.x_max - g.x_min) * np.arange(g.nx() + 1)) / g.nx()
        Y = g.y_min + ((g.y_max - g.y_min) * np.arange(g.ny() + 1)) / g.ny()
        cx = 0.25 * (((X[:-1] + X[1:]) + X[:-1]) + X[1:])
        cy = 0.25 * (((Y[:-1] + Y[:-1]) + Y[1:]) + Y[1:])
        return np.repeat(cx, g.ny()), np.tile(cy, g.nx())

    def _require_solver(self):
        if self.solver is None:
            raise ZgError(-3, "no solver fields on this mesh: call SmFluid.add_types(mesh) first")

    def set_state(self, rho, vx, vy, p, e):
        """Write the primitive state (field `init`) of every cell."""
        self._require_solver()
        n = self.n_cells()
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (rho, vx, vy, p, e)]
        for a in arrs:
            if a.shape != (n,):
                raise ZgError(-1, f"state arrays must have shape ({n},)")
        ptrs = [a.ctypes.data_as(C.POINTER(C.c_double)) for a in arrs]
        check(self.ctx, self._lib.zg_state_upload(self.ctx, *ptrs))
        check(self.ctx, self._lib.zg_synchronize(self.ctx))

    def get_state(self):
        """(density, vx, vy, pressure, energy) host arrays of the field `init`."""
        self._require_solver()
        n = self.n_cells()
        out = [np.empty(n) for _ in range(5)]
        check(self.ctx, self._lib.zg_state_download(self.ctx, *[a.ctypes.data_as(C.POINTER(C.c_double))
                                                                 for a in out]))
        return out

    def set_wait(self, wait):
        self._require_solver()
        w = np.ascontiguousarray(wait, dtype=np.int32)
        check(self.ctx, self._lib.zg_wait_upload(self.ctx, w.ctypes.data_as(C.POINTER(C.c_int))))
        check(self.ctx, self._lib.zg_synchronize(self.ctx))

    def get_wait(self):
        self._require_solver()
        w = np.empty(self.n_cells(), np.int32)
        check(self.ctx, self._lib.zg_wait_download(self.ctx, w.ctypes.data_as(C.POINTER(C.c_int))))
        return w

    # ---- adaptation (eu_mesh.h: set_max_level, set_distributor, refine) ----
    def set_max_level(self, max_level: int, capacity: int | None = None):
        """EuMesh::set_max_level on a rectangle mesh: the cells get the AMR
        layout on the device with room for `capacity` cells (default
        max(16 n, 2^20)).  Call before SmFluid.add_types."""
        n = self.n_cells()
        if capacity is None:
            capacity = min(max(16 * n, 1 << 20), (2 ** 31 - 1) // 16)
        check(self.ctx, self._lib.zg_amr_enable(self.ctx, int(max_level), int(capacity)))
        self._amr = True

    def max_level(self) -> int:
        return self.amr_info().max_level

    def adaptive(self) -> bool:  # eu_mesh.cpp:170-172
        return self.max_level() > 0

    def set_distributor(self, kind):
        """EuMesh::set_distributor(solver.distributor(type)); `kind` is the
        value of SmFluid.distributor or the type name ("const", "slope")."""
        if isinstance(kind, str):
            kind = SmFluid.DISTRIBUTORS.get(kind, -1)
        check(self.ctx, self._lib.zg_amr_set_distributor(self.ctx, int(kind)))

    def put_flags(self, flags):
        """EuCell::set_flag for every cell."""
        f = np.ascontiguousarray(flags, dtype=np.int32)
        if f.shape != (self.n_cells(),):
            raise ZgError(-1, f"flags must have shape ({self.n_cells()},)")
        check(self.ctx, self._lib.zg_amr_put_flags(self.ctx, f.ctypes.data_as(C.POINTER(C.c_int))))
        check(self.ctx, self._lib.zg_synchronize(self.ctx))

    def refine(self):  # eu_mesh.cpp:290-359
        check(self.ctx, self._lib.zg_amr_refine(self.ctx))

    def amr_info(self):
        from ._lib import AmrStats
        st = AmrStats()
        check(self.ctx, self._lib.zg_amr_info(self.ctx, C.byref(st)))
        return st

    def amr_arrays(self) -> dict:
        """Host copies of the adaptive mesh: cells (cx, cy, vol, inc, level,
        flag, b_idx, z_idx), map points (vx, vy: 9 per cell) and face slots
        (boundary, neib, nx, ny, fx, fy, area: 8 per cell)."""
        from ._lib import AmrCells
        n = self.n_cells()
        g = {k: np.empty(n) for k in ("cx", "cy", "vol", "inc")}
        g.update({k: np.empty(9 * n) for k in ("vx", "vy")})
        g.update({k: np.empty(n, np.int32) for k in ("level", "flag", "b_idx", "z_idx")})
        g.update({k: np.empty(8 * n, np.int32) for k in ("boundary", "neib")})
        g.update({k: np.empty(8 * n) for k in ("nx", "ny", "fx", "fy", "area")})
        dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
        ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int))
        view = AmrCells(dp(g["cx"]), dp(g["cy"]), dp(g["vol"]), dp(g["inc"]), dp(g["vx"]), dp(g["vy"]),
                        ip(g["level"]), ip(g["flag"]), ip(g["b_idx"]), ip(g["z_idx"]), ip(g["boundary"]),
                        ip(g["neib"]), dp(g["nx"]), dp(g["ny"]), dp(g["fx"]), dp(g["fy"]), dp(g["area"]))
        check(self.ctx, self._lib.zg_amr_download(self.ctx, C.byref(view)))
        return g

    def launch_count(self) -> int:
        n = C.c_longlong()
        check(self.ctx, self._lib.zg_launch_count(self.ctx, C.byref(n)))
        return n.value

    def synchronize(self):
        check(self.ctx, self._lib.zg_synchronize(self.ctx))

    def close(self):
        if getattr(self, "ctx", None) and self.ctx.value:
            self._lib.zg_destroy(self.ctx)
            self.ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class Parts:
    """SmFluid::Parts (sm_fluid.h:26-36): names of the solver's fields."""
    init: str = "init"
    half: str = "half"
    next: str = "next"
    d_dx: str = "d_dx"
    d_dy: str = "d_dy"
    d_dz: str = "d_dz"
    wait: str = "wait"


class SmFluid:
    """math/solver/sm_fluid.{h,cpp} on the GPU."""

    DISTRIBUTORS = {"const": 0, "slope": 1}  # enum zg_distributor

    def __init__(self, eos, precision: Precision = Precision.FP64, kernels: Kernels = Kernels.PARITY):
        self._lib = load()
        p = SmfParams()
        self._lib.zg_smf_default_params(C.byref(p))  # sm_fluid.cpp:16-23
        p.eos_kind, p.gamma, p.P0, p.e0 = eos.kind, eos.gamma, eos.P0, eos.e0
        p.precision, p.kernels = int(precision), int(kernels)
        self.params = p
        self.eos = eos
        self.mesh = None
        self.part = Parts()

    def _push(self):
        if self.mesh is not None:
            check(self.mesh.ctx, self._lib.zg_smf_configure(self.mesh.ctx, C.byref(self.params)))

    def add_types(self, mesh: EuMesh) -> Parts:  # sm_fluid.cpp:25-35
        self.mesh = mesh
        mesh.solver = self
        self._push()
        return self.part

    def set_CFL(self, CFL: float):  # sm_fluid.cpp:37-39
        self.params.CFL = max(0.0, min(float(CFL), 1.0))
        self._push()

    def set_accuracy(self, acc: int):  # sm_fluid.cpp:41-43
        self.params.accuracy = min(max(1, int(acc)), 2)
        self._push()

    def set_method(self, method: Fluxes):  # sm_fluid.cpp:49-51 -> num_flux.cpp:6-35
        if not 0 <= int(method) <= int(Fluxes.CIR2):
            raise ZgError(-1, f"numerical flux {Fluxes(method).name} is not a single-material flux")
        self.params.flux = int(method)
        self._push()

    def set_limiter(self, name: str):  # sm_fluid.cpp:53-55 -> limiter.cxx:163-252
        k = self._lib.zg_limiter_from_name(name.encode())
        if k < 0:
            raise ZgError(-1, f"Unknown limiter '{name}'")
        self.params.limiter = k
        self._push()

    def set_scheme(self, scheme: Scheme):
        self.params.scheme = int(scheme)
        self._push()

    def set_max_dt(self, dt: float):  # sm_fluid.cpp:65-67
        self.params.max_dt = float(dt)
        if self.mesh is not None:
            check(self.mesh.ctx, self._lib.zg_smf_set_max_dt(self.mesh.ctx, float(dt)))

    def CFL(self) -> float:
        return self.params.CFL

    def update(self, mesh: EuMesh, steps: int = 1):  # sm_fluid.cpp:81-102
        if mesh is not self.mesh:
            self.add_types(mesh)
        if steps == 1:
            check(mesh.ctx, self._lib.zg_smf_update(mesh.ctx))
        else:
            check(mesh.ctx, self._lib.zg_smf_update_n(mesh.ctx, int(steps)))

    def dt(self) -> float:  # sm_fluid.h:68
        if self.mesh is None:
            return float("nan")
        d = C.c_double()
        check(self.mesh.ctx, self._lib.zg_smf_dt(self.mesh.ctx, C.byref(d)))
        return d.value

    def set_flags(self, mesh: EuMesh, download: bool = True):  # sm_fluid.cpp:517-559 (flag values)
        """Flags of every cell; on an adaptive mesh they stay on the device for
        EuMesh.refine, and `download=False` skips the host copy."""
        if mesh is not self.mesh:
            self.add_types(mesh)
        if not download:
            check(mesh.ctx, self._lib.zg_smf_set_flags(mesh.ctx, None))
            return None
        f = np.empty(mesh.n_cells(), np.int32)
        check(mesh.ctx, self._lib.zg_smf_set_flags(mesh.ctx, f.ctypes.data_as(C.POINTER(C.c_int))))
        return f

    def set_flags_gradient(self, mesh: EuMesh, refine: float = 0.05, coarsen: float = 0.01, download: bool = True):
        """Flags by |grad rho| h / rho (refine above `refine`, coarsen below
        `coarsen`) on an adaptive mesh; no reference counterpart."""
        if mesh is not self.mesh:
            self.add_types(mesh)
        if not download:
            check(mesh.ctx, self._lib.zg_amr_set_flags_gradient(mesh.ctx, refine, coarsen, None))
            return None
        f = np.empty(mesh.n_cells(), np.int32)
        check(mesh.ctx, self._lib.zg_amr_set_flags_gradient(mesh.ctx, refine, coarsen,
                                                             f.ctypes.data_as(C.POINTER(C.c_int))))
        return f

    def distributor(self, type: str = "slope") -> int:  # sm_fluid.cpp:372-375
        if type not in self.DISTRIBUTORS:
            raise ZgError(-1, f"SmFluid error: unknown m_distributor type '{type}'")
        return self.DISTRIBUTORS[type]
