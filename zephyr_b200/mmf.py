"""Python mirror of zephyr's multi-material solver MmFluid
(math/solver/mm_fluid.h:45-163) and its mixture MixturePT
(phys/matter/mixture_pt.h) on top of the C ABI (``zg_mmf_*``).

    water = Material.stiffened("Water")        # StiffenedGas::create("Water")
    air = Material.ideal("Air")                # IdealGas::create("Air")
    solver = MmFluid(MixturePT([water, air]))  # MmFluid(mixture)
    solver.set_CFL(0.4)
    solver.add_types(mesh)                     # mesh: smf.EuMesh of a Rectangle
    solver.make_states(mesh, rho, vx, vy, p, beta)
    solver.update(mesh); solver.dt()

Cell states cross the boundary as 14 doubles per cell: density, velocity x,
velocity y, pressure, specific internal energy, temperature, mass fractions
[4], true densities [4] (the fields of mmf::PState, math/cfd/models.h:167-180).
There is no CPU fallback: the calls go to the CUDA library.
"""
from __future__ import annotations

import ctypes as C
import enum

import numpy as np

from ._lib import Material as _Material
from ._lib import MmfParams, ZgError, check, load
from .smf import EuMesh, Fluxes

NSTATE = 14
EOS_IDEAL, EOS_STIFFENED = 0, 1


class CrpMode(enum.IntEnum):
    """mm_fluid.h:31-37"""
    NONE = 0
    V3 = 1
    V5 = 2
    VS = 3
    PLIC = 4
    MUSCL = 5


class DirSplit(enum.IntEnum):
    """mm_fluid.h:23-28"""
    NONE = 0
    SIMPLE = 1
    STRANG = 2


class Material:
    """A material of the mixture: IdealGas(name) / StiffenedGas(name) or
    explicit parameters."""

    def __init__(self, kind, gamma, P0=0.0, e0=0.0, Cv=1.0, T0=0.0, rho_ref=float("nan")):
        self.c = _Material(kind, gamma, P0, e0, Cv, T0, rho_ref)

    @classmethod
    def _named(cls, kind, name):
        self = cls.__new__(cls)
        self.c = _Material()
        rc = load().zg_material_named(kind, name.encode(), C.byref(self.c))
        if rc != 0:
            raise ZgError(rc, f"unknown material '{name}'")
        return self

    @classmethod
    def ideal(cls, name: str) -> "Material":  # ideal_gas.cpp:14-24
        return cls._named(EOS_IDEAL, name)

    @classmethod
    def stiffened(cls, name: str) -> "Material":  # stiffened_gas.cpp:13-86
        return cls._named(EOS_STIFFENED, name)

    def __repr__(self):
        c = self.c
        kind = "StiffenedGas" if c.kind == EOS_STIFFENED else "IdealGas"
        return f"{kind}(gamma={c.gamma}, P0={c.P0}, e0={c.e0}, Cv={c.Cv}, T0={c.T0}, rho_ref={c.rho_ref})"


class MixturePT(list):
    """MixturePT{materials...} (mixture_pt.h:28-35)."""


class MmFluid:
    """MmFluid(const MixturePT&) with its setters; the fields live on the mesh's
    device context after add_types."""

    def __init__(self, mixture: MixturePT):
        self._lib = load()
        self.p = MmfParams()
        self._lib.zg_mmf_default_params(C.byref(self.p))  # mm_fluid.cpp:16-26
        if len(mixture) > 4:
            raise ValueError("at most 4 materials (Fractions::max_size)")
        self.p.n_materials = len(mixture)
        for i, m in enumerate(mixture):
            self.p.materials[i] = m.c
        self.mixture = mixture
        self.mesh = None
        self._dt = float("nan")

    def _push(self):
        if self.mesh is not None:
            check(self.mesh.ctx, self._lib.zg_mmf_configure(self.mesh.ctx, C.byref(self.p)))

    def add_types(self, mesh: EuMesh):  # mm_fluid.cpp:28-40
        self.mesh = mesh
        self._push()
        return self

    def set_precision(self, precision: int):
        """Precision.FP64 (the reference's arithmetic) or Precision.MIXED (FP32
        HLLC of the pure faces -- pure-stencil faces in first order, faces
        whose reconstructed states stay pure in second order -- FP64
        elsewhere; second order with a CRP mode only)."""
        self.p.precision = int(precision)
        self._push()

    def set_CFL(self, CFL: float):  # mm_fluid.cpp:42-44
        self.p.CFL = max(0.0, min(CFL, 1.0))
        self._push()

    def set_accuracy(self, acc: int):  # mm_fluid.cpp:46-48
        self.p.accuracy = min(max(1, acc), 2)
        self._push()

    def set_limiter(self, name: str):  # mm_fluid.cpp:72-74 -> limiter.cxx:163-252
        k = self._lib.zg_limiter_from_name(name.encode())
        if k < 0:
            raise ZgError(-1, f"unknown limiter '{name}'")
        self.p.limiter = k
        self._push()

    def set_method(self, method: Fluxes):  # mm_fluid.cpp:50-61
        if method == Fluxes.CRP:
            self.p.crp_mode = CrpMode.PLIC
        elif method == Fluxes.HLLC:
            self.p.crp_mode = CrpMode.NONE
        else:
            raise ZgError(-1, "the mixture flux is HLLC (plain or composite); other fluxes are not implemented")
        self._push()

    def set_crp_mode(self, mode: CrpMode):  # mm_fluid.cpp:63-69
        """CrpMode::MUSCL computes the volume-fraction gradients (grad_a); the
        reference defines no face fraction for it, so a step that reaches a
        composite face raises ZgError (ZG_ERR_NUMERIC) where the reference's
        assert fails (mm_fluid.cpp:245-250, 276)."""
        if mode != CrpMode.NONE:
            self.p.crp_mode = mode
            self._push()

    def set_splitting(self, split: DirSplit):  # mm_fluid.cpp:75-77
        self.p.split = int(split)
        self._push()

    def set_max_dt(self, dt: float):  # mm_fluid.cpp:91-93
        self.p.max_dt = dt
        self._push()

    def CFL(self) -> float:
        return self.p.CFL

    def _require(self, mesh):
        if mesh is not self.mesh:
            raise ZgError(-3, "call add_types(mesh) first")

    def make_states(self, mesh: EuMesh, rho, vx, vy, p, beta):
        """PState(density, velocity, pressure, Fractions(beta), mixture) for
        every cell; beta is (n_cells, n_materials) or (n_cells, 4)."""
        self._require(mesh)
        n = mesh.n_cells()
        b = np.zeros((n, 4))
        b[:, :np.asarray(beta).shape[1]] = beta
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (rho, vx, vy, p)] + [np.ascontiguousarray(b)]
        ptrs = [a.ctypes.data_as(C.POINTER(C.c_double)) for a in arrs]
        check(mesh.ctx, self._lib.zg_mmf_make_states(mesh.ctx, *ptrs))

    def set_states(self, mesh: EuMesh, cells):
        self._require(mesh)
        s = np.ascontiguousarray(cells, dtype=np.float64).reshape(-1, NSTATE)
        check(mesh.ctx, self._lib.zg_mmf_state_upload(mesh.ctx, s.ctypes.data_as(C.POINTER(C.c_double))))

    def states(self, mesh: EuMesh):
        self._require(mesh)
        s = np.empty((mesh.n_cells(), NSTATE))
        check(mesh.ctx, self._lib.zg_mmf_state_download(mesh.ctx, s.ctypes.data_as(C.POINTER(C.c_double))))
        return s

    def update(self, mesh: EuMesh, steps: int = 1):  # mm_fluid.cpp:112-137
        self._require(mesh)
        check(mesh.ctx, self._lib.zg_mmf_update_n(mesh.ctx, steps))

    def dt(self) -> float:  # mm_fluid.h:97
        d = C.c_double()
        check(self.mesh.ctx, self._lib.zg_mmf_dt(self.mesh.ctx, C.byref(d)))
        return d.value

    def set_flags(self, mesh: EuMesh):  # mm_fluid.cpp:836-885
        self._require(mesh)
        f = np.empty(mesh.n_cells(), np.int32)
        check(mesh.ctx, self._lib.zg_mmf_set_flags(mesh.ctx, f.ctypes.data_as(C.POINTER(C.c_int))))
        return f

    def grad_a(self, mesh: EuMesh):
        """part.grad_a of the last MUSCL sub-step (fractions_grad,
        mm_fluid.cpp:469-482): (n, n_materials, 2) volume-fraction gradients."""
        self._require(mesh)
        n, nm = mesh.n_cells(), self.p.n_materials
        g = np.empty((n, nm, 2))
        check(mesh.ctx, self._lib.zg_mmf_grad_a(mesh.ctx, g.ctypes.data_as(C.POINTER(C.c_double))))
        return g

    def interface(self, mesh: EuMesh):
        """interface_recovery of the current state: normals (n, nm, 2), offsets (n, nm)."""
        self._require(mesh)
        n, nm = mesh.n_cells(), self.p.n_materials
        nrm = np.empty((n, nm, 2))
        off = np.empty((n, nm))
        check(mesh.ctx, self._lib.zg_mmf_interface(mesh.ctx, nrm.ctypes.data_as(C.POINTER(C.c_double)),
                                                   off.ctypes.data_as(C.POINTER(C.c_double))))
        return nrm, off
