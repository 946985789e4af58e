"""Python mirror of zephyr's output classes (io/vtu_file.h, io/pvd_file.h,
io/variables.h) on top of the C ABI (``zg_vtu_write``, ``zg_pvd_*``): VTU
files and PVD series in the reference's byte format, packed from the device
buffers of a mesh's context.

    pvd = PvdFile("test2D", "output")
    pvd.variables = Variables(["level"])
    pvd.variables.append("density", ("smf", 0))   # the SmFluid state on the device
    pvd.variables.append("u", ("tr", 0))          # Transfer's u1
    pvd.variables.append("exact", host_array)     # any per-cell host array
    pvd.save(mesh, curr_time)
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import OutVar, ZgError, check, load
from .smf import EuMesh

# io::Variable's named variables (io/variable.cpp:11-160)
NAMED = {"level": 0, "index": 1, "rank": 2, "flag": 3, "b_idx": 4, "z_idx": 5, "center": 6, "coords": 6}
# device state fields: zg_out_source values
SOURCES = {"smf": 7, "mmf": 8, "tr": 9}
HOST = 10
# SmFluid / Transfer component names
SMF_FIELDS = {"density": 0, "vel.x": 1, "vel.y": 2, "pressure": 3, "energy": 4}
TR_FIELDS = {"u1": 0, "n.x": 1, "n.y": 2, "p.x": 3, "p.y": 4, "n": 5, "p": 6}


class Variables(list):
    """The variables to write: entries (name, source) where source is None
    for a named variable, ("smf" | "mmf" | "tr", component) for a device
    field, or a host array of one value per cell."""

    def __init__(self, names=()):
        super().__init__()
        for nm in names:
            self.append(nm)

    def append(self, name, source=None):  # noqa: D401 - mirrors Variables::append
        if source is None and name not in NAMED:
            raise ZgError(-1, f"Unknown variable '{name}'")
        super().append((name, source))

    def _pack(self, n_cells):
        keep = []
        arr = (OutVar * max(len(self), 1))()
        for k, (name, src) in enumerate(self):
            v = arr[k]
            v.name = name.encode()
            if src is None:
                v.source = NAMED[name]
            elif isinstance(src, tuple):
                v.source = SOURCES[src[0]]
                v.component = int(src[1])
            else:
                a = np.ascontiguousarray(src, dtype=np.float64)
                if a.size != n_cells:
                    raise ValueError(f"variable '{name}': one value per cell")
                keep.append(a)
                v.source = HOST
                v.host = a.ctypes.data_as(C.POINTER(C.c_double))
        return arr, keep


class VtuFile:
    """VtuFile::save(filename, mesh, variables) (vtu_file.cpp:555-584)."""

    @staticmethod
    def save(filename, mesh: EuMesh, variables: Variables = Variables()):
        arr, keep = variables._pack(mesh.n_cells())
        check(mesh.ctx, load().zg_vtu_write(mesh.ctx, str(filename).encode(), arr, len(variables)))


class PvdFile:
    """PvdFile(filename, directory) with `variables` and save(mesh, timestep)
    (pvd_file.h:12-89)."""

    def __init__(self, filename, directory="output"):
        self._lib = load()
        self.variables = Variables()
        self.h = C.c_void_p()
        rc = self._lib.zg_pvd_open(C.byref(self.h), str(filename).encode(), str(directory).encode())
        if rc != 0:
            raise ZgError(rc, f"cannot open PVD file {filename} in {directory}")

    def save(self, mesh: EuMesh, timestep: float):
        arr, keep = self.variables._pack(mesh.n_cells())
        check(mesh.ctx, self._lib.zg_pvd_save(self.h, mesh.ctx, arr, len(self.variables), timestep))

    def close(self):
        if self.h:
            self._lib.zg_pvd_close(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
