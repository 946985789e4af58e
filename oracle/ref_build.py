"""Build the reference-source checker ``oracle/_ref/libzref.so`` (TEST
INFRASTRUCTURE ONLY).

The reference's own translation units for the single-material step are
compiled where they lie under the reference tree, with g++ directly (the
reference's CMake build is not used), against the small stand-ins in
``oracle/ref_shim`` for what this machine lacks: a subset of Eigen's dense API,
two boost headers, the generated ``configuration.h``, and a plain-array
EuMesh.  ``ref_driver.cpp`` runs the reference's SmFluid on that mesh.

Outputs go to ``oracle/_ref/`` only.  The GPU box has no reference tree: the
built ``libzref.so`` travels with the repository snapshot instead.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
REF = Path(os.environ.get("ZEPHYR_REFERENCE", "/root/reference"))
SHIM = HERE / "ref_shim"
OUT_DIR = HERE / "_ref"
OBJ_DIR = OUT_DIR / "obj"
LIB = OUT_DIR / "libzref.so"

# The reference translation units the checker needs (paths in the zephyr tree).
UNITS = [
    "zephyr/math/solver/sm_fluid.cpp",
    "zephyr/math/solver/riemann.cpp",
    "zephyr/math/cfd/models.cpp",
    "zephyr/math/cfd/rotate.cpp",
    "zephyr/math/cfd/limiter.cxx",
    "zephyr/math/cfd/flux/hllc.cpp",
    "zephyr/math/cfd/flux/hll.cpp",
    "zephyr/math/cfd/flux/godunov.cpp",
    "zephyr/math/cfd/flux/rusanov.cpp",
    "zephyr/math/cfd/flux/cir.cpp",
    "zephyr/math/cfd/flux/crp_flux.cpp",
    "zephyr/math/cfd/flux/num_flux.cpp",
    "zephyr/phys/matter/eos/eos.cpp",
    "zephyr/phys/matter/eos/ideal_gas.cpp",
    "zephyr/phys/matter/eos/stiffened_gas.cpp",
    "zephyr/phys/matter/mixture_pt.cpp",
    "zephyr/phys/matter/material.cpp",
    "zephyr/phys/matter/materials.cpp",
    "zephyr/phys/matter/plast/plasticity.cpp",
    "zephyr/phys/matter/cond/conductivity.cpp",
    "zephyr/phys/matter/visc/viscosity.cpp",
    "zephyr/phys/fractions.cpp",
    "zephyr/geom/primitives/quad.cpp",
    "zephyr/geom/primitives/line.cpp",
]

FLAGS = ["-std=c++20", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-w"]


def reference_present() -> bool:
    return (REF / "zephyr" / "math" / "solver" / "sm_fluid.cpp").exists()


def build(force: bool = False, verbose: bool = False) -> Path:
    if not reference_present():
        if LIB.exists():
            return LIB
        raise FileNotFoundError(f"reference sources not found under {REF}")
    cxx = shutil.which("g++") or "g++"
    OBJ_DIR.mkdir(parents=True, exist_ok=True)
    inc = ["-I", str(SHIM), "-I", str(REF)]
    shims = list(SHIM.rglob("*"))
    newest_shim = max(p.stat().st_mtime for p in shims if p.is_file())
    objs = []
    for unit in UNITS + ["DRIVER"]:
        src = HERE / "ref_driver.cpp" if unit == "DRIVER" else REF / unit
        obj = OBJ_DIR / (src.name + ".o")
        objs.append(obj)
        if force or not obj.exists() or obj.stat().st_mtime < max(src.stat().st_mtime, newest_shim):
            cmd = [cxx, *FLAGS, "-x", "c++", *inc, "-c", str(src), "-o", str(obj)]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
    if force or not LIB.exists() or LIB.stat().st_mtime < max(o.stat().st_mtime for o in objs):
        cmd = [cxx, "-shared", "-o", str(LIB), *map(str, objs), "-pthread"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
