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
# the zephyr source tree: $ZEPHYR_REFERENCE, else a checkout named
# "reference" beside this repository
REF = Path(os.environ.get("ZEPHYR_REFERENCE", str(HERE.parent.parent / "reference")))
SHIM_COMMON = HERE / "ref_shim" / "common"          # Eigen subset, boost bits, configuration.h
SHIM_MESH = HERE / "ref_shim" / "mesh_standin"      # plain-array EuMesh for the uniform checker
OUT_DIR = HERE / "_ref"
LIB = OUT_DIR / "libzref.so"
LIB_MESH = OUT_DIR / "libzref_mesh.so"

# The reference translation units of the step (uniform checker, stand-in mesh).
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

# Directories whose every translation unit joins the real-mesh checker, and
# the units left out: solvers off this path.
MESH_DIRS = ["zephyr/mesh", "zephyr/geom", "zephyr/math/cfd", "zephyr/math/solver", "zephyr/phys", "zephyr/io"]
MESH_FILES = ["zephyr/utils/mpi.cpp", "zephyr/utils/threads.cpp", "zephyr/utils/json.cpp",
              "zephyr/utils/stopwatch.cpp", "zephyr/utils/numpy.cpp", "zephyr/math/funcs.cpp",
              "zephyr/math/random.cpp", "zephyr/math/sle/tridiagonal.cpp", "zephyr/math/calc/integrals.cpp"]
MESH_SKIP = {"zephyr/math/solver/convection.cpp"}

FLAGS = ["-std=c++20", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-w"]
# The reference relies on <cstring> and <functional> arriving through Eigen
# and Boost headers; the stand-ins do not include them.
FORCE = ["-include", "cstring", "-include", "functional"]
# sections.cpp calls unqualified abs() on doubles (quad_volume_fraction,
# quad_find_section).  With the reference's real Eigen/Boost headers the C++
# <math.h> overloads are in scope; with the stand-ins only the C int abs(int)
# would be, truncating every normal component to 0.  Force the C++ <math.h>.
UNIT_FORCE = {"sections.cpp": ["-include", "math.h"]}


def reference_present() -> bool:
    return (REF / "zephyr" / "math" / "solver" / "sm_fluid.cpp").exists()


def _compile(cxx, src, obj, inc, force, verbose, newest_shim):
    if force or not obj.exists() or obj.stat().st_mtime < max(src.stat().st_mtime, newest_shim):
        cmd = [cxx, *FLAGS, *FORCE, *UNIT_FORCE.get(src.name, []), "-x", "c++", *inc, "-c", str(src), "-o",
               str(obj)]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)


def _link(cxx, lib, objs, force, verbose):
    if force or not lib.exists() or lib.stat().st_mtime < max(o.stat().st_mtime for o in objs):
        cmd = [cxx, "-shared", "-o", str(lib), *map(str, objs), "-pthread"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)


def mesh_units():
    units = []
    for d in MESH_DIRS:
        for ext in ("*.cpp", "*.cxx"):
            for p in sorted((REF / d).rglob(ext)):
                rel = str(p.relative_to(REF))
                if rel not in MESH_SKIP:
                    units.append(rel)
    return units + MESH_FILES


DROPIN_DIR = HERE.parent / "tests" / "dropin"
DROPIN_BINS = {"dropin_smf": DROPIN_DIR / "dropin_smf.cpp", "dropin_mmf": DROPIN_DIR / "dropin_mmf.cpp"}
GPU_LIB_DIR = HERE.parent / "zephyr_b200"
INCLUDE_DIR = HERE.parent / "include"


def build_dropin(force: bool = False, verbose: bool = False) -> list:
    """The drop-in test drivers: zephyr's problem loops against the
    reference's own EuMesh / SmFluid / MmFluid (libzref_mesh.so) and the C++
    drop-ins of include/zephyr/math/solver/*_gpu.h over libzephyr_gpu.so.
    (The reference's sm_fluid.h and mm_fluid.h cannot share a translation
    unit: each pulls its own PState into zephyr::math.)"""
    gpu_lib = GPU_LIB_DIR / "libzephyr_gpu.so"
    cxx = shutil.which("g++") or "g++"
    out = []
    for name, src in DROPIN_BINS.items():
        binary = OUT_DIR / name
        out.append(binary)
        deps = [src, DROPIN_DIR / "dropin_common.h", LIB_MESH, gpu_lib, *INCLUDE_DIR.rglob("*.h")]
        if not force and binary.exists() and binary.stat().st_mtime >= max(d.stat().st_mtime for d in deps):
            continue
        cmd = [cxx, *FLAGS, *FORCE, "-I", str(SHIM_COMMON), "-I", str(REF), "-I", str(INCLUDE_DIR), str(src),
               "-o", str(binary), str(LIB_MESH), str(gpu_lib), "-pthread",
               "-Wl,-rpath,$ORIGIN:$ORIGIN/../../zephyr_b200"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return out


def build(force: bool = False, verbose: bool = False) -> Path:
    """Build both checkers; returns the uniform one's path."""
    if not reference_present():
        if LIB.exists():
            return LIB
        raise FileNotFoundError(f"reference sources not found under {REF}")
    cxx = shutil.which("g++") or "g++"
    newest_shim = max(p.stat().st_mtime for p in (HERE / "ref_shim").rglob("*") if p.is_file())
    jobs = os.cpu_count() or 4
    from concurrent.futures import ThreadPoolExecutor

    # uniform checker: stand-in mesh
    obj_dir = OUT_DIR / "obj"
    obj_dir.mkdir(parents=True, exist_ok=True)
    inc = ["-I", str(SHIM_COMMON), "-I", str(SHIM_MESH), "-I", str(REF)]
    srcs = [REF / u for u in UNITS] + [HERE / "ref_driver.cpp"]
    objs = [obj_dir / (s.name + ".o") for s in srcs]
    with ThreadPoolExecutor(jobs) as ex:
        list(ex.map(lambda so: _compile(cxx, so[0], so[1], inc, force, verbose, newest_shim), zip(srcs, objs)))
    _link(cxx, LIB, objs, force, verbose)

    # real-mesh checker: the reference's EuMesh and AMR
    obj_dir = OUT_DIR / "obj_mesh"
    obj_dir.mkdir(parents=True, exist_ok=True)
    inc = ["-I", str(SHIM_COMMON), "-I", str(REF)]
    units = mesh_units()
    drivers = ["ref_mesh_driver.cpp", "ref_mm_driver.cpp", "ref_tr_driver.cpp"]
    srcs = [REF / u for u in units] + [HERE / d for d in drivers]
    objs = [obj_dir / (u.replace("/", "_") + ".o") for u in units] + [obj_dir / (d + ".o") for d in drivers]
    with ThreadPoolExecutor(jobs) as ex:
        list(ex.map(lambda so: _compile(cxx, so[0], so[1], inc, force, verbose, newest_shim), zip(srcs, objs)))
    _link(cxx, LIB_MESH, objs, force, verbose)
    if (GPU_LIB_DIR / "libzephyr_gpu.so").exists():
        build_dropin(force, verbose)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=False))
