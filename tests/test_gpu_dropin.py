"""The C++ drop-ins of include/zephyr/math/solver/{sm,mm}_fluid_gpu.h inside
zephyr's own problem loops.

Each case runs a driver loop twice in one process: once with the reference's
solver class (zephyr::math::SmFluid / MmFluid compiled from its sources,
oracle/_ref/libzref_mesh.so) and once with the GPU drop-in, the solver type
being the only difference (tests/dropin/dropin_smf.cpp follows
problems/single-fluid/smf_test_2D.cpp:34-160: Riemann2D data, the initial
adaptation loop, update + set_flags + refine every step on the host EuMesh;
tests/dropin/dropin_mmf.cpp an air / water column problem in the manner of
problems/multi-fluid/mmf_air_water.cpp).  Every cell value and every dt must
agree bit for bit.  The drivers are built by oracle/ref_build.py.
"""
import json
import subprocess
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

REF = Path(__file__).resolve().parent.parent / "oracle" / "_ref"

# Riemann2D cases 6 (the driver's own) and 7: the others leave the end time
# unset in the reference (test_2D.cpp:9-60), so their loops would not be
# reproducible
SMF_CASES = [
    # test, nx, max_level, steps, accuracy, limiter, flux, CFL
    ("riemann6 MC HLLC amr2", (6, 24, 2, 30, 2, "MC", 3, 0.5)),
    ("riemann7 first order uniform", (7, 32, 0, 40, 1, "MC", 3, 0.4)),
    ("riemann6 van Albada HLL amr3", (6, 16, 3, 20, 2, "vanAlbada1", 2, 0.5)),
    ("riemann7 minmod Rusanov amr1", (7, 20, 1, 25, 2, "minmod", 1, 0.4)),
    # axial symmetry (Rectangle::set_axial + SmFluid::set_axial) on unrefined
    # meshes: the reference's refine computes no volume_alt for new cells
    # (mesh/amr sets only the split faces' area_alt, faces.h:80), so an
    # axisymmetric adaptive run is not defined there
    ("riemann6 axial MC second order uniform", (6, 20, 0, 20, 2, "MC", 3, 0.5, "axial")),
    ("riemann7 axial first order uniform", (7, 24, 0, 30, 1, "MC", 3, 0.4, "axial")),
    ("riemann6 CIR1 amr1", (6, 16, 1, 15, 2, "minmod", 6, 0.4)),
    ("riemann7 HLLC_M uniform", (7, 24, 0, 25, 2, "MC", 4, 0.4)),
]

MMF_CASES = [
    # nx, steps, crp_mode, accuracy, CFL
    ("plic first order", (24, 40, 4, 1, 0.4)),
    ("plain hllc first order", (24, 40, 0, 1, 0.4)),
    ("vs first order", (20, 30, 3, 1, 0.5)),
    ("plic second order", (20, 25, 4, 2, 0.4)),
]


def _run(binary, args):
    exe = REF / binary
    if not exe.exists():
        pytest.fail(f"{exe} is missing: build it with `python -m oracle.ref_build` where the reference is present")
    proc = subprocess.run([str(exe), *map(str, args)], capture_output=True, text=True, timeout=600)
    lines = [ln for ln in proc.stdout.splitlines() if ln.startswith("{")]
    assert lines, f"no result from {binary}: rc={proc.returncode} {proc.stdout[-500:]} {proc.stderr[-500:]}"
    res = json.loads(lines[-1])
    print(res)
    assert "error" not in res, res
    assert proc.returncode == 0 and res["bit_identical"], res
    return res


@pytest.mark.parametrize("name,args", SMF_CASES, ids=[c[0] for c in SMF_CASES])
def test_smfluid_dropin_in_the_reference_driver_loop(name, args):
    res = _run("dropin_smf", args)
    assert res["cells_gpu"] > 0 and res["steps"] > 0


@pytest.mark.parametrize("name,args", MMF_CASES, ids=[c[0] for c in MMF_CASES])
def test_mmfluid_dropin_in_a_reference_driver_loop(name, args):
    res = _run("dropin_mmf", args)
    assert res["cells_gpu"] == args[0] * args[0]
