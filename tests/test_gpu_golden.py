"""GPU against the golden fixtures produced by the reference's own code
(tests/golden, made by tests/golden/make_golden.py from oracle/_ref): the
parity kernels must reproduce the reference's dt sequence, states, isolation
counters and flags bit for bit (the Godunov flux to rounding: its exact
Riemann solver's powers come from CUDA's pow)."""
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"
CASES = sorted(p.stem for p in GOLDEN.glob("*.npz")
               if p.stem not in ("pointwise", "isolation_20_mc") and not p.stem.startswith(("amr_", "mm_", "adapt_", "tr_", "vtu_")))
AMR_CASES = sorted(p.stem for p in GOLDEN.glob("amr_*.npz"))


def _gpu_for(Z, g):
    nx, ny = int(g["nx"]), int(g["ny"])
    x0, x1, y0, y1 = (float(v) for v in g["box"])
    ek, gamma, P0 = g["eos"]
    gen = Z.Rectangle(x0, x1, y0, y1)
    gen.set_boundaries(Z.Boundaries(*(int(b) for b in g["bounds"])))
    gen.set_sizes(nx, ny)
    mesh = Z.EuMesh(gen)
    eos = Z.IdealGas(float(gamma)) if int(ek) == 0 else Z.StiffenedGas(float(gamma), float(P0), 0.0)
    solver = Z.SmFluid(eos)
    solver.set_accuracy(int(g["accuracy"]))
    solver.set_CFL(float(g["CFL"]))
    solver.set_limiter(str(g["limiter"]))
    solver.set_method(Z.Fluxes(int(g["flux"])))
    solver.add_types(mesh)
    return mesh, solver


@pytest.mark.parametrize("name", CASES)
def test_gpu_matches_reference_fixture(gpu_lib, name):
    Z = gpu_lib
    g = np.load(GOLDEN / f"{name}.npz", allow_pickle=False)
    mesh, solver = _gpu_for(Z, g)
    mesh.set_state(*g["init"])
    dts = []
    for _ in range(int(g["steps"])):
        solver.update(mesh)
        dts.append(solver.dt())
    final = np.array(mesh.get_state())
    if int(g["flux"]) in (0, 5):
        # Godunov: the rarefaction fans' powers come from CUDA's pow, within
        # a few ulps of glibc's; HLLC_LM: its low-Mach factor is CUDA's sin;
        # the states agree to rounding after all steps
        assert np.allclose(np.array(dts), g["dts"], rtol=1e-12, atol=0.0)
        scale = np.abs(g["final"]).max(axis=1, keepdims=True)
        worst = float((np.abs(final - g["final"]) / scale).max())
        assert worst <= 1e-11, f"largest relative difference {worst:.3e}"
    else:
        assert np.array_equal(np.array(dts), g["dts"]), "dt sequence differs from the reference"
        assert np.array_equal(final, g["final"]), f"{np.count_nonzero(final != g['final'])} values differ"
    assert np.array_equal(mesh.get_wait(), g["wait"])
    assert np.array_equal(solver.set_flags(mesh), g["flags"])


@pytest.mark.parametrize("name", AMR_CASES)
def test_gpu_matches_reference_on_refined_mesh(gpu_lib, name):
    """The parity kernels on meshes refined by the reference's refine()
    (hanging faces, up to three levels), against the reference's steps."""
    Z = gpu_lib
    g = np.load(GOLDEN / f"{name}.npz", allow_pickle=False)
    mesh = Z.EuMesh.from_arrays(g)
    solver = Z.SmFluid(Z.IdealGas(1.4))
    solver.set_accuracy(int(g["accuracy"]))
    solver.set_CFL(float(g["CFL"]))
    solver.set_limiter(str(g["limiter"]))
    solver.add_types(mesh)
    mesh.set_state(*g["init"])
    dts = []
    for _ in range(int(g["steps"])):
        solver.update(mesh)
        dts.append(solver.dt())
    assert np.array_equal(np.array(dts), g["dts"])
    final = np.array(mesh.get_state())
    assert np.array_equal(final, g["final"]), f"{np.count_nonzero(final != g['final'])} values differ"
    assert np.array_equal(solver.set_flags(mesh), g["flags"])


def test_gpu_refuses_tiled_kernels_on_slot_mesh(gpu_lib):
    Z = gpu_lib
    g = np.load(GOLDEN / f"{AMR_CASES[0]}.npz", allow_pickle=False)
    mesh = Z.EuMesh.from_arrays(g)
    solver = Z.SmFluid(Z.IdealGas(1.4), kernels=Z.Kernels.FAST)
    solver.add_types(mesh)
    mesh.set_state(*g["init"])
    with pytest.raises(Z.ZgError):
        solver.update(mesh)


def test_gpu_matches_reference_isolation(gpu_lib):
    Z = gpu_lib
    g = np.load(GOLDEN / "isolation_20_mc.npz", allow_pickle=False)
    gen = Z.Rectangle(0.0, 1.0, 0.0, 1.0)
    gen.set_boundaries(Z.Boundaries(2, 2, 2, 2))
    gen.set_nx(20)
    mesh = Z.EuMesh(gen)
    solver = Z.SmFluid(Z.IdealGas(1.4))
    solver.set_accuracy(2)
    solver.set_CFL(0.4)
    solver.set_limiter("MC")
    solver.add_types(mesh)
    mesh.set_state(*g["init"])
    mesh.set_wait(g["wait0"])
    solver.update(mesh)
    assert solver.dt() == g["dts"][0]
    assert np.array_equal(np.array(mesh.get_state()), g["final"])
    assert np.array_equal(mesh.get_wait(), g["wait"])
