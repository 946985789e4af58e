"""Axial symmetry (SmFluid::set_axial with an axisymmetric Rectangle, y the
radius) on the GPU against the reference's own EuMesh / SmFluid compiled
from its sources (oracle/_ref): the mesh arrays, volume_alt and area_alt of
the reference's axisymmetric mesh go to the GPU (zg_mesh_upload,
zg_mesh_set_axial); every step's dt and state must agree bit for bit with
the reference's (sm_fluid.cpp:127-174, 176-253, 255-366)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = [
    # box, bounds, accuracy, limiter, flux, steps
    ("off axis walls first order", (0.0, 1.0, 0.5, 1.5), (2, 2, 1, 1), 1, "MC", 3, 30),
    ("on axis second order MC", (0.0, 1.0, 0.0, 1.0), (2, 2, 1, 2), 2, "MC", 3, 25),
    ("on axis second order van Albada HLL", (0.0, 2.0, 0.0, 1.0), (1, 2, 1, 1), 2, "van Albada", 2, 25),
]


@pytest.mark.parametrize("name,box,bounds,acc,lim,flux,steps", CASES, ids=[c[0] for c in CASES])
def test_axial_step_matches_reference(gpu_lib, name, box, bounds, acc, lim, flux, steps):
    from oracle import ref_mesh as RM
    if not RM.available():
        pytest.fail("oracle/_ref/libzref_mesh.so is missing: build it with oracle/ref_build.py")
    Z = gpu_lib
    nx, ny = 24, 20
    ref = RM.RefEuMesh(nx, ny, box=box, bounds=bounds, accuracy=acc, limiter=lim, CFL=0.4, flux=flux, axial=True)
    g = ref.cells()
    g.update(ref.faces())
    g["vol_alt"], g["area_alt"] = ref.axial_geometry()
    mesh = Z.EuMesh.from_arrays(g)
    solver = Z.SmFluid(Z.IdealGas(1.4))
    solver.set_accuracy(acc)
    solver.set_limiter(lim)
    solver.set_CFL(0.4)
    solver.set_method(Z.Fluxes(flux))
    solver.add_types(mesh)
    cx, cy = np.asarray(g["cx"]), np.asarray(g["cy"])
    r = np.hypot(cx - 0.5 * (box[0] + box[1]), cy - box[2])
    rho = np.where(r < 0.3, 2.0, 1.0) + 0.1 * cx
    u = 0.1 * np.sin(3 * cy)
    v = 0.2 * np.cos(2 * cx)
    p = np.where(r < 0.3, 3.0, 1.0)
    st = (rho, u, v, p, p / (0.4 * rho))
    ref.set_state(*st)
    mesh.set_state(*st)
    for k in range(steps):
        dt_r = ref.step()
        solver.update(mesh)
        assert solver.dt() == dt_r, (k, solver.dt(), dt_r)
    a, b = np.array(ref.state()), np.array(mesh.get_state())
    assert np.array_equal(a, b), f"{np.count_nonzero(a != b)} values differ"
    assert np.array_equal(ref.wait(), mesh.get_wait())
    mesh.close()


def test_axial_is_refused_off_the_parity_kernels(gpu_lib):
    from oracle import ref_mesh as RM
    if not RM.available():
        pytest.fail("oracle/_ref/libzref_mesh.so is missing")
    Z = gpu_lib
    ref = RM.RefEuMesh(8, 8, box=(0.0, 1.0, 0.5, 1.5), axial=True)
    g = ref.cells()
    g.update(ref.faces())
    g["vol_alt"], g["area_alt"] = ref.axial_geometry()
    mesh = Z.EuMesh.from_arrays(g)
    solver = Z.SmFluid(Z.IdealGas(1.4), kernels=Z.Kernels.FAST)
    solver.set_accuracy(2)
    solver.add_types(mesh)
    n = mesh.n_cells()
    one = np.ones(n)
    mesh.set_state(one, 0 * one, 0 * one, one, one / 0.4)
    with pytest.raises(Z.ZgError):
        solver.update(mesh)
    mesh.close()
