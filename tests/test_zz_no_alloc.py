"""zg_rect_step_noalloc, the allocation-free first-order step, called through
the C ABI with caller-owned device arrays: two calls in a row must give the
same dt and states as two zg_smf_update steps of a context with the same
parameters.  Both run the parity kernels, so the tolerance is zero: the
results must agree bit for bit.

This file is collected last so that it also runs after every other GPU test
in the same process (the library is then loaded and its scratch set up by
earlier calls on the device, or not at all when the file runs alone)."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOLERANCE = 0.0  # bit-exact: same kernels, same order of operations


WATER = (4.4, 6.0e8, 0.0)  # stiffened gas: gamma, P0, e0


def _existing_path(Z, nx, ny, box, bounds, flux, CFL, state, steps, stiff=False):
    gen = Z.Rectangle(*box)
    gen.set_boundaries(Z.Boundaries(*bounds))
    gen.set_sizes(nx, ny)
    mesh = Z.EuMesh(gen)
    solver = Z.SmFluid(Z.StiffenedGas(*WATER) if stiff else Z.IdealGas(1.4))
    solver.set_accuracy(1)
    solver.set_CFL(CFL)
    solver.set_method(Z.Fluxes(flux))
    solver.add_types(mesh)
    mesh.set_state(*state)
    out = []
    for _ in range(steps):
        solver.update(mesh)
        out.append((solver.dt(), [np.array(a) for a in mesh.get_state()]))
    mesh.close()
    return out


def _noalloc_path(Z, nx, ny, box, bounds, flux, CFL, state, steps, stiff=False):
    import torch
    from zephyr_b200 import _lib

    lib = Z.load()
    p = _lib.SmfParams()
    lib.zg_smf_default_params(C.byref(p))
    if stiff:
        p.eos_kind = 1
        p.gamma, p.P0, p.e0 = WATER
    p.flux = flux
    p.CFL = CFL
    p.accuracy = 1
    dev = torch.device("cuda", 0)
    bufs = [[torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device=dev) for a in state]]
    bufs += [[torch.empty(nx * ny, dtype=torch.float64, device=dev) for _ in range(5)] for _ in range(2)]
    dts = torch.full((steps,), float("nan"), dtype=torch.float64, device=dev)
    b = (C.c_int * 4)(*bounds)
    stream = torch.cuda.current_stream(dev)
    for s in range(steps):
        src, dst = bufs[s], bufs[s + 1]
        ins = (C.c_void_p * 5)(*[t.data_ptr() for t in src])
        outs = (C.c_void_p * 5)(*[t.data_ptr() for t in dst])
        rc = lib.zg_rect_step_noalloc(0, nx, ny, *box, b, C.byref(p), ins, outs,
                                      C.c_void_p(dts.data_ptr() + 8 * s), C.c_void_p(stream.cuda_stream))
        assert rc == 0, f"zg_rect_step_noalloc returned {rc}"
    torch.cuda.synchronize(dev)
    d = dts.cpu().numpy()
    return [(float(d[s]), [t.cpu().numpy() for t in bufs[s + 1]]) for s in range(steps)]


CASES = [
    # nx, ny, box, bounds (L, R, B, T), flux, CFL, workload
    (64, 48, (0.0, 1.0, 0.0, 0.75), (2, 2, 1, 1), 3, 0.4, "random"),
    (96, 96, (0.0, 1.0, 0.0, 1.0), (3, 3, 3, 3), 2, 0.5, "fourier"),
    # the largest axis: the coordinate tables fill the scratch to its end
    (8192, 4, (0.0, 2.0, 0.0, 0.001), (2, 1, 3, 3), 3, 0.4, "random"),
    (4, 8192, (0.0, 0.001, 0.0, 2.0), (3, 3, 1, 2), 3, 0.4, "random"),
    # stiffened gas (P0, e0 and the minimum pressure from the parameters), walls and ZOE
    (40, 32, (0.0, 0.1, 0.0, 0.08), (1, 2, 2, 1), 3, 0.4, "water"),
    # the other fluxes of the parity kernels
    (48, 40, (0.0, 1.0, 0.0, 1.0), (2, 2, 1, 1), 1, 0.4, "random"),
    (48, 40, (0.0, 1.0, 0.0, 1.0), (3, 3, 2, 2), 6, 0.4, "random"),
]
IDS = ["random_64x48_hllc_walls", "fourier_96_hll_periodic", "random_8192x4_max_x", "random_4x8192_max_y",
       "water_40x32_walls_zoe", "random_48x40_rusanov", "random_48x40_cir1"]


@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_noalloc_step_matches_zg_smf_update(gpu_lib, case):
    Z = gpu_lib
    from zephyr_b200.workloads import fourier_smooth

    nx, ny, box, bounds, flux, CFL, kind = case
    stiff = kind == "water"
    if kind == "water":
        rng = np.random.default_rng(23)
        n = nx * ny
        rho = 1000.0 * (1.0 + 0.01 * rng.random(n))
        u, v = 5.0 * rng.standard_normal(n), 5.0 * rng.standard_normal(n)
        p = 1.0e5 * (1.0 + rng.random(n))
        state = (rho, u, v, p, (p + WATER[0] * WATER[1]) / ((WATER[0] - 1.0) * rho))
    elif kind == "random":
        rng = np.random.default_rng(17)
        n = nx * ny
        rho = 1.0 + 0.3 * rng.random(n)
        u, v = 0.2 * rng.standard_normal(n), 0.2 * rng.standard_normal(n)
        p = 1.0 + 0.5 * rng.random(n)
        state = (rho, u, v, p, p / (0.4 * rho))
    else:
        state = tuple(np.asarray(a) for a in fourier_smooth(nx).state)
    want = _existing_path(Z, nx, ny, box, bounds, flux, CFL, state, 2, stiff)
    got = _noalloc_path(Z, nx, ny, box, bounds, flux, CFL, state, 2, stiff)
    for (dt_w, st_w), (dt_g, st_g) in zip(want, got):
        assert abs(dt_g - dt_w) <= TOLERANCE * abs(dt_w)
        for a, b in zip(st_g, st_w):
            np.testing.assert_allclose(a, b, rtol=TOLERANCE, atol=0.0)


def test_noalloc_rejects_meshes_above_its_maximum(gpu_lib):
    from zephyr_b200 import _lib

    lib = gpu_lib.load()
    p = _lib.SmfParams()
    lib.zg_smf_default_params(C.byref(p))
    b = (C.c_int * 4)(2, 2, 2, 2)
    null5 = (C.c_void_p * 5)()
    for nx, ny in ((8193, 16), (16, 8193)):
        rc = lib.zg_rect_step_noalloc(0, nx, ny, 0.0, 1.0, 0.0, 1.0, b, C.byref(p), null5, null5, None, None)
        assert rc == -6  # ZG_ERR_TOO_LARGE
