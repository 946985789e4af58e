"""Slab decomposition on the GPU (zg_state_rows, zg_smf_cfl_min): several
slabs of one rectangle, each with its own context on the same GPU, joined by
the in-process communicator (LocalComm: the exchange copies rows through host
buffers or device tensors, no kernel waits on another), against the single-domain GPU step
with the same kernels.  Dyadic cell size: every owned cell and every dt bit
for bit."""
import numpy as np
import pytest

from zephyr_b200 import slabs as S

pytestmark = pytest.mark.gpu

CASES = [
    # nx, ny, bounds, accuracy, scheme, kernels
    ("fused periodic predictor-corrector", 128, 64, (3, 3, 3, 3), 2, 0, "FAST"),
    ("fused walls heun", 128, 32, (1, 2, 3, 3), 2, 1, "FAST"),
    ("parity zoe second order", 64, 32, (2, 2, 1, 2), 2, 0, "PARITY"),
    ("two-pass periodic", 64, 64, (3, 3, 3, 3), 2, 0, "FAST_TWO_PASS"),
]


def initial(nx, ny, seed=5):
    rng = np.random.default_rng(seed)
    n = nx * ny
    rho = 1.0 + 0.3 * rng.random(n)
    u = 0.3 * rng.standard_normal(n)
    v = 0.3 * rng.standard_normal(n)
    p = 1.0 + 0.5 * rng.random(n)
    return rho, u, v, p, p / (0.4 * rho)


@pytest.mark.parametrize("device_rows", [False, True], ids=["host rows", "device rows"])
@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("name,nx,ny,bounds,acc,scheme,kern", CASES, ids=[c[0] for c in CASES])
def test_gpu_slabs_match_the_single_domain(gpu_lib, name, nx, ny, bounds, acc, scheme, kern, world, device_rows):
    Z = gpu_lib
    steps = 8

    def configure(s):
        s.set_accuracy(acc)
        s.set_CFL(0.4)
        s.set_limiter("van Albada")
        s.set_scheme(Z.Scheme(scheme))

    st0 = initial(nx, ny)
    whole = S.GpuSlabSolver(S.Slab(nx, ny, (0.0, 1.0, 0.0, 1.0), bounds, 1, 0), Z.IdealGas(1.4), configure,
                            kernels=Z.Kernels[kern])
    whole.set_state(*st0)
    dts = []
    for _ in range(steps):
        whole.update()
        dts.append(whole.dt())
    want = np.array(whole.mesh.get_state())
    whole.close()

    comm = S.LocalComm()
    for r in range(world):
        slab = S.Slab(nx, ny, (0.0, 1.0, 0.0, 1.0), bounds, world, r, halo=S.halo_rows(acc, scheme == 1))
        loc = S.GpuSlabSolver(slab, Z.IdealGas(1.4), configure, kernels=Z.Kernels[kern], device_rows=device_rows)
        lo, hi = slab.rows
        gl, gh = slab.ghosts
        idx = np.concatenate([np.arange((i % nx) * ny, (i % nx + 1) * ny) for i in range(lo - gl, hi + gh)])
        loc.set_state(*[a[idx] for a in st0])
        comm.join(r, S.SlabStepper(slab, loc, comm, CFL=0.4))
    for k in range(steps):
        S.step_all(comm)
        got_dt = {st.dt for st in comm.members.values()}
        assert got_dt == {dts[k]}, (k, got_dt, dts[k])
    got = np.concatenate([comm.members[r].owned_state()[0] for r in range(world)], axis=1)
    bad = got != want
    assert not bad.any(), f"{int(bad.sum())} values differ"
    for st in comm.members.values():
        st.local.close()
