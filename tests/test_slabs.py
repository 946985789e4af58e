"""Slab decomposition (zephyr_b200/slabs.py) on the host: the partition, the
halo exchange of two rows per step and the global dt, with the oracle as
each rank's local solver, against the single-domain oracle.  On a dyadic
cell size the local rectangles reproduce the global coordinates, so every
owned cell and every dt must agree bit for bit.  Runs in one process
(LocalComm) and as world_size 2 and 3 gloo ranks (TorchComm)."""
import os

import numpy as np
import pytest

from oracle import oracle as O
from zephyr_b200 import slabs as S

CASES = [
    # nx, ny, bounds, accuracy, limiter id, steps
    ("periodic second order", 64, 32, (3, 3, 3, 3), 2, 5, 8),
    ("walls zoe second order", 64, 24, (1, 2, 3, 3), 2, 3, 8),
    ("zoe first order", 32, 16, (2, 2, 1, 2), 1, 3, 10),
]


class OracleSlab:
    """The oracle as the local solver of a slab."""

    def __init__(self, slab, accuracy, limiter, CFL):
        self.ny = slab.ny
        self.mesh = O.Mesh(slab.local_rows, slab.ny, *slab.local_box, bounds=slab.local_bounds)
        self.s = O.Solver(self.mesh, limiter=limiter, accuracy=accuracy, CFL=CFL)
        self._dt = float("nan")

    def set_state(self, *st):
        self.s.set_state(*st)

    def get_rows(self, row0, nrows):
        a, b = row0 * self.ny, (row0 + nrows) * self.ny
        return np.concatenate([f[a:b] for f in self.s.state()]), self.s.wait()[a:b].copy()

    def put_rows(self, row0, f, w):
        a = row0 * self.ny
        n = len(w)
        st = self.s.state()
        for k in range(5):
            st[k][a:a + n] = f[k * n:(k + 1) * n]
        wt = self.s.wait()
        wt[a:a + n] = w
        self.s.set_state(*st)
        self.s.set_wait(wt)

    def cfl_min(self):
        return self.s.cfl_min()

    def set_max_dt(self, dt):
        self.s.set_max_dt(dt)

    def update(self):
        self._dt = self.s.step()

    def dt(self):
        return self._dt


def initial(nx, ny, seed=3):
    rng = np.random.default_rng(seed)
    n = nx * ny
    rho = 1.0 + 0.3 * rng.random(n)
    u = 0.3 * rng.standard_normal(n)
    v = 0.3 * rng.standard_normal(n)
    p = 1.0 + 0.5 * rng.random(n)
    return rho, u, v, p, p / (0.4 * rho)


def reference(nx, ny, bounds, acc, lim, steps):
    s = O.Solver(O.Mesh(nx, ny, bounds=bounds), limiter=lim, accuracy=acc, CFL=0.4)
    s.set_state(*initial(nx, ny))
    dts = [s.step() for _ in range(steps)]
    return np.array(s.state()), dts


def local_slab(nx, ny, bounds, world, rank, acc, lim):
    slab = S.Slab(nx, ny, (0.0, 1.0, 0.0, 1.0), bounds, world, rank, halo=S.halo_rows(acc))
    loc = OracleSlab(slab, acc, lim, 0.4)
    lo, hi = slab.rows
    gl, gh = slab.ghosts
    rows = [(i % nx) for i in range(lo - gl, hi + gh)]
    idx = np.concatenate([np.arange(i * ny, (i + 1) * ny) for i in rows])
    loc.set_state(*[a[idx] for a in initial(nx, ny)])
    return slab, loc


def test_partition_covers_the_rows_once():
    for nx, world in ((64, 3), (10, 4), (7, 7)):
        rows = [S.Slab(nx, 4, (0, 1, 0, 1), (3, 3, 3, 3), world, r).rows for r in range(world)]
        assert rows[0][0] == 0 and rows[-1][1] == nx
        assert all(a[1] == b[0] for a, b in zip(rows, rows[1:]))
        assert max(h - l for l, h in rows) - min(h - l for l, h in rows) <= 1


@pytest.mark.parametrize("world", [2, 3, 4])
@pytest.mark.parametrize("name,nx,ny,bounds,acc,lim,steps", CASES, ids=[c[0] for c in CASES])
def test_slabs_in_one_process_match_the_single_domain(name, nx, ny, bounds, acc, lim, steps, world):
    comm = S.LocalComm()
    for r in range(world):
        slab, loc = local_slab(nx, ny, bounds, world, r, acc, lim)
        comm.join(r, S.SlabStepper(slab, loc, comm, CFL=0.4))
    want, dts = reference(nx, ny, bounds, acc, lim, steps)
    for k in range(steps):
        S.step_all(comm)
        got_dt = {st.dt for st in comm.members.values()}
        assert got_dt == {dts[k]}, (k, got_dt, dts[k])
    got = np.concatenate([comm.members[r].owned_state()[0].reshape(5, -1) for r in range(world)], axis=1)
    assert np.array_equal(got, want)


def _rank_main(rank, world, port, case, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        name, nx, ny, bounds, acc, lim, steps = case
        slab, loc = local_slab(nx, ny, bounds, world, rank, acc, lim)
        st = S.SlabStepper(slab, loc, S.TorchComm("cpu"), CFL=0.4)
        dts = [st.step() for _ in range(steps)]
        f, _ = st.owned_state()
        np.savez(os.path.join(out, f"rank{rank}.npz"), f=f, dts=np.array(dts))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("case", CASES[:2], ids=[c[0] for c in CASES[:2]])
def test_slabs_as_gloo_ranks_match_the_single_domain(tmp_path, case, world):
    import socket

    import torch.multiprocessing as mp
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    mp.start_processes(_rank_main, args=(world, port, case, str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    name, nx, ny, bounds, acc, lim, steps = case
    want, dts = reference(nx, ny, bounds, acc, lim, steps)
    parts = [np.load(tmp_path / f"rank{r}.npz") for r in range(world)]
    for p in parts:
        assert np.array_equal(p["dts"], np.array(dts))
    got = np.concatenate([p["f"] for p in parts], axis=1)
    assert np.array_equal(got, want)
