"""Slab decomposition of a rectangle across ranks, one GPU per rank.

The reference runs its step on several MPI ranks: each rank owns part of the
mesh and, before each stage, mesh.sync() refreshes the layer of neighbour
cells it reads from the other ranks (math/solver/sm_fluid.cpp:86-97,
mesh/euler/tourism.h), and compute_dt takes the minimum over ranks
(mpi::min, sm_fluid.cpp:113).  Here the rectangle is cut into slabs of whole
rows (rows run along x; cell (i, j) is i * ny + j, so a row block is
contiguous in memory):

- rank r owns rows [i_lo, i_hi) and keeps `halo` ghost rows on each side
  that has a neighbour (both sides on an x-periodic rectangle, the inner
  sides otherwise): as many rows as one step reads away from a cell
  (halo_rows: 2 for the predictor-corrector, 4 for Heun's two stages, 1 for
  first order); its local rectangle is those rows, with the global
  boundary flags on the outer sides and ZOE at the ghost ends (the ghost
  rows' own updates are never used);
- once per step the ghost rows are refreshed from the neighbours' owned rows
  (zg_state_rows out, a send / receive, zg_state_rows in): one exchange of
  the step's reach replaces the reference's three syncs of one layer (the
  ghost rows' own updates are garbage and are never read);
- dt: every rank computes the CFL minimum of its rows (owned and ghost, all
  current after the exchange; zg_smf_cfl_min), the ranks take the minimum
  (all-reduce MIN), and each local step is capped at CFL times it
  (zg_smf_set_max_dt), so all ranks take the reference's global dt.

A rank's result equals the single-domain step's on its owned rows: bit for
bit when the local rectangles reproduce the global mesh's coordinates (a
dyadic cell size), to rounding otherwise.

The communicator is pluggable: `TorchComm` uses torch.distributed (NCCL on
GPU buffers, gloo on host buffers; one process per GPU), `LocalComm` runs
several slabs in one process (tests).  A local solver needs get_rows /
put_rows / cfl_min / set_max_dt / update / dt (`GpuSlabSolver` wraps the C
ABI; the tests wrap the oracle the same way).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

HALO = 2
ZOE = 2
PERIODIC = 3


def halo_rows(accuracy: int, heun: bool = False) -> int:
    """Ghost rows one exchange per step needs: the rows a step reads away
    from a cell -- 1 for first order, 2 for the predictor-corrector
    (gradients, then the corrector's faces), 4 for Heun's two stages of
    gradients and faces."""
    if accuracy == 1:
        return 1
    return 4 if heun else 2


@dataclass(frozen=True)
class Slab:
    """The rows of one rank.  Global mesh: nx x ny cells over box, boundary
    flags (left, right, bottom, top) with PERIODIC on both x sides for an
    x-periodic rectangle."""
    nx: int
    ny: int
    box: tuple
    bounds: tuple
    world: int
    rank: int
    halo: int = HALO

    @property
    def xper(self) -> bool:
        return self.bounds[0] == PERIODIC or self.bounds[1] == PERIODIC

    @property
    def rows(self) -> tuple:
        """[i_lo, i_hi): the owned rows, as even as the division allows."""
        base, extra = divmod(self.nx, self.world)
        lo = self.rank * base + min(self.rank, extra)
        return lo, lo + base + (1 if self.rank < extra else 0)

    @property
    def left(self):
        """Rank owning the rows below i_lo, or None."""
        if self.world == 1:
            return None
        if self.rank == 0:
            return self.world - 1 if self.xper else None
        return self.rank - 1

    @property
    def right(self):
        if self.world == 1:
            return None
        if self.rank == self.world - 1:
            return 0 if self.xper else None
        return self.rank + 1

    @property
    def ghosts(self) -> tuple:
        """Ghost rows below and above the owned rows."""
        return (self.halo if self.left is not None else 0, self.halo if self.right is not None else 0)

    @property
    def local_rows(self) -> int:
        lo, hi = self.rows
        gl, gh = self.ghosts
        return hi - lo + gl + gh

    @property
    def local_box(self) -> tuple:
        lo, hi = self.rows
        gl, gh = self.ghosts
        x0, x1, y0, y1 = self.box
        h = (x1 - x0) / self.nx
        return (x0 + (lo - gl) * h, x0 + (hi + gh) * h, y0, y1)

    @property
    def local_bounds(self) -> tuple:
        """Global flags on outer sides; ZOE at ghost ends (a world of one
        keeps the global flags, periodic included)."""
        if self.world == 1:
            return tuple(self.bounds)
        left = ZOE if self.left is not None else self.bounds[0]
        right = ZOE if self.right is not None else self.bounds[1]
        return (left, right, self.bounds[2], self.bounds[3])

    def owned_local(self) -> tuple:
        """[first, last) local rows that this rank owns."""
        gl, _ = self.ghosts
        lo, hi = self.rows
        return gl, gl + hi - lo


class LocalComm:
    """All slabs of a run in one process: the exchange copies rows between
    the local solvers directly."""

    def __init__(self):
        self.members = {}

    def join(self, rank, stepper):
        self.members[rank] = stepper

    def exchange_all(self):
        inbox = {r: {} for r in self.members}
        for r, st in self.members.items():
            for dest, rows in st.outgoing():
                inbox[dest].setdefault(r, []).append(rows)
        for r, st in self.members.items():
            st.incoming(inbox[r])


class TorchComm:
    """torch.distributed: point-to-point sends of the ghost rows and an
    all-reduce MIN of the CFL minimum.  Buffers live on `device` (a CUDA
    device for NCCL, "cpu" for gloo)."""

    def __init__(self, device="cpu", group=None):
        import torch
        self.torch = torch
        self.device = torch.device(device)
        self.group = group

    def exchange(self, stepper):
        torch = self.torch
        dist = torch.distributed
        ops, recvs = [], []
        for dest, (f, w) in stepper.outgoing():
            tf = torch.as_tensor(f, device=self.device)
            tw = torch.as_tensor(w, device=self.device)
            ops += [dist.P2POp(dist.isend, tf, dest, self.group), dist.P2POp(dist.isend, tw, dest, self.group)]
        for src, shape_f, shape_w in stepper.expected():
            rf = torch.empty(shape_f, dtype=torch.float64, device=self.device)
            rw = torch.empty(shape_w, dtype=torch.int32, device=self.device)
            ops += [dist.P2POp(dist.irecv, rf, src, self.group), dist.P2POp(dist.irecv, rw, src, self.group)]
            recvs.append((src, rf, rw))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()
        device_rows = getattr(stepper.local, "device_rows", False) and self.device.type == "cuda"
        inbox = {}
        for src, rf, rw in recvs:  # in posting order: messages of one peer stay in the order sent
            inbox.setdefault(src, []).append((rf, rw) if device_rows else (rf.cpu().numpy(), rw.cpu().numpy()))
        stepper.incoming(inbox)

    def min_all(self, value: float) -> float:
        t = self.torch.tensor([value], dtype=self.torch.float64, device=self.device)
        self.torch.distributed.all_reduce(t, op=self.torch.distributed.ReduceOp.MIN, group=self.group)
        return float(t.item())


class SlabStepper:
    """One rank's slab: its local solver, the halo exchange and the global
    dt.  With a LocalComm, call `LocalComm.exchange_all` and `step_all`
    instead of `step`."""

    def __init__(self, slab: Slab, local, comm, CFL: float, max_dt: float = float(np.finfo(np.float64).max)):
        self.slab, self.local, self.comm = slab, local, comm
        self.CFL, self.max_dt = CFL, max_dt
        self.dt = float("nan")

    # -- rows leaving and entering this slab --------------------------------
    def outgoing(self):
        """(destination rank, (fields, wait)) of the owned rows each
        neighbour keeps as ghosts.  A neighbour on both sides (two ranks,
        periodic) gets two messages, low side first."""
        s, H = self.slab, self.slab.halo
        first, last = s.owned_local()
        out = []
        if s.left is not None:
            out.append((s.left, self.local.get_rows(first, H)))
        if s.right is not None:
            out.append((s.right, self.local.get_rows(last - H, H)))
        return out

    def expected(self):
        s, H = self.slab, self.slab.halo
        n = H * s.ny
        return [(r, (5 * n,), (n,)) for r in (s.left, s.right) if r is not None]

    def incoming(self, msgs):
        """Rows from the neighbours into the ghost rows; msgs maps a source
        rank to its messages in the order sent.  A left neighbour sends its
        high rows (our low ghosts), a right one its low rows (our high
        ghosts); one neighbour on both sides (two ranks, periodic) sends its
        low rows first, then its high rows."""
        s, H = self.slab, self.slab.halo
        first, last = s.owned_local()
        if s.left is not None and s.left == s.right:
            lo_msg, hi_msg = msgs[s.left]
            self.local.put_rows(last, *lo_msg)
            self.local.put_rows(first - H, *hi_msg)
            return
        if s.left is not None:
            self.local.put_rows(first - H, *msgs[s.left][0])
        if s.right is not None:
            self.local.put_rows(last, *msgs[s.right][0])

    # -- the step ----------------------------------------------------------
    def step(self):
        """Halo exchange, global dt, local step (torch.distributed comm)."""
        self.comm.exchange(self)
        dmin = self.comm.min_all(self.local.cfl_min())
        self._advance(dmin)
        return self.dt

    def _advance(self, dmin_global):
        self.local.set_max_dt(min(self.CFL * dmin_global, self.max_dt))
        self.local.update()
        self.dt = self.local.dt()

    def owned_state(self):
        """(fields (5, rows * ny), wait) of the owned rows, in host memory."""
        first, last = self.slab.owned_local()
        f, w = self.local.get_rows(first, last - first)
        if hasattr(f, "cpu"):
            f, w = f.cpu().numpy(), w.cpu().numpy()
        return np.asarray(f).reshape(5, -1), np.asarray(w)


def step_all(comm: LocalComm):
    """One step of every slab of an in-process run."""
    comm.exchange_all()
    dmin = min(st.local.cfl_min() for st in comm.members.values())
    for st in comm.members.values():
        st._advance(dmin)


class GpuSlabSolver:
    """The local solver of a slab on one GPU, through the C ABI (FP64 FAST or
    PARITY kernels): a rectangle of the slab's local rows, zg_state_rows for
    the ghost rows, zg_smf_cfl_min, zg_smf_set_max_dt.

    device_rows: the rows leave and enter as torch tensors on the slab's GPU
    (zg_state_rows copies device to device), so a TorchComm on that device
    sends them with NCCL without a host round trip; otherwise they are numpy
    arrays in host memory."""

    def __init__(self, slab: Slab, eos, configure, precision=None, kernels=None, device=0, stream=None,
                 device_rows=False):
        from . import smf as Z
        gen = Z.Rectangle(*slab.local_box)
        gen.set_boundaries(Z.Boundaries(*slab.local_bounds))
        gen.set_sizes(slab.local_rows, slab.ny)
        self.Z = Z
        self.mesh = Z.EuMesh(gen, device=device, stream=stream)
        self.solver = Z.SmFluid(eos, precision=precision or Z.Precision.FP64,
                                kernels=kernels if kernels is not None else Z.Kernels.FAST)
        configure(self.solver)
        self.solver.add_types(self.mesh)
        self.ny = slab.ny
        self.device = device
        self.device_rows = device_rows

    def set_state(self, rho, u, v, p, e, wait=None):
        self.mesh.set_state(rho, u, v, p, e)
        if wait is not None:
            self.mesh.set_wait(wait)

    def get_rows(self, row0, nrows):
        n = nrows * self.ny
        if self.device_rows:
            import torch
            dev = torch.device("cuda", self.device)
            f = torch.empty(5 * n, dtype=torch.float64, device=dev)
            w = torch.empty(n, dtype=torch.int32, device=dev)
        else:
            f = np.empty(5 * n)
            w = np.empty(n, np.int32)
        self._rows(row0, nrows, f, w, 0)
        return f, w

    def put_rows(self, row0, f, w):
        if hasattr(f, "data_ptr"):  # torch tensors (device or host)
            f = f.to(dtype=self._torch().float64).contiguous()
            w = w.to(dtype=self._torch().int32).contiguous()
            nrows = w.numel() // self.ny
        else:
            f = np.ascontiguousarray(f, dtype=np.float64)
            w = np.ascontiguousarray(w, dtype=np.int32)
            nrows = len(w) // self.ny
        self._rows(row0, nrows, f, w, 1)

    @staticmethod
    def _torch():
        import torch
        return torch

    def _rows(self, row0, nrows, f, w, put):
        from ._lib import check
        if hasattr(f, "data_ptr"):
            # the copies run on the library's stream; the tensors must be
            # complete on torch's stream first (zg_state_rows synchronises
            # its own stream before it returns)
            if f.is_cuda:
                self._torch().cuda.current_stream(f.device).synchronize()
            fp = C.cast(C.c_void_p(f.data_ptr()), C.POINTER(C.c_double))
            wp = C.cast(C.c_void_p(w.data_ptr()), C.POINTER(C.c_int))
        else:
            fp = f.ctypes.data_as(C.POINTER(C.c_double))
            wp = w.ctypes.data_as(C.POINTER(C.c_int))
        check(self.mesh.ctx, self.mesh._lib.zg_state_rows(self.mesh.ctx, int(row0), int(nrows), fp, wp, int(put)))

    def cfl_min(self):
        from ._lib import check
        d = C.c_double()
        check(self.mesh.ctx, self.mesh._lib.zg_smf_cfl_min(self.mesh.ctx, C.byref(d)))
        return d.value

    def set_max_dt(self, dt):
        self.solver.set_max_dt(dt)

    def update(self):
        self.solver.update(self.mesh)

    def dt(self):
        return self.solver.dt()

    def close(self):
        self.mesh.close()
