"""Shared driver of the adaptation tests (test harness only): one schedule of
SmFluid::set_flags / EuMesh::refine / SmFluid::update calls and random flag
rounds, run on any mesh object with the same methods -- the GPU mesh
(zephyr_b200.smf.EuMesh + SmFluid) or the reference's EuMesh compiled from
its sources (oracle.ref_mesh.RefEuMesh) -- and digests of the adapted mesh
after every call, so that a run can be pinned to the reference's by
fixture."""
from __future__ import annotations

import hashlib

import numpy as np

CELL_KEYS = ("cx", "cy", "vol", "inc", "level", "flag", "b_idx", "z_idx")
MAP_KEYS = ("vx", "vy")
FACE_KEYS = ("boundary", "neib", "nx", "ny", "fx", "fy", "area")
MESH_KEYS = CELL_KEYS + MAP_KEYS + FACE_KEYS
STATE_KEYS = ("rho", "vx", "vy", "p", "e", "wait")


def init_state(cx, cy, gamma=1.4):
    """A blast (p = 10 inside r < 0.12 around (0.45, 0.55), 0.1 outside) over
    a smooth density and velocity field, so that every limited gradient the
    slope distributor uses is non-zero."""
    r = np.hypot(cx - 0.45, cy - 0.55)
    rho = 1.0 + 0.3 * np.sin(2 * np.pi * cx) * np.cos(2 * np.pi * cy) + 0.5 * (r < 0.2)
    u = 0.2 * np.cos(2 * np.pi * cy)
    v = -0.15 * np.sin(2 * np.pi * cx)
    p = np.where(r < 0.12, 10.0, 0.1)
    return rho, u, v, p, p / ((gamma - 1.0) * rho)


def random_flags(n, seed):
    """Seeded flags in {-1, 0, 1}, mostly -1 (coarsening), some out of range."""
    rng = np.random.default_rng(seed)
    f = rng.integers(-1, 2, n).astype(np.int32)
    f[rng.random(n) < 0.45] = -1
    f[rng.random(n) < 0.02] = 3
    f[rng.random(n) < 0.02] = -4
    return f


def canonical(g):
    """Arrays of a mesh with the UNDEFINED face slots' contents zeroed and
    signed zeros folded (int64 / float64)."""
    act = np.asarray(g["boundary"]) != -1
    out = {}
    for k in MESH_KEYS:
        a = np.asarray(g[k])
        if k in FACE_KEYS[1:]:
            a = np.where(act, a, 0)
        out[k] = a.astype(np.float64) + 0.0 if a.dtype.kind == "f" else a.astype(np.int64)
    return out


def digest(arrays):
    return {k: hashlib.sha256(np.ascontiguousarray(v).tobytes()).hexdigest()[:20] for k, v in arrays.items()}


class RefAdapter:
    """oracle.ref_mesh.RefEuMesh behind the schedule's methods."""

    def __init__(self, ref):
        self.r = ref

    def n(self):
        return self.r.n

    def mesh(self):
        g = self.r.cells()
        g.update(self.r.faces())
        g["vx"], g["vy"] = self.r.verts()
        return g

    def state(self):
        s = self.r.state()
        return dict(zip(STATE_KEYS, [*s, self.r.wait()]))

    def set_state(self, *s):
        self.r.set_state(*s)

    def set_flags(self):
        return self.r.solver_flags()

    def put_flags(self, f):
        self.r.put_flags(f)

    def refine(self):
        self.r.refine()

    def step(self):
        return self.r.step()


class GpuAdapter:
    """zephyr_b200.smf.EuMesh with its SmFluid behind the schedule's methods."""

    def __init__(self, mesh, solver):
        self.m, self.s = mesh, solver

    def n(self):
        return self.m.n_cells()

    def mesh(self):
        return self.m.amr_arrays()

    def state(self):
        s = self.m.get_state()
        return dict(zip(STATE_KEYS, [*s, self.m.get_wait()]))

    def set_state(self, *s):
        self.m.set_state(*s)

    def set_flags(self):
        return self.s.set_flags(self.m)

    def put_flags(self, f):
        self.m.put_flags(f)

    def refine(self):
        self.m.refine()

    def step(self):
        self.s.update(self.m)
        return self.s.dt()


def schedule(cycles, steps_per_cycle, random_rounds, seed=100):
    """The calls of one run: `cycles` times set_flags, refine and
    `steps_per_cycle` steps; then `random_rounds` refines with random flags;
    then two steps."""
    ops = []
    for _ in range(cycles):
        ops += ["set_flags", "refine"] + ["step"] * steps_per_cycle
    ops += [f"random:{seed + k}" for k in range(random_rounds)]
    ops += ["step", "step"]
    return ops


def run(adapter, ops, on_event=None):
    """Run `ops` from the base mesh with init_state at the cell centres.
    After the base mesh and after every call, on_event(label, adapter) is
    called; the run returns the list of (label, n, mesh digest, state digest,
    flags or dt)."""
    g = adapter.mesh()
    adapter.set_state(*init_state(g["cx"], g["cy"]))
    log = []

    def event(label, extra=None):
        g = adapter.mesh()
        entry = (label, adapter.n(), digest(canonical(g)), digest(adapter.state()), extra)
        log.append(entry)
        if on_event:
            on_event(label, adapter, g)

    event("base")
    for k, op in enumerate(ops):
        if op == "set_flags":
            f = adapter.set_flags()
            event(f"{k}:set_flags", digest({"flags": np.asarray(f, np.int64)})["flags"])
        elif op == "refine":
            adapter.refine()
            event(f"{k}:refine")
        elif op == "step":
            dt = adapter.step()
            event(f"{k}:step", float(dt))
        elif op.startswith("random:"):
            adapter.put_flags(random_flags(adapter.n(), int(op.split(":")[1])))
            adapter.refine()
            event(f"{k}:{op}")
        else:
            raise ValueError(op)
    return log
