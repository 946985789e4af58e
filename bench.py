#!/usr/bin/env python
"""Benchmark of the finite-volume step (cell-updates/s) on one or more GPUs.

Default workload (the config the metric is quoted on): 2048 x 2048 periodic
cells, smooth seeded Fourier data, second order (LSM gradients + van Albada
limiting + HLLC), CFL 0.4, FP64.  One step = SmFluid::update on every cell.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--scheme pc|heun] [--workload fourier2048|riemann256]

Multi-GPU (torchrun): every rank runs an independent replica of the whole
workload (weak scaling); the timed region is bracketed by a barrier and a
device synchronise, and the time is the maximum over ranks.

Output: one JSON line on rank 0.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "cell-updates/s"
PEAKS_FILE = ROOT / "MEASURED_PEAKS.json"
TRAFFIC_FILE = ROOT / "profiles" / "traffic_per_cell.txt"
FALLBACK_HBM_GBS = 6650.0

# Algorithmic bytes per cell and launch (the model: each pass reads the
# persistent state it needs once and writes its result once; 2-D conserved
# state = 4 doubles).  Kernels that the model folds into others carry 0.
B_ALG_KERNEL = {"dt": 0, "flux1": 64, "grad": 0, "stage1": 64, "stage2": 96, "heun_a": 64, "heun_b": 96,
                "flags": 0, "step": 160}
# (the two-pass predictor "stage1" is fused with the gradients; the corrector
# "stage2" carries the next step's CFL minimum; the fused FAST/MIXED kernel
# "step" is the whole predictor-corrector step of a rectangle in one launch,
# so one launch processes the model's two passes: 160 B per cell)
B_ALG_STEP = {1: 64, 2: 160}
# FP64 pipe of B200: 64 FP64 thread-instructions per SM and cycle
FP64_INST_PER_SM_CYCLE = 64
N_SM = 148


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["fourier2048", "riemann256"], default="fourier2048")
    ap.add_argument("--size", type=int, default=0, help="override the mesh size (n x n) for small profiling runs")
    ap.add_argument("--scheme", choices=["pc", "heun"], default="pc")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    # profiling aids: one section alone on a smaller case (not the bench line)
    ap.add_argument("--only", choices=["forms", "amr", "mm", "adjoint", "transfer", "vtu"], default=None,
                    help="run one section alone and print its JSON (for ncu captures)")
    ap.add_argument("--amr-base", type=int, default=0, help="AMR base cells per side (default 512)")
    ap.add_argument("--tr-nx", type=int, default=0, help="transport mesh cells along x (default 4096)")
    ap.add_argument("--amr-kernels", choices=["fast", "mixed", "parity"], default="fast")
    ap.add_argument("--mm-accuracy", type=int, choices=[1, 2], default=1, help="MmFluid order with --only mm")
    ap.add_argument("--amr-criterion", choices=["gradient", "reference"], default="gradient")
    return ap.parse_args()


def workload(name, size=0):
    from zephyr_b200.workloads import fourier_smooth, riemann2d_case3
    if name == "fourier2048":
        return fourier_smooth(size or 2048), dict(acc=2, lim="van Albada", CFL=0.4, lim_id=5, bounds=(3, 3, 3, 3))
    return riemann2d_case3(size or 256), dict(acc=1, lim="MC", CFL=0.4, lim_id=3, bounds=(2, 2, 2, 2))


def config_of(args, w, cfg, n_gpus):
    return {
        "workload": f"{w.name} {w.gen.nx()}x{w.gen.ny()}",
        "cells": w.gen.nx() * w.gen.ny(),
        "accuracy": cfg["acc"],
        "scheme": "predictor-corrector (reference)" if args.scheme == "pc" else "heun (extension)",
        "flux": "HLLC",
        "limiter": cfg["lim"],
        "CFL": cfg["CFL"],
        "boundaries": "periodic" if cfg["bounds"][0] == 3 else "transmissive (ZOE)",
        "l2": "working set larger than L2 (no flush)",
        "parallelism": f"replicas x{n_gpus}",
    }


# ---------------------------------------------------------------------------
class ClockSampler:
    """SM clocks and clock-event (throttle) reasons sampled through NVML in a
    background thread while the timed region runs (read-only queries)."""

    REASONS = {"hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40,
               "sw_power_cap": 0x4, "hw_power_brake_slowdown": 0x80}

    def __init__(self, index):
        self.index = index
        self.samples = []
        self.stop_flag = threading.Event()
        self.thread = None

    def start(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = None
            try:  # the CUDA device's own GPU, whatever CUDA_VISIBLE_DEVICES maps it to
                import torch
                uuid = str(torch.cuda.get_device_properties(self.index).uuid)
                self.h = pynvml.nvmlDeviceGetHandleByUUID(("GPU-" + uuid).encode())
            except Exception:
                self.h = pynvml.nvmlDeviceGetHandleByIndex(self.index)
            self.max_sm = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
        except Exception:
            self.nv = None
            return
        self.thread = threading.Thread(target=self._run, daemon=True)
        self.thread.start()

    def _run(self):
        nv = self.nv
        while not self.stop_flag.is_set():
            try:
                sm = nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)
                rs = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                self.samples.append((sm, rs))
            except Exception:
                pass
            time.sleep(0.002)

    def stop(self):
        if self.thread is None:
            return None
        self.stop_flag.set()
        self.thread.join(timeout=2)
        if not self.samples:
            return None
        sm = [s for s, _ in self.samples]
        reasons = sorted({name for _, r in self.samples for name, bit in self.REASONS.items() if r & bit})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": self.max_sm, "reasons": reasons,
                "samples": len(sm), "source": "NVML during the timed region"}


# ---------------------------------------------------------------------------
def hbm_peak():
    try:
        d = json.loads(PEAKS_FILE.read_text())
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def traffic_per_cell(kernel, column=1):
    """dram read+write bytes per cell of `kernel` (column 1), or its FP64
    thread-instructions per cell (column 2) and FP64 pipe activity in per cent
    (column 3), from the committed ncu summaries."""
    try:
        for ln in TRAFFIC_FILE.read_text().splitlines():
            parts = ln.split()
            if len(parts) > column and parts[0] == kernel and not ln.startswith("#"):
                return float(parts[column])
    except (OSError, ValueError):
        pass
    return None


def cpu_solver(w, cfg, scheme, threads):
    """The reference's own SmFluid compiled from its sources (oracle/_ref,
    kind "reference") when that build exists and the scheme is the
    reference's; otherwise the oracle restatement (kind "port")."""
    gen = w.gen
    if scheme == "pc":
        from oracle import ref as R
        if R.available():
            r = R.RefSolver(gen.nx(), gen.ny(), box=(gen.x_min, gen.x_max, gen.y_min, gen.y_max),
                            bounds=cfg["bounds"], accuracy=cfg["acc"], limiter=cfg["lim"], CFL=cfg["CFL"])
            r.set_threads(threads)
            r.set_state(*w.state)
            return r, "reference", "zephyr's SmFluid::update compiled from its sources (oracle/_ref)"
    from oracle import oracle as O
    om = O.Mesh(gen.nx(), gen.ny(), gen.x_min, gen.x_max, gen.y_min, gen.y_max, cfg["bounds"])
    osv = O.Solver(om, gamma=1.4, flux=O.FLUX_HLLC, limiter=cfg["lim_id"], accuracy=cfg["acc"],
                   scheme=0 if scheme == "pc" else 1, CFL=cfg["CFL"], threads=threads)
    osv.set_state(*w.state)
    osv._keep = om
    return osv, "port", "oracle restatement of the reference step"


def cpu_baseline(w, cfg, scheme, budget_s=12.0):
    """The reference's CPU path on this host's cores, on a bounded sample."""
    threads = os.cpu_count() or 1
    solver, kind, what = cpu_solver(w, cfg, scheme, threads)
    t0 = time.perf_counter()
    solver.step()
    t1 = time.perf_counter()
    steps = 1
    per = t1 - t0
    extra = max(0, min(20, int(budget_s / max(per, 1e-3)) - 1))
    if extra:
        t0 = time.perf_counter()
        solver.steps(extra)
        t1 = time.perf_counter()
        steps = extra
        per = (t1 - t0) / extra
    cells = w.gen.nx() * w.gen.ny()
    return {"value": cells / per, "unit": METRIC, "cores": threads, "kind": kind,
            "sample": f"{steps} step(s) of the full {w.gen.nx()}x{w.gen.ny()} workload after 1 untimed step; "
                      f"{what}; {threads} std::threads"}


# ---------------------------------------------------------------------------
def run_reference(args, rank, world):
    if rank != 0:
        return
    w, cfg = workload(args.workload, args.size)
    threads = os.cpu_count() or 1
    solver, kind, what = cpu_solver(w, cfg, args.scheme, threads)
    for _ in range(args.warmup):
        solver.step()
    t0 = time.perf_counter()
    solver.steps(args.steps)
    t1 = time.perf_counter()
    cells = w.gen.nx() * w.gen.ny()
    sec = t1 - t0
    value = cells * args.steps / sec
    sample = f"{args.steps} full steps of the {w.gen.nx()}x{w.gen.ny()} workload; {what}; {threads} std::threads"
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": 0,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sec / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config_of(args, w, cfg, 1),
        "cpu_baseline": {"value": value, "unit": METRIC, "cores": threads, "kind": kind, "sample": sample},
        "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference is a CMake C++ project with no Python packaging (pip cannot install it); its "
                "own step code is compiled from its sources against stand-ins for Eigen/Boost and run on the "
                "host cores",
    }
    print(json.dumps(line), flush=True)


def _solver(Z, w, cfg, args, local_rank, stream, precision, kernels):
    mesh = Z.EuMesh(w.gen, device=local_rank, stream=stream.cuda_stream)
    solver = Z.SmFluid(w.eos, precision=precision, kernels=kernels)
    solver.set_accuracy(cfg["acc"])
    solver.set_CFL(cfg["CFL"])
    solver.set_limiter(cfg["lim"])
    solver.set_method(Z.Fluxes.HLLC)
    solver.set_scheme(Z.Scheme.HEUN if args.scheme == "heun" else Z.Scheme.PREDICTOR_CORRECTOR)
    solver.add_types(mesh)
    mesh.set_state(*w.state)
    return mesh, solver


def _timed_steps(torch, lib, mesh, solver, steps, dev, stream, barrier, clocks=False, per_kernel=True):
    """K steps between a barrier + synchronise and CUDA events on the
    library's stream; returns (ms, per-kernel dict, launches, clocks).  With
    per_kernel the library brackets every launch with its own events (the
    split by kernel); without, the steps run bare."""
    from zephyr_b200._lib import KERNEL_KINDS
    sampler = ClockSampler(torch.cuda.current_device()) if clocks else None
    if sampler:
        sampler.start()
    lib.zg_set_timing(mesh.ctx, 1 if per_kernel else 0)
    n0 = mesh.launch_count()
    barrier()
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    solver.update(mesh, steps=steps)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    barrier()
    ms = e0.elapsed_time(e1)
    launches = mesh.launch_count() - n0
    kms = (C.c_double * len(KERNEL_KINDS))()
    kcount = (C.c_longlong * len(KERNEL_KINDS))()
    lib.zg_kernel_times(mesh.ctx, kms, kcount)
    lib.zg_set_timing(mesh.ctx, 0)
    kernels = {}
    tot = max(sum(kms), 1e-12)
    for k, name in enumerate(KERNEL_KINDS):
        if kcount[k]:
            kernels[name] = {"launches": int(kcount[k]), "ms_total": kms[k], "ms_avg": kms[k] / kcount[k],
                             "share": kms[k] / tot}
    return ms, kernels, launches, (sampler.stop() if sampler else None)


HORIZON = 500      # steps of the configuration (accuracy of the mixed form over them)
MM_SIZE = 1024     # shock / water-column problem, cells per side
MM_B_ALG = 160     # bytes per cell and step: 10 FP64 state fields read once and written once
MM2_B_ALG = 320    # second order: the state read by both stages, the half-step state written and read, the next state written


def mm_cpu_reference(w, steps_budget_s=10.0, accuracy=1):
    """The reference's own MmFluid (oracle/_ref) on this host's cores, a few
    steps of the full problem; None when that build is absent."""
    from oracle import ref_mm as RM
    if not RM.available():
        return None
    threads = os.cpu_count() or 1
    r = RM.RefMmFluid(w.nx, w.ny, box=w.box, bounds=w.bounds, materials="stiffened:Water,ideal:Air", CFL=0.4,
                      accuracy=accuracy, crp_mode=4)
    r.set_threads(threads)
    r.make_states(w.rho, w.vx, w.vy, w.p, w.beta)
    t0 = time.perf_counter()
    r.step()
    per = time.perf_counter() - t0
    steps = max(1, min(10, int(steps_budget_s / max(per, 1e-3))))
    t0 = time.perf_counter()
    for _ in range(steps):
        r.step()
    per = (time.perf_counter() - t0) / steps
    return {"value": w.nx * w.ny / per, "unit": METRIC, "cores": threads, "kind": "reference",
            "sample": f"{steps} step(s) of the {w.nx}x{w.ny} problem after 1 untimed step; zephyr's "
                      f"MmFluid::update (accuracy {accuracy}) compiled from its sources (oracle/_ref); "
                      f"{threads} threads"}


def mm_variant(torch, lib, dev, stream, barrier, K, W, local_rank, want_cpu, precision=None, accuracy=1):
    """The multi-material step (MmFluid, CRP + PLIC) on the two-material
    shock / water-column problem, 1024 x 1024; first order in FP64
    (bit-exact) or the mixed form, or second order (FP64, bit-exact, MC
    limiter)."""
    import zephyr_b200 as Z
    from zephyr_b200.mmf import Material, MixturePT, MmFluid
    from zephyr_b200.workloads import shock_water_column
    w = shock_water_column(MM_SIZE)
    gen = Z.Rectangle(*w.box)
    gen.set_boundaries(Z.Boundaries(*w.bounds))
    gen.set_sizes(w.nx, w.ny)
    mesh = Z.EuMesh(gen, device=local_rank, stream=stream.cuda_stream)
    solver = MmFluid(MixturePT([Material.stiffened("Water"), Material.ideal("Air")]))
    solver.set_CFL(0.4)
    solver.set_accuracy(accuracy)
    solver.add_types(mesh)
    if precision is not None:
        solver.set_precision(precision)
    solver.make_states(mesh, w.rho, w.vx, w.vy, w.p, w.beta)
    solver.update(mesh, W)
    mesh.synchronize()
    # timed bare; the kernel split from the next K steps with per-kernel events
    ms, _, launches, _ = _timed_steps(torch, lib, mesh, solver, K, dev, stream, barrier, per_kernel=False)
    _, kernels, _, _ = _timed_steps(torch, lib, mesh, solver, K, dev, stream, barrier)
    solver.dt()  # raises if a step produced a state the reference rejects
    cells = w.nx * w.ny
    out = {"workload": f"shock_water_column {w.nx}x{w.ny} (water column in air, planar shock, "
                       "StiffenedGas Water + IdealGas Air)",
           "form": (("mixed (FP32 pure-stencil face arithmetic)" if precision == Z.Precision.MIXED else
                     "FP64, bit-exact with the reference") +
                    f" (MmFluid {('first', 'second')[accuracy - 1]} order"
                    f"{', MC limiter' if accuracy == 2 else ''}, CRP + PLIC, CFL 0.4)"),
           "ms": ms, "kernels": kernels, "launches": launches, "cells": cells,
           "final": solver.states(mesh) if precision is not None else None}
    mesh.close()
    if want_cpu:
        out["cpu_baseline"] = mm_cpu_reference(w, accuracy=accuracy)
    return out


AMR_BASE = 512         # quadtree AMR blast: base mesh cells per side
AMR_LEVELS = 3         # refinement levels above the base
AMR_CAPACITY = 8 << 20  # device room for cells (live + those held during a refine)
# untimed steps (adapting every AMR_EVERY) before the timed window: by step
# 7000 the gradient criterion holds 1.1-1.2 M live cells (the 1-3 M window of
# the configuration; steps 100-500 have about 0.3 M)
AMR_WARM_STEPS = 7000
AMR_TIMED_STEPS = 400  # steps 7000 to 7400
AMR_EVERY = 10         # set_flags + refine every AMR_EVERY steps
AMR_SPLIT_STEPS = 100  # steps after the timed window that give the per-kernel split
AMR_B_ALG = 160 + 36   # bytes per cell-update: the FP64 two-stage step plus the slot-mesh neighbour indices
AMR_CELL_BYTES = 600   # bytes of one cell's AmrCells arrays (63 doubles, 22 ints, 16 bytes)
AMR_KERNELS = "fast"   # kernel family of the AMR step: "fast" (slot FAST) or "parity" (bit-exact)


def _amr_flags(solver, mesh, criterion):
    if criterion == "gradient":  # |grad rho| h / rho: refine above 0.05, coarsen below 0.01
        solver.set_flags_gradient(mesh, 0.05, 0.01, download=False)
    else:  # SmFluid::set_flags (neighbour jumps)
        solver.set_flags(mesh, download=False)


def _amr_setup(Z, init_state, mesh, solver, criterion="reference"):
    """smf_test_2D.cpp:112-117: max_level + 3 rounds of (initial data by cell
    means, set_flags, refine), then the initial data once more."""
    for _ in range(AMR_LEVELS + 3):
        g = init_state()
        mesh.set_state(*g)
        _amr_flags(solver, mesh, criterion)
        mesh.refine()
    mesh.set_state(*init_state())


def amr_cpu_reference(budget_s=12.0):
    """The reference's own EuMesh / SmFluid (oracle/_ref) on this host's
    cores: the same setup, then steps with an adaptation every AMR_EVERY
    steps; None when that build is absent."""
    from oracle import ref_mesh as RM
    from zephyr_b200.workloads import blast_cell_means
    if not RM.available():
        return None
    threads = os.cpu_count() or 1
    RM.lib().zm_threads(threads)
    r = RM.RefEuMesh(AMR_BASE, AMR_BASE, bounds=(2, 2, 2, 2), accuracy=2, limiter="van Albada 1", CFL=0.4,
                     max_level=AMR_LEVELS, distributor="slope")

    def init():
        vx, vy = r.verts()
        return blast_cell_means(vx, vy)

    for _ in range(AMR_LEVELS + 3):
        r.set_state(*init())
        r.solver_flags()
        r.refine()
    r.set_state(*init())
    t0 = time.perf_counter()
    updates, steps = 0, 0
    while steps < AMR_EVERY or (time.perf_counter() - t0 < budget_s and steps < 4 * AMR_EVERY):
        updates += r.n
        r.step()
        steps += 1
        if steps % AMR_EVERY == 0:
            r.solver_flags()
            r.refine()
    sec = time.perf_counter() - t0
    RM.lib().zm_threads(0)
    return {"value": updates / sec, "unit": METRIC, "cores": threads, "kind": "reference",
            "sample": f"steps 0-{steps} after the initial adaptation ({r.n} live cells at the end), "
                      f"set_flags + refine every {AMR_EVERY} steps (the reference has the neighbour-jump "
                      f"criterion only); zephyr's EuMesh / SmFluid compiled from its "
                      f"sources (oracle/_ref); {threads} std::threads"}


def amr_variant(torch, lib, dev, stream, local_rank, want_cpu, kernels_name=None, criterion="reference"):
    """The quadtree AMR blast: base 512^2, 3 levels, the benchmark's
    |grad rho| h / rho criterion or the reference's SmFluid::set_flags, slope
    distributor, adaptation every 10 steps; the FP64 step on the slot mesh
    with the FAST kernels (derived face geometry), the MIXED kernels, or the
    PARITY kernels (bit-exact with the reference).  Times steps 7000-7400
    including every set_flags + refine."""
    import zephyr_b200 as Z
    from zephyr_b200._lib import KERNEL_KINDS
    from zephyr_b200.workloads import blast_cell_means
    gen = Z.Rectangle(0.0, 1.0, 0.0, 1.0)
    gen.set_boundaries(Z.Boundaries(Z.Boundary.ZOE, Z.Boundary.ZOE, Z.Boundary.ZOE, Z.Boundary.ZOE))
    gen.set_sizes(AMR_BASE, AMR_BASE)
    mesh = Z.EuMesh(gen, device=local_rank, stream=stream.cuda_stream)
    mesh.set_max_level(AMR_LEVELS, AMR_CAPACITY)
    kernels_name = kernels_name or AMR_KERNELS
    kernels = Z.Kernels.PARITY if kernels_name == "parity" else Z.Kernels.FAST
    precision = Z.Precision.MIXED if kernels_name == "mixed" else Z.Precision.FP64
    solver = Z.SmFluid(Z.IdealGas(1.4), precision=precision, kernels=kernels)
    solver.add_types(mesh)
    solver.set_accuracy(2)
    solver.set_CFL(0.4)
    solver.set_limiter("van Albada 1")
    solver.set_method(Z.Fluxes.HLLC)
    mesh.set_distributor(solver.distributor("slope"))

    def init():
        g = mesh.amr_arrays()
        return blast_cell_means(g["vx"], g["vy"])

    _amr_setup(Z, init, mesh, solver, criterion)
    for s in range(AMR_WARM_STEPS):
        solver.update(mesh)
        if (s + 1) % AMR_EVERY == 0:
            _amr_flags(solver, mesh, criterion)
            mesh.refine()
    torch.cuda.synchronize(dev)
    n0 = mesh.launch_count()
    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731
    e0, e1 = ev(), ev()
    adapt_ev = []
    live, held = [], []
    e0.record(stream)
    for s in range(AMR_TIMED_STEPS):
        live.append(mesh.n_cells())
        solver.update(mesh)
        if (s + 1) % AMR_EVERY == 0:
            a0, a1 = ev(), ev()
            a0.record(stream)
            _amr_flags(solver, mesh, criterion)
            mesh.refine()
            a1.record(stream)
            adapt_ev.append((a0, a1))
            st = mesh.amr_info()
            held.append((st.n_before, st.n_large))
    e1.record(stream)
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1)
    adapt_ms = [a.elapsed_time(b) for a, b in adapt_ev]
    launches = mesh.launch_count() - n0
    # the per-kernel split from the AMR_SPLIT_STEPS steps after the window,
    # with an event pair around every launch
    lib.zg_set_timing(mesh.ctx, 1)
    for s in range(AMR_SPLIT_STEPS):
        solver.update(mesh)
        if (s + 1) % AMR_EVERY == 0:
            _amr_flags(solver, mesh, criterion)
            mesh.refine()
    kms = (C.c_double * len(KERNEL_KINDS))()
    kcount = (C.c_longlong * len(KERNEL_KINDS))()
    lib.zg_kernel_times(mesh.ctx, kms, kcount)
    lib.zg_set_timing(mesh.ctx, 0)
    kernels = {name: {"launches": int(kcount[k]), "ms_total": kms[k], "ms_avg": kms[k] / kcount[k]}
               for k, name in enumerate(KERNEL_KINDS) if kcount[k]}
    solver.dt()
    final = (mesh.get_state()[0], mesh.amr_arrays()["level"])
    mesh.close()
    updates = int(sum(live))
    step_ms = ms - sum(adapt_ms)
    refine_bytes = sum(AMR_CELL_BYTES * (a + b) for a, b in held)
    out = {
        "workload": f"AMR blast, base {AMR_BASE}x{AMR_BASE}, max_level {AMR_LEVELS}, ZOE; rho = 1, u = v = 0, "
                    f"p = 1e-5 except p = 1e3 for r < 0.01 at (0.5, 0.5), 20x20 sub-sampled cell means",
        "form": {"fast": "FP64 FAST kernels on the slot mesh (face geometry from centre and level, fused "
                         "multiply-adds, cells in Morton order, face-once corrector; within 1e-12 of the parity "
                         "form per step)",
                 "mixed": "MIXED kernels on the slot mesh (FP32 states, gradients and fluxes; FP64 conserved "
                          "sums, update, pressure recovery and dt; cells in Morton order, face-once corrector)",
                 "parity": "FP64 PARITY kernels on the slot mesh, bit-exact with the reference"}[kernels_name] +
                " -- SmFluid second order, predictor-corrector, HLLC, van Albada 1, CFL 0.4; set_flags criterion; "
                "slope distributor",
        "criterion": ("|grad rho| h / rho: refine above 0.05, coarsen below 0.01" if criterion == "gradient" else
                      "SmFluid::set_flags (neighbour jumps 0.05 / 0.4x, sm_fluid.cpp:517-559)"),
        "value": updates / (ms / 1e3), "unit": METRIC, "timed_steps": AMR_TIMED_STEPS,
        "window": f"steps {AMR_WARM_STEPS}-{AMR_WARM_STEPS + AMR_TIMED_STEPS}", "adapt_every": AMR_EVERY,
        "ms_total": ms, "ms_per_step_incl_adapt": ms / AMR_TIMED_STEPS,
        "step_only_value": updates / (step_ms / 1e3),
        "adapt_ms_avg": sum(adapt_ms) / max(len(adapt_ms), 1), "adaptations": len(adapt_ms),
        "live_cells": {"min": min(live), "max": max(live), "mean": updates / len(live)},
        "cells_held_max": max(b for _, b in held) if held else None,
        "refine_GBs": refine_bytes / (sum(adapt_ms) / 1e3) / 1e9 if adapt_ms else None,
        "refine_bytes_rule": f"{AMR_CELL_BYTES} B per cell over the cells before plus the cells held "
                             "(all cell and face arrays read once, new arrays written once)",
        "algorithmic_bytes_per_cell_update": AMR_B_ALG,
        "step_achieved_GBs": AMR_B_ALG * updates / (step_ms / 1e3) / 1e9,
        "gpu_launches": int(launches), "kernels": kernels,
        "kernels_window": f"the {AMR_SPLIT_STEPS} steps after the timed window, with per-launch events",
        "final": final,
    }
    if want_cpu:
        out["cpu_baseline"] = amr_cpu_reference()
    return out


def amr_mixed_accuracy(torch, dev, stream, local_rank):
    """The MIXED form's error on the adaptive blast, on the same mesh as the
    FP64 FAST form: both run the same schedule in lockstep (the initial
    adaptation, then AMR_WARM_STEPS + AMR_TIMED_STEPS steps adapting every
    AMR_EVERY steps), and every adaptation uses the FP64 run's flags
    (|grad rho| h / rho) for both meshes, so the two meshes stay identical
    cell for cell.  L1 / Linf of the density relative to the FP64 form at
    the end."""
    import zephyr_b200 as Z
    from zephyr_b200.workloads import blast_cell_means
    runs = []
    for prec in (Z.Precision.FP64, Z.Precision.MIXED):
        gen = Z.Rectangle(0.0, 1.0, 0.0, 1.0)
        gen.set_boundaries(Z.Boundaries(Z.Boundary.ZOE, Z.Boundary.ZOE, Z.Boundary.ZOE, Z.Boundary.ZOE))
        gen.set_sizes(AMR_BASE, AMR_BASE)
        mesh = Z.EuMesh(gen, device=local_rank, stream=stream.cuda_stream)
        mesh.set_max_level(AMR_LEVELS, AMR_CAPACITY)
        solver = Z.SmFluid(Z.IdealGas(1.4), precision=prec, kernels=Z.Kernels.FAST)
        solver.add_types(mesh)
        solver.set_accuracy(2)
        solver.set_CFL(0.4)
        solver.set_limiter("van Albada 1")
        solver.set_method(Z.Fluxes.HLLC)
        mesh.set_distributor(solver.distributor("slope"))
        runs.append((mesh, solver))
    (m64, s64), (mmx, smx) = runs

    def adapt():
        # each form computes its own gradients (the slope distributor's),
        # then both take the FP64 form's flags
        f = s64.set_flags_gradient(m64, 0.05, 0.01, download=True)
        smx.set_flags_gradient(mmx, 0.05, 0.01, download=False)
        for m in (m64, mmx):
            m.put_flags(f)
            m.refine()

    for _ in range(AMR_LEVELS + 3):
        g = m64.amr_arrays()
        st = blast_cell_means(g["vx"], g["vy"])
        m64.set_state(*st)
        mmx.set_state(*st)
        adapt()
    g = m64.amr_arrays()
    st = blast_cell_means(g["vx"], g["vy"])
    m64.set_state(*st)
    mmx.set_state(*st)
    steps = AMR_WARM_STEPS + AMR_TIMED_STEPS
    for k in range(steps):
        s64.update(m64)
        smx.update(mmx)
        if (k + 1) % AMR_EVERY == 0:
            adapt()
    r64, rmx = m64.get_state()[0], mmx.get_state()[0]
    same = bool(np.array_equal(m64.amr_arrays()["level"], mmx.amr_arrays()["level"]))
    out = {"steps": steps, "same_mesh_as_fp64": same, "live_cells": int(len(r64)),
           "l1_rel_density_err_vs_fp64": float(np.sum(np.abs(rmx - r64)) / np.sum(np.abs(r64))),
           "linf_rel_density_err_vs_fp64": float(np.max(np.abs(rmx - r64)) / np.max(np.abs(r64))),
           "how": "both forms adapt with the FP64 run's flags, so the meshes are identical"}
    for m, _ in runs:
        m.close()
    return out


ADJ_SIZE = 1024  # the smooth periodic problem at 1024^2, 100 Heun steps, checkpoints every 10


def adjoint_variant(torch, dev, stream, local_rank):
    """The adjoint mode on the smooth periodic problem: time of one forward
    run (J) and of one gradient run (J, dJ/drho_0, dJ/dgamma with the
    checkpointed reverse sweep), and the gradient against central finite
    differences of the FP64 forward along 16 Gaussian directions (seed 5,
    eps 1e-6)."""
    from zephyr_b200.adjoint import Adjoint
    from zephyr_b200.workloads import fourier_smooth
    w = fourier_smooth(ADJ_SIZE)
    r, u, v, p = [torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device=dev) for a in w.state[:4]]
    adj = Adjoint(ADJ_SIZE, ADJ_SIZE, device=local_rank, stream=stream.cuda_stream)
    dt = adj.cfl_dt(1.4, 0.4, r, u, v, p)
    prm = Adjoint.params(steps=100, checkpoint_every=10, dt=dt)
    grad = torch.empty_like(r)
    adj.forward(prm, r, u, v, p)
    adj.gradient(prm, r, u, v, p, grad)
    torch.cuda.synchronize(dev)

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        out = fn()
        e1.record(stream)
        torch.cuda.synchronize(dev)
        return e0.elapsed_time(e1), out

    n0 = adj.launch_count()
    ms_f, J = timed(lambda: adj.forward(prm, r, u, v, p))
    ms_g, (J2, dg) = timed(lambda: adj.gradient(prm, r, u, v, p, grad))
    # the mixed form: FP64 primal, FP32 slopes and reverse-sweep face arithmetic
    pmx = Adjoint.params(steps=100, checkpoint_every=10, dt=dt, precision=1)
    gmx = torch.empty_like(r)
    adj.forward(pmx, r, u, v, p)
    adj.gradient(pmx, r, u, v, p, gmx)
    ms_fm, Jm = timed(lambda: adj.forward(pmx, r, u, v, p))
    ms_gm, (_, dgm) = timed(lambda: adj.gradient(pmx, r, u, v, p, gmx))
    launches = adj.launch_count() - n0
    rng = np.random.default_rng(5)
    eps = 1e-6
    errs, errs_m = [], []
    for _ in range(16):
        d = torch.tensor(rng.standard_normal(ADJ_SIZE * ADJ_SIZE), dtype=torch.float64, device=dev)
        fd = (adj.forward(prm, r + eps * d, u, v, p) - adj.forward(prm, r - eps * d, u, v, p)) / (2 * eps)
        ad = float(torch.dot(grad, d))
        errs.append(abs(fd - ad) / abs(ad))
        errs_m.append(abs(fd - float(torch.dot(gmx, d))) / abs(ad))
    fd_g = (adj.forward(Adjoint.params(steps=100, checkpoint_every=10, dt=dt, gamma=1.4 + eps), r, u, v, p) -
            adj.forward(Adjoint.params(steps=100, checkpoint_every=10, dt=dt, gamma=1.4 - eps), r, u, v, p)) / (2 * eps)
    adj.close()
    return {"workload": f"smooth periodic problem {ADJ_SIZE}x{ADJ_SIZE}, J = mean p over [0.6,0.7]^2 after 100 "
                        "Heun steps at the CFL 0.4 dt of the initial state, smooth van Albada (eps 1e-8), HLLC",
            "forward_ms": ms_f, "gradient_ms": ms_g, "adjoint_over_forward": ms_g / ms_f,
            "checkpoint_every": 10, "J": J, "dJ_dgamma": dg,
            "fd_rel_err_max": max(errs), "fd_rel_err_median": float(np.median(errs)), "fd_directions": 16,
            "fd_rel_err_gamma": abs(fd_g - dg) / abs(dg), "gpu_launches": int(launches),
            "mixed": {"form": "FP64 primal step with FP32 slopes (from FP64 neighbour differences); reverse "
                              "sweep with FP32 slope partials, face states, HLLC reverse and face cotangents, "
                              "FP64 adjoint states, cotangent sums, primitive map and gamma",
                      "forward_ms": ms_fm, "gradient_ms": ms_gm, "adjoint_over_forward": ms_gm / ms_fm,
                      "gradient_speedup_vs_fp64": ms_g / ms_gm, "J_rel_err_vs_fp64": abs(Jm - J) / abs(J),
                      "grad_l2_rel_err_vs_fp64": float(torch.linalg.norm(gmx - grad) / torch.linalg.norm(grad)),
                      "dJ_dgamma_rel_err_vs_fp64": abs(dgm - dg) / abs(dg),
                      "fd_rel_err_max": max(errs_m), "fd_rel_err_median": float(np.median(errs_m))},
            "note": "gradient time includes the checkpointed forward, the segment recomputation and the reverse "
                    "sweep; FD: central differences of the FP64 forward, eps 1e-6, Gaussian directions seed 5"}


def _max_over_ranks(torch, vals, dev, world):
    t = torch.tensor(vals, dtype=torch.float64, device=dev)
    if world > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return [float(x) for x in t]


TR_NX = 4096             # VOF transport: cells along x of [0, 1] x [0, 0.7]
TR_DISKS = 64            # seeded disks of the transport workload
# bytes per cell and split step (two sub-steps), each sub-step: face fluxes
# read u1, n, p (40) and write two fluxes per face (16); the update reads the
# two fluxes and u1 and writes u1 (32); the normals read u1 and write n, p
# (40); three smoothing passes read u1, n, p and write n, p (3 x 72)
TR_B_ALG = 2 * (56 + 32 + 40 + 216)


def tr_cpu_reference(box, budget_s=10.0):
    """The reference's own Transfer (oracle/_ref; its loops are serial) on a
    512 x 358 sample of the workload; None when that build is absent."""
    from oracle import ref_tr as RT
    from zephyr_b200.workloads import transfer_disk_field
    if not RT.available():
        return None
    nx, ny = 512, 358
    r = RT.RefTransfer(nx, ny, box=box, method="VOF", CFL=0.5, vel=("translation", 0.7, -0.35))
    r.set_u(transfer_disk_field(nx, ny, box, count=TR_DISKS, seed=7))
    r.update_interface(3)

    def step():
        r.set_dt(r.compute_dt())
        r.update(1)
        r.update(2)

    t0 = time.perf_counter()
    step()
    per = time.perf_counter() - t0
    steps = max(1, min(20, int(budget_s / max(per, 1e-3))))
    t0 = time.perf_counter()
    for _ in range(steps):
        step()
    per = (time.perf_counter() - t0) / steps
    return {"value": nx * ny / per, "unit": METRIC, "cores": 1, "kind": "reference",
            "sample": f"{steps} split step(s) of a {nx}x{ny} mesh of the same disk field after 1 untimed step; "
                      "zephyr's Transfer (VOF) compiled from its sources (oracle/_ref); serial loops"}


def transfer_variant(torch, lib, dev, stream, barrier, K, W, local_rank, want_cpu, nx=0):
    """The scalar VOF transport (Transfer, method VOF with direction
    splitting, the transfer problem's translation velocity) on a field of
    disks, bit-exact with the reference; the transfer problem's time loop runs
    on the device (zg_tr_advance)."""
    import zephyr_b200 as Z
    from zephyr_b200._lib import KERNEL_KINDS
    from zephyr_b200.transfer import Method, Transfer
    from zephyr_b200.workloads import transfer_disk_field
    box = (0.0, 1.0, 0.0, 0.7)
    nx = nx or TR_NX
    ny = int(round(nx * 0.7))
    u0 = transfer_disk_field(nx, ny, box, count=TR_DISKS, seed=7)
    gen = Z.Rectangle(*box)
    gen.set_boundaries(Z.Boundaries(Z.Boundary.ZOE, Z.Boundary.ZOE, Z.Boundary.ZOE, Z.Boundary.ZOE))
    gen.set_sizes(nx, ny)
    mesh = Z.EuMesh(gen, device=local_rank, stream=stream.cuda_stream)
    s = Transfer()
    s.set_method(Method.VOF)
    s.set_CFL(0.5)
    s.set_velocity_translation(0.7, -0.35)
    s.add_types(mesh)
    s.set_u1(mesh, u0)
    s.update_interface(mesh)
    t = s.advance(mesh, W, 0.0, 1.0e9, splitting=True)
    n0 = mesh.launch_count()
    barrier()
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    t = s.advance(mesh, K, t, 1.0e9, splitting=True)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    barrier()
    ms = e0.elapsed_time(e1)
    launches = mesh.launch_count() - n0
    u = s.u1(mesh)  # raises if a polygon overflowed the kernels' capacity
    # per-kernel times over K more steps (events around every launch)
    lib.zg_set_timing(mesh.ctx, 1)
    s.advance(mesh, K, t, 1.0e9, splitting=True)
    kms = (C.c_double * len(KERNEL_KINDS))()
    kcount = (C.c_longlong * len(KERNEL_KINDS))()
    lib.zg_kernel_times(mesh.ctx, kms, kcount)
    lib.zg_set_timing(mesh.ctx, 0)
    tot = max(sum(kms), 1e-12)
    kernels = {name: {"launches": int(kcount[k]), "ms_total": kms[k], "ms_avg": kms[k] / kcount[k],
                      "share": kms[k] / tot} for k, name in enumerate(KERNEL_KINDS) if kcount[k]}
    cells = nx * ny
    out = {"workload": f"transfer_disks {nx}x{ny} ([0,1]x[0,0.7], {TR_DISKS} seeded disks, ZOE walls)",
           "form": "FP64, bit-exact with the reference (Transfer VOF, CFL 0.5, translation (0.7, -0.35), "
                   "split X then Y, 3 smoothing passes)",
           "ms": ms, "kernels": kernels, "launches": launches, "cells": cells,
           "mixed_cells": int(((u > 0.0) & (u < 1.0)).sum())}
    mesh.close()
    if want_cpu:
        out["cpu_baseline"] = tr_cpu_reference(box)
    return out


VTU_SIZE = 1024   # output: cells per side of the mesh written


def vtu_variant(torch, local_rank, stream, want_cpu):
    """VTU output (zg_vtu_write) of a 1024^2 mesh with the level and the five
    SmFluid state fields as the single-fluid driver writes them: time of the
    whole call (device packing, copies, file write) into a temporary
    directory, and the reference's VtuFile::save (oracle/_ref) on the same
    mesh and values."""
    import tempfile
    import zephyr_b200 as Z
    from zephyr_b200.io import Variables, VtuFile
    from zephyr_b200.workloads import fourier_smooth
    w = fourier_smooth(VTU_SIZE)
    gen = Z.Rectangle(0.0, 1.0, 0.0, 1.0)  # ZOE walls: the reference's adaptive EuMesh rejects periodic axes
    gen.set_sizes(VTU_SIZE, VTU_SIZE)
    mesh = Z.EuMesh(gen, device=local_rank, stream=stream.cuda_stream)
    solver = Z.SmFluid(w.eos)
    solver.add_types(mesh)
    mesh.set_state(*w.state)
    names = ("density", "vel.x", "vel.y", "pressure", "energy")
    v = Variables(["level"])
    for k, nm in enumerate(names):
        v.append(nm, ("smf", k))
    out = {"workload": f"fourier_smooth {VTU_SIZE}x{VTU_SIZE}: level + 5 FP64 state fields, quadrilateral cells"}
    with tempfile.TemporaryDirectory() as d:
        f = Path(d) / "out.vtu"
        times = []
        for _ in range(4):
            t0 = time.perf_counter()
            VtuFile.save(f, mesh, v)
            times.append(time.perf_counter() - t0)
        size = f.stat().st_size
        ms = 1e3 * statistics.median(times[1:])
        out.update(ms=ms, bytes=size, GBs=size / (ms / 1e3) / 1e9, gpu_launches=4 * (2 + 1))
        if want_cpu:
            from oracle import ref_mesh as RME
            if RME.available():
                n = VTU_SIZE
                r = RME.RefEuMesh(n, n, bounds=(2, 2, 2, 2))
                r.set_state(*w.state)
                t0 = time.perf_counter()
                r.write_vtu(Path(d) / "ref.vtu", names=("level",), with_state=True)
                ref_s = time.perf_counter() - t0
                same = (Path(d) / "ref.vtu").read_bytes() == f.read_bytes()
                out["cpu_baseline"] = {"ms": 1e3 * ref_s, "kind": "reference", "cores": 1,
                                       "sample": "one VtuFile::save of the same mesh and values (oracle/_ref)",
                                       "same_bytes": same}
    mesh.close()
    return out


def run_ours(args, rank, world, local_rank):
    import torch
    import zephyr_b200 as Z

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    # A dedicated (non-default) stream: the library queues its kernels on it
    # and the timing events are recorded on it.
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    lib = Z.load()

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    K, W = args.steps, max(args.warmup, 3)
    if args.only and args.only != "forms":
        global AMR_BASE, AMR_CAPACITY
        if args.amr_base:
            AMR_BASE = args.amr_base
            AMR_CAPACITY = max(1 << 20, 32 * AMR_BASE * AMR_BASE)
        if args.only == "amr":
            out = amr_variant(torch, lib, dev, stream, local_rank, want_cpu=False, kernels_name=args.amr_kernels,
                              criterion=args.amr_criterion)
            out.pop("final")
        elif args.only == "vtu":
            out = vtu_variant(torch, local_rank, stream, want_cpu=True)
        elif args.only == "transfer":
            out = transfer_variant(torch, lib, dev, stream, barrier, K, W, local_rank, want_cpu=False, nx=args.tr_nx)
        elif args.only == "mm":
            out = mm_variant(torch, lib, dev, stream, barrier, K, W, local_rank, want_cpu=False,
                             precision=Z.Precision.MIXED if args.amr_kernels == "mixed" else Z.Precision.FP64,
                             accuracy=args.mm_accuracy)
            out.pop("final")
        else:
            out = adjoint_variant(torch, dev, stream, local_rank)
        if rank == 0:
            print(json.dumps({"only": args.only, **out}, default=str), flush=True)
        return

    w, cfg = workload(args.workload, args.size)
    cells = w.gen.nx() * w.gen.ny()

    # ---- headline: the FP64 step (FAST kernels), inputs resident in HBM ----
    # timed bare (no per-kernel events); the split by kernel comes from a
    # second run of K steps with the library's per-launch events
    mesh, solver = _solver(Z, w, cfg, args, local_rank, stream, Z.Precision.FP64, Z.Kernels.FAST)
    solver.update(mesh, steps=W)
    mesh.synchronize()
    ms, _, launches, clocks = _timed_steps(torch, lib, mesh, solver, K, dev, stream, barrier, clocks=True,
                                           per_kernel=False)
    dt_last = solver.dt()
    _, kernels, _, _ = _timed_steps(torch, lib, mesh, solver, K, dev, stream, barrier)

    # ---- end to end through the public API with host buffers ---------------
    pin = [torch.empty(cells, dtype=torch.float64, pin_memory=True) for _ in range(5)]
    for t, a in zip(pin, mesh.get_state()):
        t.numpy()[:] = a
    outp = [torch.empty(cells, dtype=torch.float64, pin_memory=True) for _ in range(5)]
    P = C.POINTER(C.c_double)
    inp_ptrs = [C.cast(C.c_void_p(t.data_ptr()), P) for t in pin]
    out_ptrs = [C.cast(C.c_void_p(t.data_ptr()), P) for t in outp]
    e2e_steps = max(3, min(K, 10))
    barrier()
    torch.cuda.synchronize(dev)
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(e2e_steps):
        Z._lib.check(mesh.ctx, lib.zg_state_upload(mesh.ctx, *inp_ptrs))
        Z._lib.check(mesh.ctx, lib.zg_smf_update(mesh.ctx))
        Z._lib.check(mesh.ctx, lib.zg_state_download(mesh.ctx, *out_ptrs))
    f1.record(stream)
    torch.cuda.synchronize(dev)
    barrier()
    e2e_ms = f0.elapsed_time(f1)
    mesh.close()

    # ---- the other forms on the same workload ------------------------------
    variants = {}
    other_scheme = "heun" if args.scheme == "pc" else "pc"
    for name, prec, kern, scheme in (("fp64_parity", Z.Precision.FP64, Z.Kernels.PARITY, args.scheme),
                                     ("mixed", Z.Precision.MIXED, Z.Kernels.FAST, args.scheme),
                                     ("fp64_two_pass", Z.Precision.FP64, Z.Kernels.FAST_TWO_PASS, args.scheme),
                                     ("fp64_" + other_scheme, Z.Precision.FP64, Z.Kernels.FAST, other_scheme),
                                     ("mixed_" + other_scheme, Z.Precision.MIXED, Z.Kernels.FAST, other_scheme)):
        a2 = argparse.Namespace(**{**vars(args), "scheme": scheme})
        m2, s2 = _solver(Z, w, cfg, a2, local_rank, stream, prec, kern)
        s2.update(m2, steps=W)
        m2.synchronize()
        v_ms, _, v_launch, _ = _timed_steps(torch, lib, m2, s2, K, dev, stream, barrier, per_kernel=False)
        _, v_kernels, _, _ = _timed_steps(torch, lib, m2, s2, K, dev, stream, barrier)
        variants[name] = {"ms": v_ms, "kernels": v_kernels, "launches": v_launch, "mesh": m2, "solver": s2,
                          "scheme": scheme}
    if args.only == "forms":  # the step's forms on the 2048^2 workload alone
        for v in variants.values():
            v["mesh"].close()
        if rank == 0:
            print(json.dumps({"only": "forms", "headline_ms_per_step": ms / K, "headline_kernels": kernels,
                              **{n: {"ms_per_step": v["ms"] / K, "kernels": v["kernels"]}
                                 for n, v in variants.items()}}), flush=True)
        return

    # accuracy over the configuration's horizon: density after HORIZON steps
    # of the mixed form (and of the FAST FP64 form) against the bit-exact FP64
    # parity form run for the same steps from the same initial state
    acc = {}
    for scheme in ("pc", "heun"):
        a2 = argparse.Namespace(**{**vars(args), "scheme": scheme})
        rho = {}
        for name, prec, kern in (("parity", Z.Precision.FP64, Z.Kernels.PARITY),
                                 ("mixed", Z.Precision.MIXED, Z.Kernels.FAST),
                                 ("fast", Z.Precision.FP64, Z.Kernels.FAST)):
            m3, s3 = _solver(Z, w, cfg, a2, local_rank, stream, prec, kern)
            s3.update(m3, steps=HORIZON)
            rho[name] = m3.get_state()[0]
            m3.close()
        o = rho["parity"]
        acc[scheme] = {f"{k}_{nm}": v for nm in ("mixed", "fast") for k, v in (
            ("l1_rel_density_err_vs_fp64_parity", float(np.sum(np.abs(rho[nm] - o)) / np.sum(np.abs(o)))),
            ("linf_rel_density_err_vs_fp64_parity", float(np.max(np.abs(rho[nm] - o)) / np.max(np.abs(o)))))}
    l1 = acc[args.scheme]["l1_rel_density_err_vs_fp64_parity_mixed"]
    linf = acc[args.scheme]["linf_rel_density_err_vs_fp64_parity_mixed"]

    mm = mm_variant(torch, lib, dev, stream, barrier, K, W, local_rank,
                    want_cpu=(rank == 0 and world == 1 and not args.no_cpu_baseline), precision=Z.Precision.FP64)
    mm_mx = mm_variant(torch, lib, dev, stream, barrier, K, W, local_rank, want_cpu=False,
                       precision=Z.Precision.MIXED)
    mm2 = mm_variant(torch, lib, dev, stream, barrier, K, W, local_rank,
                     want_cpu=(rank == 0 and world == 1 and not args.no_cpu_baseline), precision=Z.Precision.FP64,
                     accuracy=2)
    mm2_mx = mm_variant(torch, lib, dev, stream, barrier, K, W, local_rank, want_cpu=False,
                        precision=Z.Precision.MIXED, accuracy=2)
    z2, z2mx = mm2.pop("final"), mm2_mx.pop("final")
    mm2_err = {f"l1_rel_{name}_err_vs_fp64": float(np.sum(np.abs(z2mx[:, k] - z2[:, k])) / np.sum(np.abs(z2[:, k])))
               for name, k in (("density", 0), ("pressure", 3))}
    z64, zmx = mm.pop("final"), mm_mx.pop("final")
    mm_err = {f"l1_rel_{name}_err_vs_fp64": float(np.sum(np.abs(zmx[:, k] - z64[:, k])) / np.sum(np.abs(z64[:, k])))
              for name, k in (("density", 0), ("pressure", 3))}
    adjv = adjoint_variant(torch, dev, stream, local_rank)
    trv = transfer_variant(torch, lib, dev, stream, barrier, K, W, local_rank,
                           want_cpu=(rank == 0 and world == 1 and not args.no_cpu_baseline))
    vtuv = vtu_variant(torch, local_rank, stream, want_cpu=(rank == 0 and world == 1 and not args.no_cpu_baseline))
    # the benchmark's criterion (|grad rho| h / rho) for the FP64 FAST and
    # MIXED forms; the reference's own set_flags for the bit-exact form
    amr = amr_variant(torch, lib, dev, stream, local_rank,
                      want_cpu=(rank == 0 and world == 1 and not args.no_cpu_baseline), kernels_name="fast",
                      criterion="gradient")
    amr_par = amr_variant(torch, lib, dev, stream, local_rank, want_cpu=False, kernels_name="parity",
                          criterion="reference")
    amr_mx = amr_variant(torch, lib, dev, stream, local_rank, want_cpu=False, kernels_name="mixed",
                         criterion="gradient")
    amr.pop("final"), amr_mx.pop("final"), amr_par.pop("final")
    amr_acc = amr_mixed_accuracy(torch, dev, stream, local_rank)
    amr_mx["l1_rel_density_err_vs_fp64"] = amr_acc["l1_rel_density_err_vs_fp64"]
    amr_mx["linf_rel_density_err_vs_fp64"] = amr_acc["linf_rel_density_err_vs_fp64"]
    amr_mx["same_mesh_as_fp64"] = amr_acc["same_mesh_as_fp64"]
    amr_mx["error_run"] = amr_acc

    vnames = list(variants)
    vals = _max_over_ranks(torch, [ms, e2e_ms, mm["ms"], amr["ms_total"], amr_par["ms_total"], mm_mx["ms"],
                                   amr_mx["ms_total"], trv["ms"], mm2["ms"], mm2_mx["ms"]] +
                           [variants[v]["ms"] for v in vnames], dev, world)
    ms, e2e_ms, ms_mm, ms_amr, ms_amr_par, ms_mm_mx, ms_amr_mx, ms_tr, ms_mm2, ms_mm2_mx = vals[:10]
    vms = dict(zip(vnames, vals[10:]))
    ms_par, ms_mix = vms["fp64_parity"], vms["mixed"]
    amr_mx["value"] = world * amr_mx["value"] * amr_mx["ms_total"] / ms_amr_mx
    amr_mx["speedup_vs_fp64"] = ms_amr / ms_amr_mx
    amr["value"] = world * amr["value"] * amr["ms_total"] / ms_amr
    amr_par["value"] = world * amr_par["value"] * amr_par["ms_total"] / ms_amr_par
    for v in variants.values():
        v["mesh"].close()
    if rank != 0:
        return

    value = world * cells * K / (ms / 1e3)
    e2e_value = world * cells * e2e_steps / (e2e_ms / 1e3)
    top = max(kernels, key=lambda n: kernels[n]["ms_total"])
    peak, peak_kind = hbm_peak()
    balg = B_ALG_KERNEL[top] * cells
    achieved = balg / (kernels[top]["ms_avg"] / 1e3) / 1e9
    tpc = traffic_per_cell(top)
    roof = {"bound": "hbm", "kernel": top, "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_source": peak_kind,
            "traffic": (tpc * cells) if tpc is not None else None,
            "algorithmic_bytes_per_launch": balg,
            "step_achieved": B_ALG_STEP[cfg["acc"]] * cells * K / (ms / 1e3) / 1e9}
    roof["step_frac"] = roof["step_achieved"] / peak
    # the FP64 pipe beside it: FP64 thread-instructions per cell of the top
    # kernel (ncu, committed summary) at this run's duration, against the
    # pipe's issue rate at the SM clock sampled during the timed region
    f64_per_cell = traffic_per_cell(top, 2)
    if f64_per_cell is not None:
        mhz = (clocks or {}).get("sm_mhz") or 1965.0
        f64_peak = FP64_INST_PER_SM_CYCLE * N_SM * mhz * 1e6
        f64_rate = f64_per_cell * cells / (kernels[top]["ms_avg"] / 1e3)
        roof["fp64_pipe"] = {"inst_per_cell": f64_per_cell, "achieved_inst_per_s": f64_rate,
                             "peak_inst_per_s": f64_peak, "frac": f64_rate / f64_peak,
                             "ncu_pipe_active_pct": traffic_per_cell(top, 3),
                             "source": "profiles/traffic_per_cell.txt (ncu --set full of the same kernel)"}
    mixed_balg = {1: 64, 2: 144}[cfg["acc"]]
    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": K,
        "warmup": args.warmup, "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": dict(config_of(args, w, cfg, world),
                       form="FP64 (FAST kernels: one fused kernel per step, face-once tiles in shared memory)",
                       timing="headline timed without per-kernel events; the kernel split from a second run"),
        "roofline": roof, "kernels": kernels,
        "gpu_launches": int(launches + sum(v["launches"] for v in variants.values()) +
                            mm["launches"] + mm_mx["launches"] + mm2["launches"] + mm2_mx["launches"] +
                            adjv["gpu_launches"] + amr["gpu_launches"] +
                            amr_par["gpu_launches"] + amr_mx["gpu_launches"] + trv["launches"] +
                            vtuv["gpu_launches"]),
        "gpu_launches_headline": int(launches), "clocks": clocks,
        "e2e": {"value": e2e_value, "unit": METRIC, "h2d_bytes_per_step": 5 * 8 * cells,
                "d2h_bytes_per_step": 5 * 8 * cells, "steps": e2e_steps,
                "note": "per step: upload of the whole state from pinned host memory, zg_smf_update, "
                        "download of the whole state"},
        "variants": {
            "fp64_parity": {"value": world * cells * K / (ms_par / 1e3), "ms_per_step": ms_par / K,
                            "note": "bit-exact with the reference (gather form, no FMA)",
                            "kernels": variants["fp64_parity"]["kernels"]},
            "mixed": {"value": world * cells * K / (ms_mix / 1e3), "ms_per_step": ms_mix / K,
                      "speedup_vs_fp64": ms / ms_mix, "speedup_vs_fp64_parity": ms_par / ms_mix,
                      "l1_rel_density_err_vs_fp64": l1, "linf_rel_density_err_vs_fp64": linf,
                      "err_after_steps": HORIZON,
                      "err_reference": "the bit-exact FP64 parity form after the same steps",
                      "step_achieved_GBs": mixed_balg * cells * K / (ms_mix / 1e3) / 1e9,
                      "step_frac": mixed_balg * cells * K / (ms_mix / 1e3) / 1e9 / peak,
                      "kernels": variants["mixed"]["kernels"]},
            "fp64_two_pass": {"value": world * cells * K / (vms["fp64_two_pass"] / 1e3),
                              "ms_per_step": vms["fp64_two_pass"] / K,
                              "note": "the earlier FAST form: gradients + predictor stored in HBM, then the "
                                      "face pass", "kernels": variants["fp64_two_pass"]["kernels"]},
            "fp64_" + other_scheme: {"value": world * cells * K / (vms["fp64_" + other_scheme] / 1e3),
                                     "ms_per_step": vms["fp64_" + other_scheme] / K,
                                     "scheme": "heun (extension)" if other_scheme == "heun" else
                                               "predictor-corrector (reference)",
                                     "kernels": variants["fp64_" + other_scheme]["kernels"]},
            "mixed_" + other_scheme: {"value": world * cells * K / (vms["mixed_" + other_scheme] / 1e3),
                                      "ms_per_step": vms["mixed_" + other_scheme] / K,
                                      "speedup_vs_fp64": vms["fp64_" + other_scheme] / vms["mixed_" + other_scheme],
                                      "l1_rel_density_err_vs_fp64": acc[other_scheme][
                                          "l1_rel_density_err_vs_fp64_parity_mixed"],
                                      "linf_rel_density_err_vs_fp64": acc[other_scheme][
                                          "linf_rel_density_err_vs_fp64_parity_mixed"],
                                      "err_after_steps": HORIZON,
                                      "kernels": variants["mixed_" + other_scheme]["kernels"]},
            "accuracy_over_horizon": {"steps": HORIZON, "vs": "FP64 parity form (bit-exact with the reference)",
                                      "predictor_corrector": acc["pc"], "heun": acc["heun"]},
            "multimaterial": {
                "value": world * mm["cells"] * K / (ms_mm / 1e3), "unit": METRIC, "ms_per_step": ms_mm / K,
                "workload": mm["workload"], "form": mm["form"], "steps": K, "warmup": W,
                "step_achieved_GBs": MM_B_ALG * mm["cells"] * K / (ms_mm / 1e3) / 1e9,
                "step_frac": MM_B_ALG * mm["cells"] * K / (ms_mm / 1e3) / 1e9 / peak,
                "algorithmic_bytes_per_cell": MM_B_ALG, "gpu_launches": int(mm["launches"]),
                "kernels": mm["kernels"], "cpu_baseline": mm.get("cpu_baseline")},
            "multimaterial_mixed": {
                "value": world * mm_mx["cells"] * K / (ms_mm_mx / 1e3), "unit": METRIC,
                "ms_per_step": ms_mm_mx / K, "speedup_vs_fp64": ms_mm / ms_mm_mx,
                "form": "FP32 face states, wave speeds and HLLC fluxes of the pure-stencil faces (IEEE, no FMA); "
                        "FP64 accumulation, update, EoS pressure recovery, composite Riemann fluxes, "
                        "PT closure, PLIC and dt",
                **mm_err, "err_after_steps": W + 2 * K, "kernels": mm_mx["kernels"],
                "gpu_launches": int(mm_mx["launches"])},
            "multimaterial_second_order": {
                "value": world * mm2["cells"] * K / (ms_mm2 / 1e3), "unit": METRIC, "ms_per_step": ms_mm2 / K,
                "workload": mm2["workload"], "form": mm2["form"], "steps": K, "warmup": W,
                "step_achieved_GBs": MM2_B_ALG * mm2["cells"] * K / (ms_mm2 / 1e3) / 1e9,
                "step_frac": MM2_B_ALG * mm2["cells"] * K / (ms_mm2 / 1e3) / 1e9 / peak,
                "algorithmic_bytes_per_cell": MM2_B_ALG, "gpu_launches": int(mm2["launches"]),
                "kernels": mm2["kernels"], "cpu_baseline": mm2.get("cpu_baseline")},
            "multimaterial_second_order_mixed": {
                "value": world * mm2_mx["cells"] * K / (ms_mm2_mx / 1e3), "unit": METRIC,
                "ms_per_step": ms_mm2_mx / K, "speedup_vs_fp64": ms_mm2 / ms_mm2_mx,
                "form": "FP32 HLLC of the faces whose reconstructed states stay pure; FP64 reconstruction and "
                        "closures, composite Riemann fluxes, sums, update, PLIC and dt",
                **mm2_err, "err_after_steps": W + 2 * K, "kernels": mm2_mx["kernels"],
                "gpu_launches": int(mm2_mx["launches"])},
            "adjoint": adjv,
            "vtu_write": vtuv,
            "transfer": {
                "value": world * trv["cells"] * K / (ms_tr / 1e3), "unit": METRIC, "ms_per_step": ms_tr / K,
                "workload": trv["workload"], "form": trv["form"], "steps": K, "warmup": W,
                "mixed_cells_at_end": trv["mixed_cells"],
                "step_achieved_GBs": TR_B_ALG * trv["cells"] * K / (ms_tr / 1e3) / 1e9,
                "step_frac": TR_B_ALG * trv["cells"] * K / (ms_tr / 1e3) / 1e9 / peak,
                "algorithmic_bytes_per_cell": TR_B_ALG, "gpu_launches": int(trv["launches"]),
                "kernels": trv["kernels"], "cpu_baseline": trv.get("cpu_baseline")},
            "amr": amr,
            "amr_parity": {k: amr_par[k] for k in ("form", "criterion", "value", "unit", "ms_per_step_incl_adapt",
                                                     "step_only_value", "adapt_ms_avg", "live_cells",
                                                     "gpu_launches", "kernels")},
            "amr_mixed": {k: amr_mx[k] for k in ("form", "criterion", "value", "unit", "ms_per_step_incl_adapt",
                                                  "speedup_vs_fp64",
                                                  "l1_rel_density_err_vs_fp64", "linf_rel_density_err_vs_fp64",
                                                  "same_mesh_as_fp64", "error_run",
                                                  "step_only_value", "adapt_ms_avg", "live_cells", "gpu_launches",
                                                  "kernels")},
        },
        "dt_last": dt_last,
    }
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(w, cfg, args.scheme)
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    import datetime

    import torch
    if world > 1:
        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                             device_id=torch.device("cuda", local_rank))
    try:
        run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
