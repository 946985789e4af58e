"""Generate the golden fixtures of tests/golden from the reference's own code.

The outputs come from oracle/_ref/libzref.so: zephyr's SmFluid, fluxes,
limiters and EoS compiled from the reference sources (oracle/ref_build.py).
Run here, where the reference tree exists:

    python tests/golden/make_golden.py

Each fixture stores its inputs and the reference's outputs, so that the
tests (oracle and GPU) need neither the reference tree nor its build.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import ref as R  # noqa: E402
from zephyr_b200.workloads import fourier_smooth, riemann2d_case3  # noqa: E402

OUT = Path(__file__).resolve().parent

LIMITER_NAMES = ["none", "unit", "minmod", "MC", "van Leer", "van Albada 1", "van Albada 2", "CHARM", "HCUS",
                 "HQUICK", "Koren", "smart", "superbee"]


def random_state(n, seed, kind="gas"):
    rng = np.random.default_rng(seed)
    if kind == "water":
        rho = 1000.0 * (1.0 + 0.01 * rng.random(n))
        u = 5.0 * rng.standard_normal(n)
        v = 5.0 * rng.standard_normal(n)
        p = 1.0e5 * (1.0 + rng.random(n))
        e = (p + 4.4 * 6.0e8) / (3.4 * rho)  # stiffened_gas.cpp:121-128 with e0 = 0
        return rho, u, v, p, e
    rho = 1.0 + 0.3 * rng.random(n)
    u = 0.2 * rng.standard_normal(n)
    v = 0.2 * rng.standard_normal(n)
    p = 1.0 + 0.5 * rng.random(n)
    return rho, u, v, p, p / (0.4 * rho)


# name: (nx, ny, box, bounds, eos(kind, gamma, P0), flux, limiter, accuracy, CFL, steps, state)
CASES = {
    "c1_riemann3_32_first_order": (32, 32, (0, 1, 0, 1), (2, 2, 2, 2), (0, 1.4, 0.0), 3, "MC", 1, 0.4, 40,
                                   lambda: riemann2d_case3(32).state),
    "riemann3_32_mc": (32, 32, (0, 1, 0, 1), (2, 2, 2, 2), (0, 1.4, 0.0), 3, "MC", 2, 0.4, 40,
                       lambda: riemann2d_case3(32).state),
    "fourier_32_vanalbada_periodic": (32, 32, (0, 1, 0, 1), (3, 3, 3, 3), (0, 1.4, 0.0), 3, "van Albada", 2, 0.4,
                                      40, lambda: fourier_smooth(32).state),
    "walls_hll_24_first_order": (24, 24, (0, 1, 0, 1), (1, 1, 1, 1), (0, 1.4, 0.0), 2, "MC", 1, 0.5, 40,
                                 lambda: riemann2d_case3(24).state),
    "nonsquare_37x19_minmod": (37, 19, (0.0, 2.0, -0.5, 0.5), (1, 1, 3, 3), (0, 1.4, 0.0), 3, "minmod", 2, 0.45,
                               25, lambda: random_state(37 * 19, 7)),
    "stiffened_16_vanalbada": (16, 16, (0.0, 0.1, 0.0, 0.1), (2, 2, 1, 1), (1, 4.4, 6.0e8), 3, "van Albada", 2,
                               0.4, 15, lambda: random_state(256, 11, "water")),
    "superbee_20_zoe": (20, 20, (0, 1, 0, 1), (2, 2, 2, 2), (0, 1.4, 0.0), 3, "superbee", 2, 0.4, 20,
                        lambda: random_state(400, 3)),
    # the exact-Riemann Godunov flux (shocks, rarefactions and fans across faces) and Rusanov
    "godunov_riemann3_32_first_order": (32, 32, (0, 1, 0, 1), (2, 2, 2, 2), (0, 1.4, 0.0), 0, "MC", 1, 0.4, 40,
                                        lambda: riemann2d_case3(32).state),
    "godunov_stiffened_16_mc": (16, 16, (0.0, 0.1, 0.0, 0.1), (2, 2, 1, 1), (1, 4.4, 6.0e8), 0, "MC", 2, 0.4, 15,
                                lambda: random_state(256, 12, "water")),
    "rusanov_fourier_32_vanalbada": (32, 32, (0, 1, 0, 1), (3, 3, 3, 3), (0, 1.4, 0.0), 1, "van Albada", 2, 0.4,
                                     30, lambda: fourier_smooth(32).state),
    # HLLC_M, HLLC_LM (low Mach numbers: the sine branch), CIR1 and CIR2
    "hllcm_riemann3_24_mc": (24, 24, (0, 1, 0, 1), (2, 2, 2, 2), (0, 1.4, 0.0), 4, "MC", 2, 0.4, 25,
                             lambda: riemann2d_case3(24).state),
    "hllclm_random_24_vanalbada": (24, 24, (0, 1, 0, 1), (1, 1, 3, 3), (0, 1.4, 0.0), 5, "van Albada", 2, 0.4, 25,
                                   lambda: random_state(576, 21)),
    "cir1_riemann3_24_first_order": (24, 24, (0, 1, 0, 1), (2, 2, 2, 2), (0, 1.4, 0.0), 6, "MC", 1, 0.4, 30,
                                     lambda: riemann2d_case3(24).state),
    "cir1_fourier_24_mc_periodic": (24, 24, (0, 1, 0, 1), (3, 3, 3, 3), (0, 1.4, 0.0), 6, "MC", 2, 0.4, 25,
                                    lambda: fourier_smooth(24).state),
    "cir2_stiffened_16_minmod": (16, 16, (0.0, 0.1, 0.0, 0.1), (2, 2, 1, 1), (1, 4.4, 6.0e8), 7, "minmod", 2, 0.4,
                                 15, lambda: random_state(256, 13, "water")),
}
NEW_FLUX_CASES = ("hllcm_riemann3_24_mc", "hllclm_random_24_vanalbada", "cir1_riemann3_24_first_order",
                  "cir1_fourier_24_mc_periodic", "cir2_stiffened_16_minmod")


def make_case(name, spec):
    nx, ny, box, bounds, (ek, g, P0), flux, lim, acc, CFL, steps, init = spec
    st0 = [np.asarray(a, dtype=np.float64) for a in init()]
    r = R.RefSolver(nx, ny, box=box, bounds=bounds, eos_kind=ek, gamma=g, P0=P0, flux=flux, limiter=lim,
                    accuracy=acc, CFL=CFL)
    r.set_state(*st0)
    dts = np.array([r.step() for _ in range(steps)])
    st = r.state()
    flags = r.set_flags()
    np.savez_compressed(OUT / f"{name}.npz", nx=nx, ny=ny, box=np.array(box, float), bounds=np.array(bounds),
                        eos=np.array([ek, g, P0], float), flux=flux, limiter=lim, accuracy=acc, CFL=CFL,
                        steps=steps, init=np.array(st0), dts=dts, final=np.array(st), flags=flags,
                        wait=r.wait())


def make_isolation():
    """Isolation counters planted on the host (sm_fluid.cpp:179-182, 293-297)."""
    n = 20
    rng = np.random.default_rng(5)
    st0 = [np.asarray(a) for a in riemann2d_case3(n).state]
    wait0 = np.zeros(n * n, np.int32)
    # Counters of 2 or 3: the reference's corrector reads its neighbours'
    # counters while the same loop decrements them (sm_fluid.cpp:293 vs
    # 361-363); starting at 2 or more, no counter reaches 0 during this one
    # step, so every read sees "isolated" exactly as a snapshot would.
    wait0[rng.choice(n * n, 60, replace=False)] = rng.integers(2, 4, 60)
    r = R.RefSolver(n, n, bounds=(2, 2, 2, 2), accuracy=2, limiter="MC", CFL=0.4)
    r.set_state(*st0)
    r.set_wait(wait0)
    dts = np.array([r.step()])
    np.savez_compressed(OUT / "isolation_20_mc.npz", init=np.array(st0), wait0=wait0, dts=dts,
                        final=np.array(r.state()), wait=r.wait())


def make_pointwise():
    rng = np.random.default_rng(2024)
    m = 256
    zL = np.zeros((m, 6))
    zR = np.zeros((m, 6))
    for z in (zL, zR):
        z[:, 0] = 0.1 + 2.0 * rng.random(m)
        z[:, 1] = 1.5 * rng.standard_normal(m)
        z[:, 2] = 1.0 * rng.standard_normal(m)
        z[:, 4] = 0.05 + 2.0 * rng.random(m)
        z[:, 5] = z[:, 4] / (0.4 * z[:, 0])
    out = {}
    for kind, tag in ((3, "hllc"), (2, "hll")):
        out[tag] = np.array([R.flux(kind, a, b) for a, b in zip(zL, zR)])
    vals = np.array([-5.0, -1.0, -1e-3, -1e-300, 0.0, 1e-300, 1e-3, 0.5, 1.0, 2.0, 5.0, np.inf, -np.inf])
    lim = np.array([[[R.limiter(nm, a, b) for b in vals] for a in vals] for nm in LIMITER_NAMES])
    np.savez_compressed(OUT / "pointwise.npz", zL=zL, zR=zR, limiter_values=vals, limiter_names=LIMITER_NAMES,
                        limiter_table=lim, **out)


def blast(cx, cy, p_in=10.0):
    r = np.hypot(cx - 0.5, cy - 0.5)
    rho = np.ones_like(cx)
    p = np.where(r < 0.1, p_in, 0.1)
    return rho, np.zeros_like(cx), np.zeros_like(cx), p, p / (0.4 * rho)


def make_amr(name, n, acc, limiter, bounds, max_level, steps, adapt_rounds):
    """A mesh refined by the reference's EuMesh::refine (flags from
    SmFluid::set_flags on blast data, as in smf_test_2D.cpp:112-117), then
    `steps` steps of the reference's SmFluid::update on it."""
    from oracle import ref_mesh as RM
    R = RM.RefEuMesh(n, n, bounds=bounds, accuracy=acc, limiter=limiter, CFL=0.4, max_level=max_level)
    for _ in range(adapt_rounds):
        c = R.cells()
        R.set_state(*blast(c["cx"], c["cy"]))
        R.solver_flags()
        R.refine()
    c = R.cells()
    R.set_state(*blast(c["cx"], c["cy"]))
    g = R.mesh_arrays()
    init = np.array(R.state())
    dts = np.array([R.step() for _ in range(steps)])
    final = np.array(R.state())
    flags = R.solver_flags()
    np.savez_compressed(OUT / f"{name}.npz", steps=steps, accuracy=acc, limiter=limiter, CFL=0.4,
                        init=init, dts=dts, final=final, flags=flags, wait=R.wait(),
                        **{k: g[k] for k in ("cx", "cy", "vol", "inc", "level", "z_idx", "b_idx", "boundary",
                                             "neib", "nx", "ny", "fx", "fy", "area")})


def make_amr_cycle(name, n, bounds, max_level, distributor, acc, limiter, cycles, steps_per_cycle, random_rounds):
    """The reference's EuMesh / SmFluid through one adaptation schedule
    (tests/amr_cycle.py): set_flags, refine and steps with the solver's
    distributor, then refines with random flags.  Stores the digests of the
    mesh, state and flags after every call."""
    import json
    from oracle import ref_mesh as RM
    sys.path.insert(0, str(ROOT / "tests"))
    import amr_cycle as AC
    R = RM.RefEuMesh(n, n, bounds=bounds, accuracy=acc, limiter=limiter, CFL=0.4, max_level=max_level,
                     distributor=distributor)
    ad = AC.RefAdapter(R)
    ops = AC.schedule(cycles, steps_per_cycle, random_rounds)
    log = AC.run(ad, ops)
    np.savez_compressed(OUT / f"{name}.npz", n=n, bounds=np.array(bounds), max_level=max_level,
                        distributor=distributor, accuracy=acc, limiter=limiter, CFL=0.4, cycles=cycles,
                        steps_per_cycle=steps_per_cycle, random_rounds=random_rounds, log=json.dumps(log))
    return log


MM_MATERIALS = "stiffened:Water,ideal:Air"


def make_mm(name, n, crp_mode, steps, split=0, acc=1, limiter="MC"):
    """The reference's MmFluid (first order, CFL 0.4, direction splitting
    `split`: 0 NONE, 1 SIMPLE, 2 STRANG) on the shock / water column problem
    at n x n: initial states through the reference's mixture closure, the
    interface reconstruction of the first step, `steps` steps, and the
    refinement flags at the end."""
    from oracle import ref_mm as RM
    from zephyr_b200.workloads import shock_water_column
    w = shock_water_column(n)
    r = RM.RefMmFluid(n, n, box=w.box, bounds=w.bounds, materials=MM_MATERIALS, CFL=0.4, accuracy=acc,
                      crp_mode=crp_mode)
    r.set_splitting(split)
    r.set_limiter(limiter)
    r.make_states(w.rho, w.vx, w.vy, w.p, w.beta)
    init = r.states()
    nrm, off = r.interface()
    dts = np.array([r.step() for _ in range(steps)])
    np.savez_compressed(OUT / f"{name}.npz", n=n, box=np.array(w.box), bounds=np.array(w.bounds), crp_mode=crp_mode,
                        split=split, acc=acc, limiter=limiter, CFL=0.4, steps=steps, inputs=np.stack([w.rho, w.vx, w.vy, w.p]), beta=w.beta, init=init,
                        normals=nrm, offsets=off, dts=dts, final=r.states(), flags=r.flags())


# Transfer fixtures: name -> (nx, ny, method, velocity, split, steps).  The
# transfer problem (problems/transfer.cpp): a disk of radius 0.1 at
# (0.15, 0.5) in [0, 1] x [0, 0.7] with ZOE walls, CFL 0.5.
TR_TRANSLATION = ("translation", 0.7, -0.35)
TR_ROTATION = ("rotation", 0.5, 0.5, float(np.pi))
TR_CASES = {
    "tr_disk_40x28_vof_translation_split": (40, 28, "VOF", TR_TRANSLATION, True, 30),
    "tr_disk_40x28_vof_rotation_any": (40, 28, "VOF", TR_ROTATION, False, 30),
    "tr_disk_36x25_vofcrp_rotation_split": (36, 25, "VOF_CRP", TR_ROTATION, True, 25),
    "tr_disk_32x22_crpn1_translation_split": (32, 22, "CRP_N1", TR_TRANSLATION, True, 25),
    "tr_disk_32x22_crpn2_rotation_any": (32, 22, "CRP_N2", TR_ROTATION, False, 25),
    "tr_disk_30x21_crpse_translation_any": (30, 21, "CRP_SE", TR_TRANSLATION, False, 20),
    "tr_disk_30x21_crpv3_rotation_split": (30, 21, "CRP_V3", TR_ROTATION, True, 20),
    "tr_disk_30x21_crpv5_translation_split": (30, 21, "CRP_V5", TR_TRANSLATION, True, 20),
}
# the MUSCL and WENO families (make_golden.py --transfer-high-order)
TR_HIGH_ORDER_CASES = {
    "tr_disk_32x22_muscld_rotation_split": (32, 22, "MUSCLd", TR_ROTATION, True, 25),
    "tr_disk_32x22_muscln_translation_any": (32, 22, "MUSCLn", TR_TRANSLATION, False, 25),
    "tr_disk_30x21_muscldcrp_translation_split": (30, 21, "MUSCLd_CRP", TR_TRANSLATION, True, 20),
    "tr_disk_30x21_musclncrp_rotation_any": (30, 21, "MUSCLn_CRP", TR_ROTATION, False, 20),
    "tr_disk_30x21_musclmc_rotation_split": (30, 21, "MUSCL_MC", TR_ROTATION, True, 20),
    "tr_disk_30x21_musclmccrp_translation_any": (30, 21, "MUSCL_MC_CRP", TR_TRANSLATION, False, 20),
    "tr_disk_30x21_weno_rotation_split": (30, 21, "WENO", TR_ROTATION, True, 20),
    "tr_disk_30x21_wenocrp_translation_any": (30, 21, "WENO_CRP", TR_TRANSLATION, False, 20),
}


def make_tr(name, nx, ny, method, vel, split, steps):
    """The reference's Transfer on the transfer problem: the disk's exact
    cell fractions (BodyDisk::initial), the interface of update_interface,
    `steps` iterations of the problem's time loop (compute_dt, set_dt,
    update X then Y, or ANY), and the refinement flags at the end."""
    from oracle import ref_tr as RT
    box = (0.0, 1.0, 0.0, 0.7)
    r = RT.RefTransfer(nx, ny, box=box, bounds=(2, 2, 2, 2), method=method, CFL=0.5, vel=vel)
    u0 = r.disk(0.15, 0.5, 0.1)
    r.set_u(u0)
    r.update_interface(3 if method.startswith(("VOF", "MUSCL", "WENO")) else 0)
    _, n0, p0 = r.get()
    dts = []
    for _ in range(steps):
        dt = r.compute_dt()
        r.set_dt(dt)
        for d in ((1, 2) if split else (0,)):
            r.update(d)
        dts.append(dt)
    u, n, p = r.get()
    np.savez_compressed(OUT / f"{name}.npz", nx=nx, ny=ny, box=np.array(box), bounds=np.array((2, 2, 2, 2)),
                        method=method, vel_kind=vel[0], vel=np.array(vel[1:], float), split=split, steps=steps,
                        CFL=0.5, u0=u0, n0=n0, p0=p0, dts=np.array(dts), u=u, n=n, p=p, flags=r.flags())


def make_trs(cases=TR_CASES):
    for name, spec in cases.items():
        make_tr(name, *spec)
    print("wrote transfer cases")


VTU_NAMES = ("level", "index", "center", "rank", "flag", "b_idx", "z_idx")


def make_vtu():
    """The reference's VtuFile::save and PvdFile on a rectangle and on a
    refined mesh, with the named cell variables and the SmFluid state as the
    single-fluid driver writes it (density, vel.x, vel.y, pressure, energy).
    Stores the inputs (state, refine flags) and the files' bytes."""
    import shutil
    from oracle import ref_mesh as RME
    tmp = OUT / "_vtu_tmp"
    shutil.rmtree(tmp, ignore_errors=True)
    tmp.mkdir()
    rng = np.random.default_rng(21)
    try:
        # a rectangle with a random state, then a PVD series of two saves
        nx, ny, box = 6, 4, (0.0, 1.0, 0.0, 0.5)
        r = RME.RefEuMesh(nx, ny, box=box, bounds=(2, 1, 2, 1))
        st = [1.0 + rng.random(nx * ny), rng.random(nx * ny) - 0.5, rng.random(nx * ny) - 0.5,
              1.0 + rng.random(nx * ny), 2.5 + rng.random(nx * ny)]
        r.set_state(*st)
        r.write_vtu(tmp / "rect.vtu", names=VTU_NAMES, with_state=True)
        pvd = RME.RefPvd("series", tmp / "out")
        pvd.save(r, 0.0, names=("level",), with_state=True)
        pvd.save(r, 0.125, names=("level",), with_state=True)
        del pvd
        np.savez_compressed(OUT / "vtu_rect_6x4.npz", nx=nx, ny=ny, box=np.array(box), bounds=np.array((2, 1, 2, 1)),
                            state=np.array(st), names=np.array(VTU_NAMES),
                            vtu=np.frombuffer((tmp / "rect.vtu").read_bytes(), np.uint8),
                            pvd=np.frombuffer((tmp / "out" / "series.pvd").read_bytes(), np.uint8),
                            pvd_vtu0=np.frombuffer((tmp / "out" / "series_0.vtu").read_bytes(), np.uint8),
                            pvd_vtu1=np.frombuffer((tmp / "out" / "series_1.vtu").read_bytes(), np.uint8),
                            timesteps=np.array([0.0, 0.125]))
        # an adaptive rectangle after one refine (const distributor)
        n = 8
        a = RME.RefEuMesh(n, n, box=(0.0, 1.0, 0.0, 1.0), bounds=(2, 2, 2, 2), max_level=2, distributor="const")
        st = [1.0 + rng.random(n * n), rng.random(n * n) - 0.5, rng.random(n * n) - 0.5,
              1.0 + rng.random(n * n), 2.5 + rng.random(n * n)]
        a.set_state(*st)
        flags = np.zeros(n * n, np.int32)
        flags[rng.random(n * n) < 0.3] = 1
        a.put_flags(flags)
        a.refine()
        cells = a.cells()
        mvx, mvy = a.verts()
        a.write_vtu(tmp / "amr.vtu", names=VTU_NAMES, with_state=True)
        np.savez_compressed(OUT / "vtu_amr_8_refined.npz", n=n, state=np.array(st), flags=flags, max_level=2,
                            names=np.array(VTU_NAMES), map_x=mvx, map_y=mvy, level=cells["level"],
                            flag=cells["flag"], b_idx=cells["b_idx"], z_idx=cells["z_idx"], cx=cells["cx"],
                            cy=cells["cy"], state_after=np.array(a.state()),
                            vtu=np.frombuffer((tmp / "amr.vtu").read_bytes(), np.uint8))
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    print("wrote vtu cases")


def make_mm_pointwise():
    """Mixture closure, sound speed, mixture HLLC and CRP fluxes of the
    reference on states taken from a running shock / water-column problem,
    and the PLIC helpers on a grid of arguments."""
    from oracle import ref_mm as RM
    from zephyr_b200.workloads import shock_water_column
    n = 48
    w = shock_water_column(n)
    r = RM.RefMmFluid(n, n, box=w.box, bounds=w.bounds, materials=MM_MATERIALS, CFL=0.4, accuracy=1, crp_mode=4)
    r.make_states(w.rho, w.vx, w.vy, w.p, w.beta)
    for _ in range(70):
        dt = r.step()
    s = r.states()
    beta = s[:, 6:10]
    mixed = np.where(((beta > 0).sum(axis=1) > 1))[0]
    # pairs (cell, right neighbour) touching a mixed cell: the +x face, local frame = global
    pairs = [(i, i + n) for i in range(n * (n - 1)) if i in set(mixed) or (i + n) in set(mixed)]
    pairs = pairs[:96]
    h = 0.1 / n
    sl = np.array([s[a] for a, _ in pairs])
    sr = np.array([s[b] for _, b in pairs])
    hllc = np.array([r.hllc(a, b) for a, b in zip(sl, sr)])
    crp, crp_args = [], []
    for a, b in zip(sl, sr):
        # master material: the larger volume fraction on the upwind side (mm_fluid.cpp:201-226)
        up = a if 0.5 * (a[1] + b[1]) > 0.0 else b
        al = [min(max(up[6 + k] * up[0] / up[10 + k], 0.0), 1.0) if up[6 + k] > 0 and not np.isnan(up[10 + k]) else 0.0
              for k in range(2)]
        iA = int(np.argmax(al))
        aL = min(max(a[6 + iA] * a[0] / a[10 + iA], 0.0), 1.0) if not np.isnan(a[10 + iA]) else 0.0
        aR = min(max(b[6 + iA] * b[0] / b[10 + iA], 0.0), 1.0) if not np.isnan(b[10 + iA]) else 0.0
        a_sig = 0.5 * (aL + aR)
        crp_args.append((h, h, iA, a_sig, dt))
        crp.append(r.crp_flux(a, b, h, h, iA, a_sig, dt))
    sound = np.array([r.sound_speed(x) for x in s[mixed]])
    # closure from conservative states (models.cpp:190-204): q of each mixed cell, guesses from its state
    q = np.zeros((len(mixed), 8))
    z = s[mixed]
    q[:, 0] = z[:, 0]
    q[:, 1] = z[:, 0] * z[:, 1]
    q[:, 2] = z[:, 0] * z[:, 2]
    q[:, 3] = z[:, 0] * (z[:, 4] + 0.5 * (z[:, 1] ** 2 + z[:, 2] ** 2))
    q[:, 4:8] = z[:, 0:1] * z[:, 6:10]
    q *= 1.0 + 1.0e-3 * np.sin(np.arange(q.size).reshape(q.shape))  # perturbed, as after an update
    guess = np.concatenate([z[:, 3:4], z[:, 5:6], z[:, 10:14]], axis=1)
    closure = np.array([r.state_from_q(a, g) for a, g in zip(q, guess)])
    al = np.array([0.0, 1e-9, 0.03, 0.2, 0.5, 0.7, 0.97, 1.0 - 1e-9, 1.0])
    ff = np.array([[RM.face_fraction(a, b) for b in al] for a in al])
    cosv = np.array([-1.0, -0.8, -0.3, 0.0, 0.25, 0.6, 0.99, 1.0])
    cflv = np.array([0.0, 0.05, 0.3, 0.9])
    avg = np.array([[[RM.average_flux(a, c, k) for k in cflv] for c in cosv] for a in al])
    nv = np.array([[0.6, 0.8], [1.0, 0.0], [-0.28, 0.96], [0.0, -1.0], [0.70710678, -0.70710678]])
    qfs = np.array([[RM.quad_find_section(a, x, y, 1.0, 0.5) for a in al] for x, y in nv])
    pv = np.linspace(-0.8, 0.8, 17)
    qvf = np.array([[RM.quad_volume_fraction(p, x, y, 1.0, 0.5) for p in pv] for x, y in nv])
    np.savez_compressed(OUT / "mm_pointwise.npz", sl=sl, sr=sr, hllc=hllc, crp=np.array(crp),
                        crp_args=np.array(crp_args), sound_states=s[mixed], sound=sound, q=q, guess=guess,
                        closure=closure, alphas=al, face_fraction=ff, cos=cosv, cfl=cflv, average_flux=avg,
                        normals=nv, quad_find_section=qfs, p=pv, quad_volume_fraction=qvf)


def main():
    for name, spec in CASES.items():
        make_case(name, spec)
        print("wrote", name)
    make_isolation()
    make_pointwise()
    print("wrote isolation, pointwise")
    make_amr("amr_blast_16_first_order", 16, 1, "MC", (2, 2, 1, 1), 2, 20, 4)
    make_amr("amr_blast_16_vanalbada", 16, 2, "van Albada", (2, 2, 2, 2), 2, 20, 4)
    make_amr("amr_blast_12_mc_3levels", 12, 2, "MC", (1, 1, 1, 1), 3, 10, 5)
    print("wrote amr cases")
    make_mm("mm_shock_column_32_plic", 32, 4, 200)
    make_mm("mm_shock_column_24_hllc", 24, 0, 120)
    make_mm("mm_shock_column_24_vs", 24, 3, 120)
    make_mm("mm_shock_column_24_strang_plic", 24, 4, 80, split=2)
    make_mm("mm_shock_column_24_simple_vs", 24, 3, 80, split=1)
    make_mm("mm_shock_column_32_second_order_plic", 32, 4, 60, acc=2, limiter="MC")
    make_mm("mm_shock_column_24_second_order_hllc_minmod", 24, 0, 50, acc=2, limiter="minmod")
    make_mm("mm_shock_column_24_second_order_strang_vs", 24, 3, 40, split=2, acc=2, limiter="van Albada")
    make_mm_pointwise()
    print("wrote multi-material cases")
    make_amr_cycles()
    make_trs()
    make_vtu()


AMR_CYCLES = {
    "adapt_cycle_16_slope_mc": (16, (2, 1, 1, 2), 3, "slope", 2, "MC", 8, 2, 6),
    "adapt_cycle_14_const_first_order": (14, (1, 2, 2, 1), 2, "const", 1, "MC", 6, 3, 5),
}


def make_amr_cycles():
    for name, spec in AMR_CYCLES.items():
        log = make_amr_cycle(name, *spec)
        print("wrote", name, "cells", [e[1] for e in log if "refine" in e[0] or "random" in e[0]])


if __name__ == "__main__":
    if "--transfer-high-order" in sys.argv:
        make_trs(TR_HIGH_ORDER_CASES)
    elif "--transfer" in sys.argv:
        make_trs()
    elif "--vtu" in sys.argv:
        make_vtu()
    elif "--fluxes2" in sys.argv:
        for name in NEW_FLUX_CASES:
            make_case(name, CASES[name])
            print("wrote", name)
    elif "--fluxes" in sys.argv:
        for name in ("godunov_riemann3_32_first_order", "godunov_stiffened_16_mc", "rusanov_fourier_32_vanalbada"):
            make_case(name, CASES[name])
    elif "--amr-cycle" in sys.argv:
        make_amr_cycles()
    elif "--mm2" in sys.argv:
        make_mm("mm_shock_column_32_second_order_plic", 32, 4, 60, acc=2, limiter="MC")
        make_mm("mm_shock_column_24_second_order_hllc_minmod", 24, 0, 50, acc=2, limiter="minmod")
        make_mm("mm_shock_column_24_second_order_strang_vs", 24, 3, 40, split=2, acc=2, limiter="van Albada")
    elif "--mm-split" in sys.argv:
        make_mm("mm_shock_column_24_strang_plic", 24, 4, 80, split=2)
        make_mm("mm_shock_column_24_simple_vs", 24, 3, 80, split=1)
    elif "--mm" in sys.argv:
        make_mm("mm_shock_column_32_plic", 32, 4, 200)
        make_mm("mm_shock_column_24_hllc", 24, 0, 120)
        make_mm("mm_shock_column_24_vs", 24, 3, 120)
        make_mm_pointwise()
    else:
        main()
