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
}


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


if __name__ == "__main__":
    main()
