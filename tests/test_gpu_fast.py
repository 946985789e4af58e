"""FAST (FP64, face-once tiles) and MIXED (FP32 faces, FP64 conserved) kernel
families against the oracle.

FAST: each step starts from the oracle's state and must land within 1e-12
relative of the oracle's next state in the conserved fields (the per-step
tolerance of the FP64 form; momenta are scaled by the field's magnitude).  The isolation
counters and the dt sequence must match.

MIXED: after many steps the L1 density error relative to the FP64 oracle
must stay within 1e-5 (the stated target of the mixed form); L-infinity is
reported.
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

REL_TOL = 1e-12
L1_TOL_MIXED = 1e-5
LIMS = {"MC": 3, "van Albada": 5, "minmod": 2, "superbee": 12}


def _setup(Z, nx, ny, bounds, box=(0.0, 1.0, 0.0, 1.0), acc=2, lim="van Albada", scheme=0, CFL=0.4, eos=None,
           precision=None, flux=3, kernels=None, threads=8):
    eos = eos or Z.IdealGas(1.4)
    gen = Z.Rectangle(*box)
    gen.set_boundaries(Z.Boundaries(*bounds))
    gen.set_sizes(nx, ny)
    mesh = Z.EuMesh(gen)
    solver = Z.SmFluid(eos, precision=precision or Z.Precision.FP64, kernels=kernels or Z.Kernels.FAST)
    solver.set_accuracy(acc)
    solver.set_CFL(CFL)
    solver.set_limiter(lim)
    solver.set_method(Z.Fluxes(flux))
    solver.set_scheme(Z.Scheme(scheme))
    solver.add_types(mesh)
    osv = O.Solver(O.Mesh(nx, ny, *box, bounds=bounds), eos_kind=eos.kind, gamma=eos.gamma, P0=eos.P0,
                   e0=eos.e0, flux=flux, limiter=LIMS[lim], accuracy=acc, scheme=scheme, CFL=CFL, threads=threads)
    return mesh, solver, osv


def _rel(a, b, k):
    scale = np.maximum(np.abs(b), 1e-300)
    if k in (1, 2):
        scale = np.maximum(scale, np.max(np.abs(b)))
    return float(np.max(np.abs(a - b) / scale))


def _cons(z):
    rho, u, v, p, e = z
    return [rho, rho * u, rho * v, rho * (e + 0.5 * (u * u + v * v))]


def _rel_cons(g, o):
    """Largest relative difference of the conserved fields (momenta scaled
    by their field's magnitude, since they pass through zero)."""
    cg, co = _cons(g), _cons(o)
    return max(_rel(cg[k], co[k], k) for k in range(4))


def _per_step(mesh, solver, osv, state, steps, what):
    osv.set_state(*state)
    worst = 0.0
    for s in range(steps):
        z = osv.state()
        w = osv.wait()
        mesh.set_state(*z)
        mesh.set_wait(w)
        solver.update(mesh)
        dt_g = solver.dt()
        dt_o = osv.step()
        assert abs(dt_g - dt_o) <= REL_TOL * dt_o, f"{what} step {s}: dt {dt_g} vs {dt_o}"
        g, o = mesh.get_state(), osv.state()
        r = _rel_cons(g, o)
        worst = max(worst, r)
        assert r <= REL_TOL, f"{what} step {s}: conserved fields rel diff {r:.3e}"
        assert np.array_equal(mesh.get_wait(), osv.wait()), f"{what} step {s}: isolation counters"
    return worst


CASES = [
    ("first order riemann", dict(nx=64, ny=64, bounds=(2, 2, 2, 2), acc=1, lim="MC"), "riemann"),
    ("MC riemann", dict(nx=64, ny=64, bounds=(2, 2, 2, 2), lim="MC"), "riemann"),
    ("van Albada fourier periodic", dict(nx=64, ny=64, bounds=(3, 3, 3, 3)), "fourier"),
    ("superbee walls", dict(nx=48, ny=48, bounds=(1, 1, 1, 1), lim="superbee"), "riemann"),
    ("minmod nonsquare", dict(nx=37, ny=19, bounds=(1, 1, 3, 3), box=(0.0, 2.0, -0.5, 0.5), lim="minmod"),
     "random"),
    ("heun fourier", dict(nx=64, ny=64, bounds=(3, 3, 3, 3), scheme=1), "fourier"),
    ("heun riemann walls", dict(nx=40, ny=40, bounds=(1, 2, 1, 2), scheme=1, lim="MC"), "riemann"),
    ("hll first order", dict(nx=40, ny=40, bounds=(2, 2, 1, 1), acc=1, flux=2), "riemann"),
    ("godunov first order riemann", dict(nx=48, ny=48, bounds=(2, 2, 2, 2), acc=1, lim="MC", flux=0), "riemann"),
    ("godunov MC riemann", dict(nx=48, ny=48, bounds=(2, 2, 1, 1), lim="MC", flux=0), "riemann"),
    ("rusanov fourier periodic", dict(nx=48, ny=48, bounds=(3, 3, 3, 3), flux=1), "fourier"),
    # tile edges of the fused kernels (30 x 14 interior cells per block):
    # sizes that leave partial tiles, thin periodic axes, mixed boundaries
    ("tiles periodic 43x61", dict(nx=43, ny=61, bounds=(3, 3, 3, 3)), "random"),
    ("tiles walls zoe 29x95", dict(nx=29, ny=95, bounds=(1, 2, 2, 1), lim="MC"), "random"),
    ("tiles thin periodic 3x70", dict(nx=3, ny=70, bounds=(3, 3, 1, 1)), "random"),
    ("tiles thin periodic 70x2", dict(nx=70, ny=2, bounds=(2, 2, 3, 3), lim="minmod"), "random"),
    ("tiles hll 31x31", dict(nx=31, ny=31, bounds=(1, 1, 2, 2), flux=2, lim="MC"), "random"),
    ("tiles heun 57x33 walls", dict(nx=57, ny=33, bounds=(1, 1, 1, 1), scheme=1), "random"),
    ("tiles heun periodic 15x31", dict(nx=15, ny=31, bounds=(3, 3, 3, 3), scheme=1, lim="superbee"), "random"),
]


def _state(kind, nx, ny):
    from zephyr_b200.workloads import fourier_smooth, riemann2d_case3
    if kind == "riemann":
        return riemann2d_case3(nx).state
    if kind == "fourier":
        return fourier_smooth(nx).state
    rng = np.random.default_rng(7)
    n = nx * ny
    rho = 1.0 + 0.3 * rng.random(n)
    u = 0.2 * rng.standard_normal(n)
    v = 0.2 * rng.standard_normal(n)
    p = 1.0 + 0.5 * rng.random(n)
    return rho, u, v, p, p / (0.4 * rho)


@pytest.mark.parametrize("family", ["FAST", "FAST_TWO_PASS"])
@pytest.mark.parametrize("name,cfg,kind", CASES, ids=[c[0] for c in CASES])
def test_fast_within_tolerance_per_step(gpu_lib, name, cfg, kind, family):
    Z = gpu_lib
    mesh, solver, osv = _setup(Z, **cfg, kernels=Z.Kernels[family])
    _per_step(mesh, solver, osv, _state(kind, cfg["nx"], cfg["ny"]), 12, name)


@pytest.mark.parametrize("family", ["FAST", "FAST_TWO_PASS"])
@pytest.mark.parametrize("scheme", [0, 1], ids=["predictor_corrector", "heun"])
def test_fast_headline_size_per_step(gpu_lib, family, scheme):
    """The benchmark's own workload (2048 x 2048 periodic smooth data, van
    Albada, HLLC, CFL 0.4) through the FAST kernels: each step starts from the
    oracle's state and must land within 1e-12 of the oracle's next state."""
    import os
    Z = gpu_lib
    from zephyr_b200.workloads import fourier_smooth
    n = 2048
    mesh, solver, osv = _setup(Z, n, n, (3, 3, 3, 3), scheme=scheme, kernels=Z.Kernels[family],
                               threads=max(8, os.cpu_count() or 8))
    worst = _per_step(mesh, solver, osv, fourier_smooth(n).state, 2, f"2048^2 {family} scheme {scheme}")
    print(f"2048^2 {family} scheme {scheme}: worst conserved rel diff per step {worst:.3e}")


@pytest.mark.parametrize("scheme", [0, 1], ids=["predictor_corrector", "heun"])
def test_mixed_headline_size_one_step(gpu_lib, scheme):
    """One mixed-form step of the benchmark's workload from the oracle's
    state: density within 1e-6 relative of the FP64 oracle's next state (FP32
    face arithmetic, FP64 update)."""
    import os
    Z = gpu_lib
    from zephyr_b200.workloads import fourier_smooth
    n = 2048
    mesh, solver, osv = _setup(Z, n, n, (3, 3, 3, 3), scheme=scheme, precision=Z.Precision.MIXED,
                               threads=max(8, os.cpu_count() or 8))
    st = fourier_smooth(n).state
    mesh.set_state(*st)
    osv.set_state(*st)
    solver.update(mesh)
    dt_o = osv.step()
    assert abs(solver.dt() - dt_o) <= 1e-12 * dt_o
    g, o = mesh.get_state(), osv.state()
    r = float(np.max(np.abs(g[0] - o[0]) / np.abs(o[0])))
    print(f"2048^2 mixed scheme {scheme}: one-step max rel density difference {r:.3e}")
    assert r <= 1e-6


@pytest.mark.parametrize("scheme", [0, 1], ids=["predictor_corrector", "heun"])
def test_mixed_l1_at_headline_size_and_horizon(gpu_lib, scheme):
    """The mixed form over the full configuration: 2048 x 2048 periodic smooth
    data, 500 steps.  Its density is compared with the FP64 parity form after
    the same 500 steps (the parity kernels are bit-exact with the reference's
    step); L1 relative error within 1e-5."""
    Z = gpu_lib
    from zephyr_b200.workloads import fourier_smooth
    n, steps = 2048, 500
    w = fourier_smooth(n)
    res = {}
    for name, prec, kern in (("mixed", Z.Precision.MIXED, Z.Kernels.FAST),
                             ("parity", Z.Precision.FP64, Z.Kernels.PARITY)):
        gen = Z.Rectangle(0.0, 1.0, 0.0, 1.0)
        gen.set_boundaries(Z.Boundaries(3, 3, 3, 3))
        gen.set_sizes(n, n)
        mesh = Z.EuMesh(gen)
        solver = Z.SmFluid(Z.IdealGas(1.4), precision=prec, kernels=kern)
        solver.set_accuracy(2)
        solver.set_CFL(0.4)
        solver.set_limiter("van Albada")
        solver.set_scheme(Z.Scheme(scheme))
        solver.add_types(mesh)
        mesh.set_state(*w.state)
        solver.update(mesh, steps=steps)
        res[name] = mesh.get_state()[0]
        del solver, mesh
    g, o = res["mixed"], res["parity"]
    l1 = float(np.sum(np.abs(g - o)) / np.sum(np.abs(o)))
    linf = float(np.max(np.abs(g - o)) / np.max(np.abs(o)))
    print(f"mixed scheme={scheme} 2048^2 x {steps}: L1 rel density error {l1:.3e}, Linf {linf:.3e}")
    assert l1 <= L1_TOL_MIXED


def test_fast_stiffened(gpu_lib):
    Z = gpu_lib
    eos = Z.StiffenedGas(4.4, 6.0e8, 0.0)
    n = 32
    rng = np.random.default_rng(11)
    N = n * n
    rho = 1000.0 * (1.0 + 0.01 * rng.random(N))
    u = 5.0 * rng.standard_normal(N)
    v = 5.0 * rng.standard_normal(N)
    p = 1.0e5 * (1.0 + rng.random(N))
    e = eos.energy_rP(rho, p)
    mesh, solver, osv = _setup(Z, n, n, (2, 2, 1, 1), box=(0.0, 0.1, 0.0, 0.1), eos=eos)
    _per_step(mesh, solver, osv, (rho, u, v, p, e), 8, "stiffened")


def test_fast_isolation(gpu_lib):
    Z = gpu_lib
    from zephyr_b200.workloads import riemann2d_case3
    mesh, solver, osv = _setup(Z, 40, 40, (2, 2, 2, 2), lim="MC")
    rng = np.random.default_rng(3)
    wait = np.zeros(1600, np.int32)
    wait[rng.choice(1600, 200, replace=False)] = rng.integers(1, 4, 200)
    osv.set_state(*riemann2d_case3(40).state)
    osv.set_wait(wait)
    for s in range(4):
        z, w = osv.state(), osv.wait()
        mesh.set_state(*z)
        mesh.set_wait(w)
        solver.update(mesh)
        osv.step()
        assert np.array_equal(mesh.get_wait(), osv.wait())
        assert _rel_cons(mesh.get_state(), osv.state()) <= REL_TOL


def test_fast_many_steps_stay_close(gpu_lib):
    """Free-running FAST vs oracle over 100 steps on smooth data."""
    Z = gpu_lib
    from zephyr_b200.workloads import fourier_smooth
    w = fourier_smooth(128)
    mesh, solver, osv = _setup(Z, 128, 128, (3, 3, 3, 3))
    mesh.set_state(*w.state)
    osv.set_state(*w.state)
    for s in range(100):  # dt comes from the corrector's fused CFL minimum after step 0
        solver.update(mesh)
        dt_g, dt_o = solver.dt(), osv.step()
        assert abs(dt_g - dt_o) <= 1e-10 * dt_o, f"step {s}: dt {dt_g} vs {dt_o}"
    g, o = mesh.get_state(), osv.state()
    assert _rel(g[0], o[0], 0) < 1e-10
    assert _rel(g[3], o[3], 3) < 1e-10


def test_fast_conservation_full_size(gpu_lib):
    Z = gpu_lib
    from zephyr_b200.workloads import fourier_smooth
    w = fourier_smooth(2048)
    mesh, solver, _ = _setup(Z, 16, 16, (3, 3, 3, 3))  # oracle unused
    mesh = Z.EuMesh(w.gen)
    solver.add_types(mesh)
    mesh.set_state(*w.state)

    def totals(st):
        rho, u, v, p, e = st
        return np.array([rho.sum(), (rho * u).sum(), (rho * v).sum(),
                         (rho * (e + 0.5 * (u * u + v * v))).sum()])

    t0 = totals(w.state)
    solver.update(mesh, steps=20)
    t1 = totals(mesh.get_state())
    scale = np.array([t0[0], t0[0], t0[0], t0[3]])
    assert np.all(np.abs(t1 - t0) / scale < 1e-11), (t1 - t0) / scale


@pytest.mark.parametrize("scheme", [0, 1])
def test_mixed_l1_error_vs_fp64_oracle(gpu_lib, scheme):
    """The mixed form's density after 100 steps of the smooth periodic
    problem: L1 error relative to the FP64 oracle within 1e-5."""
    Z = gpu_lib
    from zephyr_b200.workloads import fourier_smooth
    n = 256
    w = fourier_smooth(n)
    mesh, solver, osv = _setup(Z, n, n, (3, 3, 3, 3), scheme=scheme, precision=Z.Precision.MIXED)
    mesh.set_state(*w.state)
    osv.set_state(*w.state)
    steps = 100
    solver.update(mesh, steps=steps)
    osv.steps(steps)
    g, o = mesh.get_state(), osv.state()
    l1 = float(np.sum(np.abs(g[0] - o[0])) / np.sum(np.abs(o[0])))
    linf = float(np.max(np.abs(g[0] - o[0])) / np.max(np.abs(o[0])))
    print(f"mixed scheme={scheme}: L1 rel density error {l1:.3e}, Linf {linf:.3e}")
    assert l1 <= L1_TOL_MIXED
    assert linf <= 1e-3


def test_mixed_riemann_stays_physical(gpu_lib):
    """Strong shocks in FP32 faces: the state stays finite and positive and
    close to the FP64 oracle in L1."""
    Z = gpu_lib
    from zephyr_b200.workloads import riemann2d_case3
    n = 128
    mesh, solver, osv = _setup(Z, n, n, (2, 2, 2, 2), lim="MC", precision=Z.Precision.MIXED)
    st = riemann2d_case3(n).state
    mesh.set_state(*st)
    osv.set_state(*st)
    solver.update(mesh, steps=60)
    osv.steps(60)
    g, o = mesh.get_state(), osv.state()
    assert np.all(np.isfinite(g[0])) and np.all(g[0] > 0) and np.all(g[3] > 0)
    l1 = float(np.sum(np.abs(g[0] - o[0])) / np.sum(np.abs(o[0])))
    print(f"mixed riemann: L1 rel density error {l1:.3e}")
    assert l1 <= 1e-4


def test_mixed_wait_and_flags_paths(gpu_lib):
    Z = gpu_lib
    from zephyr_b200.workloads import riemann2d_case3
    mesh, solver, osv = _setup(Z, 32, 32, (2, 2, 2, 2), lim="MC", precision=Z.Precision.MIXED)
    mesh.set_state(*riemann2d_case3(32).state)
    osv.set_state(*riemann2d_case3(32).state)
    wait = np.zeros(1024, np.int32)
    wait[::7] = 2
    mesh.set_wait(wait)
    osv.set_wait(wait)
    solver.update(mesh)
    osv.step()
    assert np.array_equal(mesh.get_wait(), osv.wait())
    f = solver.set_flags(mesh)
    assert set(np.unique(f)) <= {-1, 0, 1}
