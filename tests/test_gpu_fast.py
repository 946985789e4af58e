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
           precision=None, flux=3):
    eos = eos or Z.IdealGas(1.4)
    gen = Z.Rectangle(*box)
    gen.set_boundaries(Z.Boundaries(*bounds))
    gen.set_sizes(nx, ny)
    mesh = Z.EuMesh(gen)
    solver = Z.SmFluid(eos, precision=precision or Z.Precision.FP64, kernels=Z.Kernels.FAST)
    solver.set_accuracy(acc)
    solver.set_CFL(CFL)
    solver.set_limiter(lim)
    solver.set_method(Z.Fluxes(flux))
    solver.set_scheme(Z.Scheme(scheme))
    solver.add_types(mesh)
    osv = O.Solver(O.Mesh(nx, ny, *box, bounds=bounds), eos_kind=eos.kind, gamma=eos.gamma, P0=eos.P0,
                   e0=eos.e0, flux=flux, limiter=LIMS[lim], accuracy=acc, scheme=scheme, CFL=CFL, threads=8)
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


@pytest.mark.parametrize("name,cfg,kind", CASES, ids=[c[0] for c in CASES])
def test_fast_within_tolerance_per_step(gpu_lib, name, cfg, kind):
    Z = gpu_lib
    mesh, solver, osv = _setup(Z, **cfg)
    _per_step(mesh, solver, osv, _state(kind, cfg["nx"], cfg["ny"]), 12, name)


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
