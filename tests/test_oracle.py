"""The oracle on its own (CPU): pointwise formulas against independent
restatements, and size-independent properties of the step."""
import math

import numpy as np
import pytest

from oracle import oracle as O


def py_limiter(kind, a, b):
    """limiter.cxx binary forms, restated in Python."""
    if kind == 0:
        return 0.0
    if kind == 1:
        return 1.0
    if kind == 2:
        return 0.0 if a * b <= 0 else min(a / b, 1.0)
    if kind == 3:
        r = a / b if b != 0 else (math.copysign(math.inf, a) if a != 0 else math.nan)
        if math.isnan(r):
            return 0.0
        return max(0.0, min(2 * r, min(0.5 * (1.0 + r), 2.0)))
    if kind == 5:
        if a * b <= 0:
            return 0.0
        return a * (a + b) / (a * a + b * b)
    raise ValueError(kind)


@pytest.mark.parametrize("kind", [0, 1, 2, 3, 5])
def test_limiters_against_python(kind):
    vals = [-5.0, -1.0, -1e-3, 0.0, 1e-3, 0.5, 1.0, 2.0, 5.0]
    for a in vals:
        for b in vals:
            if kind in (2, 3) and b == 0.0:
                continue
            assert O.limiter(kind, a, b) == py_limiter(kind, a, b), (kind, a, b)


def test_vanalbada1_table():
    # phi(a, b) = a (a + b) / (a^2 + b^2) for a b > 0, 0 otherwise (limiter.cxx:77-82)
    assert O.limiter(5, 1.0, 2.0) == 0.6
    assert O.limiter(5, 2.0, 1.0) == 1.2
    assert O.limiter(5, -1.0, 2.0) == 0.0
    assert O.limiter(5, 3.0, 3.0) == 1.0


def phys_flux(z, gamma=1.4):
    rho, u, v, w, p, e = z
    E = rho * (e + 0.5 * (u * u + v * v + w * w))
    return np.array([rho * u, rho * u * u + p, rho * u * v, rho * u * w, (E + p) * u])


def test_hllc_consistency_and_supersonic():
    z = np.array([1.3, 0.2, -0.4, 0.0, 0.9, 0.9 / (0.4 * 1.3)])
    F = O.flux(O.FLUX_HLLC, z, z)
    assert np.allclose(F, phys_flux(z), rtol=1e-13, atol=1e-15)
    zs = z.copy()
    zs[1] = 5.0  # supersonic to the right: upwind flux of the left state, exactly
    assert np.array_equal(O.flux(O.FLUX_HLLC, zs, zs * np.array([1, 1, 1, 1, 1.1, 1.1])), phys_flux(zs))


def test_hll_consistency():
    z = np.array([0.7, -0.3, 0.1, 0.0, 2.0, 2.0 / (0.4 * 0.7)])
    assert np.allclose(O.flux(O.FLUX_HLL, z, z), phys_flux(z), rtol=1e-13, atol=1e-15)


def test_eos_consistency():
    # ideal: e(rho, p(rho, e)) == e; stiffened "Water": gamma 4.4, P0 6e8
    for kind, g, P0 in ((0, 1.4, 0.0), (1, 4.4, 6.0e8)):
        rho, e = 998.0, 1.0e6
        p, _, _ = O.eos(kind, g, P0, 0.0, rho, e)
        _, e2, c = O.eos(kind, g, P0, 0.0, rho, p)
        assert abs(e2 - e) <= 1e-12 * abs(e)
        assert c > 0


def _state(n, seed=1):
    rng = np.random.default_rng(seed)
    N = n * n
    rho = 1.0 + 0.2 * rng.random(N)
    u = 0.1 * rng.standard_normal(N)
    v = 0.1 * rng.standard_normal(N)
    p = 1.0 + 0.2 * rng.random(N)
    return rho, u, v, p, p / (0.4 * rho)


def _totals(st):
    rho, u, v, p, e = st
    return np.array([rho.sum(), (rho * u).sum(), (rho * v).sum(), (rho * (e + 0.5 * (u * u + v * v))).sum()])


@pytest.mark.parametrize("acc,scheme", [(1, 0), (2, 0), (2, 1)])
def test_periodic_conservation(acc, scheme):
    n = 24
    m = O.Mesh(n, n, bounds=(O.BC_PERIODIC,) * 4)
    s = O.Solver(m, limiter=5, accuracy=acc, scheme=scheme, CFL=0.4)
    st = _state(n)
    s.set_state(*st)
    t0 = _totals(st)
    s.steps(20)
    t1 = _totals(s.state())
    assert np.all(np.abs(t1 - t0) <= 1e-12 * np.array([t0[0], t0[0], t0[0], t0[3]]))


def test_uniform_state_is_steady():
    n = 16
    for bounds in ((O.BC_ZOE,) * 4, (O.BC_WALL,) * 4, (O.BC_PERIODIC,) * 4):
        m = O.Mesh(n, n, bounds=bounds)
        s = O.Solver(m, limiter=3, accuracy=2, CFL=0.5)
        N = n * n
        st = (np.full(N, 1.2), np.zeros(N), np.zeros(N), np.full(N, 0.8), np.full(N, 0.8 / (0.4 * 1.2)))
        s.set_state(*st)
        s.steps(5)
        out = s.state()
        for a, b in zip(out, st):
            assert np.allclose(a, b, rtol=1e-14, atol=1e-15)


def test_mirror_symmetry():
    """Data mirrored about x = 1/2 (u odd) stay mirrored to rounding."""
    n = 20
    m = O.Mesh(n, n, bounds=(O.BC_ZOE,) * 4)
    s = O.Solver(m, limiter=5, accuracy=2, CFL=0.4)
    rng = np.random.default_rng(5)
    half = rng.random((n // 2, n))
    f = np.concatenate([half, half[::-1]], axis=0)  # f[i, j] = f[n-1-i, j]
    rho = (1.0 + 0.3 * f).reshape(-1)
    p = (1.0 + 0.2 * f.T.copy().T).reshape(-1)
    uu = 0.2 * np.concatenate([half, -half[::-1]], axis=0).reshape(-1)
    v = 0.1 * f.reshape(-1)
    st = (rho, uu, v, p, p / (0.4 * rho))
    s.set_state(*st)
    s.steps(10)
    r, u, v2, pp, e = (a.reshape(n, n) for a in s.state())
    assert np.allclose(r, r[::-1], rtol=1e-12)
    assert np.allclose(u, -u[::-1], atol=1e-12)
    assert np.allclose(pp, pp[::-1], rtol=1e-12)


def test_sod_along_x_matches_along_y():
    """The same 1-D Riemann problem along x and along y gives transposed fields."""
    n = 32
    N = n * n
    X = (np.arange(n) + 0.5) / n
    left = X < 0.5
    rho1 = np.where(left, 1.0, 0.125)
    p1 = np.where(left, 1.0, 0.1)
    res = []
    for axis in (0, 1):
        rho = np.repeat(rho1, n) if axis == 0 else np.tile(rho1, n)
        p = np.repeat(p1, n) if axis == 0 else np.tile(p1, n)
        m = O.Mesh(n, n, bounds=(O.BC_ZOE,) * 4)
        s = O.Solver(m, limiter=3, accuracy=2, CFL=0.4)
        s.set_state(rho, np.zeros(N), np.zeros(N), p, p / (0.4 * rho))
        s.steps(15)
        res.append(s.state())
    rx = res[0][0].reshape(n, n)
    ry = res[1][0].reshape(n, n)
    assert np.allclose(rx, ry.T, rtol=1e-13)
    assert np.allclose(res[0][1].reshape(n, n), res[1][2].reshape(n, n).T, atol=1e-13)


def test_flags_values():
    n = 16
    m = O.Mesh(n, n, bounds=(O.BC_ZOE,) * 4)
    s = O.Solver(m, limiter=3, accuracy=2)
    N = n * n
    rho = np.ones(N)
    rho[: N // 2] = 2.0  # jump across i = n/2
    s.set_state(rho, np.zeros(N), np.zeros(N), np.ones(N), 1.0 / (0.4 * rho))
    f = s.set_flags().reshape(n, n)
    assert np.all(f[n // 2 - 1] == 1) and np.all(f[n // 2] == 1)
    assert np.all(f[: n // 2 - 1] == -1) and np.all(f[n // 2 + 1:] == -1)
