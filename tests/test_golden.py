"""Pin the oracle to the reference: the oracle (CPU restatement) against the
golden fixtures that tests/golden/make_golden.py produced from the
reference's own SmFluid, fluxes and limiters compiled from its sources.
Bit-exact equality is required."""
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O

GOLDEN = Path(__file__).resolve().parent / "golden"
LIM_ID = {"none": 0, "unit": 1, "minmod": 2, "MC": 3, "van Leer": 4, "van Albada 1": 5, "van Albada": 5,
          "van Albada 2": 6, "CHARM": 7, "HCUS": 8, "HQUICK": 9, "Koren": 10, "smart": 11, "superbee": 12}
CASES = sorted(p.stem for p in GOLDEN.glob("*.npz")
               if p.stem not in ("pointwise", "isolation_20_mc") and not p.stem.startswith(("amr_", "mm_", "adapt_", "tr_", "vtu_")))
AMR_CASES = sorted(p.stem for p in GOLDEN.glob("amr_*.npz"))


def load(name):
    return np.load(GOLDEN / f"{name}.npz", allow_pickle=False)


def oracle_for(g):
    nx, ny = int(g["nx"]), int(g["ny"])
    box = tuple(float(x) for x in g["box"])
    ek, gamma, P0 = g["eos"]
    m = O.Mesh(nx, ny, *box, bounds=tuple(int(b) for b in g["bounds"]))
    s = O.Solver(m, eos_kind=int(ek), gamma=float(gamma), P0=float(P0), flux=int(g["flux"]),
                 limiter=LIM_ID[str(g["limiter"])], accuracy=int(g["accuracy"]), CFL=float(g["CFL"]))
    return m, s


def test_fixtures_present():
    assert len(CASES) >= 7
    assert (GOLDEN / "pointwise.npz").exists()


@pytest.mark.parametrize("name", CASES)
def test_oracle_matches_reference_step(name):
    g = load(name)
    m, s = oracle_for(g)
    s.set_state(*g["init"])
    dts = np.array([s.step() for _ in range(int(g["steps"]))])
    assert np.array_equal(dts, g["dts"]), "dt sequence differs from the reference"
    final = np.array(s.state())
    assert np.array_equal(final, g["final"]), f"{np.count_nonzero(final != g['final'])} values differ"
    assert np.array_equal(s.wait(), g["wait"])
    assert np.array_equal(s.set_flags(), g["flags"]), "refinement flags differ"


@pytest.mark.parametrize("name", AMR_CASES)
def test_oracle_matches_reference_on_refined_mesh(name):
    """Meshes refined by the reference's EuMesh::refine (hanging faces, up to
    three levels) and stepped by the reference's SmFluid: the oracle must
    reproduce dt, states and flags bit for bit."""
    g = load(name)
    m = O.Mesh.from_arrays(g)
    s = O.Solver(m, limiter=LIM_ID[str(g["limiter"])], accuracy=int(g["accuracy"]), CFL=float(g["CFL"]))
    s.set_state(*g["init"])
    dts = np.array([s.step() for _ in range(int(g["steps"]))])
    assert np.array_equal(dts, g["dts"])
    assert np.array_equal(np.array(s.state()), g["final"])
    assert np.array_equal(s.set_flags(), g["flags"])
    assert (g["boundary"] == -1).any() and (g["level"] > 0).any()


def test_oracle_matches_reference_isolation():
    g = load("isolation_20_mc")
    m = O.Mesh(20, 20, bounds=(2, 2, 2, 2))
    s = O.Solver(m, limiter=3, accuracy=2, CFL=0.4)
    s.set_state(*g["init"])
    s.set_wait(g["wait0"])
    assert s.step() == g["dts"][0]
    assert np.array_equal(np.array(s.state()), g["final"])
    assert np.array_equal(s.wait(), g["wait"])


def test_oracle_fluxes_match_reference():
    g = load("pointwise")
    for kind, tag in ((O.FLUX_HLLC, "hllc"), (O.FLUX_HLL, "hll")):
        got = np.array([O.flux(kind, a, b) for a, b in zip(g["zL"], g["zR"])])
        assert np.array_equal(got, g[tag]), tag


def test_oracle_limiters_match_reference():
    g = load("pointwise")
    vals = g["limiter_values"]
    for name, table in zip(g["limiter_names"], g["limiter_table"]):
        got = np.array([[O.limiter(LIM_ID[str(name)], a, b) for b in vals] for a in vals])
        assert np.array_equal(got, table, equal_nan=True), str(name)


def test_oracle_matches_reference_build_directly():
    """When the reference-source build is present, compare on fresh inputs."""
    from oracle import ref as R
    if not R.available():
        pytest.skip("oracle/_ref/libzref.so not built (no reference tree on this machine)")
    rng = np.random.default_rng(99)
    for bounds, acc, lim in (((3, 3, 2, 2), 2, "van Albada"), ((1, 2, 1, 2), 2, "MC"), ((2, 2, 3, 3), 1, "MC")):
        n = 18
        N = n * n
        rho = 1.0 + rng.random(N)
        u = 0.5 * rng.standard_normal(N)
        v = 0.5 * rng.standard_normal(N)
        p = 0.5 + rng.random(N)
        st = (rho, u, v, p, p / (0.4 * rho))
        r = R.RefSolver(n, n, bounds=bounds, accuracy=acc, limiter=lim, CFL=0.45)
        s = O.Solver(O.Mesh(n, n, bounds=bounds), limiter=LIM_ID[lim], accuracy=acc, CFL=0.45)
        r.set_state(*st)
        s.set_state(*st)
        for _ in range(12):
            assert r.step() == s.step()
        assert np.array_equal(np.array(r.state()), np.array(s.state()))
        gr, go = r.grad(), s.grad()
        assert np.array_equal(gr[0], go[0]) and np.array_equal(gr[1], go[1])


@pytest.mark.parametrize("kind,name", [(4, "HLLC_M"), (5, "HLLC_LM"), (6, "CIR1"), (7, "CIR2")])
def test_oracle_more_fluxes_match_reference_build_directly(kind, name):
    """HLLC_M, HLLC_LM, CIR1 and CIR2 (NumFlux::create, num_flux.cpp:6-35)
    pointwise against the reference's own classes on random ideal and
    stiffened states, subsonic and supersonic, with tangential shear and
    low Mach numbers (HLLC_LM's sine branch); bit for bit."""
    from oracle import ref as R
    if not R.available():
        pytest.skip("reference-source build not present")
    rng = np.random.default_rng(40 + kind)
    for eos in [(0, 1.4, 0.0, 0.0), (1, 4.4, 6e8, 0.0), (1, 2.0, 1e5, 3.0)]:
        for _ in range(600):
            zs = []
            for _ in range(2):
                if eos[0] == 0:
                    r, p = 0.1 + 2 * rng.random(), 0.05 + 3 * rng.random()
                    scale = 10.0 ** rng.uniform(-3, 0.5)
                else:
                    r = 900 + 200 * rng.random() if eos[2] > 1e6 else 0.5 + rng.random()
                    p = 1e5 * (0.5 + 10 * rng.random())
                    scale = (100.0 if eos[2] > 1e6 else 1.0) * 10.0 ** rng.uniform(-3, 0.5)
                u, v = rng.normal() * scale, rng.normal() * scale
                e = p / ((eos[1] - 1) * r) if eos[0] == 0 else eos[3] + (p + eos[1] * eos[2]) / ((eos[1] - 1) * r)
                zs.append(np.array([r, u, v, 0.0, p, e]))
            zl, zr = zs
            a = np.asarray(O.flux(kind, zl, zr, *eos))
            b = np.asarray(R.flux(kind, zl, zr, *eos))
            assert np.array_equal(a, b, equal_nan=True), (name, eos, zl, zr, a, b)


def test_oracle_fluxes_match_reference_build_directly():
    """Godunov (exact Riemann solver) and Rusanov, pointwise, against the
    reference's own NumFlux on random ideal and stiffened states (shocks,
    rarefactions, fans on the face, vacuum); NaN where the reference's is."""
    from oracle import ref as R
    if not R.available():
        pytest.skip("reference-source build not present")
    rng = np.random.default_rng(3)
    for eos in [(0, 1.4, 0.0, 0.0), (1, 4.4, 6e8, 0.0), (1, 2.0, 1e5, 3.0)]:
        for kind in (0, 1):
            for _ in range(800):
                zs = []
                for _ in range(2):
                    if eos[0] == 0:
                        r, p = 0.1 + 2 * rng.random(), 0.05 + 3 * rng.random()
                    else:
                        r = 900 + 200 * rng.random() if eos[2] > 1e6 else 0.5 + rng.random()
                        p = 1e5 * (0.5 + 10 * rng.random())
                    u, v = rng.normal() * (100.0 if eos[2] > 1e6 else 1.0), rng.normal()
                    e = p / ((eos[1] - 1) * r) if eos[0] == 0 else eos[3] + (p + eos[1] * eos[2]) / ((eos[1] - 1) * r)
                    zs.append(np.array([r, u, v, 0.0, p, e]))
                zl, zr = zs
                if rng.random() < 0.1:
                    zl[1], zr[1] = 5.0, -5.0  # colliding: two shocks
                elif rng.random() < 0.1:
                    zl[1], zr[1] = -5.0, 5.0  # receding: rarefactions, vacuum
                a = np.asarray(O.flux(kind, zl, zr, *eos))
                b = np.asarray(R.flux(kind, zl, zr, *eos))
                assert np.array_equal(a, b, equal_nan=True), (kind, eos, zl, zr)
