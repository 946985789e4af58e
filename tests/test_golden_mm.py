"""Pin the multi-material oracle (oracle/zoracle_mm.inc) to the reference:
the golden fixtures of tests/golden/mm_*.npz were produced by the reference's
own MmFluid, MixturePT, HLLC, CRP and PLIC code compiled from its sources
(tests/golden/make_golden.py --mm).  Bit-exact equality is required; NaN
entries (true densities of absent materials) must match as NaN."""
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O

GOLDEN = Path(__file__).resolve().parent / "golden"
CASES = sorted(p.stem for p in GOLDEN.glob("mm_shock_column_*.npz"))
LIM_ID = {"minmod": 2, "MC": 3, "van Albada": 5}


def same(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return a.shape == b.shape and bool(np.all((a == b) | (np.isnan(a) & np.isnan(b))))


def solver_for(g):
    n = int(g["n"])
    m = O.Mesh(n, n, *(float(x) for x in g["box"]), bounds=tuple(int(b) for b in g["bounds"]))
    s = O.MmSolver(m, CFL=float(g["CFL"]), crp_mode=int(g["crp_mode"]))
    s.set_splitting(int(g["split"]) if "split" in g.files else 0)
    if "acc" in g.files:
        s.set_accuracy(int(g["acc"]), LIM_ID[str(g["limiter"])])
    return m, s


def test_mm_fixtures_present():
    assert len(CASES) >= 3 and (GOLDEN / "mm_pointwise.npz").exists()


@pytest.mark.parametrize("name", CASES)
def test_oracle_mm_matches_reference_steps(name):
    g = np.load(GOLDEN / f"{name}.npz")
    m, s = solver_for(g)
    rho, vx, vy, p = g["inputs"]
    s.make_states(rho, vx, vy, p, g["beta"])
    assert same(s.states(), g["init"]), "mixture closure of the initial states differs"
    nrm, off = s.interface()
    assert same(nrm, g["normals"]) and same(off, g["offsets"]), "PLIC reconstruction differs"
    dts = s.steps(int(g["steps"]))
    assert np.array_equal(dts, g["dts"]), "dt sequence differs"
    assert same(s.states(), g["final"]), "final states differ"
    assert np.array_equal(s.flags(), g["flags"])
    assert not s.bad()
    # the problem really has mixed cells
    beta = g["final"][:, 6:10]
    assert ((beta > 0).sum(axis=1) > 1).any()


def test_oracle_mm_pointwise_matches_reference():
    g = np.load(GOLDEN / "mm_pointwise.npz")
    n = 4
    s = O.MmSolver(O.Mesh(n, n, 0.0, 0.1, 0.0, 0.1, bounds=(2, 2, 1, 1)))
    for a, b, want in zip(g["sl"], g["sr"], g["hllc"]):
        assert same(s.hllc(a, b), want)
    for a, b, (hL, hR, iA, a_sig, dt), want in zip(g["sl"], g["sr"], g["crp_args"], g["crp"]):
        assert same(s.crp_flux(a, b, hL, hR, int(iA), a_sig, dt), want)
    for st, want in zip(g["sound_states"], g["sound"]):
        assert s.sound_speed(st) == want
    for q, guess, want in zip(g["q"], g["guess"], g["closure"]):
        assert same(s.state_from_q(q, guess), want)


def test_oracle_plic_helpers_match_reference():
    g = np.load(GOLDEN / "mm_pointwise.npz")
    al = g["alphas"]
    assert same([[O.mm_face_fraction(a, b) for b in al] for a in al], g["face_fraction"])
    assert same([[[O.mm_average_flux(a, c, k) for k in g["cfl"]] for c in g["cos"]] for a in al], g["average_flux"])
    assert same([[O.mm_quad_find_section(a, x, y, 1.0, 0.5) for a in al] for x, y in g["normals"]],
                g["quad_find_section"])
    assert same([[O.mm_quad_volume_fraction(p, x, y, 1.0, 0.5) for p in g["p"]] for x, y in g["normals"]],
                g["quad_volume_fraction"])


def test_oracle_mm_matches_reference_build_directly():
    """When the reference-source build is present, compare on a fresh case
    (other size, every CRP mode)."""
    from oracle import ref_mm as R
    if not R.available():
        pytest.skip("oracle/_ref/libzref_mesh.so not built (no reference tree on this machine)")
    from zephyr_b200.workloads import shock_water_column
    n = 40
    w = shock_water_column(n)
    for crp in (O.CRP_NONE, O.CRP_V3, O.CRP_V5, O.CRP_VS, O.CRP_PLIC):
        r = R.RefMmFluid(n, n, box=w.box, bounds=w.bounds, CFL=0.45, accuracy=1, crp_mode=crp)
        s = O.MmSolver(O.Mesh(n, n, *w.box, bounds=w.bounds), CFL=0.45, crp_mode=crp)
        r.make_states(w.rho, w.vx, w.vy, w.p, w.beta)
        s.make_states(w.rho, w.vx, w.vy, w.p, w.beta)
        for _ in range(90):
            assert r.step() == s.step()
        assert same(r.states(), s.states()), crp
