"""Pin the transport oracle (oracle/zoracle_tr.inc) to the reference: the
golden fixtures tests/golden/tr_*.npz were produced by the reference's own
Transfer, InterfaceRecovery and Polygon code compiled from its sources
(tests/golden/make_golden.py --transfer).  Bit-exact equality is required."""
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O

GOLDEN = Path(__file__).resolve().parent / "golden"
CASES = sorted(p.stem for p in GOLDEN.glob("tr_disk_*.npz"))


def same(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return a.shape == b.shape and bool(np.all((a == b) | (np.isnan(a) & np.isnan(b))))


def vel_of(g):
    return (str(g["vel_kind"]), *map(float, g["vel"]))


def test_tr_fixtures_present():
    assert len(CASES) >= 8


@pytest.mark.parametrize("name", CASES)
def test_oracle_transfer_matches_reference(name):
    g = np.load(GOLDEN / f"{name}.npz")
    nx, ny = int(g["nx"]), int(g["ny"])
    method = str(g["method"])
    m = O.Mesh(nx, ny, *map(float, g["box"]), bounds=tuple(int(b) for b in g["bounds"]))
    s = O.TrSolver(m, method=method, CFL=float(g["CFL"]), vel=vel_of(g))
    s.set_u(g["u0"])
    s.update_interface(3 if method.startswith(("VOF", "MUSCL", "WENO")) else 0)
    _, n0, p0 = s.get()
    assert same(n0, g["n0"]) and same(p0, g["p0"]), "initial reconstruction differs"
    dirs = (1, 2) if bool(g["split"]) else (0,)
    for k, want in enumerate(g["dts"]):
        dt = s.compute_dt()
        assert dt == want, f"dt of step {k}"
        s.set_dt(dt)
        for d in dirs:
            s.update(d)
    u, n, p = s.get()
    assert same(u, g["u"]) and same(n, g["n"]) and same(p, g["p"])
    assert np.array_equal(s.flags(), g["flags"])
    # the body has really moved through mixed cells
    assert ((u > 0) & (u < 1)).sum() > 10 and not np.array_equal(u, g["u0"])


def test_oracle_transfer_matches_reference_build_directly():
    """When the reference-source build is present, compare on fresh cases:
    every method, both velocity fields, split and unsplit, including a
    velocity parallel to the y faces (normal velocity exactly 0 there)."""
    from oracle import ref_tr as RT
    if not RT.available():
        pytest.skip("reference-source build not present")
    box = (0.0, 1.0, 0.0, 0.7)
    vels = [("translation", 0.7, -0.35), ("rotation", 0.5, 0.5, float(np.pi)), ("translation", 1.0, 0.0)]
    for method in O.TR_METHODS:
        for vel in vels:
            for split in (False, True):
                r = RT.RefTransfer(22, 15, box=box, method=method, vel=vel)
                s = O.TrSolver(O.Mesh(22, 15, *box), method=method, vel=vel)
                u0 = r.disk(0.3, 0.4, 0.15)
                r.set_u(u0)
                s.set_u(u0)
                sm = 3 if method.startswith(("VOF", "MUSCL", "WENO")) else 0
                r.update_interface(sm)
                s.update_interface(sm)
                for _ in range(6):
                    dt = r.compute_dt()
                    assert s.compute_dt() == dt
                    r.set_dt(dt)
                    s.set_dt(dt)
                    for d in ((1, 2) if split else (0,)):
                        r.update(d)
                        s.update(d)
                for a, b in zip(r.get(), s.get()):
                    assert same(a, b), (method, vel, split)
