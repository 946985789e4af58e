"""The adaptation fixtures (tests/golden/adapt_cycle_*.npz) against a fresh
run of the reference's EuMesh / SmFluid (oracle/_ref/libzref_mesh.so) through
the same schedule, and the schedule helpers themselves."""
import json
from pathlib import Path

import numpy as np
import pytest

import amr_cycle as AC

GOLDEN = Path(__file__).resolve().parent / "golden"
CASES = sorted(p.stem for p in GOLDEN.glob("adapt_cycle_*.npz"))


def test_canonical_folds_undefined_slots_and_signed_zeros():
    g = {k: np.zeros(1) for k in AC.CELL_KEYS + AC.MAP_KEYS}
    g.update({k: np.array([-0.0, 5.0]) for k in AC.FACE_KEYS})
    g["boundary"] = np.array([0, -1])
    g["neib"] = np.array([3, 9])
    c = AC.canonical(g)
    assert c["nx"].tolist() == [0.0, 0.0] and np.signbit(c["nx"]).tolist() == [False, False]
    assert c["neib"].tolist() == [3, 0] and c["boundary"].tolist() == [0, -1]


def test_random_flags_are_seeded():
    assert np.array_equal(AC.random_flags(100, 4), AC.random_flags(100, 4))
    f = AC.random_flags(5000, 1)
    assert set(np.unique(f)) <= {-4, -1, 0, 1, 3} and (f < 0).mean() > 0.4


@pytest.mark.parametrize("case", CASES)
def test_fixture_reproduces_with_the_reference(case):
    from oracle import ref_mesh as RM
    if not RM.available():
        pytest.skip("the reference's build is not present")
    z = np.load(GOLDEN / f"{case}.npz")
    ref = RM.RefEuMesh(int(z["n"]), int(z["n"]), bounds=tuple(int(b) for b in z["bounds"]),
                       accuracy=int(z["accuracy"]), limiter=str(z["limiter"]), CFL=float(z["CFL"]),
                       max_level=int(z["max_level"]), distributor=str(z["distributor"]))
    ops = AC.schedule(int(z["cycles"]), int(z["steps_per_cycle"]), int(z["random_rounds"]))
    log = json.loads(json.dumps(AC.run(AC.RefAdapter(ref), ops)))
    assert log == json.loads(str(z["log"]))
    assert ref.check_refined() == 0  # EuMesh::check_refined on the final mesh
