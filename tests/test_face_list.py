"""The face list of the FAST and MIXED steps on an adaptive rectangle,
restated on the meshes of the AMR fixtures (the reference's own EuMesh after
adaptation, hanging faces included).

`computes_face` (zephyr_b200/csrc/smf_struct.cuh) picks the cell that
evaluates a face; `k_own_list` and `k_face_index` (smf_slot_order.cu) list
those faces and tell every other slot where to find its face: in the
neighbour's full slot of the opposite side, with the opposite sign.  These
checks hold the mesh to the properties that rule relies on: every face is
evaluated exactly once, the slot a cell reads points back to it, and the two
cells see the same face (centre and area)."""
from pathlib import Path

import numpy as np
import pytest

GOLD = Path(__file__).parent / "golden"
UNDEFINED, INNER, PERIODIC = -1, 0, 3  # amr_faces.h face flags


def is_boundary(flag):  # amr_faces.h:157-161
    return flag not in (INNER, PERIODIC, UNDEFINED)


def computes_face(level, ic, s, flag, nb):
    """computes_face: a boundary face by its cell, a coarse-fine face by the
    fine cell, a same-level face by the cell on its low side."""
    if is_boundary(flag):
        return True
    if level[nb] != level[ic]:
        return level[nb] < level[ic]
    return (s & 1) == 1


@pytest.mark.parametrize("name", ["amr_blast_12_mc_3levels", "amr_blast_16_first_order", "amr_blast_16_vanalbada"])
def test_every_face_evaluated_once_and_found_by_both_cells(name):
    d = np.load(GOLD / f"{name}.npz")
    fb, fn, level = d["boundary"], d["neib"], d["level"]
    fx, fy, area = d["fx"], d["fy"], d["area"]
    n = len(level)
    # the list as k_own_list builds it (cells in order, slots ascending)
    listed = [8 * p + s for p in range(n) for s in range(8)
              if fb[8 * p + s] != UNDEFINED and computes_face(level, p, s, fb[8 * p + s], fn[8 * p + s])]
    entry = {f: t for t, f in enumerate(listed)}
    uses = np.zeros(len(listed), dtype=int)
    hanging = 0
    for p in range(n):
        for s in range(8):
            f = 8 * p + s
            flag = fb[f]
            if flag == UNDEFINED:
                continue
            if computes_face(level, p, s, flag, fn[f]):
                uses[entry[f]] += 1
                continue
            nb = int(fn[f])
            q = (s & 3) ^ 1  # the neighbour's slot of the opposite side, a full one
            g = 8 * nb + q
            assert fb[g] == INNER and fn[g] == p, (name, p, s)
            assert fb[8 * nb + q + 4] == UNDEFINED, (name, p, s)  # not split: the face is the whole side
            assert computes_face(level, nb, q, fb[g], p), (name, p, s)
            # the same face seen from both cells (the owner's full face is the
            # coarse cell's half face)
            assert fx[f] == fx[g] and fy[f] == fy[g] and area[f] == area[g], (name, p, s)
            uses[entry[g]] += 1
            hanging += level[nb] > level[p]
    inner = np.array([fb[f] == INNER for f in listed])
    assert np.all(uses[inner] == 2) and np.all(uses[~inner] == 1)
    assert hanging > 0  # coarse-fine faces present
