"""The restatement of the adaptive configuration's refinement criterion
(|grad rho| h / rho, oracle/gradient_flags.py) on refined meshes of the
reference's own EuMesh (oracle/_ref): the unlimited least-squares gradient
is exact for a linear density on every cell whose face slots all lead to
actual neighbours, whatever the refinement around it."""
import numpy as np
import pytest

import amr_cycle as AC
from oracle import gradient_flags as GF


def _ref_mesh():
    from oracle import ref_mesh as RM
    if not RM.available():
        pytest.skip("the reference's build (oracle/_ref/libzref_mesh.so) is not present")
    r = RM.RefEuMesh(16, 16, bounds=(2, 2, 2, 2), max_level=2)
    for seed in (3, 4, 5):
        r.put_flags(np.where(AC.random_flags(r.n, seed) > 0, 1, 0).astype(np.int32))
        r.refine()
    g = r.cells()
    g.update(r.faces())
    return r, g


def test_linear_density_gives_the_exact_gradient():
    r, g = _ref_mesh()
    cx, cy = np.asarray(g["cx"]), np.asarray(g["cy"])
    assert np.asarray(g["level"]).max() >= 1
    rho = 1.0 + 0.1 * cx + 0.2 * cy
    crit = GF.criterion(g, rho)
    fb = np.asarray(g["boundary"]).reshape(len(cx), 8)
    interior = ~np.any((fb != -1) & (fb != 0), axis=1)
    want = np.hypot(0.1, 0.2) * np.sqrt(np.asarray(g["vol"])) / rho
    assert interior.sum() > 100
    assert np.allclose(crit[interior], want[interior], rtol=1e-12, atol=0.0)


def test_flags_follow_the_thresholds():
    r, g = _ref_mesh()
    cx = np.asarray(g["cx"])
    rho = np.where(cx < 0.5, 1.0, 1.3)  # a jump: refine next to it, coarsen away from it
    c = GF.criterion(g, rho)
    f = GF.flags(g, rho)
    assert np.array_equal(f == 1, c > 0.05) and np.array_equal(f == -1, c < 0.01)
    assert (f == 1).any() and (f == -1).any()
