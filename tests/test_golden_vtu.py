"""Pin the VTU / PVD writer restatement (oracle/vtu.py) to the reference's own
writer: tests/golden/vtu_*.npz hold the bytes io::VtuFile::save and
io::PvdFile wrote (tests/golden/make_golden.py --vtu).  Byte equality."""
from pathlib import Path

import numpy as np

from oracle import oracle as O
from oracle import vtu as V

GOLDEN = Path(__file__).resolve().parent / "golden"
STATE_NAMES = ("density", "vel.x", "vel.y", "pressure", "energy")


def rect_map_points(nx, ny, box):
    """Map points 0, 2, 6, 8 of every cell of the rectangle (the others are
    not written), with amr_cells_gen.cpp:155-161's vertex formula."""
    x0, x1, y0, y1 = box
    X = x0 + ((x1 - x0) * np.arange(nx + 1)) / nx
    Y = y0 + ((y1 - y0) * np.arange(ny + 1)) / ny
    mx, my = np.zeros((nx * ny, 9)), np.zeros((nx * ny, 9))
    i, j = np.divmod(np.arange(nx * ny), ny)
    for q, (di, dj) in {0: (0, 0), 2: (1, 0), 6: (0, 1), 8: (1, 1)}.items():
        mx[:, q] = X[i + di]
        my[:, q] = Y[j + dj]
    return mx.ravel(), my.ravel()


def variables(names, cells, state):
    out = [V.cell_variable(nm, cells) for nm in names]
    out += [(nm, np.asarray(a, dtype=np.float64)) for nm, a in zip(STATE_NAMES, state)]
    return out


def test_vtu_rect_matches_reference():
    g = np.load(GOLDEN / "vtu_rect_6x4.npz")
    nx, ny, box = int(g["nx"]), int(g["ny"]), tuple(map(float, g["box"]))
    geo = O.Mesh(nx, ny, *box, bounds=tuple(int(b) for b in g["bounds"])).geometry()
    n = nx * ny
    cells = dict(cx=geo["cx"], cy=geo["cy"], level=np.zeros(n), flag=np.zeros(n), b_idx=np.arange(n),
                 z_idx=np.zeros(n))
    pts = V.quad_points(*rect_map_points(nx, ny, box))
    got = V.vtu_bytes(pts, variables([str(s) for s in g["names"]], cells, g["state"]))
    assert got == g["vtu"].tobytes()
    # the PVD series: two saves of level + state
    vtu0 = V.vtu_bytes(pts, variables(["level"], cells, g["state"]))
    assert vtu0 == g["pvd_vtu0"].tobytes() == g["pvd_vtu1"].tobytes()
    assert V.pvd_text("series", g["timesteps"]).encode() == g["pvd"].tobytes()


def test_vtu_amr_matches_reference():
    g = np.load(GOLDEN / "vtu_amr_8_refined.npz")
    cells = {k: g[k] for k in ("cx", "cy", "level", "flag", "b_idx", "z_idx")}
    assert (g["level"] > 0).any()
    pts = V.quad_points(g["map_x"], g["map_y"])
    got = V.vtu_bytes(pts, variables([str(s) for s in g["names"]], cells, g["state_after"]))
    assert got == g["vtu"].tobytes()
