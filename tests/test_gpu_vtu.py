"""The device-fed VTU / PVD writer (zg_vtu_write, zg_pvd_*) against the bytes
the reference's own io::VtuFile and io::PvdFile wrote for the same mesh and
state (tests/golden/vtu_*.npz), and against the oracle's restatement of the
format for the other state sources."""
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"
STATE = (("density", 0), ("vel.x", 1), ("vel.y", 2), ("pressure", 3), ("energy", 4))


def variables(names):
    from zephyr_b200.io import Variables
    v = Variables([str(s) for s in names])
    for nm, k in STATE:
        v.append(nm, ("smf", k))
    return v


def rect_mesh(Z, g):
    gen = Z.Rectangle(*map(float, g["box"]))
    gen.set_boundaries(Z.Boundaries(*(Z.Boundary(int(b)) for b in g["bounds"])))
    gen.set_sizes(int(g["nx"]), int(g["ny"]))
    mesh = Z.EuMesh(gen)
    solver = Z.SmFluid(Z.IdealGas(1.4))
    solver.add_types(mesh)
    mesh.set_state(*g["state"])
    return mesh, solver


def test_gpu_vtu_rect_matches_reference(gpu_lib, tmp_path):
    from zephyr_b200.io import VtuFile
    g = np.load(GOLDEN / "vtu_rect_6x4.npz")
    mesh, _ = rect_mesh(gpu_lib, g)
    f = tmp_path / "sub" / "rect.vtu"  # the parent directory is created as the reference does
    VtuFile.save(f, mesh, variables(g["names"]))
    assert f.read_bytes() == g["vtu"].tobytes()


def test_gpu_pvd_series_matches_reference(gpu_lib, tmp_path):
    from zephyr_b200.io import PvdFile
    g = np.load(GOLDEN / "vtu_rect_6x4.npz")
    mesh, _ = rect_mesh(gpu_lib, g)
    pvd = PvdFile("series", tmp_path / "out")
    pvd.variables = variables(["level"])
    for t in g["timesteps"]:
        pvd.save(mesh, float(t))
    pvd.close()
    out = tmp_path / "out"
    assert (out / "series.pvd").read_bytes() == g["pvd"].tobytes()
    assert (out / "series_0.vtu").read_bytes() == g["pvd_vtu0"].tobytes()
    assert (out / "series_1.vtu").read_bytes() == g["pvd_vtu1"].tobytes()


def test_gpu_vtu_adaptive_matches_reference(gpu_lib, tmp_path):
    import zephyr_b200 as Z
    from zephyr_b200.io import VtuFile
    g = np.load(GOLDEN / "vtu_amr_8_refined.npz")
    n = int(g["n"])
    gen = Z.Rectangle(0.0, 1.0, 0.0, 1.0)
    gen.set_boundaries(Z.Boundaries(*(Z.Boundary(2) for _ in range(4))))
    gen.set_sizes(n, n)
    mesh = Z.EuMesh(gen)
    mesh.set_max_level(int(g["max_level"]))
    solver = Z.SmFluid(Z.IdealGas(1.4))
    solver.add_types(mesh)
    mesh.set_distributor(solver.distributor("const"))
    mesh.set_state(*g["state"])
    mesh.put_flags(g["flags"])
    mesh.refine()
    f = tmp_path / "amr.vtu"
    VtuFile.save(f, mesh, variables(g["names"]))
    assert f.read_bytes() == g["vtu"].tobytes()


def test_gpu_vtu_transfer_mm_and_host_sources(gpu_lib, tmp_path):
    """Transfer, MmFluid and host sources: the file equals the format's
    restatement fed with the state read back through the ABI."""
    import zephyr_b200 as Z
    from oracle import vtu as V
    from zephyr_b200.io import Variables, VtuFile
    from zephyr_b200.mmf import Material, MixturePT, MmFluid
    from zephyr_b200.transfer import Transfer
    from zephyr_b200.workloads import shock_water_column, transfer_disks
    nx, ny, box = 40, 28, (0.0, 1.0, 0.0, 0.7)
    gen = Z.Rectangle(*box)
    gen.set_boundaries(Z.Boundaries(*(Z.Boundary(2) for _ in range(4))))
    gen.set_sizes(nx, ny)
    mesh = Z.EuMesh(gen)
    tr = Transfer()
    tr.set_velocity_rotation(0.5, 0.35, np.pi)
    tr.add_types(mesh)
    tr.set_u1(mesh, transfer_disks(nx, ny, box))
    tr.update_interface(mesh)
    tr.advance(mesh, 3, 0.0, 1.0, splitting=True)
    u, nrm, pt = tr.interface(mesh)
    host = np.linspace(0.0, 1.0, nx * ny)
    v = Variables(["level", "center"])
    for nm, k in (("u", 0), ("n.x", 1), ("n.y", 2), ("p.x", 3), ("p.y", 4), ("n", 5), ("p", 6)):
        v.append(nm, ("tr", k))
    v.append("host", host)
    f = tmp_path / "tr.vtu"
    VtuFile.save(f, mesh, v)
    X = box[0] + ((box[1] - box[0]) * np.arange(nx + 1)) / nx
    Y = box[2] + ((box[3] - box[2]) * np.arange(ny + 1)) / ny
    i, j = np.divmod(np.arange(nx * ny), ny)
    mx, my = np.zeros((nx * ny, 9)), np.zeros((nx * ny, 9))
    for q, (di, dj) in {0: (0, 0), 2: (1, 0), 6: (0, 1), 8: (1, 1)}.items():
        mx[:, q], my[:, q] = X[i + di], Y[j + dj]
    cx = 0.25 * (X[i] + X[i + 1] + X[i] + X[i + 1])
    cy = 0.25 * (Y[j] + Y[j] + Y[j + 1] + Y[j + 1])
    cells = dict(cx=cx, cy=cy, level=np.zeros(nx * ny), flag=np.zeros(nx * ny), b_idx=np.arange(nx * ny),
                 z_idx=np.zeros(nx * ny))
    vec = lambda a: np.stack([a[:, 0], a[:, 1], np.zeros(len(a))], axis=1)  # noqa: E731
    want = V.vtu_bytes(V.quad_points(mx.ravel(), my.ravel()),
                       [V.cell_variable("level", cells), V.cell_variable("center", cells), ("u", u),
                        ("n.x", nrm[:, 0].copy()), ("n.y", nrm[:, 1].copy()), ("p.x", pt[:, 0].copy()),
                        ("p.y", pt[:, 1].copy()), ("n", vec(nrm)), ("p", vec(pt)), ("host", host)])
    assert f.read_bytes() == want

    # the multi-material state on another mesh
    w = shock_water_column(32)
    gen = Z.Rectangle(*w.box)
    gen.set_boundaries(Z.Boundaries(*w.bounds))
    gen.set_sizes(w.nx, w.ny)
    mm_mesh = Z.EuMesh(gen)
    mm = MmFluid(MixturePT([Material.stiffened("Water"), Material.ideal("Air")]))
    mm.add_types(mm_mesh)
    mm.make_states(mm_mesh, w.rho, w.vx, w.vy, w.p, w.beta)
    mm.update(mm_mesh, 2)
    s = mm.states(mm_mesh)
    v = Variables()
    names = [("rho", 0), ("P", 3), ("T", 5), ("b0", 6), ("b1", 7), ("rho1", 9)]
    for nm, k in names:
        v.append(nm, ("mmf", k))
    f = tmp_path / "mm.vtu"
    VtuFile.save(f, mm_mesh, v)
    col = {0: 0, 3: 3, 5: 5, 6: 6, 7: 7, 9: 11}  # component -> column of the 14-double states
    data = f.read_bytes()
    for nm, k in names:
        key = f'Name="{nm}" format="appended" offset="'.encode()
        at = data.index(key) + len(key)
        off = int(data[at:data.index(b'"', at)])
        base = data.index(b"\n_") + 2 + off
        assert int(np.frombuffer(data[base:base + 4], np.uint32)[0]) == 8 * w.nx * w.ny
        got = np.frombuffer(data[base + 4:base + 4 + 8 * w.nx * w.ny], np.float64)
        assert np.array_equal(got, s[:, col[k]], equal_nan=True), nm


def test_gpu_vtu_rejects_unknown_sources(gpu_lib, tmp_path):
    from zephyr_b200 import ZgError
    from zephyr_b200.io import Variables, VtuFile
    g = np.load(GOLDEN / "vtu_rect_6x4.npz")
    mesh, _ = rect_mesh(gpu_lib, g)
    with pytest.raises(ZgError):
        Variables(["no such variable"])
    v = Variables()
    v.append("x", ("tr", 0))  # no Transfer configured on this mesh
    with pytest.raises(ZgError):
        VtuFile.save(tmp_path / "x.vtu", mesh, v)
