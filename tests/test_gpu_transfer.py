"""The scalar VOF transport on the GPU (Transfer: every method -- VOF,
VOF_CRP, the CRP, MUSCL and WENO families) against the golden fixtures produced by the reference's own Transfer
(tests/golden/tr_*.npz) and against the oracle on fresh inputs.  Bit-exact:
the kernels keep the reference's order of operations and are compiled
without fused multiply-adds."""
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"
CASES = sorted(p.stem for p in GOLDEN.glob("tr_disk_*.npz"))
METHODS = ["CRP_V3", "CRP_V5", "CRP_SE", "CRP_N1", "CRP_N2", "VOF", "VOF_CRP", "MUSCLd", "MUSCLn", "MUSCLd_CRP",
           "MUSCLn_CRP", "MUSCL_MC", "MUSCL_MC_CRP", "WENO", "WENO_CRP"]
ZOE = 2


def same(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return a.shape == b.shape and bool(np.all((a == b) | (np.isnan(a) & np.isnan(b))))


def gpu_transfer(Z, nx, ny, box, method, vel, CFL=0.5, bounds=(ZOE,) * 4):
    from zephyr_b200.transfer import Method, Transfer
    gen = Z.Rectangle(*box)
    gen.set_boundaries(Z.Boundaries(*(Z.Boundary(b) for b in bounds)))
    gen.set_sizes(nx, ny)
    mesh = Z.EuMesh(gen)
    s = Transfer()
    s.set_CFL(CFL)
    s.set_method(Method[method])
    if vel[0] == "translation":
        s.set_velocity_translation(vel[1], vel[2])
    else:
        s.set_velocity_rotation(vel[1], vel[2], vel[3])
    s.add_types(mesh)
    return mesh, s


def oracle_transfer(nx, ny, box, method, vel, CFL=0.5):
    from oracle import oracle as O
    return O.TrSolver(O.Mesh(nx, ny, *box), method=method, CFL=CFL, vel=vel)


def smoothing(method):
    return 3 if method.startswith(("VOF", "MUSCL", "WENO")) else 0


@pytest.mark.parametrize("name", CASES)
def test_gpu_transfer_matches_reference_fixture(gpu_lib, name):
    g = np.load(GOLDEN / f"{name}.npz")
    nx, ny, method = int(g["nx"]), int(g["ny"]), str(g["method"])
    vel = (str(g["vel_kind"]), *map(float, g["vel"]))
    mesh, s = gpu_transfer(gpu_lib, nx, ny, tuple(map(float, g["box"])), method, vel, float(g["CFL"]))
    s.set_u1(mesh, g["u0"])
    s.update_interface(mesh, smoothing(method))
    _, n0, p0 = s.interface(mesh)
    assert same(n0, g["n0"]) and same(p0, g["p0"]), "initial reconstruction differs"
    dirs = (1, 2) if bool(g["split"]) else (0,)
    for k, want in enumerate(g["dts"]):
        dt = s.compute_dt(mesh)
        assert dt == want, f"dt of step {k}"
        s.set_dt(dt)
        for d in dirs:
            s.update(mesh, d)
    u, n, p = s.interface(mesh)
    assert same(u, g["u"]), f"u1 differs in {int((u != g['u']).sum())} cells"
    assert same(n, g["n"]) and same(p, g["p"])
    assert np.array_equal(s.set_flags(mesh), g["flags"])


VELS = {
    "translation": ("translation", 0.7, -0.35),
    "rotation": ("rotation", 0.5, 0.5, float(np.pi)),
    "along_x": ("translation", 1.0, 0.0),     # normal velocity exactly 0 on the y faces
    "along_y": ("translation", 0.0, -0.35),   # ... and on the x faces
}


def run_both(Z, nx, ny, box, method, vel, split, steps, u0, CFL=0.5):
    mesh, g = gpu_transfer(Z, nx, ny, box, method, vel, CFL)
    o = oracle_transfer(nx, ny, box, method, vel, CFL)
    g.set_u1(mesh, u0)
    o.set_u(u0)
    g.update_interface(mesh, smoothing(method))
    o.update_interface(smoothing(method))
    for _ in range(steps):
        dg, do = g.compute_dt(mesh), o.compute_dt()
        assert dg == do
        g.set_dt(dg)
        o.set_dt(do)
        for d in ((1, 2) if split else (0,)):
            g.update(mesh, d)
            o.update(d)
    return g.interface(mesh), o.get(), (mesh, g, o)


@pytest.mark.parametrize("method", METHODS)
@pytest.mark.parametrize("vel", list(VELS))
@pytest.mark.parametrize("split", [False, True])
def test_gpu_transfer_matches_oracle(gpu_lib, method, vel, split):
    from zephyr_b200.workloads import transfer_disk_field
    nx, ny, box = 67, 45, (0.0, 1.0, 0.0, 0.7)
    u0 = transfer_disk_field(nx, ny, box, count=12, seed=3)
    (ug, ng, pg), (uo, no, po), _ = run_both(gpu_lib, nx, ny, box, method, VELS[vel], split, 8, u0)
    assert same(ug, uo), f"u1 differs in {int((ug != uo).sum())} cells"
    assert same(ng, no) and same(pg, po)


def test_gpu_transfer_advance_matches_time_loop(gpu_lib):
    """zg_tr_advance runs the transfer problem's loop on the device: dt from
    compute_dt clipped at t_end, update X then Y, time advanced by dt."""
    from zephyr_b200.workloads import transfer_disks
    nx, ny, box = 50, 35, (0.0, 1.0, 0.0, 0.7)
    vel = VELS["rotation"]
    u0 = transfer_disks(nx, ny, box)
    mesh, a = gpu_transfer(gpu_lib, nx, ny, box, "VOF", vel)
    a.set_u1(mesh, u0)
    a.update_interface(mesh)
    t_end = 0.02  # reached within the 6 steps (dt ~ 0.0046)
    t = a.advance(mesh, 6, 0.0, t_end, splitting=True)
    o = oracle_transfer(nx, ny, box, "VOF", vel)
    o.set_u(u0)
    o.update_interface(3)
    tt = 0.0
    for _ in range(6):
        dt = o.compute_dt()
        if tt + dt > t_end:
            dt = t_end - tt
        o.set_dt(dt)
        o.update(1)
        o.update(2)
        tt += dt
    assert t == tt and abs(t - t_end) < 1.0e-15
    ug, ng, pg = a.interface(mesh)
    uo, no, po = o.get()
    assert same(ug, uo) and same(ng, no) and same(pg, po)


def test_gpu_transfer_large_one_step_matches_oracle(gpu_lib):
    """A 1024 x 716 mesh, one split step of VOF on a field of disks."""
    from zephyr_b200.workloads import transfer_disk_field
    nx, ny, box = 1024, 716, (0.0, 1.0, 0.0, 0.7)
    u0 = transfer_disk_field(nx, ny, box, count=40, seed=11)
    (ug, ng, pg), (uo, no, po), _ = run_both(gpu_lib, nx, ny, box, "VOF", VELS["rotation"], True, 1, u0)
    assert same(ug, uo) and same(ng, no) and same(pg, po)


def test_gpu_transfer_full_size_properties(gpu_lib):
    """At 2048 x 2048: u1 stays in [0, 1], two runs agree bit for bit, and
    the VOF scheme keeps the body's volume to 1e-3 over 20 steps."""
    from zephyr_b200.workloads import transfer_disk_field
    nx = ny = 2048
    box = (0.0, 1.0, 0.0, 1.0)
    u0 = transfer_disk_field(nx, ny, box, count=64, seed=5)
    outs = []
    for _ in range(2):
        mesh, s = gpu_transfer(gpu_lib, nx, ny, box, "VOF", VELS["rotation"])
        s.set_u1(mesh, u0)
        s.update_interface(mesh)
        s.advance(mesh, 20, 0.0, 1.0e9, splitting=True)
        outs.append(s.interface(mesh))
    (u, n, p), (u2, n2, p2) = outs
    assert same(u, u2) and same(n, n2) and same(p, p2)
    assert u.min() >= 0.0 and u.max() <= 1.0
    assert abs(u.sum() - u0.sum()) / u0.sum() < 1.0e-3
    assert not np.array_equal(u, u0)


@pytest.mark.parametrize("nx,ny", [(1, 9), (9, 1), (2, 2)])
def test_gpu_transfer_thin_meshes(gpu_lib, nx, ny):
    rng = np.random.default_rng(nx * 10 + ny)
    u0 = rng.random(nx * ny)
    u0[rng.random(nx * ny) < 0.3] = 0.0
    for method in ("VOF", "CRP_N1"):
        (ug, ng, pg), (uo, no, po), _ = run_both(gpu_lib, nx, ny, (0.0, 1.0, 0.0, 1.0), method, VELS["rotation"],
                                                 False, 3, u0)
        assert same(ug, uo) and same(ng, no) and same(pg, po)


def test_gpu_transfer_uniform_and_static_fields(gpu_lib):
    nx, ny, box = 20, 14, (0.0, 1.0, 0.0, 0.7)
    for u0 in (np.zeros(nx * ny), np.ones(nx * ny)):
        (ug, _, _), (uo, _, _), _ = run_both(gpu_lib, nx, ny, box, "VOF", VELS["translation"], True, 3, u0)
        assert same(ug, uo)
    # zero velocity: dt = CFL * DBL_MAX and nothing moves
    from zephyr_b200.workloads import transfer_disks
    u0 = transfer_disks(nx, ny, box)
    (ug, _, _), (uo, _, _), (mesh, g, o) = run_both(gpu_lib, nx, ny, box, "VOF", ("translation", 0.0, 0.0),
                                                    False, 2, u0)
    assert same(ug, uo) and same(ug, u0)
    assert g.compute_dt(mesh) == o.compute_dt() == 0.5 * np.finfo(np.float64).max


def test_gpu_transfer_rejects_unsupported(gpu_lib):
    from zephyr_b200 import ZgError
    from zephyr_b200.transfer import Method
    with pytest.raises(ZgError):
        gpu_transfer(gpu_lib, 8, 8, (0.0, 1.0, 0.0, 1.0), "VOF", VELS["rotation"], bounds=(3, 3, ZOE, ZOE))
    mesh, s = gpu_transfer(gpu_lib, 2, 8, (0.0, 1.0, 0.0, 1.0), "VOF", VELS["rotation"])
    with pytest.raises(ZgError):  # WENO's stencil needs 3 cells per axis
        s.set_method(Method.WENO)
    with pytest.raises(ZgError):
        s.update(mesh, 3)
