"""Adaptation on the GPU (zg_amr_*): the base mesh of an adaptive rectangle,
and schedules of SmFluid::set_flags / EuMesh::refine / SmFluid::update with
random flag rounds, bit-exact with the reference's EuMesh::refine on one rank
(cell order, levels, z-indices, map points, geometry, face slots and
neighbours, distributed states, isolation counters, flags and dt).

Pinned by the digests of tests/golden/adapt_cycle_*.npz (made by the
reference, tests/golden/make_golden.py); where the reference's build
oracle/_ref/libzref_mesh.so is present, the same schedules (and a larger
one) also run side by side with it, array by array."""
import json
from pathlib import Path

import numpy as np
import pytest

import amr_cycle as AC

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"
CYCLE_CASES = sorted(p.stem for p in GOLDEN.glob("adapt_cycle_*.npz"))


def ref_available():
    from oracle import ref_mesh as RM
    return RM.available()


def gpu_mesh(n, bounds, max_level, distributor, acc, limiter, CFL, capacity=None, ny=None):
    import zephyr_b200 as Z
    gen = Z.Rectangle(0.0, 1.0, 0.0, 1.0)
    gen.set_boundaries(Z.Boundaries(*bounds))
    gen.set_sizes(n, ny or n)
    mesh = Z.EuMesh(gen)
    mesh.set_max_level(max_level, capacity)
    solver = Z.SmFluid(Z.IdealGas(1.4))
    solver.add_types(mesh)
    solver.set_accuracy(acc)
    solver.set_limiter(limiter)
    solver.set_CFL(CFL)
    mesh.set_distributor(solver.distributor(distributor))
    return mesh, solver


def compare_live(label, ref_ad, gpu_ad, g_gpu):
    g_ref = ref_ad.mesh()
    assert ref_ad.n() == gpu_ad.n(), (label, ref_ad.n(), gpu_ad.n())
    a, b = AC.canonical(g_ref), AC.canonical(g_gpu)
    for k in AC.MESH_KEYS:
        if not np.array_equal(a[k], b[k]):
            i = int(np.argmax(a[k] != b[k]))
            raise AssertionError(f"{label}: {k} differs first at {i}: ref {a[k][i]!r} gpu {b[k][i]!r}")
    sr, sg = ref_ad.state(), gpu_ad.state()
    for k in AC.STATE_KEYS:
        if not np.array_equal(sr[k], sg[k]):
            i = int(np.argmax(sr[k] != sg[k]))
            raise AssertionError(f"{label}: state {k} differs first at {i}: ref {sr[k][i]!r} gpu {sg[k][i]!r}")


@pytest.mark.parametrize("case", CYCLE_CASES)
def test_adaptation_schedule_matches_reference_digests(gpu_lib, case):
    z = np.load(GOLDEN / f"{case}.npz")
    want = json.loads(str(z["log"]))
    mesh, solver = gpu_mesh(int(z["n"]), tuple(int(b) for b in z["bounds"]), int(z["max_level"]),
                            str(z["distributor"]), int(z["accuracy"]), str(z["limiter"]), float(z["CFL"]))
    ops = AC.schedule(int(z["cycles"]), int(z["steps_per_cycle"]), int(z["random_rounds"]))
    got = AC.run(AC.GpuAdapter(mesh, solver), ops)
    assert len(got) == len(want)
    for g, w in zip(got, want):
        label = w[0]
        assert g[0] == label
        assert g[1] == w[1], (label, "cells", g[1], w[1])
        bad = [k for k in w[2] if g[2][k] != w[2][k]]
        assert not bad, (label, "mesh arrays differ", bad)
        bad = [k for k in w[3] if g[3][k] != w[3][k]]
        assert not bad, (label, "state arrays differ", bad)
        assert g[4] == w[4], (label, g[4], w[4])
    mesh.close()


@pytest.mark.parametrize("n,ny,bounds,max_level,distributor,acc,limiter,cycles,steps,rand", [
    (16, None, (2, 1, 1, 2), 3, "slope", 2, "MC", 8, 2, 6),
    (40, 28, (2, 2, 1, 1), 3, "slope", 2, "van Albada", 10, 2, 4),
    (24, None, (1, 1, 1, 1), 4, "const", 1, "MC", 6, 3, 6),
])
def test_adaptation_side_by_side_with_reference(gpu_lib, n, ny, bounds, max_level, distributor, acc, limiter,
                                                cycles, steps, rand):
    if not ref_available():
        pytest.skip("the reference's build (oracle/_ref/libzref_mesh.so) is not present; the digest test pins it")
    from oracle import ref_mesh as RM
    ref = RM.RefEuMesh(n, ny or n, bounds=bounds, accuracy=acc, limiter=limiter, CFL=0.4, max_level=max_level,
                       distributor=distributor)
    ref_ad = AC.RefAdapter(ref)
    mesh, solver = gpu_mesh(n, bounds, max_level, distributor, acc, limiter, 0.4, ny=ny)
    gpu_ad = AC.GpuAdapter(mesh, solver)
    g0 = gpu_ad.mesh()
    s0 = AC.init_state(g0["cx"], g0["cy"])
    ref_ad.set_state(*s0)
    gpu_ad.set_state(*s0)
    compare_live("base", ref_ad, gpu_ad, g0)
    for k, op in enumerate(AC.schedule(cycles, steps, rand, seed=7)):
        if op == "set_flags":
            fr, fg = ref_ad.set_flags(), gpu_ad.set_flags()
            assert np.array_equal(fr, fg), (k, "flags")
        elif op == "refine":
            ref_ad.refine()
            gpu_ad.refine()
        elif op == "step":
            assert ref_ad.step() == gpu_ad.step(), (k, "dt")
        else:
            f = AC.random_flags(ref_ad.n(), int(op.split(":")[1]))
            ref_ad.put_flags(f)
            gpu_ad.put_flags(f)
            ref_ad.refine()
            gpu_ad.refine()
        compare_live(f"{k}:{op}", ref_ad, gpu_ad, gpu_ad.mesh())
    mesh.close()


def test_capacity_overflow_leaves_the_mesh_unchanged(gpu_lib):
    import zephyr_b200 as Z
    n = 12
    mesh, solver = gpu_mesh(n, (2, 2, 2, 2), 2, "slope", 2, "MC", 0.4, capacity=n * n + 30)
    g = mesh.amr_arrays()
    mesh.set_state(*AC.init_state(g["cx"], g["cy"]))
    before = AC.digest(AC.canonical(mesh.amr_arrays()))
    state = mesh.get_state()
    mesh.put_flags(np.ones(n * n, np.int32))  # 4 children per cell: far above the capacity
    with pytest.raises(Z.ZgError) as e:
        mesh.refine()
    assert e.value.code == -6
    assert mesh.n_cells() == n * n
    after = AC.canonical(mesh.amr_arrays())
    after.pop("flag")
    before.pop("flag")
    assert AC.digest(after) == before
    assert all(np.array_equal(a, b) for a, b in zip(state, mesh.get_state()))
    # a refine that fits still works afterwards
    f = np.zeros(n * n, np.int32)
    f[5] = 1
    mesh.put_flags(f)
    mesh.refine()
    assert mesh.n_cells() == n * n + 3
    st = mesh.amr_info()
    assert (st.n_before, st.n_after, st.n_refine, st.n_coarse) == (n * n, n * n + 3, 1, 0)
    mesh.close()


def test_adaptive_mesh_rejects_periodic_and_late_enable(gpu_lib):
    import zephyr_b200 as Z
    gen = Z.Rectangle(0.0, 1.0, 0.0, 1.0)
    gen.set_boundaries(Z.Boundaries(Z.Boundary.PERIODIC, Z.Boundary.PERIODIC, Z.Boundary.WALL, Z.Boundary.WALL))
    gen.set_sizes(8, 8)
    mesh = Z.EuMesh(gen)
    with pytest.raises(Z.ZgError) as e:
        mesh.set_max_level(2)
    assert e.value.code == -1
    mesh.close()
    gen.set_boundaries(Z.Boundaries())
    mesh = Z.EuMesh(gen)
    solver = Z.SmFluid(Z.IdealGas(1.4))
    solver.add_types(mesh)
    with pytest.raises(Z.ZgError) as e:
        mesh.set_max_level(2)
    assert e.value.code == -3
    with pytest.raises(Z.ZgError):
        mesh.refine()
    mesh.close()


@pytest.mark.parametrize("acc,scheme", [(2, "pc"), (1, "pc"), (2, "heun")])
def test_fast_kernels_on_the_adaptive_mesh_match_parity(gpu_lib, acc, scheme):
    """The FAST slot kernels (derived face geometry, fused multiply-adds)
    against the bit-exact parity kernels, one step from the same state on an
    adapted mesh with hanging faces: within 1e-12 relative per step."""
    import zephyr_b200 as Z
    mesh, solver = gpu_mesh(24, (2, 1, 1, 2), 3, "slope", acc, "MC", 0.4)
    if scheme == "heun":
        solver.set_scheme(Z.Scheme.HEUN)
    g = mesh.amr_arrays()
    mesh.set_state(*AC.init_state(g["cx"], g["cy"]))
    for _ in range(4):
        solver.set_flags(mesh)
        mesh.refine()
        solver.update(mesh)
    st = mesh.amr_arrays()
    assert (st["boundary"][4::8] != -1).any()  # hanging faces present
    s0, w0 = mesh.get_state(), mesh.get_wait()
    solver.update(mesh)
    par = mesh.get_state()
    mesh.set_state(*s0)
    mesh.set_wait(w0)
    fast = Z.SmFluid(Z.IdealGas(1.4), kernels=Z.Kernels.FAST)
    fast.params = solver.params
    fast.params.kernels = int(Z.Kernels.FAST)
    fast.add_types(mesh)
    fast.update(mesh)
    got = mesh.get_state()

    def cons(z):  # rho, rho u, rho v, rho E
        r, u, v, p, e = z
        return [r, r * u, r * v, r * (e + 0.5 * (u * u + v * v))]

    for k, (a, b) in enumerate(zip(cons(par), cons(got))):
        # density and energy pointwise; momenta relative to their field's size
        scale = np.abs(a) if k in (0, 3) else np.max(np.abs(a))
        assert np.max(np.abs(a - b) / scale) <= 1e-12, (k, np.max(np.abs(a - b) / scale))
    assert fast.dt() == solver.dt() or abs(fast.dt() - solver.dt()) <= 1e-14 * solver.dt()
    mesh.close()


@pytest.mark.parametrize("acc,scheme,form", [(2, "pc", "fast"), (2, "heun", "fast"), (1, "pc", "fast"),
                                             (2, "pc", "mixed"), (1, "pc", "mixed")])
def test_fast_state_order_between_steps(gpu_lib, acc, scheme, form):
    """The FAST and MIXED adaptive steps keep the state in the Morton cell
    order between steps and every other entry point brings it back: steps
    run back to back (state held in that order, set_flags and refine
    between them) give the same bits, counters included, as the same
    schedule read out after every step."""
    import zephyr_b200 as Z

    def run(read_each_step):
        mesh, solver = gpu_mesh(24, (2, 1, 1, 2), 3, "slope", acc, "MC", 0.4)
        if scheme == "heun":
            solver.set_scheme(Z.Scheme.HEUN)
        g = mesh.amr_arrays()
        mesh.set_state(*AC.init_state(g["cx"], g["cy"]))
        fast = Z.SmFluid(Z.IdealGas(1.4), kernels=Z.Kernels.FAST)
        fast.params = solver.params
        fast.params.kernels = int(Z.Kernels.FAST)
        if form == "mixed":
            fast.params.precision = int(Z.Precision.MIXED)
        fast.add_types(mesh)
        seen = []
        for _ in range(3):
            for _ in range(4):
                fast.update(mesh)
                if read_each_step:
                    seen.append((mesh.get_state(), mesh.get_wait()))
            fast.set_flags(mesh)
            mesh.refine()
        fast.update(mesh, 3)
        out = mesh.get_state(), mesh.get_wait(), fast.dt(), mesh.n_cells()
        mesh.close()
        return out, seen

    (z0, w0, dt0, n0), _ = run(False)
    (z1, w1, dt1, n1), seen = run(True)
    assert n0 == n1 and dt0 == dt1 and len(seen) == 12
    for a, b in zip(z0, z1):
        assert np.array_equal(a, b)
    assert np.array_equal(w0, w1)


def test_refine_after_fast_steps_splits_with_the_last_steps_gradients(gpu_lib):
    """A refine with the slope distributor right after steps, with flags put
    by the caller and no gradient pass between, splits with the gradients of
    the last step (the cells' stored gradients the reference's distributor
    reads).  The FAST steps keep their gradients in the cell order and bring
    them back with the state; against the parity steps on the same schedule
    the refined states agree to the FAST form's rounding."""
    import zephyr_b200 as Z
    outs = []
    for kern in (Z.Kernels.PARITY, Z.Kernels.FAST):
        mesh, solver = gpu_mesh(24, (2, 1, 1, 2), 3, "slope", 2, "MC", 0.4)
        g = mesh.amr_arrays()
        mesh.set_state(*AC.init_state(g["cx"], g["cy"]))
        for _ in range(2):
            solver.set_flags(mesh)
            mesh.refine()
        s = Z.SmFluid(Z.IdealGas(1.4), kernels=kern)
        s.params = solver.params
        s.params.kernels = int(kern)
        s.add_types(mesh)
        s.update(mesh, 3)
        flags = np.zeros(mesh.n_cells(), dtype=np.int32)
        flags[::3] = 1
        mesh.put_flags(flags)
        mesh.refine()
        outs.append((mesh.get_state(), mesh.amr_arrays()["level"]))
        mesh.close()
    (za, la), (zb, lb) = outs
    assert np.array_equal(la, lb) and (la == 3).any()
    for k in range(4):  # rho, u, v, p
        a, b = za[k], zb[k]
        assert np.max(np.abs(a - b)) <= 1e-11 * np.max(np.abs(a)), (k, np.max(np.abs(a - b)))


def _adapted(acc=2, distributor="slope", bounds=(2, 1, 1, 2), rounds=4):
    mesh, solver = gpu_mesh(24, bounds, 3, distributor, acc, "MC", 0.4)
    g = mesh.amr_arrays()
    mesh.set_state(*AC.init_state(g["cx"], g["cy"]))
    for _ in range(rounds):
        solver.set_flags(mesh)
        mesh.refine()
        solver.update(mesh)
    return mesh, solver


@pytest.mark.parametrize("acc", [2, 1])
def test_mixed_form_on_the_adaptive_mesh_tracks_fp64(gpu_lib, acc):
    """The MIXED slot kernels (FP32 states, gradients and fluxes; FP64
    conserved sums, update and dt) against the FP64 FAST slot kernels from
    the same state on an adapted mesh with hanging faces: L1 density error
    below 1e-5 after 20 steps."""
    import zephyr_b200 as Z
    mesh, solver = _adapted(acc)
    s0, w0 = mesh.get_state(), mesh.get_wait()
    out = []
    for prec in (Z.Precision.FP64, Z.Precision.MIXED):
        mesh.set_state(*s0)
        mesh.set_wait(w0)
        s = Z.SmFluid(Z.IdealGas(1.4), precision=prec, kernels=Z.Kernels.FAST)
        s.params = solver.params
        s.params.kernels, s.params.precision = int(Z.Kernels.FAST), int(prec)
        s.add_types(mesh)
        s.update(mesh, 20)
        out.append((mesh.get_state(), s.dt()))
    (a, dta), (b, dtb) = out
    l1 = np.sum(np.abs(b[0] - a[0])) / np.sum(np.abs(a[0]))
    assert l1 <= 1e-5, l1
    assert abs(dtb - dta) <= 1e-5 * dta
    mesh.close()


def test_mixed_form_adapts_and_conserves_mass(gpu_lib):
    """Adaptation with the MIXED step (the refine works on the FP64 state,
    converted from the FP64 conserved variables and back): with walls and
    the conservative "const" distributor the total mass stays constant to
    1e-9: each cell evaluates its faces itself (gather form), and in FP32
    the flux a cell computes for a face and the one its neighbour computes
    for the same face differ in the last bits, so the FP64 sums no longer
    cancel exactly (the FP64 step holds 1e-14)."""
    import zephyr_b200 as Z
    mesh, solver = gpu_mesh(20, (1, 1, 1, 1), 3, "const", 2, "MC", 0.4)
    solver.params.kernels, solver.params.precision = int(Z.Kernels.FAST), int(Z.Precision.MIXED)
    solver._push()
    g = mesh.amr_arrays()
    mesh.set_state(*AC.init_state(g["cx"], g["cy"]))

    def mass():
        return float(np.sum(mesh.get_state()[0] * mesh.amr_arrays()["vol"]))

    m0 = mass()
    counts = []
    for _ in range(6):
        solver.set_flags(mesh)
        mesh.refine()
        counts.append(mesh.n_cells())
        solver.update(mesh, 3)
        assert abs(mass() - m0) <= 1e-9 * m0
    assert len(set(counts)) > 1  # the mesh did change
    mesh.close()


def test_gradient_criterion_flags(gpu_lib):
    """|grad rho| h / rho flags (the unlimited least-squares density
    gradient): uniform density coarsens everywhere; a density step refines
    the two columns next to it and coarsens the rest; a refine follows them."""
    mesh, solver = gpu_mesh(32, (2, 2, 2, 2), 2, "slope", 2, "MC", 0.4)
    g = mesh.amr_arrays()
    n = mesh.n_cells()
    ones = np.ones(n)
    mesh.set_state(ones, 0 * ones, 0 * ones, ones, ones / 0.4)
    assert (solver.set_flags_gradient(mesh) == -1).all()
    rho = np.where(g["cx"] < 0.5, 1.0, 1.5)
    mesh.set_state(rho, 0 * ones, 0 * ones, ones, ones / (0.4 * rho))
    f = solver.set_flags_gradient(mesh, 0.05, 0.01)
    near = np.abs(g["cx"] - 0.5) < 1.0 / 32
    far = np.abs(g["cx"] - 0.5) > 3.0 / 32
    assert (f[near] == 1).all() and (f[far] == -1).all()
    mesh.refine()
    assert mesh.n_cells() == n + 3 * int(near.sum())
    mesh.close()


def test_gradient_criterion_matches_its_restatement(gpu_lib):
    """The GPU's |grad rho| h / rho flags against the restatement of the
    criterion (oracle/gradient_flags.py) on adapted blast meshes, after each
    of a few adaptations driven by the criterion itself: equal flags on
    every cell whose criterion is not within rounding of a threshold."""
    from oracle import gradient_flags as GF
    from zephyr_b200.workloads import blast_cell_means
    mesh, solver = gpu_mesh(64, (2, 2, 2, 2), 3, "slope", 2, "van Albada", 0.4)
    g = mesh.amr_arrays()
    mesh.set_state(*blast_cell_means(g["vx"], g["vy"]))
    checked = 0
    for k in range(6):
        solver.update(mesh, steps=40)  # the blast moves density about
        g = mesh.amr_arrays()
        f = solver.set_flags_gradient(mesh, 0.05, 0.01)
        rho = mesh.get_state()[0]
        crit = GF.criterion(g, rho)
        want = GF.flags(g, rho)
        clear = (np.abs(crit - 0.05) > 1e-10 * 0.05) & (np.abs(crit - 0.01) > 1e-10 * 0.01)
        assert np.array_equal(f[clear], want[clear]), (k, int(np.count_nonzero(f[clear] != want[clear])))
        checked += int(clear.sum())
        mesh.refine()
    assert np.asarray(mesh.amr_arrays()["level"]).max() == 3 and checked > 4 * 64 * 64
    mesh.close()


def test_adaptation_at_the_blast_configuration_size_side_by_side_with_reference(gpu_lib):
    """The adaptive configuration at its own size: base mesh 512 x 512,
    three refinement levels, ZOE sides, the blast data (rho = 1, u = v = 0,
    p = 1e3 inside r < 0.01 around (0.5, 0.5), 1e-5 outside, at cell centres),
    slope distributor, van Albada, CFL 0.4.  The initial adaptation loop of
    smf_test_2D.cpp:112-117 (set the data, set_flags, refine; max_level + 3
    times), then cycles of set_flags / refine / two steps, on the GPU and in
    the reference's own EuMesh / SmFluid (oracle/_ref) side by side; every
    mesh and state array is compared after every call."""
    if not ref_available():
        pytest.fail("oracle/_ref/libzref_mesh.so is missing: build it with oracle/ref_build.py")
    from oracle import ref_mesh as RM
    n, max_level = 512, 3
    ref = RM.RefEuMesh(n, n, bounds=(2, 2, 2, 2), accuracy=2, limiter="van Albada", CFL=0.4, max_level=max_level,
                       distributor="slope")
    ref_ad = AC.RefAdapter(ref)  # one host thread: the reference's stage-2 counters are then deterministic
    mesh, solver = gpu_mesh(n, (2, 2, 2, 2), max_level, "slope", 2, "van Albada", 0.4, capacity=1 << 20)
    gpu_ad = AC.GpuAdapter(mesh, solver)

    def blast(g):
        r = np.hypot(np.asarray(g["cx"]) - 0.5, np.asarray(g["cy"]) - 0.5)
        rho = np.ones_like(r)
        p = np.where(r < 0.01, 1.0e3, 1.0e-5)
        return rho, np.zeros_like(r), np.zeros_like(r), p, p / (0.4 * rho)

    for k in range(max_level + 3):
        g = gpu_ad.mesh()
        ref_ad.set_state(*blast(g))
        gpu_ad.set_state(*blast(g))
        assert np.array_equal(ref_ad.set_flags(), gpu_ad.set_flags()), (k, "initial flags")
        ref_ad.refine()
        gpu_ad.refine()
        compare_live(f"init {k}: refine", ref_ad, gpu_ad, gpu_ad.mesh())
    g = gpu_ad.mesh()
    ref_ad.set_state(*blast(g))
    gpu_ad.set_state(*blast(g))
    levels = np.asarray(g["level"])
    assert levels.max() == max_level and len(levels) > n * n, (levels.max(), len(levels))
    for c in range(3):
        assert np.array_equal(ref_ad.set_flags(), gpu_ad.set_flags()), (c, "flags")
        ref_ad.refine()
        gpu_ad.refine()
        compare_live(f"cycle {c}: refine", ref_ad, gpu_ad, gpu_ad.mesh())
        for s in range(2):
            assert ref_ad.step() == gpu_ad.step(), (c, s, "dt")
            compare_live(f"cycle {c}: step {s}", ref_ad, gpu_ad, gpu_ad.mesh())
    mesh.close()
