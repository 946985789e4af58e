"""The adjoint mode (zg_adj_*): its forward against the CPU restatement
(oracle/adjoint_ref.py), its gradient against central finite differences of
the FP64 forward, independence from the checkpoint spacing, and the
torch.autograd.Function wrapper that exposes it to PyTorch (test harness
only)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FD_TOL = 1e-4  # relative error of the adjoint directional derivative against central differences


def smooth_state(nx, ny, seed=1):
    """rho = 1 + 0.2 f, u = 0.3 f, v = 0.3 f, p = 1 + 0.1 f with f a sum of
    seeded periodic modes (the smooth periodic problem), on nx x ny cells."""
    rng = np.random.default_rng(seed)
    x = (np.arange(nx) + 0.5) / nx
    y = (np.arange(ny) + 0.5) / ny
    X, Y = np.meshgrid(x, y, indexing="ij")

    def f():
        out = np.zeros((nx, ny))
        for m in range(1, 5):
            a, ph, ps = rng.random() / 4, 2 * np.pi * rng.random(), 2 * np.pi * rng.random()
            out += a * np.sin(2 * np.pi * m * X + ph) * np.sin(2 * np.pi * m * Y + ps)
        return out.ravel()

    return 1.0 + 0.2 * f(), 0.3 * f(), 0.3 * f(), 1.0 + 0.1 * f()


def cuda(*arrs):
    import torch
    return [torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda") for a in arrs]


class AdjointJ:
    """torch.autograd.Function over zg_adj_forward / zg_adj_gradient:
    J(rho_0, gamma) with u_0, v_0, p_0 held fixed."""

    @staticmethod
    def make(adj, prm_of, u, v, p):
        import torch

        class Fn(torch.autograd.Function):
            @staticmethod
            def forward(ctx, rho0, gamma):
                prm = prm_of(float(gamma))
                grad = torch.empty_like(rho0)
                J, dg = adj.gradient(prm, rho0.contiguous(), u, v, p, grad)
                ctx.save_for_backward(grad, torch.tensor(dg, dtype=torch.float64, device=rho0.device))
                return torch.tensor(J, dtype=torch.float64, device=rho0.device)

            @staticmethod
            def backward(ctx, gJ):
                grad, dg = ctx.saved_tensors
                return gJ * grad, gJ * dg

        return Fn.apply


def test_adjoint_forward_matches_cpu_restatement(gpu_lib):
    from oracle import adjoint_ref as AR
    from zephyr_b200.adjoint import Adjoint
    nx, ny, steps = 48, 40, 8
    st = smooth_state(nx, ny)
    adj = Adjoint(nx, ny)
    r, u, v, p = cuda(*st)
    dt = adj.cfl_dt(1.4, 0.4, r, u, v, p)
    prm = Adjoint.params(steps=steps, checkpoint_every=3, dt=dt, probe=(0.55, 0.8, 0.2, 0.45))
    J = adj.forward(prm, r, u, v, p)
    J_cpu, _ = AR.run(*st, nx, ny, dt=dt, steps=steps, probe=(0.55, 0.8, 0.2, 0.45))
    assert abs(J - J_cpu) <= 1e-12 * abs(J_cpu)
    adj.close()


@pytest.mark.parametrize("n,steps,every", [(64, 20, 5), (96, 31, 7)])
def test_adjoint_gradient_against_central_differences(gpu_lib, n, steps, every):
    import torch
    from zephyr_b200.adjoint import Adjoint
    st = smooth_state(n, n, seed=3)
    adj = Adjoint(n, n)
    r, u, v, p = cuda(*st)
    dt = adj.cfl_dt(1.4, 0.4, r, u, v, p)
    prm = Adjoint.params(steps=steps, checkpoint_every=every, dt=dt)
    grad = torch.empty_like(r)
    J, dJ_dgamma = adj.gradient(prm, r, u, v, p, grad)
    assert J == adj.forward(prm, r, u, v, p)
    rng = np.random.default_rng(5)
    eps = 1e-6
    for _ in range(4):
        d = torch.tensor(rng.standard_normal(n * n), dtype=torch.float64, device="cuda")
        Jp = adj.forward(prm, r + eps * d, u, v, p)
        Jm = adj.forward(prm, r - eps * d, u, v, p)
        fd = (Jp - Jm) / (2 * eps)
        ad = float(torch.dot(grad, d))
        assert abs(fd - ad) <= FD_TOL * abs(ad), (fd, ad)
    prm_p, prm_m = Adjoint.params(steps=steps, checkpoint_every=every, dt=dt, gamma=1.4 + eps), \
        Adjoint.params(steps=steps, checkpoint_every=every, dt=dt, gamma=1.4 - eps)
    # gamma enters the initial energy too: the same (rho, u, v, p) at another gamma
    fd_g = (adj.forward(prm_p, r, u, v, p) - adj.forward(prm_m, r, u, v, p)) / (2 * eps)
    assert abs(fd_g - dJ_dgamma) <= FD_TOL * abs(dJ_dgamma), (fd_g, dJ_dgamma)
    adj.close()


def test_adjoint_checkpoint_spacing_leaves_the_gradient_unchanged(gpu_lib):
    import torch
    from zephyr_b200.adjoint import Adjoint
    n, steps = 40, 12
    st = smooth_state(n, n, seed=7)
    adj = Adjoint(n, n)
    r, u, v, p = cuda(*st)
    dt = adj.cfl_dt(1.4, 0.4, r, u, v, p)
    out = []
    for every in (1, 5, 12, 40):
        g = torch.empty_like(r)
        J, dg = adj.gradient(Adjoint.params(steps=steps, checkpoint_every=every, dt=dt), r, u, v, p, g)
        out.append((J, dg, g.cpu().numpy()))
    for J, dg, g in out[1:]:
        assert J == out[0][0] and dg == out[0][1] and np.array_equal(g, out[0][2])
    adj.close()


def test_adjoint_through_torch_autograd(gpu_lib):
    import torch
    from zephyr_b200.adjoint import Adjoint
    n, steps = 32, 10
    st = smooth_state(n, n, seed=11)
    adj = Adjoint(n, n)
    r, u, v, p = cuda(*st)
    dt = adj.cfl_dt(1.4, 0.4, r, u, v, p)

    def prm_of(gamma):
        return Adjoint.params(steps=steps, checkpoint_every=4, dt=dt, gamma=gamma)

    J_of = AdjointJ.make(adj, prm_of, u, v, p)
    rho0 = r.clone().requires_grad_(True)
    gamma = torch.tensor(1.4, dtype=torch.float64, device="cuda", requires_grad=True)
    J = J_of(rho0, gamma)
    (2.0 * J).backward()
    g = torch.empty_like(r)
    J2, dg = adj.gradient(prm_of(1.4), r, u, v, p, g)
    assert float(J) == J2
    assert torch.equal(rho0.grad, 2.0 * g) and float(gamma.grad) == 2.0 * dg
    adj.close()


def test_mixed_adjoint_tracks_the_fp64_adjoint(gpu_lib):
    """The mixed adjoint (FP64 primal step with FP32 slopes; the reverse
    sweep's slope partials, face states, HLLC reverse and face cotangents in
    FP32, adjoint states and sums in FP64): J to 1e-9, the gradient to 1e-5
    in the L2 norm against the FP64 adjoint, and directional derivatives
    within the FP64 form's tolerance of central differences of the FP64
    forward."""
    import torch
    from zephyr_b200.adjoint import Adjoint
    n, steps = 64, 20
    st = smooth_state(n, n, seed=3)
    adj = Adjoint(n, n)
    r, u, v, p = cuda(*st)
    dt = adj.cfl_dt(1.4, 0.4, r, u, v, p)
    p64 = Adjoint.params(steps=steps, checkpoint_every=5, dt=dt)
    pmx = Adjoint.params(steps=steps, checkpoint_every=5, dt=dt, precision=1)
    g64, gmx = torch.empty_like(r), torch.empty_like(r)
    J64, dg64 = adj.gradient(p64, r, u, v, p, g64)
    Jmx, dgmx = adj.gradient(pmx, r, u, v, p, gmx)
    assert Jmx == adj.forward(pmx, r, u, v, p)
    assert abs(Jmx - J64) <= 1e-9 * abs(J64)  # FP32 slopes: 2e-10 here
    assert float(torch.linalg.norm(gmx - g64) / torch.linalg.norm(g64)) <= 1e-5
    assert abs(dgmx - dg64) <= 1e-5 * abs(dg64)
    rng = np.random.default_rng(5)
    eps = 1e-6
    for _ in range(3):
        d = torch.tensor(rng.standard_normal(n * n), dtype=torch.float64, device="cuda")
        fd = (adj.forward(p64, r + eps * d, u, v, p) - adj.forward(p64, r - eps * d, u, v, p)) / (2 * eps)
        ad = float(torch.dot(gmx, d))
        assert abs(fd - ad) <= FD_TOL * abs(ad), (fd, ad)
    adj.close()
