"""The checkpointed adjoint (ps_forward_checkpointed + ps_backward) against
forward-mode FP64 reference gradients (oracle/ps_oracle_dual.c) and FP64
central finite differences, and through a thin torch.autograd.Function."""
import numpy as np
import pytest

import psb200
from psb200 import scenes
from oracle import ps_oracle as O

pytestmark = pytest.mark.gpu
PARAMS = ("k_spring", "e_sphere", "e_zmin", "e_zmax", "e_xmin", "e_xmax", "e_ymin", "e_ymax")


def gpu_grads(sc, steps, every, precision="f64"):
    with psb200.Simulation(sc, precision) as sim:
        sim.set_state()
        sim.forward_checkpointed(steps, every)
        final = sim.get_state()
        loss, g = psb200.height_loss(final)
        grads, g0 = sim.backward(g)
        again = sim.get_state()
    assert np.array_equal(final, again)  # backward leaves the final state in place
    return loss, grads[0], g0, final


def with_params(sc, theta):
    e = tuple(theta[2:8])
    return sc.copy(k_spring=float(theta[0]), e_sphere=float(theta[1]), e_wall=e)


def theta_of(sc):
    return np.array([sc.k_spring, sc.e_sphere, *sc.e_wall])


@pytest.mark.parametrize("every", [1, 7, 25])
def test_adjoint_matches_forward_mode_reference(need_gpu, every):
    sc = scenes.pile(300, seed=21, k_spring=1.0)
    steps = 50
    loss, g_par, g0, final = gpu_grads(sc, steps, every)
    # forward mode: 8 parameter directions + 6 initial-state directions of particle 7
    nd = 8 + 6
    dp = np.zeros((nd, 8))
    dp[np.arange(8), np.arange(8)] = 1.0
    ds = np.zeros((nd, sc.n, 6))
    for c in range(6):
        ds[8 + c, 7, c] = 1.0
    st, tang = O.run_dual(sc, steps, dp, ds)
    assert np.array_equal(st, final)
    _, gl = psb200.height_loss(st)
    fm = np.array([np.sum(gl * tang[d]) for d in range(nd)])
    np.testing.assert_allclose(g_par, fm[:8], rtol=1e-8, atol=1e-12 * np.abs(fm[:8]).max())
    np.testing.assert_allclose(g0[7], fm[8:], rtol=1e-8, atol=1e-12 * np.abs(fm[8:]).max())


def test_adjoint_vs_central_fd_on_1024_sphere_pile(need_gpu):
    """FP64 central differences of the GPU forward against the adjoint on a
    1,024-sphere contact pile (spring 1, radii 0.004-0.006 on a 0.0118
    lattice, velocities N(0, 0.1^2)), 400 steps, checkpoint every 100, with
    the settling loss of the differentiation scene.  Sphere-sphere contacts
    (43 spheres overlap a neighbour from the first step) and the floor and
    side walls act inside the window, so dL/dk, dL/de_sphere, dL/de_zmin and
    dL/de_xmin are non-zero and must be; every parameter gradient is within
    1e-3 relative of the central difference (h = 1e-6 relative), and those
    the window never reaches (the ceiling's restitution) are zero on both
    sides.  The initial-velocity gradients of three spheres in contact from
    the first step are checked the same way, their y components included,
    which reach the loss only through the contact adjoint (the loss depends
    on x and z only).  Differentiated formulas: ParticleModel_kernels.cu:
    174-199 and BoxContainer_kernels.cu:24-52."""
    sc = scenes.pile(1024, seed=3, k_spring=1.0)
    steps, every = 400, 100
    loss, g_par, g0, _ = gpu_grads(sc, steps, every)
    theta = theta_of(sc)
    fd_par = np.zeros(8)
    for p in range(8):
        h = 1e-6 * max(1.0, abs(theta[p]))
        tp, tm = theta.copy(), theta.copy()
        tp[p] += h
        tm[p] -= h
        lp, _ = psb200.height_loss(psb200.simulate(with_params(sc, tp), steps, "f64"))
        lm, _ = psb200.height_loss(psb200.simulate(with_params(sc, tm), steps, "f64"))
        fd_par[p] = (lp - lm) / (2 * h)
    for name in ("k_spring", "e_sphere", "e_zmin", "e_xmin"):
        p = PARAMS.index(name)
        assert fd_par[p] != 0.0 and g_par[p] != 0.0, (name, g_par[p], fd_par[p])
    for p in range(8):
        if fd_par[p] == 0.0:
            assert g_par[p] == 0.0, (PARAMS[p], g_par[p])
        else:
            assert abs(g_par[p] - fd_par[p]) <= 1e-3 * abs(fd_par[p]), (PARAMS[p], g_par[p], fd_par[p])
    # initial velocities of spheres that overlap a neighbour from the first step
    for i in (40, 286, 593):
        for c in range(3):
            h = 1e-6
            sp, sm = sc.copy(), sc.copy()
            sp.state[i, 3 + c] += h
            sm.state[i, 3 + c] -= h
            lp, _ = psb200.height_loss(psb200.simulate(sp, steps, "f64"))
            lm, _ = psb200.height_loss(psb200.simulate(sm, steps, "f64"))
            fd = (lp - lm) / (2 * h)
            assert fd != 0.0 and g0[i, 3 + c] != 0.0, (i, c)
            assert abs(g0[i, 3 + c] - fd) <= 1e-3 * abs(fd), (i, c, g0[i, 3 + c], fd)


def test_fp32_adjoint_close_to_fp64(need_gpu):
    sc = scenes.pile(300, seed=22, k_spring=1.0)
    _, g64, v64, _ = gpu_grads(sc, 40, 10, "f64")
    _, g32, v32, _ = gpu_grads(sc, 40, 10, "f32")
    np.testing.assert_allclose(g32, g64, rtol=2e-2, atol=1e-3 * np.abs(g64).max())


def test_torch_autograd_binding(need_gpu):
    """torch.autograd.Function over the C ABI (test-only binding)."""
    import torch

    sc = scenes.pile(200, seed=23, k_spring=1.0)
    steps, every = 30, 10

    class DEMRun(torch.autograd.Function):
        @staticmethod
        def forward(ctx, theta, v0):
            s2 = with_params(sc, theta.detach().numpy())
            s2.state[:, 3:6] = v0.detach().numpy()
            sim = psb200.Simulation(s2, "f64")
            sim.set_state()
            sim.forward_checkpointed(steps, every)
            ctx.sim = sim
            return torch.from_numpy(sim.get_state()[:, :6].copy())

        @staticmethod
        def backward(ctx, grad_out):
            grads, g0 = ctx.sim.backward(grad_out.numpy())
            ctx.sim.close()
            return torch.from_numpy(grads[0]), torch.from_numpy(g0[:, 3:6].copy())

    theta = torch.tensor(theta_of(sc), requires_grad=True)
    v0 = torch.tensor(sc.state[:, 3:6].copy(), requires_grad=True)
    out = DEMRun.apply(theta, v0)
    h = 0.1 + 0.02 * torch.sin(2 * np.pi * out[:, 0] / 0.5)
    loss = torch.mean((out[:, 2] - h) ** 2)
    loss.backward()
    _, g_par, g0, _ = gpu_grads(sc, steps, every)
    np.testing.assert_allclose(theta.grad.numpy(), g_par, rtol=1e-12, atol=1e-300)
    np.testing.assert_allclose(v0.grad.numpy(), g0[:, 3:6], rtol=1e-12, atol=1e-300)


def test_backward_errors(need_gpu):
    sc = scenes.pile(50, seed=1)
    with psb200.Simulation(sc, "f64") as sim:
        sim.set_state()
        with pytest.raises(psb200.PSError, match="forward_checkpointed first"):
            sim.backward(np.zeros((sc.n, 6)))
    with psb200.Simulation(scenes.box_mesh_scene(20), "f64") as sim:
        sim.set_state()
        with pytest.raises(psb200.PSError, match="box containers"):
            sim.forward_checkpointed(5, 5)
