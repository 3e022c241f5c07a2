"""The benchmark configurations at their full sizes, bit for bit against the
oracle on the GPU.

The 1M-sphere box scene has its own test (test_gpu_headline.py).  Here:
- the 4,096-sphere lattice over its full 5,000 steps, FP32 and FP64;
- the 262,144-sphere funnel with its 20,200-triangle container, after a pour
  long enough that the container and the sphere contacts act on many
  spheres (with a soft spring that stays finite);
- the 65,536-sphere box of the gradient workload from the onset of its
  contacts, forward and through the checkpointed adjoint (gradients against
  the forward-mode FP64 oracle);
- the 256-scene batch (3.5 M spheres), every scene against the oracle alone.

The long pours run on the GPU only; the oracle then steps the same state a
few times, which is all a CPU check of 262 k spheres against 20 k triangles
can afford.  Diverged spheres (the specified springs are far stiffer than
the scheme's explicit update tolerates once spheres touch) must agree too:
NaN where the oracle has NaN.
"""
import numpy as np
import pytest

import psb200
from psb200 import scenes
from oracle import ps_oracle as O

pytestmark = pytest.mark.gpu


def gpu_run(sc, steps, prec):
    with psb200.Simulation(sc, prec) as sim:
        sim.set_state()
        if steps:
            sim.step(steps)
        sim.sync()
        return sim.get_state()


def gpu_stats(sc, prec):
    with psb200.Simulation(sc, prec) as sim:
        sim.set_state()
        return sim.stats()


def cast(a, prec):
    return a.astype(np.float32) if prec == "f32" else a


def same(got, want):
    return got.shape == want.shape and np.array_equal(got, want, equal_nan=True)


def ndiff(got, want):
    return int(np.sum(np.any(~((got == want) | (np.isnan(got) & np.isnan(want))), axis=1)))


@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_lattice_config_full_5000_steps(need_gpu, prec):
    sc = scenes.lattice_c1()
    got = cast(gpu_run(sc, 5000, prec), prec)
    want = O.run(sc, 5000, prec)
    assert same(got, want), f"{ndiff(got, want)} of {sc.n} differ"


@pytest.fixture(scope="module")
def funnel_poured():
    """The funnel scene with a soft spring (k*dt/m = 0.22, so contacts stay
    finite), poured for 60,000 steps on the GPU in FP32: the lowest layers
    are deep in the cone.  As specified (k = 2e4, k*dt/m = 885) the first
    sphere contacts throw spheres far outside the funnel, and the domain of
    a new scene made from that state (the mesh AABB widened to the spheres)
    would no longer fit in memory; its first 20,000 steps, before any
    contact, are the benchmark's mesh line."""
    sc = scenes.c3_scene().copy(k_spring=5.0)
    return sc.copy(state=gpu_run(sc, 60000, "f32").astype(np.float64))


def test_funnel_config_at_full_size(need_gpu, funnel_poured):
    mid = funnel_poured
    assert mid.n == 262144 and mid.tri.shape[0] == 20200
    assert np.all(np.isfinite(mid.state))
    # the container acts on many spheres in the next step: the oracle's own
    # integrate + container pass moves them, against integrate alone
    after_mesh = O.pre_grid_state(mid, mid.state, "f32")
    free = mid.copy(tri=None, box_min=(-10.0, -10.0, -10.0), box_max=(10.0, 10.0, 10.0))
    after_free = O.pre_grid_state(free, mid.state, "f32")
    hit = np.any(after_mesh != after_free, axis=1) & np.all(np.isfinite(after_mesh), axis=1)
    assert hit.sum() > 500, f"only {hit.sum()} spheres touch the funnel"
    assert gpu_stats(mid, "f32").n_collided > 1000  # spheres pile up in the cone
    got = cast(gpu_run(mid, 2, "f32"), "f32")
    want = O.run(mid, 2, "f32")
    assert same(got, want), f"{ndiff(got, want)} of {mid.n} differ"
    got64 = gpu_run(mid, 1, "f64")
    want64 = O.run(mid, 1, "f64")
    assert same(got64, want64), f"{ndiff(got64, want64)} of {mid.n} differ (FP64)"


@pytest.fixture(scope="module")
def gradient_box_states():
    """The gradient workload's box (65,536 spheres) run on the GPU: as
    specified to the onset of its contacts (step 1,300), and with the soft
    spring to step 3,000, when about 380 spheres touch another (the oracle's
    count on the same run)."""
    spec = scenes.c4_scene()
    soft = scenes.c4_scene(k_spring=5.0)
    return {"spec": spec.copy(state=gpu_run(spec, 1300, "f64")),
            "soft": soft.copy(state=gpu_run(soft, 3000, "f64"))}


@pytest.mark.parametrize("prec", ["f32", "f64"])
@pytest.mark.parametrize("which", ["soft", "spec"])
def test_gradient_config_forward_at_full_size(need_gpu, gradient_box_states, which, prec):
    mid = gradient_box_states[which]
    assert mid.n == 65536
    if prec == "f32":
        mid = mid.copy(state=mid.state.astype(np.float32).astype(np.float64))
    got = cast(gpu_run(mid, 30, prec), prec)
    want = O.run(mid, 30, prec)
    assert same(got, want), f"{ndiff(got, want)} of {mid.n} differ"
    if which == "soft":
        assert gpu_stats(mid, prec).n_collided > 200


def test_gradient_config_adjoint_at_full_size(need_gpu, gradient_box_states):
    """Checkpointed forward + backward over 100 contact steps of all 65,536
    spheres: the forward state equals the plain run, and the eight parameter
    gradients equal the forward-mode FP64 oracle's."""
    mid = gradient_box_states["soft"]
    steps = 100
    with psb200.Simulation(mid, "f64") as sim:
        sim.set_state()
        sim.forward_checkpointed(steps, 25)
        final = sim.get_state()
        _, g = psb200.height_loss(final)
        grads, g0 = sim.backward(g)
    st, tang = O.run_dual(mid, steps, np.eye(8), np.zeros((8, mid.n, 6)))
    assert np.array_equal(final, st)
    _, gl = psb200.height_loss(st)
    fm = np.array([np.sum(gl * tang[d]) for d in range(8)])
    assert np.count_nonzero(fm) >= 3  # spring, sphere restitution and at least the floor act
    np.testing.assert_allclose(grads[0], fm, rtol=1e-6, atol=1e-12 * np.abs(fm).max())
    assert np.all(np.isfinite(g0))


@pytest.mark.parametrize("k_range", [(0.25, 2.5), (5e3, 5e4)], ids=["soft", "spec"])
def test_batch_config_at_full_size(need_gpu, k_range):
    batch = scenes.c5_scenes(256, k_range=k_range)
    assert len(batch) == 256
    with psb200.Simulation(batch, "f32") as sim:
        sim.set_state()
        sim.step(3)
        joint = sim.get_state()
    off = 0
    for k, sc in enumerate(batch):
        got = joint[off:off + sc.n].astype(np.float32)
        want = O.run(sc, 3, "f32")
        assert same(got, want), f"scene {k}: {ndiff(got, want)} of {sc.n} differ"
        off += sc.n
    assert off == joint.shape[0]
