"""Neighbour-list mode (ps_set_neighbor_lists) against the grid path: the
same scenes, stepped in the same calls, must give the same state bit for bit
in FP32 and FP64 -- stable and diverging scenes, batches, triangle
containers, lists rebuilt almost every step, and calls that overflow the
lists and are repeated on the grid path."""
import os
import subprocess

import numpy as np
import pytest

import psb200
from psb200 import scenes
from oracle import ps_oracle as O

pytestmark = pytest.mark.gpu

CALLS = (1, 37, 200, 63)  # one-step call, a graph block and ragged remainders


def run(scene, prec, calls=CALLS, skin=None, cap=48):
    with psb200.Simulation(scene, prec) as sim:
        sim.set_state()
        if skin is not None:
            sim.set_neighbor_lists(skin, cap)
        for n in calls:
            sim.step(n)
        return sim.get_state(), (sim.list_stats() if skin is not None else (0, 0))


def same(a, b):
    return a.shape == b.shape and np.array_equal(a, b, equal_nan=True)


@pytest.mark.parametrize("prec", ["f32", "f64"])
@pytest.mark.parametrize("make", [lambda: scenes.pile(1500, seed=11, k_spring=1.0),
                                  lambda: scenes.settle_pile(side=10),
                                  lambda: scenes.lattice_c1(side=12)],
                         ids=["pile", "settle", "lattice"])
def test_lists_equal_grid(need_gpu, make, prec):
    sc = make()
    want, _ = run(sc, prec)
    got, (_, fb) = run(sc, prec, skin=0.3)
    assert fb == 0
    assert same(got, want)


def test_lists_equal_oracle(need_gpu):
    sc = scenes.pile(800, seed=12, k_spring=1.0)
    got, (_, fb) = run(sc, "f32", calls=(90, 30), skin=0.25)
    assert fb == 0
    assert np.array_equal(got.astype(np.float32), O.run(sc, 120, "f32"))


@pytest.mark.parametrize("skin", [0.02, 1.0])
def test_lists_skin_extremes(need_gpu, skin):
    # a thin skin makes the device ask for rebuilds inside the calls; a
    # full-cell skin reaches two cells out
    sc = scenes.pile(1200, seed=13, k_spring=1.0)
    want, _ = run(sc, "f32")
    got, (rebuilds, fb) = run(sc, "f32", skin=skin, cap=160)
    assert fb == 0
    # rebuilds inside the calls: the gated cooperative rebuild kernel ran
    assert rebuilds > 0 or skin > 0.1
    assert same(got, want)


@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_lists_diverging_scene(need_gpu, prec):
    # spring 1e4 with dt 1e-5: k dt / m >> 1, the scene goes non-finite
    sc = scenes.pile(1000, seed=14, k_spring=1e4)
    want, _ = run(sc, prec, calls=(150, 150))
    assert not np.isfinite(want).all()
    got, _ = run(sc, prec, calls=(150, 150), skin=0.3, cap=200)
    assert same(got, want)


def test_lists_back_off_to_grid_on_a_fast_scene(need_gpu):
    # spheres that cross half the skin every step or two: after a window of
    # 256 list steps the next 1,024 steps run on the grid path, with the same
    # states
    sc = scenes.pile(1000, seed=21, k_spring=1.0)
    st = sc.state.copy()
    st[:, 3:6] *= 50.0
    sc = sc.copy(state=st)
    calls = (150, 150, 150, 150)
    want, _ = run(sc, "f32", calls=calls)
    with psb200.Simulation(sc, "f32") as sim:
        sim.set_state()
        sim.set_neighbor_lists(0.01, 200)
        for n in calls:
            sim.step(n)
        got = sim.get_state()
        rebuilds, _, grid_steps = sim.list_stats_all()
    assert rebuilds * 4 > 300 and grid_steps == 300
    assert same(got, want)


def test_lists_batch(need_gpu):
    batch = [scenes.pile(300, seed=15, k_spring=0.5), scenes.settle_pile(side=8),
             scenes.pile(900, seed=16, k_spring=2.0), scenes.pile(64, seed=17, k_spring=1e4)]
    for prec in ("f32", "f64"):
        want, _ = run(batch, prec)
        got, _ = run(batch, prec, skin=0.4)
        assert same(got, want)


@pytest.mark.parametrize("prec", ["f32", "f64"])
@pytest.mark.parametrize("make", [lambda: scenes.box_mesh_scene(), lambda: scenes.funnel_wall_scene(1500)],
                         ids=["box_mesh", "funnel"])
def test_lists_triangle_containers(need_gpu, make, prec):
    sc = make()
    want, _ = run(sc, prec, calls=(120, 80))
    got, (_, fb) = run(sc, prec, calls=(120, 80), skin=0.3)
    assert fb == 0
    assert same(got, want)


def test_lists_batch_with_a_triangle_container(need_gpu):
    # a mesh scene and box scenes in one launch (the multi-scene mesh variant)
    batch = [scenes.pile(300, seed=28, k_spring=1.0), scenes.box_mesh_scene(), scenes.pile(500, seed=29, k_spring=1.0)]
    for prec in ("f32", "f64"):
        want, _ = run(batch, prec, calls=(60, 90))
        got, (_, fb) = run(batch, prec, calls=(60, 90), skin=0.2)
        assert fb == 0
        assert same(got, want)


def test_list_overflow_repeats_call_on_grid(need_gpu):
    sc = scenes.pile(1000, seed=18, k_spring=1.0)
    want, _ = run(sc, "f32", calls=(50, 50))
    got, (_, fb) = run(sc, "f32", calls=(50, 50), skin=0.3, cap=2)
    assert fb == 2
    assert same(got, want)


def test_lists_switch_on_and_off(need_gpu):
    sc = scenes.pile(1200, seed=19, k_spring=1.0)
    want, _ = run(sc, "f64", calls=(40, 40, 40, 40))
    with psb200.Simulation(sc, "f64") as sim:
        sim.set_state()
        sim.set_neighbor_lists(0.3, 48)
        sim.step(40)
        sim.set_neighbor_lists(0.0, 0)
        sim.step(40)
        sim.set_neighbor_lists(0.5, 64)  # new capacity: new buffers and graphs
        sim.step(40)
        st = sim.stats(0)  # regrids from the at-rest state
        assert np.isfinite(st.kinetic_energy) and st.kinetic_energy > 0.0
        sim.step(40)
        got = sim.get_state()
    assert same(got, want)


def test_tune_neighbor_lists_restores_state_and_keeps_parity(need_gpu):
    sc = scenes.pile(1500, seed=22, k_spring=1.0)
    want, _ = run(sc, "f32", calls=(60,))
    with psb200.Simulation(sc, "f32") as sim:
        sim.set_state()
        before = sim.get_state()
        res = sim.tune_neighbor_lists(trial_steps=20, skins=(0.0, 0.05, 0.3), max_neighbours=96)
        assert len(res["ms_table"]) == 3 and all(t > 0 for t in res["ms_table"])
        assert res["skin_fraction"] == res["skins"][int(np.argmin(res["ms_table"]))]
        assert np.array_equal(sim.get_state(), before)
        assert sim.list_stats_all() == (0, 0, 0)
        sim.step(60)
        got = sim.get_state()
    assert same(got, want)
    with psb200.Simulation(sc, "f32") as sim:
        sim.set_state()
        with pytest.raises(psb200.PSError, match="skin_fraction"):
            sim.tune_neighbor_lists(trial_steps=5, skins=(0.005,))


def test_list_arguments(need_gpu):
    sc = scenes.pile(100, seed=20)
    with psb200.Simulation(sc, "f32") as sim:
        sim.set_state()
        for bad in (1.5, 0.005, -0.1, float("nan")):
            with pytest.raises(psb200.PSError, match="skin_fraction"):
                sim.set_neighbor_lists(bad, 32)
        with pytest.raises(psb200.PSError, match="max_neighbours"):
            sim.set_neighbor_lists(0.3, 0)
        sim.set_neighbor_lists(0.0, 0)
        assert sim.list_stats_all() == (0, 0, 0)


@pytest.mark.parametrize("setting,steps", [("auto", 10000), ("auto", 400), ("0.05", 400)])
def test_cli_with_neighbor_lists_writes_the_same_csv(need_gpu, tmp_path, setting, steps):
    """runSimulateCUDA with PSB200_NEIGHBOR_LISTS: the output CSV is the
    grid path's, byte for byte.  "auto" tunes only for runs of 10,000 steps
    or more; a shorter run keeps the grid path and says so."""
    sc = scenes.pile(2000, seed=23, k_spring=1.0)
    csv_in = tmp_path / "in.csv"
    with open(csv_in, "w") as f:
        f.write("x,y,z,r\n")
        for p in sc.state:
            f.write("%.17g,%.17g,%.17g,%.17g\n" % (p[0], p[1], p[2], p[6]))
    outs = {}
    for tag, env_value in (("grid", None), ("lists", setting)):
        out = tmp_path / f"{tag}.csv"
        cmd = [psb200.CLI_PATH, "--lib", psb200.LIB_PATH, str(csv_in), "--cuda", "--max-steps", str(steps),
               "--box-min", *map(str, sc.box_min), "--box-max", *map(str, sc.box_max), "--dt", "1e-05",
               "--coeff-of-spring", "1", "--coeff-of-restitution-sphere", "0.5",
               "--coeff-of-restitution-wall", *["0.7"] * 6, "--gravity", "0", "0", "-9.8",
               "--initial-velocity", "0.05", "0", "-0.1", "--density", "1000", "--out-csv-path", str(out)]
        env = dict(os.environ)
        env.pop("PSB200_NEIGHBOR_LISTS", None)
        if env_value is not None:
            env["PSB200_NEIGHBOR_LISTS"] = env_value
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, env=env)
        assert r.returncode == 0, r.stdout + r.stderr
        if env_value == "auto" and steps < 10000:
            assert "off for runs under 10,000 steps" in r.stdout
        elif env_value is not None:
            assert "neighbour-list skin" in r.stdout
        outs[tag] = out.read_text()
    assert outs["lists"] == outs["grid"]


@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_adjoint_after_a_forward_on_lists(need_gpu, prec):
    # ps_forward_checkpointed steps through ps_step, so with lists on its
    # forward pass runs on them; checkpoints, final state and gradients must
    # equal the grid path's bit for bit
    sc = scenes.pile(1000, seed=24, k_spring=1.0)
    out = {}
    for skin in (None, 0.05):
        with psb200.Simulation(sc, prec) as sim:
            sim.set_state()
            if skin is not None:
                sim.set_neighbor_lists(skin, 64)
            sim.forward_checkpointed(300, 50)
            final = sim.get_state()
            _, g = psb200.height_loss(final)
            grads, g0 = sim.backward(g)
            out[skin] = (final, grads[0], g0)
    assert same(out[0.05][0], out[None][0])
    assert np.array_equal(out[0.05][1], out[None][1]) and np.array_equal(out[0.05][2], out[None][2])


@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_lists_batch_with_empty_and_single_sphere_scenes(need_gpu, prec):
    one = scenes.pile(1, seed=25)
    empty = one.copy(state=np.zeros((0, 8)))
    batch = [scenes.pile(400, seed=26, k_spring=1.0), empty, one, scenes.pile(200, seed=27, k_spring=1.0), empty]
    want, _ = run(batch, prec, calls=(1, 50, 30))
    got, (_, fb) = run(batch, prec, calls=(1, 50, 30), skin=0.05)
    assert fb == 0
    assert same(got, want)


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_lists_over_a_40000_step_settling_run(need_gpu, prec):
    # the lattice collapses into a pile and comes close to rest: thousands of
    # contacts change order and lists are rebuilt many times; the end state
    # must still be the grid path's bit for bit
    sc = scenes.settle_pile(side=16)
    calls = (10000,) * 4
    want, _ = run(sc, prec, calls=calls)
    with psb200.Simulation(sc, prec) as sim:
        sim.set_state()
        sim.set_neighbor_lists(0.05, 64)
        for n in calls:
            sim.step(n)
        got = sim.get_state()
        rebuilds, fallbacks, grid_steps = sim.list_stats_all()
    print(f"\nsettling pile {prec}: {rebuilds} rebuilds, {fallbacks} fallbacks, {grid_steps} steps on the grid path")
    assert rebuilds > 10
    assert same(got, want)
