"""GPU parity of the DEM step against the oracle, through the C ABI.

The device kernels perform the oracle's floating-point operations in the
oracle's order, so trajectories are compared bit for bit, in FP32 and FP64,
and the grid (cell counts, exclusive offsets, canonical order) exactly.
"""
import numpy as np
import pytest

import psb200
from psb200 import scenes
from oracle import ps_oracle as O

pytestmark = pytest.mark.gpu


def run_gpu(sc, steps, precision, chunks=None):
    with psb200.Simulation(sc, precision) as sim:
        sim.set_state()
        for c in (chunks or [steps]):
            sim.step(c)
        sim.sync()
        return sim.get_state()


def as_prec(a, precision):
    return a.astype(np.float32) if precision == "f32" else a


@pytest.mark.parametrize("precision", ["f32", "f64"])
@pytest.mark.parametrize("steps", [1, 2, 17, 120])
def test_pile_bitexact(need_gpu, precision, steps):
    sc = scenes.pile(1024, seed=3, k_spring=1.0)
    got = as_prec(run_gpu(sc, steps, precision), precision)
    want = O.run(sc, steps, precision)
    assert np.array_equal(got, want), f"{np.sum(np.any(got != want, axis=1))} particles differ"


@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_step_chunking_is_invisible(need_gpu, precision):
    """ps_step(a) then ps_step(b) equals ps_step(a+b), across graph blocks."""
    sc = scenes.pile(700, seed=5, k_spring=2.0)
    a = run_gpu(sc, 250, precision)
    b = run_gpu(sc, 250, precision, chunks=[1, 33, 200, 16])
    assert np.array_equal(a, b)


@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_lattice_c1_bitexact(need_gpu, precision):
    sc = scenes.lattice_c1()
    got = as_prec(run_gpu(sc, 300, precision), precision)
    want = O.run(sc, 300, precision)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_buckets_exact(need_gpu, precision):
    """Cell counts, exclusive offsets and the canonical order after one step
    equal the oracle's count / scan / stable order on the same positions."""
    sc = scenes.pile(1500, seed=7, k_spring=1.0)
    with psb200.Simulation(sc, precision) as sim:
        sim.set_state()
        sim.step(1)
        counts, offsets, order = sim.buckets()
        g = sim.grid(0)
    pre = O.pre_grid_state(sc, sc.state, precision)
    og = O.grid_for(sc)
    assert (g.nb[0], g.nb[1], g.nb[2]) == tuple(og.nb) and g.interval == og.interval
    cell = O.cell_ids(pre, og)
    c_o, off_o, ord_o = O.count_scan_order(cell, og.n_cells)
    assert np.array_equal(counts, c_o)
    assert np.array_equal(offsets, off_o[:-1])
    assert np.array_equal(order, ord_o)


@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_buckets_before_first_step(need_gpu, precision):
    sc = scenes.pile(400, seed=8)
    with psb200.Simulation(sc, precision) as sim:
        sim.set_state()
        counts, offsets, order = sim.buckets()
        st = sim.get_state()
    og = O.grid_for(sc)
    cell = O.cell_ids(sc.state.astype(np.float32) if precision == "f32" else sc.state, og)
    c_o, off_o, ord_o = O.count_scan_order(cell, og.n_cells)
    assert np.array_equal(counts, c_o) and np.array_equal(order, ord_o)
    assert np.array_equal(as_prec(st, precision), as_prec(sc.state, precision))


def test_multi_scene_equals_single(need_gpu):
    """A batch of uneven scenes advances exactly as each scene alone."""
    batch = scenes.c5_scenes(5, seed=9, n_lo=200, n_hi=3000)
    joint = None
    with psb200.Simulation(batch, "f32") as sim:
        sim.set_state()
        sim.step(40)
        joint = sim.get_state()
    off = 0
    for sc in batch:
        alone = run_gpu(sc, 40, "f32")
        assert np.array_equal(joint[off:off + sc.n], alone)
        want = O.run(sc, 40, "f32")
        assert np.array_equal(alone.astype(np.float32), want)
        off += sc.n


def test_simulate_one_shot(need_gpu):
    sc = scenes.pile(300, seed=12)
    a = psb200.simulate(sc, 25, "f64")
    assert np.array_equal(a, O.run(sc, 25, "f64"))


def test_stats_match_oracle(need_gpu):
    sc = scenes.pile(800, seed=13, k_spring=1.0)
    with psb200.Simulation(sc, "f64") as sim:
        sim.set_state()
        sim.step(10)
        st = sim.get_state()
        s = sim.stats(0)
    o = O.stats(st)
    assert s.n_collided == o.n_collided
    assert s.max_overlap == pytest.approx(o.max_overlap, rel=1e-12, abs=0)
    assert s.kinetic_energy == pytest.approx(o.kinetic_energy, rel=1e-12)
    assert list(s.min_pos) == list(o.min_pos) and list(s.max_pos) == list(o.max_pos)


@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_diverging_scene_and_nonfinite_particles(need_gpu, precision):
    """The reference's kick k*overlap/m is not scaled by dt, so a spring of
    1e4 on these masses makes the scheme diverge within a few steps; with
    particles also placed at NaN and infinite coordinates, the trajectories,
    non-finite values included, still equal the oracle's.  Non-finite
    particles hash to the cells the reference puts them in and take part in
    no contact."""
    sc = scenes.pile(1024, seed=11, k_spring=1e4)
    st = sc.state.copy()
    st[5, 0] = np.nan
    st[17, 1] = np.inf
    st[40, 2] = -np.inf
    st[41, 3] = np.nan
    sc = sc.copy(state=st)
    for steps in (1, 40, 150):
        got = as_prec(run_gpu(sc, steps, precision), precision)
        want = O.run(sc, steps, precision)
        assert np.array_equal(got, want, equal_nan=True), steps
    with psb200.Simulation(sc, precision) as sim:
        sim.set_state()
        sim.step(40)
        counts, offsets, order = sim.buckets()
    # the grid of step 40 is built from step 39's state after integrate + walls
    pre = O.pre_grid_state(sc, O.run(sc, 39, precision), precision)
    og = O.grid_for(sc)
    c_o, off_o, ord_o = O.count_scan_order(O.cell_ids(pre, og), og.n_cells)
    assert np.array_equal(counts, c_o)
    assert np.array_equal(offsets, off_o[:-1])
    assert np.array_equal(order, ord_o)


def test_empty_and_single_particle(need_gpu):
    one = scenes.pile(1, seed=1)
    got = run_gpu(one, 5, "f64")
    assert np.array_equal(got, O.run(one, 5, "f64"))
    empty = one.copy(state=np.zeros((0, 8)))
    with psb200.Simulation(empty, "f32") as sim:
        sim.set_state()
        sim.step(3)
        assert sim.get_state().shape == (0, 8)


def test_bad_inputs_are_errors(need_gpu):
    sc = scenes.pile(10, seed=1)
    with psb200.Simulation(sc, "f32") as sim:
        with pytest.raises(psb200.PSError):
            sim.step(1)  # no state yet
        bad = sc.state.copy()
        bad[3, 7] = -1.0  # negative mass
        with pytest.raises(psb200.PSError):
            sim.set_state(bad)
    with pytest.raises(psb200.PSError):
        psb200.Simulation(sc.copy(interval=1e-4), "f32").set_state()  # cell smaller than 2 r_max


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_later_uploads_are_checked_on_the_device(need_gpu, precision):
    # after the first upload sizes the grids, a new state is checked on the
    # device: every particle must fit its scene's cell (2 r <= edge) and have
    # a positive mass; the lowest failing index is reported and the previous
    # state stays in place
    batch = [scenes.pile(300, seed=2), scenes.pile(500, seed=3)]
    rounded = (lambda a: a.astype(np.float32).astype(np.float64)) if precision == "f32" else (lambda a: a)
    with psb200.Simulation(batch, precision) as sim:
        sim.set_state()
        sim.step(5)
        before = sim.get_state()
        edge = sim.grid(1).interval
        for idx, col, val in ((420, 6, 0.51 * edge), (733, 7, 0.0), (301, 6, np.nan), (12, 7, -2.0)):
            bad = before.copy()
            bad[idx, col] = val
            bad[idx + 40, col] = val  # a later failing particle is not the one reported
            with pytest.raises(psb200.PSError, match=f"particle {idx} does not fit"):
                sim.set_state(bad)
            assert np.array_equal(sim.get_state(), before)
        ok = before.copy()
        ok[420, 6] = 0.5 * edge  # exactly fits
        sim.set_state(ok)
        assert np.array_equal(sim.get_state(), rounded(ok))
