"""Every entry point on the smallest simulations: no particle at all, one
particle, and a batch that mixes empty, one-particle and ordinary scenes.
Each call succeeds, and what can be compared with the oracle is equal to it
bit for bit (the one-particle and mixed batches; an empty simulation has
zero gradients)."""
import numpy as np
import pytest

import psb200
from psb200 import scenes
from oracle import ps_oracle as O

pytestmark = pytest.mark.gpu


def one():
    return scenes.pile(1, seed=31)


def empty():
    return one().copy(state=np.zeros((0, 8)))


SIMS = {
    "empty": lambda: [empty()],
    "one": lambda: [one()],
    "mixed": lambda: [empty(), one(), scenes.pile(60, seed=32, k_spring=1.0), empty()],
}


def oracle_state(batch, steps, prec):
    parts = [O.run(sc, steps, prec) for sc in batch if sc.n > 0]
    want = np.concatenate(parts) if parts else np.zeros((0, 8))
    return want.astype(np.float32) if prec == "f32" else want


def cast(a, prec):
    return a.astype(np.float32) if prec == "f32" else a


@pytest.mark.parametrize("prec", ["f32", "f64"])
@pytest.mark.parametrize("name", sorted(SIMS))
def test_every_entry_point_on_small_simulations(need_gpu, name, prec):
    batch = SIMS[name]()
    n = sum(sc.n for sc in batch)
    with psb200.Simulation(batch, prec) as sim:
        sim.set_state()
        sim.checkpoint_save(0)
        sim.step(7)
        assert np.array_equal(cast(sim.get_state(), prec), oracle_state(batch, 7, prec))
        for k in range(len(batch)):
            sim.stats(k)
            sim.grid(k)
        counts, offsets, order = sim.buckets()
        assert order.shape == (n,) and int(counts.sum()) == n
        sim.checkpoint_load(0)
        assert sim.time_steps(5) >= 0.0
        sim.checkpoint_load(0)
        prof = sim.profile_steps(5)
        assert set(prof) == set(psb200.KERNEL_KINDS)
        sim.checkpoint_load(0)
        for walk, block in psb200.CONTACT_KERNELS:
            sim.set_contact_kernel(walk, block)
            sim.checkpoint_load(0)
            sim.step(7)
            assert np.array_equal(cast(sim.get_state(), prec), oracle_state(batch, 7, prec))
        sim.set_contact_kernel(*psb200.CONTACT_KERNELS[1])
        sim.checkpoint_load(0)
        tuned = sim.autotune(trial_steps=3, cell_factors=(1.05,), graph_blocks=(5, 10))  # the default cell: oracle order
        assert tuned["graph_block"] in (5, 10)
        sim.checkpoint_load(0)
        sim.set_neighbor_lists(0.3)
        sim.step(7)
        assert np.array_equal(cast(sim.get_state(), prec), oracle_state(batch, 7, prec))
        sim.tune_neighbor_lists(trial_steps=3, skins=(0.0, 0.1))
        sim.set_neighbor_lists(0.0)
        sim.checkpoint_load(0)
        sim.forward_checkpointed(12, 5)
        final = sim.get_state()
        assert np.array_equal(cast(final, prec), oracle_state(batch, 12, prec))
        _, g = psb200.height_loss(final) if n else (0.0, np.zeros((0, 6)))
        grads, g0 = sim.backward(g)
        assert len(grads) == len(batch) and g0.shape == (n, 6)
        assert all(np.all(np.isfinite(gr)) for gr in grads) and np.all(np.isfinite(g0))
        if n == 0:
            assert all(np.all(gr == 0.0) for gr in grads)
        sim.sync()
