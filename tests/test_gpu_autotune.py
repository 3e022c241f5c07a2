"""ps_autotune: the cell-size factor, graph block and contact kernel (walk
and CTA size) chosen by timing, on a batch of three scenes.  The tuner must
restore the state it started from, report full timing tables, and leave a
simulation whose trajectories are exactly the oracle's with the chosen cell
sizes (bit for bit, FP32).  Every contact kernel variant gives the same
states bit for bit."""
import numpy as np
import pytest

import psb200
from psb200 import scenes
from oracle import ps_oracle as O

pytestmark = pytest.mark.gpu


def test_autotune_choice_restores_state_and_keeps_parity(need_gpu):
    batch = [scenes.pile(n, seed=30 + k, k_spring=1.0) for k, n in enumerate((300, 700, 1500))]
    factors, blocks = (1.0, 1.5, 2.0), (5, 20)
    with psb200.Simulation(batch, "f32") as sim:
        sim.set_state()
        before = sim.get_state()
        res = sim.autotune(trial_steps=10, cell_factors=factors, graph_blocks=blocks)
        table = np.array(res["ms_table"])
        assert table.shape == (3, 2) and np.all(table > 0) and res["before_ms_per_step"] > 0
        assert res["cell_factor"] in factors and res["graph_block"] in blocks
        assert res["ms_per_step"] == min(table.min(), min(res["contact_ms"]))
        assert len(res["contact_ms"]) == len(psb200.CONTACT_KERNELS) and min(res["contact_ms"]) > 0
        assert res["contact_kernel"] == psb200.CONTACT_KERNELS[int(np.argmin(res["contact_ms"]))]
        assert sim.contact_kernel() == res["contact_kernel"]
        assert np.array_equal(sim.get_state(), before)
        grids = [sim.grid(k) for k in range(len(batch))]
        sim.step(30)
        got = sim.get_state()
    off = 0
    for sc, g in zip(batch, grids):
        r_max = float(np.float32(sc.r_max()))
        assert g.interval == pytest.approx(res["cell_factor"] * 2.0 * r_max, rel=1e-12)
        want = O.run(sc.copy(interval=g.interval), 30, "f32")
        assert np.array_equal(got[off:off + sc.n].astype(np.float32), want)
        off += sc.n


@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_every_contact_kernel_gives_the_same_states(need_gpu, precision):
    """The five contact kernels (per-lane walk with 128, 256 and 512 threads
    per CTA, warp and adaptive walks with 256) on a batch of a dense pile, a sparse
    lattice and a triangle container: states bit-identical to each other
    and to the oracle after 40 steps."""
    batch = [scenes.pile(1500, seed=41, k_spring=1.0), scenes.lattice_c1(side=10), scenes.box_mesh_scene()]
    states = []
    for walk, block in psb200.CONTACT_KERNELS:
        with psb200.Simulation(batch, precision) as sim:
            sim.set_contact_kernel(walk, block)
            assert sim.contact_kernel() == (walk, block)
            sim.set_state()
            sim.step(40)
            states.append(sim.get_state())
    for st in states[1:]:
        assert np.array_equal(st, states[0])
    off = 0
    for sc in batch:
        want = O.run(sc, 40, precision)
        got = states[0][off:off + sc.n]
        assert np.array_equal(got.astype(np.float32) if precision == "f32" else got, want)
        off += sc.n


def test_autotune_rejects_bad_arguments(need_gpu):
    sc = scenes.pile(100, seed=3)
    with psb200.Simulation(sc, "f32") as sim:
        with pytest.raises(psb200.PSError, match="ps_set_state first"):
            sim.autotune(trial_steps=2)
        sim.set_state()
        with pytest.raises(psb200.PSError, match=">= 1"):
            sim.autotune(trial_steps=2, cell_factors=(0.5,))
        with pytest.raises(psb200.PSError, match="bad argument"):
            sim.autotune(trial_steps=0)
        with pytest.raises(psb200.PSError, match="walk/block"):
            sim.set_contact_kernel(psb200.WALK_WARP, 128)
        with pytest.raises(psb200.PSError, match="walk/block"):
            sim.set_contact_kernel(psb200.WALK_LANE, 1024)
        with pytest.raises(psb200.PSError, match="walk/block"):
            sim.set_contact_kernel(psb200.WALK_ADAPTIVE, 512)
