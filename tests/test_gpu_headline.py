"""Parity at the benchmark's own size: the 1,048,576-sphere box scene as
benchmarked (spring 5e4, log-normal radii, 126 x 126 x 501 cells) stepped on
the GPU and by the oracle (oracle/ps_oracle_impl.inc), compared bit for bit
in FP32 and FP64 after 10 steps, on both neighbour walks of the contact
kernel, together with the grid of the last step (cell counts, offsets and
the canonical sorted order).  Within these 10 steps the scheme's kick
(k * overlap / m, not scaled by dt) already blows a few contacts apart, so
the comparison covers fast, far-travelling spheres as well."""
import numpy as np
import pytest

import psb200
from psb200 import scenes
from oracle import ps_oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def c2():
    return scenes.c2_scene()


@pytest.mark.parametrize("precision", ["f32", "f64"])
@pytest.mark.parametrize("kernel", [psb200.CONTACT_KERNELS[1], psb200.CONTACT_KERNELS[3], psb200.CONTACT_KERNELS[4]],
                         ids=["lane256", "warp256", "adaptive256"])
def test_1m_sphere_scene_bitexact(need_gpu, c2, precision, kernel):
    steps = 10
    with psb200.Simulation(c2, precision) as sim:
        sim.set_contact_kernel(*kernel)
        sim.set_state()
        sim.step(steps)
        got = sim.get_state()
        counts, offsets, order = sim.buckets()
    want = O.run(c2, steps, precision)
    got = got.astype(np.float32) if precision == "f32" else got
    assert np.array_equal(got, want), f"{np.sum(np.any(got != want, axis=1))} of {c2.n} spheres differ"
    # the grid of the last step, built from the state after step 9
    prev = O.run(c2, steps - 1, precision)
    pre = O.pre_grid_state(c2, prev, precision)
    og = O.grid_for(c2)
    wc, wo, word = O.count_scan_order(O.cell_ids(pre, og), og.n_cells)
    assert np.array_equal(counts, wc)
    assert np.array_equal(offsets, wo[:-1])
    assert np.array_equal(order, word)
    speed = np.linalg.norm(want[:, 3:6].astype(np.float64), axis=1)
    assert np.isfinite(speed).all() and speed.max() > 10.0  # contacts have kicked spheres hard
