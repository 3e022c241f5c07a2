"""The new path against the reference's own CUDA simulator, built from its
unmodified sources for sm_100a (oracle/_ref/libref_cuda.so) and driven per
step by the harness in oracle/ref_driver_cuda.cu.

The reference orders particles inside a cell by atomicAdd and sums
velocity kicks with FP64 atomics, so its bucket lists are compared as
per-cell sets and its trajectories within a tolerance; cell counts and scan
offsets are deterministic and compared exactly (FP64 runs)."""
import os

import numpy as np
import pytest

import psb200
from psb200 import scenes
from oracle import ps_oracle as O

pytestmark = pytest.mark.gpu

needs_ref = pytest.mark.skipif(not os.path.exists(O.REF_CUDA_SO),
                               reason="oracle/_ref/libref_cuda.so was not built (reference sources absent)")


def ref_buckets(r, h, n, n_cells):
    import ctypes as C
    counts = np.empty(n_cells, dtype=np.uint32)
    offs = np.empty(n_cells, dtype=np.uint32)
    bucket = np.empty(n, dtype=np.int64)
    r.lib.refc_get_buckets(h, C.c_void_p(counts.ctypes.data), C.c_void_p(offs.ctypes.data),
                           C.c_void_p(bucket.ctypes.data))
    return counts, offs, bucket


@needs_ref
@pytest.mark.parametrize("make", [lambda: scenes.lattice_c1(), lambda: scenes.pile(2000, seed=21, k_spring=1.0)])
@pytest.mark.parametrize("steps", [1, 6])
def test_counts_offsets_sets_equal_reference(need_gpu, make, steps):
    sc = make()
    r = O.ref_cuda()
    h = r.create(sc)
    try:
        r.step(h, steps)
        ref_state = r.state(h, sc.n)
        og = O.grid_for(sc)
        rc, ro, rb = ref_buckets(r, h, sc.n, og.n_cells)
    finally:
        r.destroy(h)
    with psb200.Simulation(sc, "f64") as sim:
        sim.set_state()
        sim.step(steps)
        counts, offsets, order = sim.buckets()
        st = sim.get_state()
    assert np.array_equal(counts, rc)
    assert np.array_equal(offsets, ro)
    # same members per cell; ours in ascending index
    nz = np.nonzero(rc)[0]
    for c in nz[:: max(1, len(nz) // 2000)]:
        a, b = ro[c], ro[c] + rc[c]
        assert np.array_equal(np.sort(rb[a:b]), order[a:b].astype(np.int64))
    # trajectories: the reference's atomic summation order differs from ours
    scale = np.abs(ref_state).max(axis=0) + 1e-300
    rel = (np.abs(st - ref_state) / scale).max()
    assert rel < 1e-12, rel
