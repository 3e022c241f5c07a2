"""The seeded workload generators (CPU): shapes, distributions, no initial overlaps."""
import numpy as np
import pytest
from scipy.spatial import cKDTree

from psb200 import scenes


def assert_no_overlap(st):
    tree = cKDTree(st[:, :3])
    pairs = tree.query_pairs(2.0 * st[:, 6].max(), output_type="ndarray")
    if len(pairs):
        d = np.linalg.norm(st[pairs[:, 0], :3] - st[pairs[:, 1], :3], axis=1)
        assert np.all(d >= st[pairs[:, 0], 6] + st[pairs[:, 1], 6])


def test_c2_scene_1m():
    sc = scenes.c2_scene()
    assert sc.n == 1 << 20
    r = sc.state[:, 6]
    assert r.min() >= 0.001 and r.max() <= 0.004 and abs(np.median(r) - 0.002) < 2e-5
    assert np.all(sc.state[:, :3] - r[:, None] >= 0) and np.all(sc.state[:, 0:2] + r[:, None] <= 1)
    assert np.all(sc.state[:, 2] + r <= 4)
    assert abs(sc.state[:, 3:6].std() - 0.05) < 1e-3
    assert sc.interval == 0.008 and sc.k_spring == 5e4 and sc.dt == 5e-6
    assert_no_overlap(sc.state)


def test_lattice_and_pile():
    c1 = scenes.lattice_c1()
    assert c1.n == 4096 and np.all(c1.state[:, 2] > 0.5)
    assert_no_overlap(c1.state)
    p = scenes.pile(1000, seed=2)
    assert p.n == 1000


def test_c3_and_c4():
    c3 = scenes.c3_scene()
    assert c3.n == 262144 and c3.tri.shape[1] == 9 and c3.widen_domain == 1
    assert np.all(c3.state[:, 2] > 1.0)
    lo, hi = c3.domain()
    assert hi[2] > 1.0  # widened over the spawn lattice
    c4 = scenes.c4_scene()
    assert c4.n == 65536 and np.all(c4.state[:, :3] < 0.5)
    assert_no_overlap(c4.state)


def test_c5_scenes():
    b = scenes.c5_scenes(16, seed=3)
    assert len(b) == 16
    for sc in b:
        assert 1 <= sc.n <= 65536 and 0.2 <= sc.box_max[0] <= 1.0
        assert 5e3 <= sc.k_spring <= 5e4 and 0.3 <= sc.e_sphere <= 0.9
        assert_no_overlap(sc.state)
