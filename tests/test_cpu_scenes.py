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


def test_c4_and_c5_stable_variants():
    """The soft-spring variants differ from the specified scenes only in
    the spring, and keep k dt / m below 1 for every sphere."""
    c4 = scenes.c4_scene(k_spring=5.0)
    assert np.array_equal(c4.state, scenes.c4_scene().state)
    assert c4.k_spring * c4.dt / c4.state[:, 7].min() < 0.25
    big = scenes.c4_scene(1 << 20, edge=0.95, k_spring=5.0)
    assert big.n == 1 << 20 and np.all(big.state[:, :3] < 0.95)
    with pytest.raises(ValueError):
        scenes.c4_scene(1 << 20)  # does not fit the 0.5 box
    spec = scenes.c5_scenes(8, seed=3)
    soft = scenes.c5_scenes(8, seed=3, k_range=(0.25, 2.5))
    for a, b in zip(spec, soft):
        assert np.array_equal(a.state, b.state) and a.e_wall == b.e_wall and a.e_sphere == b.e_sphere
        assert 0.25 <= b.k_spring <= 2.5 and b.k_spring * b.dt / b.state[:, 7].min() <= 0.38


def test_slab_packing_fraction_and_height_histogram():
    r = 0.01
    box_lo, box_hi = (0.0, 0.0, 0.0), (0.1, 0.1, 1.0)
    one = np.array([[0.05, 0.05, 0.5, 0, 0, 0, r, 1.0]])
    ball = 4.0 / 3.0 * np.pi * r ** 3
    # whole sphere inside the slab
    assert scenes.slab_packing_fraction(one, box_lo, box_hi, 0.4, 0.6) == pytest.approx(ball / (0.01 * 0.2))
    # the slab cuts the sphere through its centre: half the volume
    assert scenes.slab_packing_fraction(one, box_lo, box_hi, 0.5, 0.7) == pytest.approx(0.5 * ball / (0.01 * 0.2))
    # a cap of height h = r/2 has volume pi h^2 (3r - h) / 3
    h = r / 2
    cap = np.pi * h * h * (3 * r - h) / 3
    z_lo = 0.5 + r - h
    assert scenes.slab_packing_fraction(one, box_lo, box_hi, z_lo, 0.9) == pytest.approx(cap / (0.01 * (0.9 - z_lo)))
    assert scenes.slab_packing_fraction(one, box_lo, box_hi, 0.6, 0.9) == 0.0
    hist = scenes.height_histogram(np.vstack([one, one]), 1.0, bins=4)
    assert np.array_equal(hist, [0.0, 0.0, 1.0, 0.0])


def test_settle_pile():
    sc = scenes.settle_pile()
    assert sc.n == 4096 and sc.k_spring * sc.dt / sc.state[:, 7].min() < 0.1
    assert_no_overlap(sc.state)
    assert np.all(sc.state[:, 3:6] == 0.0)
