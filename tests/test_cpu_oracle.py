"""The oracle, pinned (CPU only).

1. Against the reference's own CPU simulator: tests/golden holds states the
   unmodified reference sources produced (tests/golden/make_golden.py); the
   oracle's CPU-semantics mode must reproduce them bit for bit.
2. Against the reference's own CUDA simulator: tests/golden/ref_cuda_*.npz
   (make_golden_cuda.py, run on a B200) holds its bucket arrays and states;
   the oracle's CUDA scheme must give the same cell counts and offsets, the
   same per-cell member sets, and states within FP64 rounding (the reference
   sums contact kicks with atomics in arbitrary order).
3. Known-answer tests written from the reference formulas by hand.
"""
import glob
import math
import os

import numpy as np
import pytest

from oracle import ps_oracle as O
from psb200 import scenes
from conftest import GOLDEN


def golden(name):
    path = os.path.join(GOLDEN, name)
    if not os.path.exists(path):
        pytest.fail(f"missing golden fixture {path}")
    return np.load(path)


def box_scene(init, box, e, k, es, dt):
    return scenes.Scene(init.copy(), tuple(box[0]), tuple(box[1]), (0, 0, -9.8), tuple(e), float(k), float(es),
                        float(dt))


# ---- 1. CPU simulator, bit for bit -----------------------------------------
def test_oracle_cpu_semantics_pile_bitexact():
    g = golden("ref_cpu_box.npz")
    sc = box_scene(g["pile_init"], g["pile_box"], g["pile_e"], g["pile_k"], g["pile_es"], g["pile_dt"])
    for i, s in enumerate(g["steps"]):
        out = O.run(sc, int(s), "f64", cpu_semantics=True)
        assert np.array_equal(out, g["pile_out"][i]), f"step {s}"


def test_oracle_cpu_semantics_lattice_bitexact():
    g = golden("ref_cpu_box.npz")
    sc = scenes.lattice_c1(side=6)
    assert np.array_equal(sc.state, g["lat_init"])
    for i, s in enumerate(g["steps"]):
        assert np.array_equal(O.run(sc, int(s), "f64", cpu_semantics=True), g["lat_out"][i])


def test_oracle_cpu_semantics_mesh_bitexact():
    g = golden("ref_cpu_mesh.npz")
    sc = scenes.Scene(g["init"].copy(), (-0.1, -0.1, 0), (0.1, 0.1, 0.25), (0, 0, -9.8), tuple(g["e_wall"]),
                      float(g["k"]), float(g["es"]), float(g["dt"]), tri=g["tri"])
    for i, s in enumerate(g["steps"]):
        assert np.array_equal(O.run(sc, int(s), "f64", cpu_semantics=True), g["out"][i]), f"step {s}"


# ---- 2. CUDA simulator --------------------------------------------------------
CUDA_FIXTURES = sorted(glob.glob(os.path.join(GOLDEN, "ref_cuda_*.npz")))


def fixture_scene(g):
    """Scene of a reference CUDA fixture: a box, or a triangle container read
    from OBJ (grid domain = the mesh AABB, the reference's edge pick)."""
    sc = box_scene(g["init"], g["box"], g["e_wall"], g["k"], g["es"], g["dt"])
    if "tri" in g.files:
        sc = sc.copy(tri=g["tri"], edge_quirk=1, widen_domain=0)
    return sc


def test_reference_cuda_fixtures_cover_both_containers():
    names = {os.path.basename(p) for p in CUDA_FIXTURES}
    assert {"ref_cuda_lattice.npz", "ref_cuda_pile.npz", "ref_cuda_mesh_box.npz", "ref_cuda_mesh_funnel.npz",
            "ref_cuda_mesh_fan.npz"} <= names


def test_reference_cuda_fan_fixture_has_a_sphere_on_every_fan_triangle():
    """In the fan fixture the reference's container moved the centre sphere
    by one 1e-5 correction per fan triangle: 300 hits in one step."""
    g = np.load(os.path.join(GOLDEN, "ref_cuda_mesh_fan.npz"))
    sc = fixture_scene(g)
    lifted = O.pre_grid_state(sc, sc.state, "f64")[0, 2] - O.pre_grid_state(
        sc.copy(tri=None, box_min=(-1, -1, -1), box_max=(1, 1, 2)), sc.state, "f64")[0, 2]
    assert round(lifted / 1e-5) == 300


@pytest.mark.parametrize("path", CUDA_FIXTURES, ids=[os.path.basename(p) for p in CUDA_FIXTURES])
def test_oracle_cuda_semantics_vs_reference_cuda(path):
    g = np.load(path)
    sc = fixture_scene(g)
    og = O.grid_for(sc)
    assert tuple(og.nb) == tuple(g["nb"]) and og.interval == float(g["interval"])
    for i, s in enumerate(g["steps"]):
        s = int(s)
        state = O.run(sc, s - 1, "f64") if s > 1 else sc.state.copy()
        pre = O.pre_grid_state(sc, state, "f64")
        cell = O.cell_ids(pre, og)
        counts, offsets, order = O.count_scan_order(cell, og.n_cells)
        assert np.array_equal(counts, g["counts"][i])
        assert np.array_equal(offsets[:-1], g["offsets"][i])
        rb = g["bucket"][i]
        for c in np.nonzero(counts)[0]:
            a, b = offsets[c], offsets[c] + counts[c]
            assert np.array_equal(np.sort(rb[a:b]), order[a:b].astype(np.int64))
        out = O.run(sc, s, "f64")
        scale = np.abs(g["out"][i]).max(axis=0) + 1e-300
        assert (np.abs(out - g["out"][i]) / scale).max() < 1e-12


# ---- 3. known-answer tests ------------------------------------------------------
def _two_spheres(d=0.019, v1=(0.1, 0, 0), v2=(-0.2, 0.05, 0), r=0.01, m1=2.0, m2=3.0):
    st = np.array([[0.5, 0.5, 0.5, *v1, r, m1], [0.5 + d, 0.5, 0.5, *v2, r, m2]], dtype=np.float64)
    return scenes.Scene(st, (0, 0, 0), (1, 1, 1), (0, 0, 0), (1,) * 6, 7.0, 0.6, 0.0)


def test_kat_two_sphere_contact():
    """dv_i = [k*ov/(|d| m_i) - 2 m_j e ((v_i-v_j).d)/((m_i+m_j)|d|^2)] d
    (ParticleModel_kernels.cu:174-199), with dt = 0 so only contacts act."""
    sc = _two_spheres()
    out = O.run(sc, 1, "f64")
    x1, x2 = sc.state[0, :3], sc.state[1, :3]
    v1, v2 = sc.state[0, 3:6], sc.state[1, 3:6]
    for (xi, xj, vi, vj, mi, mj, o) in ((x1, x2, v1, v2, 2.0, 3.0, out[0]), (x2, x1, v2, v1, 3.0, 2.0, out[1])):
        d = xi - xj
        dist = np.linalg.norm(d)
        ov = 0.02 - dist
        f = 7.0 * ov / (dist * mi) - 2 * mj * 0.6 * np.dot(vi - vj, d) / ((mi + mj) * dist ** 2)
        np.testing.assert_allclose(o[3:6], vi + f * d, rtol=1e-14, atol=1e-17)
    # apart: nothing happens
    far = O.run(_two_spheres(d=0.0201), 1, "f64")
    np.testing.assert_array_equal(far[:, 3:6], _two_spheres(d=0.0201).state[:, 3:6])


def test_kat_damping_acts_when_separating():
    """The reference applies the restitution term whatever the approach sign."""
    sc = _two_spheres(v1=(-1.0, 0, 0), v2=(1.0, 0, 0))
    sc_k0 = sc.copy(k_spring=0.0)
    out = O.run(sc_k0, 1, "f64")
    assert out[0, 3] > -1.0  # separating pair is slowed


def test_kat_walls_order_and_sign():
    """Six clamps in the order xmin, ymin, zmin, xmax, ymax, zmax on the
    pre-clamp extents; v <- -v e regardless of its sign
    (BoxContainer_kernels.cu:17-52)."""
    e = (0.1, 0.2, 0.3, 0.4, 0.5, 0.6)  # zMin zMax xMin xMax yMin yMax
    st = np.array([
        [-0.5, 0.5, 0.5, 2.0, 0, 0, 0.1, 1],     # below xmin, moving away from the wall
        [0.5, 1.2, 0.5, 0, -3.0, 0, 0.1, 1],     # above ymax
        [0.5, 0.5, 0.05, 0, 0, -1.0, 0.1, 1],    # touching zmin
        [0.5, 0.5, 0.5, 1.0, 1.0, 1.0, 0.6, 1],  # larger than the box: min and max both fire
    ])
    sc = scenes.Scene(st, (0, 0, 0), (1, 1, 1), (0, 0, 0), e, 0.0, 0.0, 0.0)
    out = st.copy()
    O.lib().or_walls_f64(O._p(out), 4, O._d3(sc.box_min), O._d3(sc.box_max), (O.C.c_double * 6)(*e))
    np.testing.assert_allclose(out[0, [0, 3]], [0.1, -2.0 * 0.3])
    np.testing.assert_allclose(out[1, [1, 4]], [0.9, 3.0 * 0.6])
    np.testing.assert_allclose(out[2, [2, 5]], [0.1, 1.0 * 0.1])
    # xmin then xmax: x = min + r, then x = max - r; v = -(-v*e_xmin)*e_xmax
    np.testing.assert_allclose(out[3, [0, 3]], [1 - 0.6, 1.0 * 0.3 * 0.4])


def test_kat_cell_ids_at_exact_boundaries():
    g = O.OrGrid()
    O.lib().or_grid_init(O._d3((0, 0, 0)), O._d3((1, 1, 1)), O.C.c_double(0.25), O.C.byref(g))
    assert tuple(g.nb) == (5, 5, 5) and g.n_cells == 125
    pts = np.zeros((6, 8))
    pts[:, :3] = [[0, 0, 0], [0.25, 0, 0], [0.2499999, 0.5, 0.75], [1.0, 1.0, 1.0], [-0.1, 2.0, np.nan],
                  [0.999, 0.0, 0.26]]
    cid = O.cell_ids(pts, g)
    assert list(cid) == [0, 25, 0 * 25 + 2 * 5 + 3, 4 * 25 + 4 * 5 + 4, 0 * 25 + 4 * 5 + 0, 3 * 25 + 0 + 1]


def test_kat_scan_and_order():
    a = np.array([3, 0, 0, 2, 1, 0], dtype=np.uint32)
    assert list(O.exclusive_scan(a)) == [0, 3, 3, 3, 5, 6]
    assert O.exclusive_scan(np.zeros(0, dtype=np.uint32)).shape == (0,)
    w = np.full(3, 0xFFFFFFFF, dtype=np.uint32)
    assert list(O.exclusive_scan(w)) == [0, 0xFFFFFFFF, 0xFFFFFFFE]
    cell = np.array([2, 0, 2, 1, 0, 2])
    counts, offs, order = O.count_scan_order(cell, 3)
    assert list(counts) == [2, 1, 3] and list(offs) == [0, 2, 3, 6]
    assert list(order) == [1, 4, 3, 0, 2, 5]


def test_kat_grid_intervals():
    assert O.lib().or_interval_cuda(O.C.c_double(0.01)) == 0.01 * 2.0 * 1.05
    assert O.lib().or_interval_cpu(O.C.c_double(0.01)) == 0.01 * 2.0 * float(np.float32(1.05))
    assert O.lib().or_interval_cuda(O.C.c_double(0.01)) != O.lib().or_interval_cpu(O.C.c_double(0.01))


def _one_triangle_scene(p, v=(0.0, 0.0, -1.0), quirk=1):
    tri = np.array([[0.0, 0.0, 0.0, 0.0, 1.0, 0.0, 1.0, 0.0, 0.0]])  # normal (v1-v0)x(v2-v0) = (0,0,-1)
    st = np.array([[*p, *v, 0.1, 1.0]])
    return scenes.Scene(st, (0, 0, 0), (1, 1, 1), (0, 0, 0), (0.5,) * 6, 0.0, 0.0, 0.0, tri=tri, edge_quirk=quirk)


def _mesh_once(sc, precision="f64"):
    out = sc.state.copy()
    t = np.ascontiguousarray(sc.tri)
    O.lib().or_mesh_f64(O._p(out), 1, O._p(t), 1, O.C.c_double(sc.e_wall[0]), O.C.c_int32(sc.edge_quirk),
                        O.C.c_int32(0))
    return out[0]


def test_kat_triangle_face_edge_vertex_and_miss():
    """Face: closest point is the projection; velocity = e*reflect(v, n);
    position += -(r - dot(-n, x - v0)) n with the outward normal (0,0,-1)
    (PolygonContainerCUDA_kernels.cu:220-294)."""
    face = _mesh_once(_one_triangle_scene((0.25, 0.25, -0.05)))
    np.testing.assert_allclose(face[3:6], [0.0, 0.0, 0.5 * 1.0], atol=1e-15)  # reflect (0,0,-1) about n -> (0,0,1)
    # dot(-n, x - v0) = -0.05: the centre sits on the +n side; the correction
    # -(r - (-0.05)) n moves it to the -n side at distance r from the plane
    np.testing.assert_allclose(face[:3], [0.25, 0.25, 0.1], atol=1e-15)
    # near vertex v0 at distance 0.0707 < r: the true nearest point is v0 (hit)
    vertex = _mesh_once(_one_triangle_scene((-0.05, -0.05, 0.0), quirk=0))
    assert vertex[3:6].tolist() != [0.0, 0.0, -1.0]
    miss = _mesh_once(_one_triangle_scene((-0.09, -0.09, 0.0), quirk=0))
    np.testing.assert_array_equal(miss[3:6], [0.0, 0.0, -1.0])  # |x - v0| = 0.127 > r


def test_kat_edge_quirk_differs_from_true_nearest():
    """The reference picks the edge point with the smallest dot(center,
    point) (PolygonContainerCUDA_kernels.cu:130-150), not the nearest one:
    at (-0.05, -0.05, 0) it chooses the midpoint (0.5, 0.5, 0) of edge BC
    (dot = -0.05 < 0) over the vertex v0 (dot = 0) and misses the triangle."""
    p = (-0.05, -0.05, 0.0)
    q = _mesh_once(_one_triangle_scene(p, quirk=1))
    e = _mesh_once(_one_triangle_scene(p, quirk=0))
    np.testing.assert_array_equal(q[3:6], [0.0, 0.0, -1.0])  # quirk: no hit
    assert not np.array_equal(q, e)


def test_funnel_normals_point_outward():
    tri = scenes.funnel_triangles()
    assert 19000 <= tri.shape[0] <= 21000
    t = tri.reshape(-1, 3, 3)
    n = np.cross(t[:, 1] - t[:, 0], t[:, 2] - t[:, 0])
    c = t.mean(axis=1)
    radial = np.stack([c[:, 0], c[:, 1], np.zeros(len(c))], 1)
    wall = np.linalg.norm(radial, axis=1) > 0.079
    bottom = ~wall
    assert np.all(np.einsum("ij,ij->i", n[wall], radial[wall]) > 0)
    assert np.all(n[bottom, 2] < 0)


# Stated FP32 trajectory tolerance over 1,000 steps against the FP64 scheme,
# per particle: position within POS_TOL * (largest box edge), velocity within
# VEL_TOL * (largest speed component).  Contact-rich pile: measured 7e-5 and
# 1e-2 (chaotic growth of rounding differences); contact-free lattice:
# measured 4e-7 and 6e-6.
FP32_TOL = {"pile": (2e-4, 3e-2), "lattice": (1e-6, 1e-4)}


@pytest.mark.parametrize("name", ["pile", "lattice"])
def test_fp32_run_tracks_fp64_run(name):
    sc = scenes.pile(512, seed=17, k_spring=1.0) if name == "pile" else scenes.lattice_c1(side=8)
    a = O.run(sc, 1000, "f32").astype(np.float64)
    b = O.run(sc, 1000, "f64")
    pos_tol, vel_tol = FP32_TOL[name]
    L = max(sc.box_max)
    vs = np.abs(b[:, 3:6]).max()
    assert np.abs(a[:, :3] - b[:, :3]).max() < pos_tol * L
    assert np.abs(a[:, 3:6] - b[:, 3:6]).max() < vel_tol * vs


# ---- 4. the forward-mode gradient oracle against central differences ---------
def test_dual_oracle_vs_central_fd_on_contact_pile():
    """oracle/ps_oracle_dual.c (forward-mode FP64, the reference gradient of
    the GPU adjoint) against FP64 central differences of the oracle's own
    forward run, on the 1,024-sphere contact pile over 400 steps: each
    non-zero parameter derivative of the settling loss within 1e-3
    relative; the contact spring, sphere restitution and floor restitution
    derivatives are non-zero."""
    import psb200

    sc = scenes.pile(1024, seed=3, k_spring=1.0)
    steps = 400
    st, tang = O.run_dual(sc, steps, np.eye(8), np.zeros((8, sc.n, 6)))
    _, gl = psb200.height_loss(st)
    fm = np.array([np.sum(gl * tang[d]) for d in range(8)])
    theta = np.array([sc.k_spring, sc.e_sphere, *sc.e_wall])
    for p in range(8):
        h = 1e-6 * max(1.0, abs(theta[p]))
        tp, tm = theta.copy(), theta.copy()
        tp[p] += h
        tm[p] -= h
        lp = psb200.height_loss(O.run(sc.copy(k_spring=tp[0], e_sphere=tp[1], e_wall=tuple(tp[2:])), steps))[0]
        lm = psb200.height_loss(O.run(sc.copy(k_spring=tm[0], e_sphere=tm[1], e_wall=tuple(tm[2:])), steps))[0]
        fd = (lp - lm) / (2 * h)
        if p in (0, 1, 2):
            assert fd != 0.0
        if fd == 0.0:
            assert fm[p] == 0.0
        else:
            assert abs(fm[p] - fd) <= 1e-3 * abs(fd), (p, fm[p], fd)
