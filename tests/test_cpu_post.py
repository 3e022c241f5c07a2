"""The CLI's steps after the path, in the library's host code, against the
reference's own implementations built from its sources
(oracle/_ref/libref_cpu.so): ParticleModel::resolveOverlaps (positions bit
for bit, along each axis), its closing overlap check (against a direct
O(N^2) evaluation) and ObjData::write (byte-identical file)."""
import hashlib
import os

import numpy as np
import pytest

import psb200
from psb200 import scenes
from oracle import ps_oracle as O

needs_ref = pytest.mark.skipif(not os.path.exists(O.REF_CPU_SO),
                               reason="oracle/_ref/libref_cpu.so was not built (reference sources absent)")


def cloud(n, seed, edge=0.1):
    rng = np.random.default_rng(seed)
    pos = rng.uniform(0.0, edge, size=(n, 3))
    r = rng.uniform(0.004, 0.006, size=n)
    return scenes._state(pos, np.zeros((n, 3)), r, 1000.0)


def brute_stats(st):
    d = st[:, None, :3] - st[None, :, :3]
    dist = np.sqrt((d[..., 0] * d[..., 0] + d[..., 1] * d[..., 1]) + d[..., 2] * d[..., 2])
    cd = st[:, 6][:, None] + st[:, 6][None, :] - dist
    upper = np.triu(np.ones(cd.shape, dtype=bool), 1)
    hit = (cd > 0.0) & upper
    return int(hit.any(axis=1).sum()), float(cd[hit].max()) if hit.any() else 0.0


@needs_ref
@pytest.mark.parametrize("axis", [0, 1, 2])
@pytest.mark.parametrize("make", [lambda: scenes.pile(800, seed=4).state, lambda: cloud(1000, 1),
                                  lambda: cloud(600, 2, edge=0.05)])
def test_resolve_overlaps_equals_reference(make, axis):
    st = make()
    want = O.ref_resolve_overlaps(st, axis)
    got, n_collided, max_overlap = psb200.resolve_overlaps(st, axis)
    assert np.array_equal(got, want)
    assert (n_collided, max_overlap) == brute_stats(want)


def test_overlap_stats_against_direct_evaluation():
    st = cloud(700, 3)
    assert psb200.overlap_stats(st) == brute_stats(st)
    # particles with a non-finite coordinate overlap nothing
    st[5, 0] = np.nan
    st[9, 2] = np.inf
    keep = np.ones(st.shape[0], dtype=bool)
    keep[[5, 9]] = False
    n_c, m = psb200.overlap_stats(st)
    n_ref, m_ref = brute_stats(st[keep])
    assert m == m_ref
    assert n_c == n_ref or n_c == brute_stats(np.nan_to_num(st, nan=1e9, posinf=1e9))[0]


def test_resolve_overlaps_rejects_bad_input():
    st = cloud(10, 4)
    with pytest.raises(psb200.PSError, match="axis"):
        psb200.resolve_overlaps(st, 3)
    st[2, 1] = np.nan
    with pytest.raises(psb200.PSError, match="non-finite"):
        psb200.resolve_overlaps(st, 2)
    empty, n_c, m = psb200.resolve_overlaps(np.zeros((0, 8)), 2)
    assert empty.shape == (0, 8) and n_c == 0 and m == 0.0


def _sha(path):
    h = hashlib.sha256()
    with open(path, "rb") as f:
        for chunk in iter(lambda: f.read(1 << 22), b""):
            h.update(chunk)
    return h.hexdigest()


@needs_ref
def test_obj_spheres_byte_identical_to_reference(tmp_path):
    # two particles: the reference sizes the sphere mesh for about a million
    # vertices in total, so any count gives files of a few hundred MB
    st = cloud(2, 5)
    st[1, 6] = 0.0123
    ours = tmp_path / "sub" / "ours.obj"  # the writer creates missing directories, as the reference does
    ref = tmp_path / "ref.obj"
    psb200.write_obj_spheres(str(ours), st)
    O.ref_write_obj(str(ref), st)
    try:
        assert os.path.getsize(ours) == os.path.getsize(ref)
        assert _sha(ours) == _sha(ref)
    finally:
        for p in (ours, ref):
            if p.exists():
                p.unlink()
