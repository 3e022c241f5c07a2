"""The bounds-checked build (lib_debug/, compiled with -DPS_DEBUG_BOUNDS).

In that build every device index into the bucket arrays (count, offset,
the scatter's scratch order), the sorted state, the triangle bins and the
neighbour lists is checked before the access; an index out of range is
skipped and sets PS_DEVERR_BOUNDS, which the next syncing call returns as
PS_ERR_DEVICE.  These tests run the scenes of the parity suite through that
build in a child process (so the product library stays the one loaded
here): every run must finish without a device error and give the oracle's
states bit for bit, which shows that no checked index left its array.
"""
import os
import subprocess
import sys

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

CHILD = r"""
import sys
import numpy as np
import psb200
from psb200 import scenes
from oracle import ps_oracle as O

psb200.LIB_PATH = psb200.DEBUG_LIB_PATH
assert psb200.bounds_checked(), "lib_debug is not the bounds-checked build"


def run(sc, steps, prec, calls=None, skin=None, walk=None):
    with psb200.Simulation(sc, prec) as sim:
        sim.set_state()
        if walk is not None:
            sim.set_contact_kernel(*walk)
        if skin is not None:
            sim.set_neighbor_lists(skin, 48)
        for c in (calls or [steps]):
            sim.step(c)
        sim.sync()
        return sim.get_state()


def check(name, got, want):
    assert got.shape == want.shape and np.array_equal(got, want), \
        f"{name}: {np.sum(np.any(got != want, axis=1))} particles differ"
    print("ok", name, flush=True)


def cast(a, prec):
    return a.astype(np.float32) if prec == "f32" else a


case = sys.argv[1]
if case == "grid":
    for prec in ("f32", "f64"):
        sc = scenes.pile(1024, seed=3, k_spring=1.0)
        check(f"pile {prec}", cast(run(sc, 120, prec, calls=[1, 33, 86]), prec), O.run(sc, 120, prec))
        for walk in psb200.CONTACT_KERNELS:
            check(f"pile {prec} contact kernel {walk}", cast(run(sc, 30, prec, walk=walk), prec), O.run(sc, 30, prec))
    sc = scenes.lattice_c1()
    check("lattice f64", run(sc, 200, "f64"), O.run(sc, 200, "f64"))
    sc = scenes.c2_scene()
    check("c2 1M f32", cast(run(sc, 4, "f32"), "f32"), O.run(sc, 4, "f32"))
elif case == "mesh":
    for prec in ("f32", "f64"):
        sc = scenes.box_mesh_scene()
        check(f"box mesh {prec}", cast(run(sc, 60, prec), prec), O.run(sc, 60, prec))
        sc = scenes.funnel_wall_scene(1500, seed=9)
        check(f"funnel {prec}", cast(run(sc, 40, prec), prec), O.run(sc, 40, prec))
elif case == "batch":
    one = scenes.pile(1, seed=4)
    empty = one.copy(state=np.zeros((0, 8)))
    batch = scenes.c5_scenes(5, seed=9, n_lo=200, n_hi=3000) + [empty, one, empty]
    with psb200.Simulation(batch, "f32") as sim:
        sim.set_state()
        sim.step(40)
        joint = sim.get_state()
    off = 0
    for k, sc in enumerate(batch):
        if sc.n == 0:
            continue
        check(f"batch scene {k}", joint[off:off + sc.n].astype(np.float32), O.run(sc, 40, "f32"))
        off += sc.n
elif case == "lists":
    for prec in ("f32", "f64"):
        sc = scenes.pile(800, seed=12, k_spring=1.0)
        check(f"lists {prec}", cast(run(sc, 120, prec, calls=[90, 30], skin=0.25), prec), O.run(sc, 120, prec))
        check(f"lists thin skin {prec}", cast(run(sc, 120, prec, calls=[120], skin=0.02), prec), O.run(sc, 120, prec))
    sc = scenes.funnel_wall_scene(1500, seed=9)
    check("lists funnel f32", cast(run(sc, 40, "f32", skin=0.3), "f32"), O.run(sc, 40, "f32"))
elif case == "adjoint":
    sc = scenes.pile(300, seed=21, k_spring=1.0)
    steps = 50
    with psb200.Simulation(sc, "f64") as sim:
        sim.set_state()
        sim.forward_checkpointed(steps, 7)
        final = sim.get_state()
        _, g = psb200.height_loss(final)
        grads, g0 = sim.backward(g)
    dp = np.eye(8)
    st, tang = O.run_dual(sc, steps, dp, np.zeros((8, sc.n, 6)))
    check("adjoint forward", final, st)
    _, gl = psb200.height_loss(st)
    fm = np.array([np.sum(gl * tang[d]) for d in range(8)])
    np.testing.assert_allclose(grads[0], fm, rtol=1e-8, atol=1e-12 * np.abs(fm).max())
    print("ok adjoint gradients", flush=True)
print("DONE", flush=True)
"""


def child_env():
    env = dict(os.environ)
    paths = [ROOT, os.path.join(ROOT, "particle-stabilizer_b200", "python")]
    env["PYTHONPATH"] = os.pathsep.join(paths + [env.get("PYTHONPATH", "")])
    return env


@pytest.mark.parametrize("case", ["grid", "mesh", "batch", "lists", "adjoint"])
def test_bounds_checked_build_runs_clean_and_bitexact(need_gpu, case):
    import psb200

    if not os.path.exists(psb200.DEBUG_LIB_PATH):
        pytest.fail(f"{psb200.DEBUG_LIB_PATH} is missing: build it with `make -C particle-stabilizer_b200 debug`")
    r = subprocess.run([sys.executable, "-c", CHILD, case], cwd=ROOT, env=child_env(), capture_output=True,
                       text=True, timeout=900)
    assert r.returncode == 0 and r.stdout.rstrip().endswith("DONE"), r.stdout[-3000:] + r.stderr[-3000:]
