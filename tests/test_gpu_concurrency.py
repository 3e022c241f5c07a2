"""Several simulations at once in one process.

Each ps_sim owns its stream, buffers, graphs and device error word, and
ctypes releases the GIL for the duration of every library call, so
simulations driven from different host threads run their calls
concurrently.  Their results must equal the same simulations run one after
another, bit for bit, and error messages stay with the thread that caused
them (ps_last_error is per thread)."""
import threading

import numpy as np
import pytest

import psb200
from psb200 import scenes

pytestmark = pytest.mark.gpu

CASES = [
    (lambda: scenes.pile(3000, seed=1, k_spring=1.0), "f32", (1, 50, 149)),
    (lambda: scenes.pile(2000, seed=2, k_spring=1.0), "f64", (200,)),
    (lambda: scenes.funnel_wall_scene(1500, seed=9), "f32", (7, 33)),
    (lambda: scenes.c5_scenes(8, seed=4, n_lo=500, n_hi=4000, k_range=(0.25, 2.5)), "f32", (60, 40)),
]


def run(make, prec, calls, rounds=3):
    out = []
    with psb200.Simulation(make(), prec) as sim:
        for _ in range(rounds):
            sim.set_state()
            for c in calls:
                sim.step(c)
            out.append(sim.get_state())
    return out


def test_simulations_on_several_host_threads_equal_sequential_runs(need_gpu):
    want = [run(*c) for c in CASES]
    got = [None] * len(CASES)
    errors = []

    def worker(k):
        try:
            got[k] = run(*CASES[k])
        except Exception as e:  # reported below, on the main thread
            errors.append((k, repr(e)))

    threads = [threading.Thread(target=worker, args=(k,)) for k in range(len(CASES))]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=600)
    assert not errors, errors
    for k in range(len(CASES)):
        assert len(got[k]) == len(want[k])
        for a, b in zip(got[k], want[k]):
            assert np.array_equal(a, b), f"case {k} differs from its sequential run"


def test_errors_stay_with_their_thread(need_gpu):
    """A failing call on one thread leaves the other thread's last error
    untouched."""
    msgs = {}
    barrier = threading.Barrier(2)

    def bad():
        with psb200.Simulation(scenes.pile(100, seed=3), "f32") as sim:
            sim.set_state()
            barrier.wait(timeout=60)
            with pytest.raises(psb200.PSError):
                sim.set_state(np.zeros((5, 8)))  # wrong particle count
            msgs["bad"] = psb200.lib().ps_last_error().decode()
            barrier.wait(timeout=60)

    def good():
        with psb200.Simulation(scenes.pile(100, seed=4), "f32") as sim:
            sim.set_state()
            barrier.wait(timeout=60)
            sim.step(10)
            sim.sync()
            barrier.wait(timeout=60)
            msgs["good"] = psb200.lib().ps_last_error().decode()

    ts = [threading.Thread(target=bad), threading.Thread(target=good)]
    for t in ts:
        t.start()
    for t in ts:
        t.join(timeout=300)
    assert "ps_set_state" in msgs["bad"]
    assert msgs["good"] == ""
