"""Benchmark of the DEM step: particle-steps/s at 1M spheres.

Workload: the 1,048,576-sphere box scene (log-normal radii, median 0.002,
sigma 0.25, clipped to [0.001, 0.004]; box 1 x 1 x 4; spring 5e4, sphere
restitution 0.4, walls 0.7, dt 5e-6; grid cell 2 r_max -> 126 x 126 x 501
cells), FP32, one simulation per GPU.  A bench "step" is one simulation step
of all particles: integrate, walls, grid rebuild, contacts.

Under the reference's scheme the contact kick is not scaled by dt, and with
this scene's spring and its smallest spheres the explicit update is unstable:
velocities diverge within a few steps and NaN appears after about a hundred.
Every timed block of --block steps therefore starts from the scene's
initial state, restored from an on-device checkpoint outside the timed
region, so all timed steps are steps 1..block of the scene.

Reports one JSON line (rank 0): value = device time (CUDA events on the
library's stream) of exactly --steps steps, max over ranks; e2e = the same
steps through host buffers (upload, steps, download per block); roofline of
the dominant kernel from a per-kernel event pass; cpu_baseline = the
reference's own CPU simulator on a bounded sample.

--impl reference times the reference's CPU simulator (oracle/_ref, built
from the reference sources) on the same scene and prints its line.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "particle-stabilizer_b200", "python"))

METRIC = "particle-steps/s at 1M spheres (forward)"
UNIT = "particle-steps/s"
WORKLOAD = ("1,048,576 spheres, log-normal r (median 0.002, sigma 0.25, clip [0.001,0.004]), box 1x1x4, "
            "k 5e4, e 0.4, walls 0.7, dt 5e-6, cell 2 r_max")
L2_BYTES = 126 * 2 ** 20
# DRAM bytes per launch of the fused FP32 contacts kernel (adaptive walk, the
# default) on this workload, measured with ncu in steady state
# (--cache-control none, the second of two captured launches: 35.2 MB read +
# 50.9 MB written; the algorithmic bytes are 75.5 MB).
CONTACTS_TRAFFIC = 86.09e6


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.device)], stdout=open(self.path, "w"),
                                         stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        time.sleep(0.25)
        if self.proc is not None:
            self.proc.terminate()
            self.proc.wait(timeout=10)

    def summary(self) -> dict:
        rows = []
        try:
            with open(self.path) as f:
                for line in f:
                    parts = [p.strip() for p in line.split(",")]
                    if len(parts) >= 9:
                        rows.append(parts)
            os.unlink(self.path)
        except OSError:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "", 1).isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "", 1).isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    return world, rank, local, dist


def barrier(dist):
    if dist is not None:
        dist.barrier()


def _reduce(dist, x: float, op) -> float:
    if dist is None:
        return x
    import torch

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(dist, x: float) -> float:
    """Largest value over the ranks (device time: the slowest rank sets it)."""
    return _reduce(dist, x, dist.ReduceOp.MAX) if dist is not None else x


def sum_over_ranks(dist, x: float) -> float:
    return _reduce(dist, x, dist.ReduceOp.SUM) if dist is not None else x


# algorithmic bytes per particle of each kernel (FP32 state = 2 x 16 B)
def alg_bytes(kind: str, n: int, cells: int, vb: int = 16) -> float:
    st = 2 * vb
    return {
        "contacts": n * (st + st + 8),          # own state in, next state out, cell+slot out
        "rank_move": n * (st + 8 + 4 + st + 4),  # state, cell+slot, own tmp in; state, orig out
        "scatter": n * (12 + 4),                # cell, slot, orig in; tmp out
        "scan": cells * 8,                      # counts in, offsets out
        "begin": n * (st + st + 8),
    }[kind]


def step_alg_bytes(n: int, cells: int) -> float:
    """Whole-step algorithmic bytes: 128 B per particle (two passes over the
    32-B state, in and out) + 4 B per cell."""
    return 128.0 * n + 4.0 * cells


def reference_cpu_sample(scene, budget_s: float, max_steps: int, warmup: int = 0) -> dict:
    """The reference's own CPU simulator (oracle/_ref/libref_cpu.so) on the
    same scene: construction and `warmup` steps untimed, then whole steps
    until the budget or max_steps."""
    from oracle import ps_oracle as O

    if os.path.exists(O.REF_CPU_SO):
        r = O.ref_cpu()
        kind = "reference"
    else:
        r = None
        kind = "port"
    if r is not None:
        h = r.create(scene)
        if warmup > 0:
            r.step(h, warmup)
        steps, t = 0, 0.0
        while steps < max_steps and t < budget_s:
            t += r.time_steps(h, 1)
            steps += 1
        r.destroy(h)
    else:
        # the oracle (C restatement of the same scheme), one thread
        t0 = time.perf_counter()
        steps = 0
        st = scene
        while steps < max_steps and time.perf_counter() - t0 < budget_s:
            O.run(st, 1, "f64")
            steps += 1
        t = time.perf_counter() - t0
    return {"value": scene.n * steps / t, "unit": UNIT, "cores": 1, "kind": kind,
            "sample": f"{steps} full steps of the 1M-sphere scene from its initial state "
                      f"({t:.1f} s, one thread: the reference's box path is serial)",
            "seconds": t, "steps": steps}


def non_finite(state) -> int:
    """Particles with a non-finite coordinate: the reference scheme's kick
    k*overlap/m is not scaled by dt and diverges once k*dt/m is well above 1."""
    return int(np.sum(~np.isfinite(state[:, :6]).all(axis=1)))


def adjoint_measure(psb200, sc, steps, every, device, restore_block=None) -> dict:
    """Plain forward vs checkpointed forward + backward on one scene (FP32),
    device/wall time with a synchronize on both sides."""
    with psb200.Simulation(sc, "f32", device=device) as sim:
        sim.set_state()
        sim.checkpoint_save(0)
        sim.time_steps(min(steps, 20))  # warm-up: graphs captured
        sim.checkpoint_load(0)
        fwd_ms = sim.time_steps(steps)
        sim.checkpoint_load(0)
        sim.forward_checkpointed(steps, every)  # warm-up of the backward path
        _, g = psb200.height_loss(sim.get_state())
        sim.backward(g)
        sim.checkpoint_load(0)
        sim.sync()
        t0 = time.perf_counter()
        sim.forward_checkpointed(steps, every)
        t1 = time.perf_counter()
        final = sim.get_state()
        loss, g = psb200.height_loss(final)
        t2 = time.perf_counter()
        grads, _ = sim.backward(g)
        t3 = time.perf_counter()
    fwd_adj_s = (t1 - t0) + (t3 - t2)
    bad = non_finite(final)
    return {"scene": sc.name, "n_particles": sc.n, "steps": steps, "checkpoint_every": every,
            "forward_ms": fwd_ms, "forward_particle_steps_per_s": sc.n * steps / (fwd_ms * 1e-3),
            "forward_plus_adjoint_ms": 1e3 * fwd_adj_s,
            "forward_plus_adjoint_particle_steps_per_s": sc.n * steps / fwd_adj_s,
            "ratio_fwd_adj_over_fwd": fwd_adj_s / (fwd_ms * 1e-3), "loss": loss, "non_finite_at_end": bad,
            "grad_k_spring": float(grads[0][0]), "grad_e_sphere": float(grads[0][1]),
            "grad_e_wall_zmin_zmax_xmin_xmax_ymin_ymax": [float(x) for x in grads[0][2:8]],
            "k_spring": sc.k_spring}


def batch_measure(psb200, scenes_mod, device, steps: int, n_scenes: int, sequential: bool = True,
                  k_range=(5e3, 5e4), tune: bool = False) -> dict:
    """256 uneven independent scenes: one simulation advancing all of them per
    launch, against the same scenes run one after another, each as its own
    simulation (steps from each scene's initial state, FP32)."""
    batch = scenes_mod.c5_scenes(n_scenes, k_range=k_range)
    n_total = sum(s.n for s in batch)
    with psb200.Simulation(batch, "f32", device=device) as sim:
        sim.set_state()
        sim.checkpoint_save(0)
        sim.time_steps(steps)
        sim.checkpoint_load(0)
        batched_ms = sim.time_steps(steps)
        launches = sim.launches()
        bad = non_finite(sim.get_state())
        tuned = None
        if tune:
            # cell size and graph block chosen by ps_autotune, then the same steps again
            sim.checkpoint_load(0)
            choice = sim.autotune(trial_steps=20)
            sim.checkpoint_load(0)
            sim.time_steps(steps)
            sim.checkpoint_load(0)
            tuned_ms = sim.time_steps(steps)
            tuned_hash = hashlib.sha256(sim.get_state().tobytes()).hexdigest()
            # neighbour lists on the tuned grid, skin by ps_tune_neighbor_lists
            sim.checkpoint_load(0)
            lt = sim.tune_neighbor_lists(trial_steps=50, skins=(0.0, 0.02, 0.05, 0.1, 0.2))
            sim.time_steps(steps)
            sim.checkpoint_load(0)
            lists_ms = sim.time_steps(steps)
            lists = {"batched_ms": lists_ms, "skin_fraction": lt["skin_fraction"], "trial_skins": lt["skins"],
                     "trial_ms_per_step": lt["ms_table"],
                     "batched_particle_steps_per_s": n_total * steps / (lists_ms * 1e-3),
                     "identical_to_tuned_grid": hashlib.sha256(sim.get_state().tobytes()).hexdigest() == tuned_hash}
            tuned = {"batched_ms": tuned_ms, "cell_factor": choice["cell_factor"],
                     "graph_block": choice["graph_block"], "trial_ms_table": choice["ms_table"],
                     "trial_cell_factors": choice["cell_factors"], "trial_graph_blocks": choice["graph_blocks"],
                     "batched_particle_steps_per_s": n_total * steps / (tuned_ms * 1e-3),
                     "non_finite_at_end": non_finite(sim.get_state()), "neighbor_lists": lists}
    out = {"n_scenes": n_scenes, "n_particles": n_total, "k_range": list(k_range), "steps": steps,
           "batched_ms": batched_ms,
           "batched_scene_steps_per_s": n_scenes * steps / (batched_ms * 1e-3),
           "batched_particle_steps_per_s": n_total * steps / (batched_ms * 1e-3),
           "launches_batched": launches, "non_finite_at_end": bad}
    if tuned is not None:
        out["autotuned"] = tuned
    if not sequential:
        return out
    seq_ms = 0.0
    seq_launches = 0
    for sc in batch:
        with psb200.Simulation(sc, "f32", device=device) as s1:
            s1.set_state()
            s1.checkpoint_save(0)
            s1.time_steps(steps)
            s1.checkpoint_load(0)
            seq_ms += s1.time_steps(steps)
            seq_launches += s1.launches()
    out.update({"sequential_ms": seq_ms, "sequential_scene_steps_per_s": n_scenes * steps / (seq_ms * 1e-3),
                "speedup_batched_over_sequential": seq_ms / batched_ms, "launches_sequential": seq_launches})
    if "autotuned" in out:
        out["autotuned"]["speedup_over_sequential"] = seq_ms / out["autotuned"]["batched_ms"]
        nl = out["autotuned"]["neighbor_lists"]
        nl["speedup_over_sequential"] = seq_ms / nl["batched_ms"]
    return out


def mesh_measure(psb200, scenes_mod, device, steps: int) -> dict:
    """262,144 spheres poured into the 20,200-triangle funnel (grid domain
    widened over the spawn lattice), FP32, `steps` steps from the initial
    state in one timed call."""
    sc = scenes_mod.c3_scene()
    with psb200.Simulation(sc, "f32", device=device) as sim:
        sim.set_state()
        sim.checkpoint_save(0)
        sim.time_steps(200)
        sim.checkpoint_load(0)
        ms = sim.time_steps(steps)
        st = sim.get_state()
        launches = sim.launches()
    below_rim = int(np.sum(st[:, 2] < 1.0))
    return {"scene": sc.name, "n_particles": sc.n, "n_triangles": int(sc.tri.shape[0]), "steps": steps,
            "ms": ms, "particle_steps_per_s": sc.n * steps / (ms * 1e-3), "launches": launches,
            "particles_below_rim_at_end": below_rim, "non_finite_at_end": non_finite(st)}


def lists_measure(psb200, scenes_mod, device, only=None, fixed_skin=None) -> dict:
    """Neighbour-list mode against the grid path on the same steps from the
    same state (after 100 warm-up steps), with the final states compared
    bit for bit.  The skin fraction is chosen by ps_tune_neighbor_lists
    (100 trial steps per candidate, 0 = grid path) from that state, unless
    `fixed_skin` gives it (profiling runs, where the tuner's timings mean
    nothing).
    Scenes: 1M spheres with a soft spring (FP32 and FP64), the 1M-sphere
    pile of the differentiation scene with spring 5, the 256 soft batch
    scenes, 262,144 spheres poured into the 20,200-triangle funnel (20,000
    steps from the initial state), and the 1M scene as specified, which
    diverges."""
    cases = [("c2_1M_k0.25_fp32", lambda: scenes_mod.c2_scene(k_spring=0.25), "f32", 1000),
             ("c2_1M_k0.25_fp64", lambda: scenes_mod.c2_scene(k_spring=0.25), "f64", 1000),
             ("c4_1M_k5_fp32", lambda: scenes_mod.c4_scene(1 << 20, edge=0.95, k_spring=5.0), "f32", 1000),
             ("c5_256_soft_fp32", lambda: scenes_mod.c5_scenes(256, k_range=(0.25, 2.5)), "f32", 300),
             ("c3_funnel_fp32", lambda: scenes_mod.c3_scene(), "f32", 20000),
             ("c2_1M_as_specified_fp32", lambda: scenes_mod.c2_scene(), "f32", 200)]
    skins = (0.0, 0.02, 0.05, 0.1, 0.2)
    out = {}
    for name, make, prec, steps in cases:
        if only is not None and name != only:
            continue
        sc = make()
        n = sc.n if not isinstance(sc, list) else sum(x.n for x in sc)
        with psb200.Simulation(sc, prec, device=device) as sim:
            sim.set_state()
            if not name.startswith("c3_"):  # the funnel pour is timed from its initial state
                sim.step(100)
            sim.checkpoint_save(1)
            sim.time_steps(steps)
            sim.checkpoint_load(1)
            grid_ms = sim.time_steps(steps)
            want = hashlib.sha256(sim.get_state().tobytes()).hexdigest()
            sim.checkpoint_load(1)
            if fixed_skin is None:
                tune = sim.tune_neighbor_lists(trial_steps=100, skins=skins, max_neighbours=64)
                skin = tune["skin_fraction"]
            else:
                tune = {"ms_table": None}
                skin = fixed_skin
                sim.set_neighbor_lists(skin, 64)
            sim.time_steps(steps)
            sim.checkpoint_load(1)
            rb0, fb0 = sim.list_stats()
            list_ms = sim.time_steps(steps)
            launches = sim.launches()
            got = hashlib.sha256(sim.get_state().tobytes()).hexdigest()
            rebuilds, fallbacks = (a - b for a, b in zip(sim.list_stats(), (rb0, fb0)))
        out[name] = {"n_particles": n, "precision": prec, "skin_fraction": skin, "steps": steps,
                     "tuning_skins": list(skins), "tuning_ms_per_step": tune["ms_table"],
                     "grid_us_per_step": 1000.0 * grid_ms / steps, "list_us_per_step": 1000.0 * list_ms / steps,
                     "speedup": grid_ms / list_ms, "identical_to_grid": got == want, "rebuilds": rebuilds,
                     "fallbacks": fallbacks, "launches": launches,
                     "list_particle_steps_per_s": n * steps / (list_ms * 1e-3)}
    return out


def reference_cuda_measure(psb200, scenes_mod, device, steps: int = 200, warm: int = 20) -> dict:
    """The reference's own CUDA simulator (oracle/_ref/libref_cuda.so, built
    from its unmodified sources for sm_100a, driven per step) against this
    library on the same B200, in the same process.

    Scene: the 1M-sphere box scene with spring 0.25 instead of 5e4, all other
    draws identical.  With the specified spring the scheme diverges, and the
    reference's count/register kernels index out of range once positions
    stop being finite, so the reference runs only here, and only after this
    library's FP64 run of the same steps stayed finite and inside the box.
    Both time steps warm+1 .. warm+steps from the same initial state (device
    time, CUDA events)."""
    from oracle import ps_oracle as O

    if not os.path.exists(O.REF_CUDA_SO):
        return {"unavailable": "oracle/_ref/libref_cuda.so was not built (reference sources absent at build time)"}
    sc = scenes_mod.c2_scene(k_spring=0.25)
    ours = {}
    for prec in ("f32", "f64"):
        with psb200.Simulation(sc, prec, device=device) as sim:
            sim.set_state()
            sim.step(warm)
            sim.checkpoint_save(1)
            sim.time_steps(steps)  # captures the graphs of this block length
            sim.checkpoint_load(1)
            ms = sim.time_steps(steps)
            st = sim.get_state()
        inside = bool(np.isfinite(st).all() and np.all(st[:, :3] >= np.array(sc.box_min))
                      and np.all(st[:, :3] <= np.array(sc.box_max)))
        ours[prec] = {"ms_per_step": ms / steps, "particle_steps_per_s": sc.n * steps / (ms * 1e-3),
                      "finite_and_inside_box": inside}
    if not ours["f64"]["finite_and_inside_box"]:
        return {"unavailable": "this library's FP64 run left the box or went non-finite; reference not run"}
    r = O.ref_cuda()
    h = r.create(sc)
    try:
        r.step(h, warm)
        ref_s = r.time_steps(h, steps)
        ref_state = r.state(h, sc.n)
    finally:
        r.destroy(h)
    ref = sc.n * steps / ref_s
    return {"scene": "1,048,576-sphere box scene as above with spring 0.25 (stable under the reference scheme)",
            "steps": f"{warm + 1}..{warm + steps}", "reference_ms_per_step": 1e3 * ref_s / steps,
            "reference_particle_steps_per_s": ref, "reference_dtype": "f64",
            "reference_finite_at_end": bool(np.isfinite(ref_state).all()),
            "ours": ours,
            "speedup_f32": ours["f32"]["particle_steps_per_s"] / ref,
            "speedup_f64": ours["f64"]["particle_steps_per_s"] / ref}


# Secondary measurements.  The reference's contact kick k*overlap/m is not
# scaled by dt, so the scheme is stable only for k*dt/m below about 1.  The
# differentiation and batch scenes with their specified springs (k*dt/m = 373
# and 27..7,460) diverge at their first contacts, so each is measured twice:
# as specified over a window before or through its divergence (the line
# reports how many particles went non-finite), and with soft springs that keep
# every particle finite (differentiation scene k = 5; batch springs
# log-uniform in [0.25, 2.5]; all other draws identical).
def walks_measure(psb200, scenes_mod, device) -> dict:
    """The contact kernel's neighbour walks on the same states: per launch of
    the contact kernel (eager steps, CUDA events) and per graph step (best of
    three), for the per-lane walk, the warp walk and the adaptive walk (the
    default), each at 256 threads per CTA, with a hash of the final state
    (equal for every walk).  Scenes: this benchmark's 1M scene (steps 1-20),
    the soft 1M scene in FP32 and FP64 and the 1M dense pile after 100 steps,
    the 256 soft batch scenes after 100 steps and the funnel after 2,000."""
    cases = [("c2_1M_as_benchmarked", lambda: scenes_mod.c2_scene(), "f32", 0, 20),
             ("c2_1M_k0.25_fp32", lambda: scenes_mod.c2_scene(k_spring=0.25), "f32", 100, 100),
             ("c2_1M_k0.25_fp64", lambda: scenes_mod.c2_scene(k_spring=0.25), "f64", 100, 100),
             ("c4_1M_k5_fp32", lambda: scenes_mod.c4_scene(1 << 20, edge=0.95, k_spring=5.0), "f32", 100, 100),
             ("c5_256_soft_fp32", lambda: scenes_mod.c5_scenes(256, k_range=(0.25, 2.5)), "f32", 100, 100),
             ("c3_funnel_fp32", lambda: scenes_mod.c3_scene(), "f32", 2000, 100)]
    kernels = (("lane", psb200.WALK_LANE), ("warp", psb200.WALK_WARP), ("adaptive", psb200.WALK_ADAPTIVE))
    out = {}
    for name, make, prec, pre, steps in cases:
        sc = make()
        res = {}
        with psb200.Simulation(sc, prec, device=device) as sim:
            sim.set_state()
            if pre:
                sim.step(pre)
            sim.checkpoint_save(1)
            for label, walk in kernels:
                sim.set_contact_kernel(walk, 256)
                sim.checkpoint_load(1)
                sim.time_steps(steps)  # captures this walk's graph
                best = None
                for _ in range(3):
                    sim.checkpoint_load(1)
                    ms = sim.time_steps(steps)
                    best = ms if best is None else min(best, ms)
                digest = hashlib.sha256(sim.get_state().tobytes()).hexdigest()[:16]
                sim.checkpoint_load(1)
                c_ms, c_n = sim.profile_steps(steps)["contacts"]
                res[label] = {"step_us": 1000.0 * best / steps, "contacts_us": 1000.0 * c_ms / max(c_n, 1),
                              "state_sha256_16": digest}
        res["identical"] = len({v["state_sha256_16"] for v in res.values()}) == 1
        out[name] = res
    return out


EXTRAS = {
    # forward vs forward + adjoint, checkpoint every 100 steps
    "adjoint": lambda p, s, dev, a: adjoint_measure(p, s.c4_scene(k_spring=5.0), 2000, 100, dev),
    "adjoint_as_specified": lambda p, s, dev, a: adjoint_measure(p, s.c4_scene(), 1000, 100, dev),
    "adjoint_1m": lambda p, s, dev, a: adjoint_measure(p, s.c4_scene(1 << 20, edge=0.95, k_spring=5.0), 2000, 100,
                                                       dev),
    "batch": lambda p, s, dev, a: batch_measure(p, s, dev, 100, 256, sequential=not a.no_sequential,
                                                k_range=(0.25, 2.5), tune=True),
    "batch_as_specified": lambda p, s, dev, a: batch_measure(p, s, dev, 100, 256, sequential=not a.no_sequential),
    "mesh": lambda p, s, dev, a: mesh_measure(p, s, dev, a.mesh_steps),
    "lists": lambda p, s, dev, a: lists_measure(p, s, dev, a.scene, a.skin),
}
# measurements run only on request (--extra NAME), not in the default line
ON_REQUEST = {
    "walks": lambda p, s, dev, a: walks_measure(p, s, dev),
}


def run_ours(args, world, rank, local, dist):
    import psb200
    from psb200 import scenes

    sc = scenes.c2_scene()
    n = sc.n
    sim = psb200.Simulation(sc, args.precision, device=local)
    sim.set_state()
    sim.checkpoint_save(0)
    g = sim.grid(0)
    cells = int(g.n_cells)
    block = max(1, args.block)

    def blocks_of(total: int) -> list[int]:
        return [min(block, total - k) for k in range(0, total, block)]

    def timed_steps(total: int) -> tuple[float, int]:
        ms, launches = 0.0, 0
        for b in blocks_of(total):
            sim.checkpoint_load(0)
            ms += sim.time_steps(b)
            launches += sim.launches()
        return ms, launches

    # Warm-up: every block length the timed region uses runs once first, so
    # each CUDA graph is captured and instantiated outside the timed region;
    # then whole blocks until at least max(warmup, 3) steps have run.
    warm_lens = sorted(set(blocks_of(args.steps)))
    warmed = 0
    for b in warm_lens:
        timed_steps(b)
        warmed += b
    while warmed < max(args.warmup, 3):
        b = warm_lens[-1]
        timed_steps(b)
        warmed += b
    barrier(dist)
    sim.sync()
    with ClockSampler(local) as clk:
        t0 = time.perf_counter()
        dev_ms, launches = timed_steps(args.steps)
        sim.sync()
        wall = time.perf_counter() - t0
    barrier(dist)
    dev_ms_max = max_over_ranks(dist, dev_ms)
    total_particle_steps = sum_over_ranks(dist, float(n * args.steps))
    value = total_particle_steps / (dev_ms_max * 1e-3)

    # per-kernel device times (eager launches, events around each) over one block
    sim.checkpoint_load(0)
    prof = sim.profile_steps(min(block, args.steps))
    per_step = {k: (ms / max(1, min(block, args.steps)), cnt) for k, (ms, cnt) in prof.items()}
    dom = max(("contacts", "rank_move", "scatter", "scan"), key=lambda k: prof[k][0])
    dom_ms_avg = prof[dom][0] / max(1, prof[dom][1])
    peak, peak_kind = peaks()
    achieved = alg_bytes(dom, n, cells) / (dom_ms_avg * 1e-3) / 1e9
    step_ms = dev_ms / args.steps
    step_gbs = step_alg_bytes(n, cells) / (step_ms * 1e-3) / 1e9

    # End to end through the C ABI with host buffers: for every block of the
    # same decomposition as `value`, upload the scene's initial state from
    # pinned host memory, run the block, download the state.  One untimed
    # pass first (pinned-memory paths, graphs already captured above).
    import torch

    pin_in = torch.empty((n, 8), dtype=torch.float64, pin_memory=True)
    pin_out = torch.empty((n, 8), dtype=torch.float64, pin_memory=True)
    host = pin_in.numpy()
    host[:] = sc.state
    host_out = pin_out.numpy()

    def e2e_pass() -> float:
        sim.sync()
        t0 = time.perf_counter()
        for b in blocks_of(args.steps):
            sim.set_state(host)
            sim.step(b)
            sim.get_state(out=host_out)
        return time.perf_counter() - t0

    e2e_pass()
    barrier(dist)
    t_e2e = e2e_pass()
    e2e_value = sum_over_ranks(dist, float(n * args.steps)) / max_over_ranks(dist, t_e2e)
    n_blocks = len(blocks_of(args.steps))

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dev_ms_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32" if args.precision == "f32" else "f64",
        "data": "synthetic: seeded generator of the 1M-sphere scene (numpy default_rng(2))",
        "config": bench_config(n, block, world),
        "grid": {"cells_per_axis": [g.nb[0], g.nb[1], g.nb[2]], "cells": cells, "cell_edge": "2 r_max"},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": peak_kind,
                     "traffic": CONTACTS_TRAFFIC if (dom == "contacts" and args.precision == "f32") else None,
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum per launch of the fused "
                                       "contacts kernel on this workload, steady state (--cache-control none)",
                     "alg_bytes_per_launch": alg_bytes(dom, n, cells)},
        "step_roofline": {"alg_bytes_per_step": step_alg_bytes(n, cells), "achieved_gbs": step_gbs,
                          "frac": step_gbs / peak},
        "kernels_ms_per_step": {k: v[0] for k, v in per_step.items()},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 64.0 * n * n_blocks / args.steps,
                "d2h_bytes_per_step": 64.0 * n * n_blocks / args.steps,
                "how": f"per block of the same {args.steps} steps: ps_set_state(pinned host, 64 B per sphere) + "
                       f"ps_step(block) + ps_get_state(pinned host), wall clock, max over ranks"},
        "gpu_launches": launches,
        "clocks": clk.summary(),
        "wall_s": wall,
    }
    sim.close()
    if not args.no_extras:
        for name in EXTRAS:
            line[name] = EXTRAS[name](psb200, scenes, local, args)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = reference_cpu_sample(sc, args.cpu_budget, 20)
    if rank == 0 and world == 1 and not args.no_reference_cuda:
        line["reference_cuda"] = reference_cuda_measure(psb200, scenes, local)
    return line


def bench_config(n: int, block: int, world: int) -> dict:
    """The workload description shared by both arms."""
    return {"workload": WORKLOAD, "n_particles": n, "block": block, "state_restored_every": block,
            "timed_steps": "steps 1..block of the scene in every block (initial state restored between blocks)",
            "l2": "working set 205 MiB (FP32 state, cell arrays) > 126 MiB L2; no flush",
            "parallelism": f"{world} independent replica{'s' if world != 1 else ''} (one per GPU, no collective)"}


def run_reference(args, world, rank):
    """Reference arm: the reference's own CPU simulator (oracle/_ref/
    libref_cpu.so, built from its unmodified sources) on the same scene and
    the same block decomposition as this library's arm: every block starts
    from the scene's initial state (a fresh simulator; construction
    untimed).  The reference's box-container path is serial, so one host
    thread is all it can use.  Warm-up: `--warmup` whole steps on a
    simulator of their own (at most about a minute of them); timed: the
    `--steps` steps, or as many whole steps as fit `--ref-budget` seconds."""
    from oracle import ps_oracle as O
    from psb200 import scenes

    if rank != 0:
        return None
    sc = scenes.c2_scene()
    block = max(1, args.block)
    blocks = [min(block, args.steps - k) for k in range(0, args.steps, block)]
    if os.path.exists(O.REF_CPU_SO):
        r, kind = O.ref_cpu(), "reference"
    else:
        r, kind = None, "port"
    warm_done, warm_t = 0, 0.0
    steps_done, t = 0, 0.0
    if r is not None:
        h = r.create(sc)
        while warm_done < args.warmup and warm_t < 60.0:
            warm_t += r.time_steps(h, 1)
            warm_done += 1
        r.destroy(h)
        for b in blocks:
            if t >= args.ref_budget:
                break
            h = r.create(sc)
            k = 0
            while k < b and t < args.ref_budget:
                t += r.time_steps(h, 1)
                k += 1
            steps_done += k
            r.destroy(h)
    else:
        # the oracle (C restatement of the same scheme), one thread
        t0 = time.perf_counter()
        while steps_done < args.steps and time.perf_counter() - t0 < args.ref_budget:
            O.run(sc, 1, "f64")
            steps_done += 1
        t = time.perf_counter() - t0
    value = sc.n * steps_done / t
    sample = (f"{steps_done} whole steps of the 1M-sphere scene in blocks of {block} from its initial state "
              f"({t:.1f} s timed, one thread: the reference's box path is serial)")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": steps_done, "warmup": warm_done, "ms_per_step": 1e3 * t / steps_done,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic: seeded generator of the 1M-sphere scene (numpy default_rng(2))",
            "config": bench_config(sc.n, block, world),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": kind, "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if steps_done < args.steps or warm_done < args.warmup:
        line["note"] = (f"{steps_done} of the requested {args.steps} steps and {warm_done} of {args.warmup} warm-up "
                        f"steps fit the time budget")
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=200)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="f32", choices=["f32", "f64"])
    ap.add_argument("--block", type=int, default=100, help="steps per block; the state is restored between blocks")
    ap.add_argument("--cpu-budget", type=float, default=20.0, help="seconds of reference CPU stepping")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-reference-cuda", action="store_true",
                    help="skip the head-to-head with the reference's own CUDA build")
    ap.add_argument("--ref-budget", type=float, default=240.0,
                    help="seconds of timed reference CPU stepping in the --impl reference arm")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the adjoint, batch and mesh measurements")
    ap.add_argument("--extra", choices=sorted(set(EXTRAS) | set(ON_REQUEST)),
                    help="run only this secondary measurement on the local GPU and print its JSON")
    ap.add_argument("--no-sequential", action="store_true",
                    help="with --extra batch: skip the scene-by-scene comparison")
    ap.add_argument("--mesh-steps", type=int, default=20000,
                    help="steps of the funnel measurement (the mesh line; fewer for profiling runs)")
    ap.add_argument("--scene", default=None,
                    help="with --extra lists: measure only this scene (e.g. c2_1M_k0.25_fp32)")
    ap.add_argument("--skin", type=float, default=None,
                    help="with --extra lists: this skin fraction instead of the tuner's choice")
    args = ap.parse_args()
    if args.extra is not None:
        import psb200
        from psb200 import scenes
        local = int(os.environ.get("LOCAL_RANK", "0"))
        measure = EXTRAS.get(args.extra) or ON_REQUEST[args.extra]
        print(json.dumps({args.extra: measure(psb200, scenes, local, args)}), flush=True)
        return
    if args.impl == "reference":
        # rank 0 alone times the reference's CPU simulator; other ranks exit
        world = int(os.environ.get("WORLD_SIZE", "1"))
        rank = int(os.environ.get("RANK", "0"))
        line = run_reference(args, world, rank)
        if rank == 0 and line is not None:
            print(json.dumps(line), flush=True)
        return
    world, rank, local, dist = dist_setup()
    if True:
        line = run_ours(args, world, rank, local, dist)
    if rank == 0 and line is not None:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
