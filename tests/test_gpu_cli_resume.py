"""Checkpoint / resume through the command line: a run of 30 steps dumped
with --dump-state and continued for 20 more with --resume-state ends in the
state of one 50-step run, bit for bit (every record, velocities included,
and the step count), in FP64 and FP32, and equal to the oracle."""
import subprocess

import numpy as np
import pytest

import psb200
from psb200 import scenes
from oracle import ps_oracle as O

pytestmark = pytest.mark.gpu


def cli(sc, tmp_path, steps, extra, prec):
    cmd = [psb200.CLI_PATH, "--lib", psb200.LIB_PATH, "--cuda", "--max-steps", str(steps), "--dt", repr(sc.dt),
           "--coeff-of-spring", repr(sc.k_spring), "--coeff-of-restitution-sphere", repr(sc.e_sphere),
           "--coeff-of-restitution-wall", *[repr(e) for e in sc.e_wall], "--gravity", *map(repr, sc.gravity),
           "--box-min", *map(repr, sc.box_min), "--box-max", *map(repr, sc.box_max), *extra]
    if prec == "f32":
        cmd.append("--fp32")
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    return r.stdout


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_dump_and_resume_continue_bit_for_bit(need_gpu, tmp_path, prec):
    sc = scenes.pile(500, seed=29, k_spring=1.0)
    start = tmp_path / "start.bin"
    psb200.write_state_bin(str(start), sc.state, 0)
    a, b, whole = tmp_path / "a.bin", tmp_path / "b.bin", tmp_path / "whole.bin"
    cli(sc, tmp_path, 30, ["--resume-state", str(start), "--dump-state", str(a)], prec)
    out = cli(sc, tmp_path, 20, ["--resume-state", str(a), "--dump-state", str(b)], prec)
    assert "after 30 steps" in out and "after 50 steps" in out
    cli(sc, tmp_path, 50, ["--resume-state", str(start), "--dump-state", str(whole)], prec)
    sa, na = psb200.read_state_bin(str(a))
    sb, nb = psb200.read_state_bin(str(b))
    sw, nw = psb200.read_state_bin(str(whole))
    assert (na, nb, nw) == (30, 50, 50)
    assert sb.tobytes() == sw.tobytes()
    assert not np.array_equal(sa, sb)  # the second run moved the spheres
    want = O.run(sc, 50, prec)
    assert np.array_equal(sb.astype(np.float32) if prec == "f32" else sb, want)
