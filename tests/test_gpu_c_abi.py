"""The C ABI driven from a plain C program (tests/c_abi/step_lattice.c, the
usage INTEGRATION.md shows): the 4,096-sphere lattice stepped through
ps_create / ps_set_state / ps_step / ps_get_state equals the oracle bit for
bit, in FP32 and FP64."""
import subprocess

import numpy as np
import pytest

from psb200 import scenes
from oracle import ps_oracle as O
from test_cpu_abi import build_c_program

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_c_program_steps_the_lattice_like_the_oracle(need_gpu, tmp_path, prec):
    sc = scenes.lattice_c1()
    # the program's scene: box [0,1]^3, g = -9.8 z, walls 0.8, k 1e4, e 0.5, dt 1e-5
    assert (sc.box_min, sc.box_max, sc.e_wall, sc.k_spring, sc.e_sphere, sc.dt) == \
        ((0.0, 0.0, 0.0), (1.0, 1.0, 1.0), (0.8,) * 6, 1e4, 0.5, 1e-5)
    exe = build_c_program(tmp_path)
    src, dst = tmp_path / "in.bin", tmp_path / "out.bin"
    np.ascontiguousarray(sc.state, dtype=np.float64).tofile(src)
    args = [exe, str(src), "300", str(dst)] + (["fp64"] if prec == "f64" else [])
    r = subprocess.run(args, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    got = np.fromfile(dst, dtype=np.float64).reshape(-1, 8)
    want = O.run(sc, 300, prec)
    assert np.array_equal(got.astype(np.float32) if prec == "f32" else got, want)
