"""The CPU code under AddressSanitizer and UndefinedBehaviorSanitizer.

- The oracle (oracle/_build_asan/, `make -C oracle asan`): the whole oracle
  test file runs against it, so every golden-vector, reference-fixture and
  known-answer check also checks memory accesses and undefined behaviour.
- The library's host-side code, built alone without CUDA
  (particle-stabilizer_b200/build_asan/libps_host_asan.so, `make host-asan`):
  the CSV and OBJ readers and writers, the overlap statistics and
  resolveOverlaps, on the golden fixtures and on random clouds, with results
  equal to the product library's.

Each runs in a child process with the sanitizer runtimes preloaded (the
Python interpreter itself is not instrumented); a report fails the child.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

import psb200
from conftest import GOLDEN, ROOT

PKG = os.path.join(ROOT, "particle-stabilizer_b200")
ORACLE_ASAN = os.path.join(ROOT, "oracle", "_build_asan", "libps_oracle.so")
HOST_ASAN = os.path.join(PKG, "build_asan", "libps_host_asan.so")


def runtimes():
    libs = []
    for name in ("libasan.so", "libubsan.so"):
        p = subprocess.run(["gcc", f"-print-file-name={name}"], capture_output=True, text=True).stdout.strip()
        if not os.path.isabs(p) or not os.path.exists(p):
            pytest.skip(f"gcc has no {name}")
        libs.append(p)
    return " ".join(libs)


def sanitized_env(**extra):
    env = dict(os.environ)
    env["LD_PRELOAD"] = runtimes()
    env["ASAN_OPTIONS"] = "detect_leaks=0:abort_on_error=1"
    env["UBSAN_OPTIONS"] = "print_stacktrace=1:halt_on_error=1"
    env["PYTHONPATH"] = os.pathsep.join([ROOT, os.path.join(PKG, "python"), env.get("PYTHONPATH", "")])
    env.update(extra)
    return env


def check_clean(r):
    out = r.stdout + r.stderr
    assert r.returncode == 0, out[-4000:]
    assert "AddressSanitizer" not in out and "runtime error" not in out, out[-4000:]


def build(target, directory):
    subprocess.run(["make", "-s", "-C", directory, target], check=True)


def test_oracle_tests_under_sanitizers():
    build("asan", os.path.join(ROOT, "oracle"))
    env = sanitized_env(PS_ORACLE_SO=ORACLE_ASAN)
    probe = subprocess.run([sys.executable, "-c", "import ctypes; from oracle import ps_oracle as O; O.lib(); "
                            "ctypes.CDLL(None).__asan_init; print(O.ORACLE_SO)"],
                           cwd=ROOT, env=env, capture_output=True, text=True)
    check_clean(probe)
    assert probe.stdout.strip() == ORACLE_ASAN  # the instrumented build is the one loaded
    r = subprocess.run([sys.executable, "-m", "pytest", os.path.join(ROOT, "tests", "test_cpu_oracle.py"), "-x", "-q",
                        "-p", "no:cacheprovider"], cwd=ROOT, env=env, capture_output=True, text=True, timeout=1200)
    check_clean(r)
    assert " passed" in r.stdout


HOST_CHILD = r"""
import ctypes as C, os, sys
import numpy as np
import psb200
L = C.CDLL(os.environ["PS_HOST_ASAN_SO"])
C.CDLL(None).__asan_init  # the sanitizer runtime is loaded
psb200.declare_host(L)
psb200._lib = L
g = np.load(os.path.join(sys.argv[1], "ref_io.npz"))
want = np.load(sys.argv[2])
got = psb200.read_csv(os.path.join(sys.argv[1], "io_cases.csv"), tuple(g["csv_velocity"]), float(g["csv_density"]))
assert np.array_equal(got, g["csv_state"])
assert np.array_equal(psb200.read_obj(os.path.join(sys.argv[1], "cube.obj")), g["obj_tri"])
out = os.path.join(sys.argv[3], "w.csv")
psb200.write_csv(out, g["write_state"])
assert open(out).read() == str(g["write_text"])
for bad, what in ((os.path.join(sys.argv[3], "missing.csv"), "csv"), (os.path.join(sys.argv[3], "missing.obj"), "obj")):
    try:
        psb200.read_csv(bad) if what == "csv" else psb200.read_obj(bad)
        raise SystemExit("a missing file was read")
    except psb200.PSError:
        pass
for k in range(3):
    st = want[f"cloud{k}"]
    assert psb200.overlap_stats(st) == tuple(want[f"stats{k}"].tolist())
    res, nc, mo = psb200.resolve_overlaps(st, k)
    assert np.array_equal(res, want[f"resolved{k}"]) and (nc, mo) == tuple(want[f"rstats{k}"].tolist())
psb200.write_obj_spheres(os.path.join(sys.argv[3], "s.obj"), want["cloud0"][:20])
assert open(os.path.join(sys.argv[3], "s.obj"), "rb").read() == open(sys.argv[4], "rb").read()
print("clean")
"""


def test_host_code_under_sanitizers(tmp_path):
    build("host-asan", PKG)
    # expected results from the product library, in this process
    rng = np.random.default_rng(7)
    want = {}
    for k in range(3):
        n = (300, 700, 1200)[k]
        st = np.zeros((n, 8))
        st[:, :3] = rng.uniform(0.0, 0.08, size=(n, 3))
        st[:, 6] = rng.uniform(0.004, 0.006, size=n)
        st[:, 7] = 1.0
        want[f"cloud{k}"] = st
        want[f"stats{k}"] = np.array(psb200.overlap_stats(st), dtype=float)
        res, nc, mo = psb200.resolve_overlaps(st, k)
        want[f"resolved{k}"] = res
        want[f"rstats{k}"] = np.array([nc, mo], dtype=float)
    np.savez(tmp_path / "want.npz", **want)
    sphere_obj = tmp_path / "want_spheres.obj"
    psb200.write_obj_spheres(str(sphere_obj), want["cloud0"][:20])
    work = tmp_path / "work"
    work.mkdir()
    r = subprocess.run([sys.executable, "-c", HOST_CHILD, GOLDEN, str(tmp_path / "want.npz"), str(work),
                        str(sphere_obj)], cwd=ROOT, env=sanitized_env(PS_HOST_ASAN_SO=HOST_ASAN),
                       capture_output=True, text=True, timeout=600)
    check_clean(r)
    assert r.stdout.strip().endswith("clean")
