"""bench.py's reference arm on the CPU: the reference's own CPU simulator
(oracle/_ref, or the oracle where it was not built) on the 1M-sphere scene,
one bounded step.  Under torchrun only rank 0 works and prints; the line
carries the same metric, unit and workload as the library's arm."""
import json
import os
import subprocess
import sys

from conftest import ROOT

sys.path.insert(0, ROOT)
import bench  # noqa: E402


def _run(env_extra, *args):
    env = dict(os.environ, **env_extra)
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", *args],
                          capture_output=True, text=True, env=env, timeout=600, cwd=ROOT)


def test_other_ranks_exit_without_work():
    r = _run({"RANK": "1", "WORLD_SIZE": "2"}, "--steps", "1", "--warmup", "0")
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""


def test_rank_zero_prints_one_reference_line():
    r = _run({"RANK": "0", "WORLD_SIZE": "1"}, "--steps", "1", "--warmup", "0", "--ref-budget", "5")
    assert r.returncode == 0, r.stderr
    lines = [ln for ln in r.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["impl"] == "reference"
    assert (line["metric"], line["unit"], line["higher_is_better"]) == (bench.METRIC, bench.UNIT, True)
    assert line["config"] == bench.bench_config(1 << 20, 100, 1)
    assert line["steps"] == 1 and line["value"] > 0
    cb = line["cpu_baseline"]
    assert cb["value"] == line["value"] and cb["cores"] == 1 and cb["kind"] in ("reference", "port") and cb["sample"]
    assert line["e2e"] == {"value": line["value"], "unit": bench.UNIT, "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
