"""The reference's own command line driving this library.

oracle/_ref/ref_main is the reference's unmodified `main`
(src/App/ParticleStabilizerMain.cpp) and DynamicLoader
(src/ParticleStabilizer/DynamicLoader.cpp), linked by oracle/Makefile with
its CSV/OBJ/overlap code.  With --cuda it does
dlopen("./libparticle_stabilizer_cuda.so") in its working directory and
calls runSimulateCUDA through its own function-pointer type
(ParticleStabilizerMain.cpp:24-35, 235-256), with its own glm, std::vector
and std::string arguments.  Here that file is this repository's library, so
the test exercises the drop-in exactly as the reference's users would.  The
CSV it writes must be byte-identical to the one this repository's CLI
writes for the same scene, and equal to the oracle's FP64 run written in the
same format, for a box scene and for an OBJ container.

One quirk of the reference's parser shows here.  It builds the wall
restitutions as CoefficientOfRestitutionWall(std::stod(argv[++i]), ... six
times) (ParticleStabilizerMain.cpp:121-127); the evaluation order of
function arguments is unspecified in C++, and g++ evaluates them right to
left, so the reference binary applies the six values in reverse of its
documented Z_MIN Z_MAX X_MIN X_MAX Y_MIN Y_MAX.  (The brace-initialised
vectors, --gravity and the rest, are evaluated left to right.)  This
repository's CLI reads the documented order, so it is given the reversed
list to run the same scene."""
import os
import subprocess

import numpy as np
import pytest

import psb200
from psb200 import scenes
from oracle import ps_oracle as O

pytestmark = pytest.mark.gpu

REF_MAIN = os.path.join(os.path.dirname(O.REF_CPU_SO), "ref_main")
needs_ref_main = pytest.mark.skipif(not os.path.exists(REF_MAIN),
                                    reason="oracle/_ref/ref_main was not built (reference sources absent)")


def write_input(path, sc):
    with open(path, "w") as f:
        f.write("x,y,z,r\n")
        for p in sc.state:
            f.write("%.17g,%.17g,%.17g,%.17g\n" % (p[0], p[1], p[2], p[6]))


CASES = {
    "box": dict(make=lambda: scenes.pile(400, seed=19, k_spring=1.0), steps=40, obj=False,
                args=["--dt", "1e-05", "--coeff-of-spring", "1", "--coeff-of-restitution-sphere", "0.5",
                      "--gravity", "0", "0", "-9.8", "--initial-velocity", "0.05", "0", "-0.1", "--density", "1000"],
                walls=("0.8", "0.7", "0.6", "0.75", "0.65", "0.55"), vel=(0.05, 0.0, -0.1)),
    "obj": dict(make=lambda: scenes.box_mesh_scene(60, seed=5), steps=25, obj=True,
                args=["--dt", "0.0001", "--coeff-of-spring", "2", "--coeff-of-restitution-sphere", "0.5",
                      "--gravity", "0", "0", "-9.8", "--initial-velocity", "0.1", "-0.2", "0.05", "--density", "1000"],
                walls=("0.7", "0.6", "0.6", "0.6", "0.6", "0.6"), vel=(0.1, -0.2, 0.05)),
}


@needs_ref_main
@pytest.mark.parametrize("case", sorted(CASES))
def test_reference_cli_loads_this_library(need_gpu, tmp_path, case):
    c = CASES[case]
    sc = c["make"]()
    csv_in = tmp_path / "in.csv"
    write_input(csv_in, sc)
    args = [str(csv_in), "--cuda", "--max-steps", str(c["steps"]), *c["args"]]
    walls = list(c["walls"])
    applied = tuple(float(x) for x in reversed(walls))  # what the g++-built reference parser applies
    if c["obj"]:
        obj = tmp_path / "container.obj"
        scenes.write_obj(str(obj), sc.tri)
        args += ["--container", str(obj)]
    else:
        args += ["--box-min", *map(str, sc.box_min), "--box-max", *map(str, sc.box_max)]
    run_dir = tmp_path / "ref_run"
    run_dir.mkdir()
    os.symlink(os.path.abspath(psb200.LIB_PATH), run_dir / "libparticle_stabilizer_cuda.so")
    out_ref = tmp_path / "out_ref.csv"
    r = subprocess.run([REF_MAIN, *args, "--coeff-of-restitution-wall", *walls, "--out-csv-path", str(out_ref)],
                       cwd=run_dir, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    # the reference's own log lines are discarded by the logging stand-in;
    # this one is printed by this library's runSimulateCUDA
    assert "Number of collided particles" in r.stdout, r.stdout
    out_ours = tmp_path / "out_ours.csv"
    r2 = subprocess.run([psb200.CLI_PATH, "--lib", psb200.LIB_PATH, *args, "--coeff-of-restitution-wall",
                         *map(repr, applied), "--out-csv-path", str(out_ours)], capture_output=True, text=True,
                        timeout=600)
    assert r2.returncode == 0, r2.stdout + r2.stderr
    assert out_ref.read_bytes() == out_ours.read_bytes()
    start = psb200.read_csv(str(csv_in), c["vel"], 1000.0)
    want = O.run(sc.copy(state=start, e_wall=applied), c["steps"], "f64")
    want_csv = tmp_path / "want.csv"
    psb200.write_csv(str(want_csv), want)
    assert out_ref.read_text() == want_csv.read_text()
    assert not np.array_equal(start[:, :3], want[:, :3])  # the run moved the spheres
