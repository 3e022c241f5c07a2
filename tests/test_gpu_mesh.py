"""Triangle container on the GPU (binned mesh) against the oracle's
all-pairs restatement of PolygonContainerCUDA, bit for bit, and the CLI /
runSimulateCUDA path with an OBJ container."""
import os
import subprocess

import numpy as np
import pytest

import psb200
from psb200 import scenes
from oracle import ps_oracle as O

pytestmark = pytest.mark.gpu


def run_gpu(sc, steps, precision):
    with psb200.Simulation(sc, precision) as sim:
        sim.set_state()
        sim.step(steps)
        sim.sync()
        return sim.get_state()


def cast(a, precision):
    return a.astype(np.float32) if precision == "f32" else a


@pytest.mark.parametrize("precision", ["f32", "f64"])
@pytest.mark.parametrize("steps", [1, 7, 60])
def test_box_mesh_bitexact(need_gpu, precision, steps):
    sc = scenes.box_mesh_scene()
    got = cast(run_gpu(sc, steps, precision), precision)
    want = O.run(sc, steps, precision)
    assert np.array_equal(got, want), f"{np.sum(np.any(got != want, axis=1))} of {sc.n} differ"


@pytest.mark.parametrize("precision", ["f32", "f64"])
@pytest.mark.parametrize("quirk", [1, 0])
def test_funnel_wall_bitexact(need_gpu, precision, quirk):
    sc = scenes.funnel_wall_scene(1500, seed=9).copy(edge_quirk=quirk)
    got = cast(run_gpu(sc, 40, precision), precision)
    want = O.run(sc, 40, precision)
    # the same step with the container replaced by a loose box (no walls reached)
    loose = sc.copy(tri=None, box_min=(-0.6, -0.6, -0.1), box_max=(0.6, 0.6, 1.2))
    moved = np.any(O.run(loose, 1, precision) != O.run(sc, 1, precision), axis=1)
    assert moved.sum() > 100  # the container acts on many particles every step
    assert np.array_equal(got, want), f"{np.sum(np.any(got != want, axis=1))} of {sc.n} differ"


def test_full_funnel_mesh_runs_with_widened_domain(need_gpu):
    sc = scenes.funnel_wall_scene(800, seed=3, coarse=False)
    got = run_gpu(sc, 12, "f32").astype(np.float32)
    want = O.run(sc, 12, "f32")
    assert np.array_equal(got, want)


def test_cli_runs_the_path_with_an_obj_container(need_gpu, tmp_path):
    """runSimulateCUDA through the command line: CSV in, OBJ container,
    CSV out equal to the oracle's FP64 state written in the same format."""
    sc = scenes.box_mesh_scene(60, seed=5)
    obj = tmp_path / "box.obj"
    scenes.write_obj(str(obj), sc.tri)
    csv_in = tmp_path / "in.csv"
    with open(csv_in, "w") as f:
        f.write("x,y,z,r\n")
        for p in sc.state:
            f.write("%.17g,%.17g,%.17g,%.17g\n" % (p[0], p[1], p[2], p[6]))
    csv_out = tmp_path / "out.csv"
    lib = psb200.LIB_PATH
    cmd = [psb200.CLI_PATH, "--lib", lib, str(csv_in), "--cuda", "--container", str(obj), "--max-steps", "25",
           "--dt", "0.0001", "--coeff-of-spring", "2", "--coeff-of-restitution-sphere", "0.5",
           "--coeff-of-restitution-wall", "0.7", "0.7", "0.7", "0.7", "0.7", "0.7", "--gravity", "0", "0", "-9.8",
           "--initial-velocity", "0.1", "-0.2", "0.05", "--density", "1000", "--out-csv-path", str(csv_out)]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "Number of collided particles" in r.stdout and "nPolygons = " in r.stdout
    start = psb200.read_csv(str(csv_in), (0.1, -0.2, 0.05), 1000.0)
    want = O.run(sc.copy(state=start), 25, "f64")
    ref_csv = tmp_path / "want.csv"
    psb200.write_csv(str(ref_csv), want)
    assert csv_out.read_text() == ref_csv.read_text()


def test_cli_resolves_overlaps_and_writes_obj(need_gpu, tmp_path):
    """--resolve-overlap-axis and --out-obj-path after the run, in the
    reference's order: the CSV equals the oracle's FP64 state after the
    reference's own resolveOverlaps (or this library's, which the CPU tests
    show identical, when the reference build is absent)."""
    sc = scenes.pile(400, seed=19, k_spring=1.0)
    csv_in = tmp_path / "in.csv"
    with open(csv_in, "w") as f:
        f.write("x,y,z,r\n")
        for p in sc.state:
            f.write("%.17g,%.17g,%.17g,%.17g\n" % (p[0], p[1], p[2], p[6]))
    csv_out, obj_out = tmp_path / "out.csv", tmp_path / "objdir" / "out.obj"
    lo, hi = sc.box_min, sc.box_max
    cmd = [psb200.CLI_PATH, "--lib", psb200.LIB_PATH, str(csv_in), "--cuda", "--max-steps", "30",
           "--box-min", *map(str, lo), "--box-max", *map(str, hi), "--dt", "1e-05", "--coeff-of-spring", "1",
           "--coeff-of-restitution-sphere", "0.5", "--coeff-of-restitution-wall", *["0.7"] * 6,
           "--gravity", "0", "0", "-9.8", "--initial-velocity", "0", "0", "0", "--density", "1000",
           "--resolve-overlap-axis", "2", "--out-csv-path", str(csv_out), "--out-obj-path", str(obj_out)]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "Number of collided particles" in r.stdout and "Max collision distance" in r.stdout
    start = psb200.read_csv(str(csv_in), (0.0, 0.0, 0.0), 1000.0)
    stepped = O.run(sc.copy(state=start, e_wall=(0.7,) * 6), 30, "f64")
    if os.path.exists(O.REF_CPU_SO):
        want = O.ref_resolve_overlaps(stepped, 2)
    else:
        want, _, _ = psb200.resolve_overlaps(stepped, 2)
    ref_csv = tmp_path / "want.csv"
    psb200.write_csv(str(ref_csv), want)
    assert csv_out.read_text() == ref_csv.read_text()
    with open(obj_out) as f:
        assert f.readline() == "o Generated particles\n"
    obj_out.unlink()


@pytest.mark.parametrize("precision", ["f32", "f64"])
@pytest.mark.parametrize("quirk", [1, 0])
@pytest.mark.parametrize("n_fan", [64, 68, 128, 132, 300])
def test_sphere_touching_more_triangles_than_one_pass_holds(need_gpu, precision, quirk, n_fan):
    """A sphere resting on the centre of a fan floor touches every fan
    triangle at once.  The device keeps 64 hits per pass and takes further
    passes for the rest, in ascending triangle order; the oracle sums every
    hit in one ascending loop.  Fan sizes sit on either side of one and two
    full passes."""
    sc = scenes.fan_floor_scene(n_fan=n_fan).copy(edge_quirk=quirk)
    # the oracle's own container pass: the centre sphere gets one 1e-5
    # correction per hit, so its lift counts the hits
    lifted = O.pre_grid_state(sc, sc.state, "f64")[0, 2] - O.pre_grid_state(
        sc.copy(tri=None, box_min=(-1, -1, -1), box_max=(1, 1, 2)), sc.state, "f64")[0, 2]
    assert round(lifted / 1e-5) == n_fan
    for steps in (1, 30):
        got = cast(run_gpu(sc, steps, precision), precision)
        want = O.run(sc, steps, precision)
        assert np.array_equal(got, want), f"{np.sum(np.any(got != want, axis=1))} of {sc.n} differ after {steps}"


def write_xyzr_csv(path, state):
    with open(path, "w") as f:
        f.write("x,y,z,r\n")
        for p in state:
            f.write("%.17g,%.17g,%.17g,%.17g\n" % (p[0], p[1], p[2], p[6]))


@pytest.mark.parametrize("flags", ["fp32", "cell_size", "widen_fp32", "zero_steps"])
def test_cli_extra_flags(need_gpu, tmp_path, flags):
    """The CLI's own flags reach the library unchanged: --fp32, --cell-size
    (a value with more than six significant digits), --widen-domain (the
    funnel, spheres above its rim), and --max-steps 0, which takes one step
    as the reference's loop does.  The CSV equals the oracle's state written
    by the same writer."""
    funnel = flags == "widen_fp32"
    sc = scenes.funnel_wall_scene(400, seed=21, z_max=1.05, widen=True) if funnel else scenes.pile(300, seed=23,
                                                                                                   k_spring=1.0)
    csv_in, csv_out = tmp_path / "in.csv", tmp_path / "out.csv"
    write_xyzr_csv(csv_in, sc.state)
    steps = 0 if flags == "zero_steps" else 20
    cmd = [psb200.CLI_PATH, "--lib", psb200.LIB_PATH, str(csv_in), "--cuda", "--max-steps", str(steps),
           "--dt", repr(sc.dt), "--coeff-of-spring", repr(sc.k_spring), "--coeff-of-restitution-sphere",
           repr(sc.e_sphere), "--coeff-of-restitution-wall", *[repr(e) for e in sc.e_wall],
           "--gravity", *map(repr, sc.gravity), "--initial-velocity", "0.1", "-0.2", "0.05", "--density", "1000",
           "--out-csv-path", str(csv_out)]
    if funnel:
        obj = tmp_path / "funnel.obj"
        scenes.write_obj(str(obj), sc.tri)
        cmd += ["--container", str(obj), "--widen-domain", "--fp32"]
    else:
        cmd += ["--box-min", *map(repr, sc.box_min), "--box-max", *map(repr, sc.box_max)]
    want_sc = sc
    prec = "f64"
    if flags == "fp32":
        cmd.append("--fp32")
        prec = "f32"
    if funnel:
        prec = "f32"
    if flags == "cell_size":
        cell = 2.1 * sc.r_max() * 1.2345678901
        cmd += ["--cell-size", repr(cell)]
        want_sc = sc.copy(interval=cell)
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    start = psb200.read_csv(str(csv_in), (0.1, -0.2, 0.05), 1000.0)
    want = O.run(want_sc.copy(state=start), max(steps, 1), prec).astype(np.float64)
    ref_csv = tmp_path / "want.csv"
    psb200.write_csv(str(ref_csv), want)
    assert csv_out.read_text() == ref_csv.read_text()
