"""The C ABI library without a GPU: exports, error behaviour, file formats.

Every function declared in include/*.h must be exported by
libparticle_stabilizer_cuda.so.  The CSV and OBJ readers/writer run on the
host and are compared with what the reference's own code produced
(tests/golden/ref_io.npz, from tests/golden/make_golden.py).
"""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

import psb200
from conftest import GOLDEN, ROOT, gpu_available


def declared_functions():
    names = set()
    for h in ("particle_stabilizer_b200.h", "ps_runsimulate.hpp"):
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = re.sub(r"//[^\n]*", "", text)
        for m in re.finditer(r"\b(ps_[a-z0-9_]+|runSimulateCUDA)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


def test_every_declared_symbol_is_exported():
    names = declared_functions()
    assert "ps_create" in names and "runSimulateCUDA" in names and len(names) >= 20
    lib = psb200.lib()
    for n in names:
        getattr(lib, n)  # raises AttributeError if missing
    out = subprocess.run(["nm", "-D", "--defined-only", psb200.LIB_PATH], capture_output=True, text=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    assert set(names) <= exported
    assert set(psb200.EXPORTED) <= exported
    # nothing else leaks out of the library
    assert all(e.startswith("ps_") or e == "runSimulateCUDA" for e in exported)


@pytest.mark.skipif(gpu_available(), reason="checks the no-GPU error path")
def test_create_without_gpu_is_a_clean_error():
    sc = psb200.scenes.pile(16)
    with pytest.raises(psb200.PSError) as e:
        psb200.Simulation(sc)
    assert "ps_create" in str(e.value)
    assert psb200.lib().ps_last_error()  # message recorded


def test_bad_arguments_rejected_before_any_cuda_call():
    h = C.c_void_p()
    assert psb200.lib().ps_create(None, 1, 0, 0, C.byref(h)) == -1
    assert psb200.lib().ps_step(None, 1) == -1
    assert psb200.lib().ps_destroy(None) == 0
    assert psb200.exclusive_scan_scratch_bytes(0) == 8


def test_read_csv_matches_reference_reader():
    g = np.load(os.path.join(GOLDEN, "ref_io.npz"))
    got = psb200.read_csv(os.path.join(GOLDEN, "io_cases.csv"), tuple(g["csv_velocity"]), float(g["csv_density"]))
    assert np.array_equal(got, g["csv_state"])


def test_write_csv_matches_reference_writer(tmp_path):
    g = np.load(os.path.join(GOLDEN, "ref_io.npz"))
    out = tmp_path / "sub" / "w.csv"  # the writer creates missing directories, as the reference does
    psb200.write_csv(str(out), g["write_state"])
    assert out.read_text() == str(g["write_text"])


def test_read_obj_matches_reference_deindexing():
    g = np.load(os.path.join(GOLDEN, "ref_io.npz"))
    got = psb200.read_obj(os.path.join(GOLDEN, "cube.obj"))
    assert np.array_equal(got, g["obj_tri"])


def test_io_errors(tmp_path):
    with pytest.raises(psb200.PSError, match="Could not open"):
        psb200.read_csv(str(tmp_path / "missing.csv"))
    bad = tmp_path / "bad.csv"
    bad.write_text("x,y,z,r\n1,2,abc,4\n")
    with pytest.raises(psb200.PSError, match="bad number"):
        psb200.read_csv(str(bad))
    with pytest.raises(psb200.PSError, match="Unable to open"):
        psb200.read_obj(str(tmp_path / "missing.obj"))
    obj = tmp_path / "bad.obj"
    obj.write_text("v 0 0 0\nf 1 2 3\n")
    with pytest.raises(psb200.PSError, match="out of range"):
        psb200.read_obj(str(obj))


def test_obj_roundtrip_of_the_funnel(tmp_path):
    tri = psb200.scenes.funnel_triangles(n_seg=24, n_cone=4, n_cyl=2, n_ring=2)
    p = tmp_path / "f.obj"
    psb200.scenes.write_obj(str(p), tri)
    assert np.array_equal(psb200.read_obj(str(p)), tri)


def test_cli_help_and_missing_input(tmp_path):
    exe = psb200.CLI_PATH
    r = subprocess.run([exe, "-h"], capture_output=True, text=True, cwd=tmp_path)
    assert r.returncode == 0 and "--coeff-of-restitution-wall" in r.stdout
    lib = os.path.dirname(psb200.LIB_PATH)
    r = subprocess.run([exe, "--lib", os.path.join(lib, "libparticle_stabilizer_cuda.so"), "missing.csv", "--cuda"],
                       capture_output=True, text=True, cwd=tmp_path)
    assert r.returncode != 0 and "Could not open file" in (r.stderr + r.stdout)
    r = subprocess.run([exe, "--lib", str(tmp_path / "nolib.so"), "x.csv"], capture_output=True, text=True,
                       cwd=tmp_path)
    assert r.returncode != 0 and "Cannot open library" in r.stderr


def test_bounds_checked_build_exports_the_same_symbols():
    """lib_debug/ (make debug) is the same C ABI compiled with
    -DPS_DEBUG_BOUNDS; ps_bounds_checked tells the two builds apart."""
    assert os.path.exists(psb200.DEBUG_LIB_PATH), "build it with `make -C particle-stabilizer_b200 debug`"
    out = subprocess.run(["nm", "-D", "--defined-only", psb200.DEBUG_LIB_PATH], capture_output=True, text=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    assert set(declared_functions()) <= exported and set(psb200.EXPORTED) <= exported
    assert psb200.bounds_checked() is False
    code = ("import psb200; psb200.LIB_PATH = psb200.DEBUG_LIB_PATH; "
            "assert psb200.bounds_checked() is True; print('checked')")
    env = dict(os.environ)
    env["PYTHONPATH"] = os.pathsep.join([ROOT, os.path.join(ROOT, "particle-stabilizer_b200", "python")])
    r = subprocess.run(["python3", "-c", code], capture_output=True, text=True, env=env)
    assert r.returncode == 0 and "checked" in r.stdout, r.stderr


C_PROGRAM = os.path.join(ROOT, "tests", "c_abi", "step_lattice.c")


def build_c_program(out_dir):
    """The header compiles as strict C11 and the program links against the
    library (tests/c_abi/step_lattice.c, the C usage INTEGRATION.md shows)."""
    exe = os.path.join(str(out_dir), "step_lattice")
    lib_dir = os.path.dirname(psb200.LIB_PATH)
    subprocess.run(["gcc", "-std=c11", "-Wall", "-Wextra", "-Werror", "-pedantic", "-I", os.path.join(ROOT, "include"),
                    C_PROGRAM, "-o", exe, "-L", lib_dir, "-lparticle_stabilizer_cuda", f"-Wl,-rpath,{lib_dir}"],
                   check=True)
    return exe


def test_header_compiles_as_c_and_the_c_program_links(tmp_path):
    exe = build_c_program(tmp_path)
    assert os.access(exe, os.X_OK)


def test_state_file_round_trip_and_bad_files(tmp_path):
    """ps_write_state_bin / ps_read_state_bin keep every record bit for bit
    (signed zeros, subnormals, infinities and NaN payloads included) and the
    step count; files that are not state files, or are cut short, are
    errors, not garbage."""
    rng = np.random.default_rng(5)
    st = rng.normal(size=(257, 8))
    st[0, :4] = [-0.0, 5e-324, np.inf, -np.inf]
    st[1, 0] = np.frombuffer(np.uint64(0x7FF8_0000_0000_1234).tobytes(), dtype=np.float64)[0]  # a NaN payload
    p = tmp_path / "sub" / "s.bin"  # the writer creates missing directories
    psb200.write_state_bin(str(p), st, 12345)
    got, steps = psb200.read_state_bin(str(p))
    assert steps == 12345 and got.tobytes() == st.tobytes()
    assert os.path.getsize(p) == 32 + 64 * st.shape[0]
    empty = tmp_path / "e.bin"
    psb200.write_state_bin(str(empty), np.zeros((0, 8)), 0)
    got, steps = psb200.read_state_bin(str(empty))
    assert got.shape == (0, 8) and steps == 0
    cut = tmp_path / "cut.bin"
    cut.write_bytes(p.read_bytes()[:-8])
    with pytest.raises(psb200.PSError, match="truncated"):
        psb200.read_state_bin(str(cut))
    csv = tmp_path / "x.csv"
    csv.write_text("x,y,z,r\n1,2,3,4\n")
    with pytest.raises(psb200.PSError, match="not a state file"):
        psb200.read_state_bin(str(csv))
    with pytest.raises(psb200.PSError, match="Could not open"):
        psb200.read_state_bin(str(tmp_path / "missing.bin"))


def test_python_structs_match_the_header_layout(tmp_path):
    """Every struct of include/particle_stabilizer_b200.h that the Python
    binding passes by pointer has the same size and field offsets on both
    sides (a mismatch would corrupt memory silently)."""
    pairs = {"ps_scene_desc": psb200.SceneDesc, "ps_stats": psb200.Stats, "ps_grid_info": psb200.GridInfo,
             "ps_grad": psb200.Grad, "ps_tune_result": psb200.TuneResult}
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "particle_stabilizer_b200.h"', "int main(void) {"]
    for cname, pytype in pairs.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in pytype._fields_:
            lines.append(f'  printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = str(tmp_path / "layout")
    subprocess.run(["gcc", "-std=c11", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), str(src), "-o", exe],
                   check=True)
    got = {}
    for line in subprocess.run([exe], capture_output=True, text=True, check=True).stdout.splitlines():
        cname, what, value = line.split()
        got[(cname, what)] = int(value)
    for cname, pytype in pairs.items():
        assert got[(cname, "size")] == C.sizeof(pytype), cname
        for fname, _ in pytype._fields_:
            assert got[(cname, fname)] == getattr(pytype, fname).offset, (cname, fname)
