"""Generate the golden fixtures of tests/golden from the reference's own code.

Run in a container where the reference sources are present and
`make -C oracle ref` has built oracle/_ref/libref_cpu.so (the reference CPU
simulator compiled from its unmodified sources):

    python tests/golden/make_golden.py

Writes, next to this script:
  ref_cpu_box.npz   initial states and the reference CPU simulator's states
                    after several steps (contact-rich pile, jittered lattice)
  ref_cpu_mesh.npz  a small closed triangle container, its particles and the
                    reference CPU simulator's states after several steps
  ref_io.npz        a CSV exercising the reader's edge cases, the reference
                    reader's output, and the reference writer's text for a state
  io_cases.csv      that CSV
  cube.obj          an OBJ with quads, slashes and negative indices, and in
                    ref_io.npz its de-indexed triangles as the reference reads them

The GPU-side fixtures of the reference CUDA simulator come from
make_golden_cuda.py, which needs a GPU.
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "particle-stabilizer_b200", "python"))

from oracle import ps_oracle as O  # noqa: E402
from psb200 import scenes  # noqa: E402

BOX_STEPS = (1, 3, 10, 40)
MESH_STEPS = (1, 5, 25)


def cube_mesh(lo=(-0.1, -0.1, 0.0), hi=(0.1, 0.1, 0.25), n=4) -> np.ndarray:
    """Closed axis-aligned box triangulated into n x n quads per face, two
    triangles each, normals pointing out."""
    lo = np.asarray(lo, dtype=np.float64)
    hi = np.asarray(hi, dtype=np.float64)
    tris = []
    for axis in range(3):
        u, v = [a for a in range(3) if a != axis]
        for side, sign in ((lo[axis], -1.0), (hi[axis], 1.0)):
            for i in range(n):
                for j in range(n):
                    def pt(a, b):
                        p = np.zeros(3)
                        p[axis] = side
                        p[u] = lo[u] + (hi[u] - lo[u]) * a / n
                        p[v] = lo[v] + (hi[v] - lo[v]) * b / n
                        return p
                    p00, p10, p01, p11 = pt(i, j), pt(i + 1, j), pt(i, j + 1), pt(i + 1, j + 1)
                    t1, t2 = [p00, p10, p11], [p00, p11, p01]
                    nrm = np.cross(t1[1] - t1[0], t1[2] - t1[0])
                    if np.sign(nrm[axis]) != sign:
                        t1, t2 = [p00, p11, p10], [p00, p01, p11]
                    tris.append(np.concatenate(t1))
                    tris.append(np.concatenate(t2))
    return np.asarray(tris).astype(np.float32).astype(np.float64)


def mesh_scene(seed=41) -> scenes.Scene:
    rng = np.random.default_rng(seed)
    tri = cube_mesh()
    n = 120
    g = np.stack(np.meshgrid(np.arange(5), np.arange(5), np.arange(5), indexing="ij"), -1).reshape(-1, 3)[:n]
    # outer layers overlap the side walls and the floor from the first step
    pos = np.array([-0.092, -0.092, 0.006]) + g * 0.046 + rng.uniform(-0.002, 0.002, size=(n, 3))
    vel = rng.normal(0, 0.5, size=(n, 3))
    r = np.full(n, 0.012)
    st = np.concatenate([pos, vel, r[:, None], scenes.mass_of(r, 1000.0)[:, None]], axis=1)
    return scenes.Scene(st, (-0.1, -0.1, 0.0), (0.1, 0.1, 0.25), (0, 0, -9.8), (0.7,) * 6, 2.0, 0.5, 1e-4, tri=tri,
                        name="cube_mesh")


def run_ref(sc, steps_list, obj_path=None):
    r = O.ref_cpu()
    h = r.create(sc, obj_path)
    out, done = [], 0
    for s in steps_list:
        r.step(h, s - done)
        done = s
        out.append(r.state(h, sc.n))
    r.destroy(h)
    return np.stack(out)


def main():
    # --- box scenes ---
    pile = scenes.pile(256, seed=31, k_spring=1.0)
    lat = scenes.lattice_c1(side=6)
    np.savez_compressed(os.path.join(HERE, "ref_cpu_box.npz"), steps=np.array(BOX_STEPS),
                        pile_init=pile.state, pile_out=run_ref(pile, BOX_STEPS),
                        pile_box=np.array([pile.box_min, pile.box_max]), pile_e=np.array(pile.e_wall),
                        pile_k=pile.k_spring, pile_es=pile.e_sphere, pile_dt=pile.dt,
                        lat_init=lat.state, lat_out=run_ref(lat, BOX_STEPS))
    # --- mesh scene ---
    ms = mesh_scene()
    with tempfile.TemporaryDirectory() as d:
        obj = os.path.join(d, "c.obj")
        scenes.write_obj(obj, ms.tri)
        mesh_out = run_ref(ms, MESH_STEPS, obj)
    np.savez_compressed(os.path.join(HERE, "ref_cpu_mesh.npz"), steps=np.array(MESH_STEPS), tri=ms.tri,
                        init=ms.state, out=mesh_out, k=ms.k_spring, es=ms.e_sphere, dt=ms.dt,
                        e_wall=np.array(ms.e_wall))
    # --- I/O ---
    csv_path = os.path.join(HERE, "io_cases.csv")
    with open(csv_path, "w") as f:
        f.write("x,y,z,r\n")
        f.write("1.5,-2.25,3.0,0.5\n")
        f.write("  -0.125, 7e-3 ,1E2,2\n")            # spaces, exponents
        f.write("1,2,3\n")                             # 3 tokens: skipped
        f.write("4,5,null,6,7\n")                      # 'null' dropped -> 4 tokens
        f.write("8,,9,10,11\n")                        # empty token dropped -> 4 tokens
        f.write("1,2,3,4,5\n")                         # 5 tokens: skipped
        f.write("0.001,0.002,0.003,0.0004\r\n")        # CRLF
        f.write("\n")                                  # blank
        f.write("-12.5,13.75,-0.0,1.25\n")
    r = O.ref_cpu()
    import ctypes as C
    cap = 64
    out = np.zeros((cap, 8))
    vel = (C.c_double * 3)(0.1, -0.2, 0.3)
    n = r.lib.refh_read_csv(csv_path.encode(), vel, 2500.0, C.c_void_p(out.ctypes.data), cap)
    state = out[:n].copy()
    wstate = np.array([[1.0, -2.5, 123.456789, 0, 0, 0, 0.25, 1.0],
                       [-0.000123, 99999.5, -1234567.0, 0, 0, 0, 5.0, 1.0],
                       [0.1, 0.2, -0.3, 0, 0, 0, 12.0, 1.0]])
    with tempfile.TemporaryDirectory() as d:
        w = os.path.join(d, "w.csv")
        r.lib.refh_write_csv(C.c_void_p(wstate.ctypes.data), wstate.shape[0], w.encode())
        text = open(w).read()
    obj_path = os.path.join(HERE, "cube.obj")
    with open(obj_path, "w") as f:
        f.write("# unit quad faces with texture/normal indices and a negative-index face\n")
        for v in [(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)]:
            f.write("v %g %g %g\n" % v)
        f.write("vt 0 0\nvn 0 0 1\n")
        f.write("f 1/1/1 4/1/1 3/1/1 2/1/1\n")
        f.write("f 5//1 6//1 7//1 8//1\n")
        f.write("f -8 -7 -3 -4\n")
        f.write("f 2 3 7\n")
    tri = np.zeros((64, 9))
    nt = r.lib.refh_read_obj(obj_path.encode(), C.c_void_p(tri.ctypes.data), 64)
    np.savez_compressed(os.path.join(HERE, "ref_io.npz"), csv_state=state, csv_velocity=np.array([0.1, -0.2, 0.3]),
                        csv_density=2500.0, write_state=wstate, write_text=np.array(text), obj_tri=tri[:nt].copy())
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
