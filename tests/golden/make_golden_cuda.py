"""Generate tests/golden/ref_cuda_*.npz from the reference's own CUDA simulator.

Needs a GPU and oracle/_ref/libref_cuda.so (the reference CUDA sources
compiled for sm_100a by `make -C oracle ref`):

    python tests/golden/make_golden_cuda.py OUTDIR [NAME,NAME,...]

For two small box scenes whose dynamics stay tame (a jittered lattice and a
soft contact-rich pile) and three triangle containers read from OBJ files
(a closed triangulated box whose outer spheres touch its walls and floor,
spheres pressing on the cone wall of a coarse funnel, and a box whose floor
is a 300-triangle fan with one sphere touching every fan triangle at once;
every centre inside the mesh AABB, which is the reference's grid domain),
it records after
several step counts the reference's bucket arrays (per-cell counts,
exclusive offsets, particle index list) and its particle states.  The CPU
tests pin the oracle's CUDA scheme to these, and the mesh fixtures its
triangle semantics (PolygonContainerCUDA.cpp:130-226,
PolygonContainerCUDA_kernels.cu:114-294: the edge pick by smallest
dot(center, point), the velocity mean of the reflections, the position
corrections summed from the pre-container position).
"""
from __future__ import annotations

import ctypes as C
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

STEPS = (1, 5, 30)


def record(sc, name, outdir):
    r = O.ref_cuda()
    with tempfile.TemporaryDirectory() as d:  # the container reads its OBJ file at construction
        obj = None
        if sc.tri is not None:
            obj = os.path.join(d, "container.obj")
            scenes.write_obj(obj, sc.tri)
        h = r.create(sc, obj)
    nb = (C.c_int32 * 3)()
    iv = C.c_double()
    lo = (C.c_double * 3)()
    r.lib.refc_get_grid(h, nb, C.byref(iv), lo)
    n_cells = nb[0] * nb[1] * nb[2]
    counts, offsets, buckets, states = [], [], [], []
    done = 0
    for s in STEPS:
        r.step(h, s - done)
        done = s
        c = np.empty(n_cells, dtype=np.uint32)
        o = np.empty(n_cells, dtype=np.uint32)
        b = np.empty(sc.n, dtype=np.int64)
        r.lib.refc_get_buckets(h, C.c_void_p(c.ctypes.data), C.c_void_p(o.ctypes.data), C.c_void_p(b.ctypes.data))
        counts.append(c)
        offsets.append(o)
        buckets.append(b)
        states.append(r.state(h, sc.n))
    r.destroy(h)
    np.savez_compressed(os.path.join(outdir, f"ref_cuda_{name}.npz"), steps=np.array(STEPS), init=sc.state,
                        box=np.array([sc.box_min, sc.box_max]), e_wall=np.array(sc.e_wall), k=sc.k_spring,
                        es=sc.e_sphere, dt=sc.dt, nb=np.array(list(nb)), interval=iv.value,
                        counts=np.stack(counts), offsets=np.stack(offsets), bucket=np.stack(buckets),
                        out=np.stack(states), **({} if sc.tri is None else {"tri": sc.tri}))


SCENES = {
    "lattice": lambda: scenes.lattice_c1(side=8),
    "pile": lambda: scenes.pile(600, seed=51, k_spring=1.0),
    "mesh_box": lambda: scenes.box_mesh_scene(),
    "mesh_funnel": lambda: scenes.funnel_wall_scene(600, seed=17, z_max=0.95, widen=False),
    "mesh_fan": lambda: scenes.fan_floor_scene(),
}


def main():
    outdir = sys.argv[1] if len(sys.argv) > 1 else HERE
    names = sys.argv[2].split(",") if len(sys.argv) > 2 else list(SCENES)
    os.makedirs(outdir, exist_ok=True)
    for name in names:
        record(SCENES[name](), name, outdir)
    print("reference CUDA fixtures written to", outdir, ":", ", ".join(names))


if __name__ == "__main__":
    main()
