"""ctypes binding of the C oracle and of the reference builds under oracle/_ref.

TEST INFRASTRUCTURE: imported only by tests/, __graft_entry__.smoke() and
bench.py's cpu_baseline / reference legs, to check results.  The product path
never imports this module.

State arrays are (n, 8) in the reference's ParticlePrimitive layout
(include/ParticleStabilizer/ParticleModel.hpp:7-25): x, y, z, vx, vy, vz,
radius, mass; float64 for the FP64 scheme and the reference builds, float32
for the FP32 scheme.
"""
from __future__ import annotations

import ctypes as C
import os
import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# PS_ORACLE_SO selects another build of the same sources (the sanitizer
# build, oracle/_build_asan/, in tests/test_cpu_sanitizers.py)
ORACLE_SO = os.environ.get("PS_ORACLE_SO") or os.path.join(HERE, "_build", "libps_oracle.so")
REF_CPU_SO = os.path.join(HERE, "_ref", "libref_cpu.so")
REF_CUDA_SO = os.path.join(HERE, "_ref", "libref_cuda.so")

# wall restitution order of the reference (ContainerBase.hpp:10-34)
ZMIN, ZMAX, XMIN, XMAX, YMIN, YMAX = range(6)


class OrGrid(C.Structure):
    _fields_ = [("min", C.c_double * 3), ("max", C.c_double * 3), ("interval", C.c_double),
                ("nb", C.c_int32 * 3), ("n_cells", C.c_int64)]


class OrParams(C.Structure):
    _fields_ = [("box_min", C.c_double * 3), ("box_max", C.c_double * 3), ("gravity", C.c_double * 3),
                ("e_wall", C.c_double * 6), ("k_spring", C.c_double), ("e_sphere", C.c_double),
                ("dt", C.c_double), ("tri", C.POINTER(C.c_double)), ("n_tri", C.c_int64),
                ("e_poly", C.c_double), ("edge_quirk", C.c_int32), ("cpu_semantics", C.c_int32),
                ("grid", OrGrid)]


class OrStats(C.Structure):
    _fields_ = [("kinetic_energy", C.c_double), ("min_pos", C.c_double * 3), ("max_pos", C.c_double * 3),
                ("n_collided", C.c_int64), ("max_overlap", C.c_double)]


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            raise RuntimeError(f"oracle library missing: {ORACLE_SO} (run `make -C oracle`)")
        _lib = C.CDLL(ORACLE_SO)
        _lib.or_interval_cuda.restype = C.c_double
        _lib.or_interval_cpu.restype = C.c_double
        _lib.or_run_f64.restype = C.c_int32
        _lib.or_run_f32.restype = C.c_int32
    return _lib


def _p(a: np.ndarray) -> C.c_void_p:
    return C.c_void_p(a.ctypes.data)


def _d3(v) -> C.Array:
    return (C.c_double * 3)(*[float(x) for x in v])


# A scene is any object with the attributes of psb200.scenes.Scene: state,
# box_min, box_max, gravity, e_wall, k_spring, e_sphere, dt, tri, interval,
# edge_quirk, widen_domain, and the methods n, r_max(), domain().


def grid_for(scene: Scene, cpu_semantics: bool = False) -> OrGrid:
    L = lib()
    if scene.interval > 0:
        iv = scene.interval
    elif cpu_semantics:
        iv = L.or_interval_cpu(C.c_double(scene.r_max()))
    else:
        iv = L.or_interval_cuda(C.c_double(scene.r_max()))
    lo, hi = scene.domain()
    g = OrGrid()
    L.or_grid_init(_d3(lo), _d3(hi), C.c_double(iv), C.byref(g))
    return g


def params_for(scene: Scene, cpu_semantics: bool = False) -> tuple[OrParams, object]:
    prm = OrParams()
    prm.box_min = _d3(scene.box_min)
    prm.box_max = _d3(scene.box_max)
    prm.gravity = _d3(scene.gravity)
    prm.e_wall = (C.c_double * 6)(*scene.e_wall)
    prm.k_spring = scene.k_spring
    prm.e_sphere = scene.e_sphere
    prm.dt = scene.dt
    keep = None
    if scene.tri is not None:
        keep = np.ascontiguousarray(scene.tri, dtype=np.float64)
        prm.tri = keep.ctypes.data_as(C.POINTER(C.c_double))
        prm.n_tri = keep.shape[0]
    prm.e_poly = scene.e_wall[ZMIN]
    prm.edge_quirk = scene.edge_quirk
    prm.cpu_semantics = 1 if cpu_semantics else 0
    prm.grid = grid_for(scene, cpu_semantics)
    return prm, keep


def run(scene: Scene, steps: int, precision: str = "f64", cpu_semantics: bool = False) -> np.ndarray:
    """Advance a copy of scene.state by `steps` oracle steps."""
    prm, keep = params_for(scene, cpu_semantics)
    if precision == "f64":
        st = np.ascontiguousarray(scene.state, dtype=np.float64).copy()
        rc = lib().or_run_f64(_p(st), C.c_int64(scene.n), C.byref(prm), C.c_int64(steps))
    else:
        if cpu_semantics:
            raise ValueError("the CPU simulator is FP64 only")
        st = np.ascontiguousarray(scene.state, dtype=np.float32).copy()
        rc = lib().or_run_f32(_p(st), C.c_int64(scene.n), C.byref(prm), C.c_int64(steps))
    del keep
    if rc != 0:
        raise RuntimeError(f"oracle run failed: {rc}")
    return st


def run_dual(scene, steps: int, dparam: np.ndarray, dstate0: np.ndarray):
    """Forward-mode FP64 run: returns (state, tangents) with tangents of
    shape (nd, n, 6) for the parameter tangents dparam (nd, 8) = (k_spring,
    e_sphere, e_wall[6]) and initial state tangents dstate0 (nd, n, 6)."""
    prm, keep = params_for(scene)
    st = np.ascontiguousarray(scene.state, dtype=np.float64).copy()
    dp = np.ascontiguousarray(dparam, dtype=np.float64)
    ds = np.ascontiguousarray(dstate0, dtype=np.float64).copy()
    lib().or_run_dual_f64.restype = C.c_int32
    rc = lib().or_run_dual_f64(_p(st), C.c_int64(scene.n), C.byref(prm), C.c_int64(steps), C.c_int32(dp.shape[0]),
                               _p(dp), _p(ds))
    del keep
    if rc != 0:
        raise RuntimeError(f"oracle dual run failed: {rc}")
    return st, ds


def cell_ids(state: np.ndarray, grid: OrGrid, clamp: bool = True) -> np.ndarray:
    st = np.ascontiguousarray(state)
    out = np.empty(st.shape[0], dtype=np.int64)
    fn = lib().or_cell_ids_f64 if st.dtype == np.float64 else lib().or_cell_ids_f32
    fn(_p(st), C.c_int64(st.shape[0]), C.byref(grid), C.c_int32(1 if clamp else 0), _p(out))
    return out


def count_scan_order(cell: np.ndarray, n_cells: int):
    """Per-cell counts, exclusive offsets (n_cells+1 entries) and the
    canonical register order for the given cell ids."""
    cell = np.ascontiguousarray(cell, dtype=np.int64)
    n = cell.shape[0]
    count = np.zeros(n_cells + 1, dtype=np.uint32)
    lib().or_count(_p(cell), C.c_int64(n), C.c_int64(n_cells), _p(count))
    count[n_cells] = 0
    offset = np.empty(n_cells + 1, dtype=np.uint32)
    lib().or_exclusive_scan(_p(count), C.c_int64(n_cells + 1), _p(offset))
    order = np.empty(n, dtype=np.uint32)
    lib().or_stable_order(_p(cell), C.c_int64(n), _p(offset), C.c_int64(n_cells), _p(order))
    return count[:n_cells], offset, order


def exclusive_scan(a: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.uint32)
    out = np.empty_like(a)
    lib().or_exclusive_scan(_p(a), C.c_int64(a.shape[0]), _p(out))
    return out


def stats(state: np.ndarray) -> OrStats:
    st = np.ascontiguousarray(state, dtype=np.float64)
    s = OrStats()
    lib().or_stats_f64(_p(st), C.c_int64(st.shape[0]), C.byref(s))
    return s


# ---- the reference's own builds (oracle/_ref) ------------------------------
class _RefLib:
    def __init__(self, path: str, prefix: str):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = C.CDLL(path)
        self.prefix = prefix
        f = getattr(self.lib, prefix + "create")
        f.restype = C.c_void_p
        f.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_char_p, C.c_void_p, C.c_void_p,
                      C.c_double, C.c_double, C.c_double]
        for name in ("step", "get_state", "destroy", "time_steps"):
            getattr(self.lib, prefix + name).argtypes = [C.c_void_p] + (
                [C.c_int64] if name in ("step", "time_steps") else [C.c_void_p] if name == "get_state" else [])
        getattr(self.lib, prefix + "time_steps").restype = C.c_double

    def create(self, scene: Scene, obj_path: str | None = None):
        st = np.ascontiguousarray(scene.state, dtype=np.float64)
        h = getattr(self.lib, self.prefix + "create")(
            _p(st), scene.n, _d3(scene.box_min), _d3(scene.box_max),
            (obj_path or "").encode(), _d3(scene.gravity), (C.c_double * 6)(*scene.e_wall),
            scene.k_spring, scene.e_sphere, scene.dt)
        if not h:
            raise ValueError("reference harness rejected the scene")
        return C.c_void_p(h)

    def step(self, h, steps: int):
        getattr(self.lib, self.prefix + "step")(h, steps)

    def time_steps(self, h, steps: int) -> float:
        return float(getattr(self.lib, self.prefix + "time_steps")(h, steps))

    def state(self, h, n: int) -> np.ndarray:
        out = np.empty((n, 8), dtype=np.float64)
        getattr(self.lib, self.prefix + "get_state")(h, _p(out))
        return out

    def destroy(self, h):
        getattr(self.lib, self.prefix + "destroy")(h)


def ref_cpu() -> _RefLib:
    r = _RefLib(REF_CPU_SO, "refh_")
    r.lib.refh_read_csv.restype = C.c_int64
    r.lib.refh_read_csv.argtypes = [C.c_char_p, C.c_void_p, C.c_double, C.c_void_p, C.c_int64]
    r.lib.refh_write_csv.argtypes = [C.c_void_p, C.c_int64, C.c_char_p]
    r.lib.refh_read_obj.restype = C.c_int64
    r.lib.refh_read_obj.argtypes = [C.c_char_p, C.c_void_p, C.c_int64]
    r.lib.refh_resolve_overlaps.argtypes = [C.c_void_p, C.c_int64, C.c_int32]
    r.lib.refh_write_obj.argtypes = [C.c_char_p, C.c_void_p, C.c_int64]
    return r


def ref_resolve_overlaps(state: np.ndarray, axis: int) -> np.ndarray:
    """The reference's own ParticleModel::resolveOverlaps on a copy of state."""
    st = np.array(state, dtype=np.float64, order="C", copy=True)
    ref_cpu().lib.refh_resolve_overlaps(_p(st), st.shape[0], int(axis))
    return st


def ref_write_obj(path: str, state: np.ndarray) -> None:
    """The reference's own ObjData::write."""
    st = np.ascontiguousarray(state, dtype=np.float64)
    ref_cpu().lib.refh_write_obj(path.encode(), _p(st), st.shape[0])


def ref_cuda() -> _RefLib:
    r = _RefLib(REF_CUDA_SO, "refc_")
    r.lib.refc_get_grid.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    r.lib.refc_get_buckets.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    return r


def run_reference(which: str, scene: Scene, steps: int, obj_path: str | None = None) -> np.ndarray:
    r = ref_cpu() if which == "cpu" else ref_cuda()
    h = r.create(scene, obj_path)
    try:
        r.step(h, steps)
        return r.state(h, scene.n)
    finally:
        r.destroy(h)


def pre_grid_state(scene, state: np.ndarray, precision: str = "f64") -> np.ndarray:
    """State at the grid rebuild of one CUDA-scheme step: integrate, then the
    box walls (or the triangle container)."""
    st = np.ascontiguousarray(state, dtype=np.float64 if precision == "f64" else np.float32).copy()
    n = st.shape[0]
    L = lib()
    if precision == "f64":
        L.or_integrate_f64(_p(st), C.c_int64(n), _d3(scene.gravity), C.c_double(scene.dt), C.c_int32(0))
    else:
        L.or_integrate_f32(_p(st), C.c_int64(n), _d3(scene.gravity), C.c_double(scene.dt))
    if scene.tri is not None:
        t = np.ascontiguousarray(scene.tri, dtype=np.float64)
        if precision == "f64":
            L.or_mesh_f64(_p(st), C.c_int64(n), _p(t), C.c_int64(t.shape[0]), C.c_double(scene.e_wall[ZMIN]),
                          C.c_int32(scene.edge_quirk), C.c_int32(0))
        else:
            L.or_mesh_f32(_p(st), C.c_int64(n), _p(t), C.c_int64(t.shape[0]), C.c_double(scene.e_wall[ZMIN]),
                          C.c_int32(scene.edge_quirk))
    else:
        fn = L.or_walls_f64 if precision == "f64" else L.or_walls_f32
        fn(_p(st), C.c_int64(n), _d3(scene.box_min), _d3(scene.box_max), (C.c_double * 6)(*scene.e_wall))
    return st
