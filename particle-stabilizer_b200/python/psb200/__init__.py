"""psb200 — Python binding of libparticle_stabilizer_cuda.so (ctypes).

The library is the product: C-ABI entry points declared in
include/particle_stabilizer_b200.h, every one of which runs on the GPU.  This
module only marshals numpy arrays into those calls.  There is no CPU
fallback: if the library is missing, importing `lib()` raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .scenes import Scene  # noqa: F401

PKG_ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
LIB_PATH = os.path.join(PKG_ROOT, "lib", "libparticle_stabilizer_cuda.so")
# the bounds-checked build of the same library (`make debug`); point LIB_PATH
# at it before the first lib() call to run everything through it
DEBUG_LIB_PATH = os.path.join(PKG_ROOT, "lib_debug", "libparticle_stabilizer_cuda.so")
CLI_PATH = os.path.join(PKG_ROOT, "bin", "particle_stabilizer_main")

PS_OK = 0
PS_FP32, PS_FP64 = 0, 1

# every symbol include/particle_stabilizer_b200.h declares
EXPORTED = (
    "ps_last_error", "ps_create", "ps_set_state", "ps_get_state", "ps_step", "ps_sync", "ps_stats_get",
    "ps_grid_get", "ps_buckets_get", "ps_last_launch_count", "ps_destroy", "ps_simulate",
    "ps_exclusive_scan_scratch_bytes", "ps_exclusive_scan_u32", "ps_read_csv", "ps_write_csv", "ps_read_obj",
    "ps_checkpoint_save", "ps_checkpoint_load", "ps_time_steps", "ps_profile_steps", "ps_forward_checkpointed",
    "ps_backward", "ps_exclusive_scan_u32_noalloc", "ps_exclusive_scan_u32_noalloc_status", "ps_autotune", "ps_set_contact_kernel", "ps_get_contact_kernel", "ps_set_neighbor_lists", "ps_list_stats", "ps_tune_neighbor_lists",
    "ps_resolve_overlaps", "ps_overlap_stats",
    "ps_write_obj_spheres", "ps_bounds_checked", "ps_write_state_bin", "ps_read_state_bin", "runSimulateCUDA",
)
KERNEL_KINDS = ("begin", "scan", "scatter", "rank_move", "contacts")


class SceneDesc(C.Structure):
    _fields_ = [("n_particles", C.c_int64), ("box_min", C.c_double * 3), ("box_max", C.c_double * 3),
                ("gravity", C.c_double * 3), ("e_wall", C.c_double * 6), ("k_spring", C.c_double),
                ("e_sphere", C.c_double), ("dt", C.c_double), ("cell_size", C.c_double),
                ("tri", C.POINTER(C.c_double)), ("n_tri", C.c_int64), ("edge_quirk", C.c_int32),
                ("widen_domain", C.c_int32)]


class Stats(C.Structure):
    _fields_ = [("kinetic_energy", C.c_double), ("min_pos", C.c_double * 3), ("max_pos", C.c_double * 3),
                ("n_collided", C.c_int64), ("max_overlap", C.c_double)]


class GridInfo(C.Structure):
    _fields_ = [("min", C.c_double * 3), ("interval", C.c_double), ("nb", C.c_int32 * 3), ("n_cells", C.c_int64),
                ("cell_base", C.c_int64), ("particle_base", C.c_int64)]


class Grad(C.Structure):
    _fields_ = [("k_spring", C.c_double), ("e_sphere", C.c_double), ("e_wall", C.c_double * 6)]

    def as_array(self) -> np.ndarray:
        """(k_spring, e_sphere, e_wall[0..5]) in the reference's wall order."""
        return np.array([self.k_spring, self.e_sphere, *self.e_wall])


class TuneResult(C.Structure):
    _fields_ = [("cell_factor", C.c_double), ("graph_block", C.c_int64), ("ms_per_step", C.c_double),
                ("before_ms_per_step", C.c_double), ("contact_walk", C.c_int32), ("contact_block", C.c_int32),
                ("contact_ms", C.c_double * 5)]


WALK_LANE, WALK_WARP, WALK_ADAPTIVE = 0, 1, 2
# contact kernel variants in the order of TuneResult.contact_ms: (walk, threads per CTA)
CONTACT_KERNELS = ((WALK_LANE, 128), (WALK_LANE, 256), (WALK_LANE, 512), (WALK_WARP, 256), (WALK_ADAPTIVE, 256))


class PSError(RuntimeError):
    pass


_lib = None


def declare_host(L: C.CDLL) -> None:
    """Signatures of the host-side entry points (file formats,
    post-processing, the error message): the part of the library that runs
    without a GPU, also built alone with sanitizers (make host-asan)."""
    L.ps_last_error.restype = C.c_char_p
    L.ps_read_csv.argtypes = [C.c_char_p, C.c_void_p, C.c_double, C.c_void_p, C.c_int64, C.POINTER(C.c_int64)]
    L.ps_write_csv.argtypes = [C.c_char_p, C.c_void_p, C.c_int64]
    L.ps_read_obj.argtypes = [C.c_char_p, C.c_void_p, C.c_int64, C.POINTER(C.c_int64)]
    L.ps_resolve_overlaps.argtypes = [C.c_void_p, C.c_int64, C.c_int32, C.POINTER(C.c_int64), C.POINTER(C.c_double)]
    L.ps_overlap_stats.argtypes = [C.c_void_p, C.c_int64, C.POINTER(C.c_int64), C.POINTER(C.c_double)]
    L.ps_write_obj_spheres.argtypes = [C.c_char_p, C.c_void_p, C.c_int64]
    L.ps_write_state_bin.argtypes = [C.c_char_p, C.c_void_p, C.c_int64, C.c_int64]
    L.ps_read_state_bin.argtypes = [C.c_char_p, C.c_void_p, C.c_int64, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]


def lib() -> C.CDLL:
    """Load the CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise PSError(f"{LIB_PATH} is missing: build it with `make -C particle-stabilizer_b200`")
        L = C.CDLL(LIB_PATH)
        declare_host(L)
        L.ps_bounds_checked.restype = C.c_int32
        L.ps_create.argtypes = [C.POINTER(SceneDesc), C.c_int32, C.c_int32, C.c_int32, C.POINTER(C.c_void_p)]
        L.ps_set_state.argtypes = [C.c_void_p, C.c_void_p, C.c_int64]
        L.ps_get_state.argtypes = [C.c_void_p, C.c_void_p, C.c_int64]
        L.ps_step.argtypes = [C.c_void_p, C.c_int64]
        L.ps_sync.argtypes = [C.c_void_p]
        L.ps_stats_get.argtypes = [C.c_void_p, C.c_int32, C.POINTER(Stats)]
        L.ps_grid_get.argtypes = [C.c_void_p, C.c_int32, C.POINTER(GridInfo)]
        L.ps_buckets_get.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.ps_last_launch_count.argtypes = [C.c_void_p]
        L.ps_last_launch_count.restype = C.c_int64
        L.ps_destroy.argtypes = [C.c_void_p]
        L.ps_simulate.argtypes = [C.POINTER(SceneDesc), C.c_void_p, C.c_void_p, C.c_int64, C.c_int32]
        L.ps_exclusive_scan_scratch_bytes.argtypes = [C.c_int64]
        L.ps_exclusive_scan_scratch_bytes.restype = C.c_size_t
        L.ps_exclusive_scan_u32.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p]
        L.ps_checkpoint_save.argtypes = [C.c_void_p, C.c_int32]
        L.ps_checkpoint_load.argtypes = [C.c_void_p, C.c_int32]
        L.ps_time_steps.argtypes = [C.c_void_p, C.c_int64, C.POINTER(C.c_double)]
        L.ps_profile_steps.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p]
        L.ps_forward_checkpointed.argtypes = [C.c_void_p, C.c_int64, C.c_int64]
        L.ps_backward.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.ps_exclusive_scan_u32_noalloc.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p]
        L.ps_exclusive_scan_u32_noalloc_status.argtypes = [C.c_void_p, C.POINTER(C.c_uint32)]
        L.ps_set_neighbor_lists.argtypes = [C.c_void_p, C.c_double, C.c_int32]
        L.ps_list_stats.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.ps_tune_neighbor_lists.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_int32, C.c_int32, C.c_void_p,
                                             C.c_void_p]
        L.ps_set_contact_kernel.argtypes = [C.c_void_p, C.c_int32, C.c_int32]
        L.ps_get_contact_kernel.argtypes = [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
        L.ps_autotune.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_int32, C.c_void_p, C.c_int32, C.c_void_p,
                                  C.POINTER(TuneResult)]
        _lib = L
    return _lib


def _check(rc: int, what: str) -> None:
    if rc != PS_OK:
        raise PSError(f"{what} failed ({rc}): {lib().ps_last_error().decode()}")


def _ptr(a: np.ndarray) -> C.c_void_p:
    return C.c_void_p(a.ctypes.data)


def precision_code(precision: str) -> int:
    return {"f32": PS_FP32, "fp32": PS_FP32, "f64": PS_FP64, "fp64": PS_FP64}[precision]


def scene_desc(sc: Scene, keep: list) -> SceneDesc:
    d = SceneDesc()
    d.n_particles = sc.n
    d.box_min = (C.c_double * 3)(*sc.box_min)
    d.box_max = (C.c_double * 3)(*sc.box_max)
    d.gravity = (C.c_double * 3)(*sc.gravity)
    d.e_wall = (C.c_double * 6)(*sc.e_wall)
    d.k_spring = sc.k_spring
    d.e_sphere = sc.e_sphere
    d.dt = sc.dt
    d.cell_size = sc.interval
    if sc.tri is not None:
        t = np.ascontiguousarray(sc.tri, dtype=np.float64)
        keep.append(t)
        d.tri = t.ctypes.data_as(C.POINTER(C.c_double))
        d.n_tri = t.shape[0]
    d.edge_quirk = sc.edge_quirk
    d.widen_domain = sc.widen_domain
    return d


class Simulation:
    """One or many scenes on one GPU (ps_create ... ps_destroy)."""

    def __init__(self, scenes, precision: str = "f32", device: int = 0):
        if isinstance(scenes, Scene):
            scenes = [scenes]
        self.scenes = list(scenes)
        keep: list = []
        arr = (SceneDesc * len(self.scenes))(*[scene_desc(s, keep) for s in self.scenes])
        h = C.c_void_p()
        _check(lib().ps_create(arr, len(self.scenes), precision_code(precision), device, C.byref(h)), "ps_create")
        self.h = h
        self.n = sum(s.n for s in self.scenes)
        self.precision = precision

    def set_state(self, state: np.ndarray | None = None) -> None:
        if state is None:
            state = np.concatenate([s.state for s in self.scenes]) if self.n else np.zeros((0, 8))
        st = np.ascontiguousarray(state, dtype=np.float64)
        _check(lib().ps_set_state(self.h, _ptr(st), st.shape[0]), "ps_set_state")

    def get_state(self, out: np.ndarray | None = None) -> np.ndarray:
        """The state in original order, (n, 8) float64; `out` may be a
        C-contiguous (n, 8) float64 buffer (for example in pinned memory)."""
        if out is None:
            out = np.empty((self.n, 8), dtype=np.float64)
        if out.shape != (self.n, 8) or out.dtype != np.float64 or not out.flags.c_contiguous:
            raise ValueError("out must be a C-contiguous (n, 8) float64 array")
        _check(lib().ps_get_state(self.h, _ptr(out), self.n), "ps_get_state")
        return out

    def step(self, n_steps: int) -> None:
        _check(lib().ps_step(self.h, int(n_steps)), "ps_step")

    def sync(self) -> None:
        _check(lib().ps_sync(self.h), "ps_sync")

    def launches(self) -> int:
        return int(lib().ps_last_launch_count(self.h))

    def checkpoint_save(self, slot: int = 0) -> None:
        _check(lib().ps_checkpoint_save(self.h, slot), "ps_checkpoint_save")

    def checkpoint_load(self, slot: int = 0) -> None:
        _check(lib().ps_checkpoint_load(self.h, slot), "ps_checkpoint_load")

    def time_steps(self, n_steps: int) -> float:
        """Device milliseconds of ps_step(n_steps), CUDA events on the simulation's stream."""
        ms = C.c_double()
        _check(lib().ps_time_steps(self.h, int(n_steps), C.byref(ms)), "ps_time_steps")
        return float(ms.value)

    def profile_steps(self, n_steps: int) -> dict:
        """Per kernel kind: (summed device ms, launches) over n_steps eager steps."""
        ms = np.zeros(len(KERNEL_KINDS), dtype=np.float64)
        cnt = np.zeros(len(KERNEL_KINDS), dtype=np.int64)
        _check(lib().ps_profile_steps(self.h, int(n_steps), _ptr(ms), _ptr(cnt)), "ps_profile_steps")
        return {k: (float(ms[i]), int(cnt[i])) for i, k in enumerate(KERNEL_KINDS)}

    def stats(self, scene: int = 0) -> Stats:
        s = Stats()
        _check(lib().ps_stats_get(self.h, scene, C.byref(s)), "ps_stats_get")
        return s

    def grid(self, scene: int = 0) -> GridInfo:
        g = GridInfo()
        _check(lib().ps_grid_get(self.h, scene, C.byref(g)), "ps_grid_get")
        return g

    def buckets(self):
        """(counts, offsets, order) over all cells / particles of all scenes."""
        total = 0
        for k in range(len(self.scenes)):
            g = self.grid(k)
            total = max(total, g.cell_base + g.n_cells)
        counts = np.empty(total, dtype=np.uint32)
        offsets = np.empty(total, dtype=np.uint32)
        order = np.empty(self.n, dtype=np.uint32)
        _check(lib().ps_buckets_get(self.h, _ptr(counts), _ptr(offsets), _ptr(order)), "ps_buckets_get")
        return counts, offsets, order

    def forward_checkpointed(self, n_steps: int, every: int) -> None:
        """Advance n_steps keeping a checkpoint every `every` steps (for backward)."""
        _check(lib().ps_forward_checkpointed(self.h, int(n_steps), int(every)), "ps_forward_checkpointed")

    def set_neighbor_lists(self, skin_fraction: float = 0.3, max_neighbours: int = 48) -> None:
        """Neighbour-list mode (ps_set_neighbor_lists); 0 switches it off."""
        _check(lib().ps_set_neighbor_lists(self.h, float(skin_fraction), int(max_neighbours)),
               "ps_set_neighbor_lists")

    def list_stats(self) -> tuple[int, int]:
        """(rebuilds, fallbacks) since set_neighbor_lists (ps_list_stats)."""
        return self.list_stats_all()[:2]

    def list_stats_all(self) -> tuple[int, int, int]:
        """(rebuilds, fallbacks, steps run on the grid path by the backoff)."""
        r, f, g = C.c_int64(), C.c_int64(), C.c_int64()
        _check(lib().ps_list_stats(self.h, C.byref(r), C.byref(f), C.byref(g)), "ps_list_stats")
        return int(r.value), int(f.value), int(g.value)

    def tune_neighbor_lists(self, trial_steps: int = 100, skins=(0.0, 0.02, 0.05, 0.1, 0.2),
                            max_neighbours: int = 64) -> dict:
        """ps_tune_neighbor_lists: the fastest skin fraction (0 = grid path)."""
        sk = np.ascontiguousarray(skins, dtype=np.float64)
        table = np.zeros(len(sk), dtype=np.float64)
        best = C.c_double()
        _check(lib().ps_tune_neighbor_lists(self.h, int(trial_steps), _ptr(sk), len(sk), int(max_neighbours),
                                            _ptr(table), C.byref(best)), "ps_tune_neighbor_lists")
        return {"skin_fraction": float(best.value), "skins": [float(x) for x in sk], "ms_table": table.tolist()}

    def list_fallbacks(self) -> int:
        """ps_step calls repeated on the grid path after a list overflow."""
        return self.list_stats()[1]

    def autotune(self, trial_steps: int = 20, cell_factors=(1.0, 1.05, 1.25, 1.5, 2.0),
                 graph_blocks=(50, 100, 200)) -> dict:
        """Time `trial_steps` steps from the current state for every cell-size
        factor (cell edge = factor * 2 * r_max per scene) and graph block
        length, keep the fastest pair and restore the state (ps_autotune)."""
        f = np.ascontiguousarray(cell_factors, dtype=np.float64)
        b = np.ascontiguousarray(graph_blocks, dtype=np.int64)
        table = np.zeros((f.size, b.size), dtype=np.float64)
        res = TuneResult()
        _check(lib().ps_autotune(self.h, int(trial_steps), _ptr(f), int(f.size), _ptr(b), int(b.size), _ptr(table),
                                 C.byref(res)), "ps_autotune")
        return {"cell_factor": res.cell_factor, "graph_block": int(res.graph_block),
                "ms_per_step": res.ms_per_step, "before_ms_per_step": res.before_ms_per_step,
                "cell_factors": [float(x) for x in f], "graph_blocks": [int(x) for x in b],
                "ms_table": table.tolist(), "contact_kernel": (int(res.contact_walk), int(res.contact_block)),
                "contact_ms": [float(x) for x in res.contact_ms], "contact_kernels": list(CONTACT_KERNELS)}

    def set_contact_kernel(self, walk: int, block: int) -> None:
        """ps_set_contact_kernel: WALK_LANE with 128, 256 or 512 threads per
        CTA, or WALK_WARP or WALK_ADAPTIVE with 256 (identical results)."""
        _check(lib().ps_set_contact_kernel(self.h, int(walk), int(block)), "ps_set_contact_kernel")

    def contact_kernel(self) -> tuple[int, int]:
        w, b = C.c_int32(), C.c_int32()
        _check(lib().ps_get_contact_kernel(self.h, C.byref(w), C.byref(b)), "ps_get_contact_kernel")
        return int(w.value), int(b.value)

    def backward(self, dl_dstate: np.ndarray):
        """Gradients of a loss of the final state: dl_dstate is (n, 6) =
        dL/d(x, y, z, vx, vy, vz).  Returns (per-scene (8,) arrays of
        dL/d(k_spring, e_sphere, e_wall[6]), dL/d(initial state) (n, 6))."""
        g = np.ascontiguousarray(dl_dstate, dtype=np.float64)
        grads = (Grad * len(self.scenes))()
        out = np.empty((self.n, 6), dtype=np.float64)
        _check(lib().ps_backward(self.h, _ptr(g), grads, _ptr(out)), "ps_backward")
        return [gr.as_array() for gr in grads], out

    def close(self) -> None:
        if getattr(self, "h", None):
            lib().ps_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def height_loss(state: np.ndarray, h0: float = 0.1, amp: float = 0.02, wavelength: float = 0.5):
    """Settling loss mean_i (z_i - h(x_i))^2, h(x) = h0 + amp sin(2 pi x / wavelength),
    and its gradient with respect to the state (n, 6)."""
    x, z = state[:, 0], state[:, 2]
    w = 2.0 * np.pi / wavelength
    r = z - (h0 + amp * np.sin(w * x))
    n = state.shape[0]
    g = np.zeros((n, 6))
    g[:, 2] = 2.0 * r / n
    g[:, 0] = -2.0 * r * amp * w * np.cos(w * x) / n
    return float(np.mean(r * r)), g


def simulate(scene: Scene, steps: int, precision: str = "f32") -> np.ndarray:
    """ps_simulate: runSimulateCUDA with host buffers."""
    keep: list = []
    d = scene_desc(scene, keep)
    st = np.ascontiguousarray(scene.state, dtype=np.float64)
    out = np.empty_like(st)
    _check(lib().ps_simulate(C.byref(d), _ptr(st), _ptr(out), int(steps), precision_code(precision)), "ps_simulate")
    return out


def exclusive_scan_u32(d_in: int, d_out: int, n: int, d_scratch: int, stream: int = 0) -> None:
    """ps_exclusive_scan_u32 on device pointers (integers)."""
    _check(lib().ps_exclusive_scan_u32(C.c_void_p(d_in), C.c_void_p(d_out), int(n), C.c_void_p(d_scratch),
                                       C.c_void_p(stream)), "ps_exclusive_scan_u32")


SCAN_NOALLOC_MAX_N = 134217728


def exclusive_scan_u32_noalloc(d_in: int, d_out: int, n: int, stream: int = 0) -> None:
    """ps_exclusive_scan_u32_noalloc on device pointers: the scan without any
    allocation, using the library's fixed scratch array (n <= SCAN_NOALLOC_MAX_N)."""
    _check(lib().ps_exclusive_scan_u32_noalloc(C.c_void_p(d_in), C.c_void_p(d_out), int(n), C.c_void_p(stream)),
           "ps_exclusive_scan_u32_noalloc")


def exclusive_scan_u32_noalloc_status(stream: int = 0) -> int:
    """ps_exclusive_scan_u32_noalloc_status: the device error bits of the
    no-allocation scans since the last query (0 = all complete), cleared."""
    w = C.c_uint32()
    _check(lib().ps_exclusive_scan_u32_noalloc_status(C.c_void_p(stream), C.byref(w)),
           "ps_exclusive_scan_u32_noalloc_status")
    return int(w.value)


def bounds_checked() -> bool:
    """ps_bounds_checked: True when the loaded library is the bounds-checked
    build, whose out-of-range device indexes are skipped and reported as
    PS_ERR_DEVICE instead of faulting."""
    return bool(lib().ps_bounds_checked())


def exclusive_scan_scratch_bytes(n: int) -> int:
    return int(lib().ps_exclusive_scan_scratch_bytes(int(n)))


def read_csv(path: str, velocity=(0.0, 0.0, -10.0), density: float = 1.0) -> np.ndarray:
    n = C.c_int64()
    v = (C.c_double * 3)(*velocity)
    _check(lib().ps_read_csv(path.encode(), v, density, None, 0, C.byref(n)), "ps_read_csv")
    out = np.empty((n.value, 8), dtype=np.float64)
    _check(lib().ps_read_csv(path.encode(), v, density, _ptr(out), n.value, C.byref(n)), "ps_read_csv")
    return out


def write_csv(path: str, state: np.ndarray) -> None:
    st = np.ascontiguousarray(state, dtype=np.float64)
    _check(lib().ps_write_csv(path.encode(), _ptr(st), st.shape[0]), "ps_write_csv")


def write_state_bin(path: str, state: np.ndarray, steps: int = 0) -> None:
    """ps_write_state_bin: every particle record (n x 8) and the step count."""
    st = np.ascontiguousarray(state, dtype=np.float64)
    _check(lib().ps_write_state_bin(path.encode(), _ptr(st), st.shape[0], int(steps)), "ps_write_state_bin")


def read_state_bin(path: str):
    """ps_read_state_bin: (state n x 8, step count)."""
    n, steps = C.c_int64(), C.c_int64()
    _check(lib().ps_read_state_bin(path.encode(), None, 0, C.byref(n), C.byref(steps)), "ps_read_state_bin")
    out = np.empty((n.value, 8), dtype=np.float64)
    _check(lib().ps_read_state_bin(path.encode(), _ptr(out), n.value, C.byref(n), C.byref(steps)),
           "ps_read_state_bin")
    return out, int(steps.value)


def read_obj(path: str) -> np.ndarray:
    n = C.c_int64()
    _check(lib().ps_read_obj(path.encode(), None, 0, C.byref(n)), "ps_read_obj")
    out = np.empty((n.value, 9), dtype=np.float64)
    _check(lib().ps_read_obj(path.encode(), _ptr(out), n.value, C.byref(n)), "ps_read_obj")
    return out


# ---- after the path (host code in the library) --------------------------------
def resolve_overlaps(state: np.ndarray, axis: int = 2):
    """ParticleModel::resolveOverlaps on a copy of `state` (n x 8 records):
    returns (new state, particles still overlapping a higher index, largest
    remaining overlap)."""
    st = np.array(state, dtype=np.float64, order="C", copy=True)
    nc = C.c_int64()
    mo = C.c_double()
    _check(lib().ps_resolve_overlaps(_ptr(st), st.shape[0], int(axis), C.byref(nc), C.byref(mo)),
           "ps_resolve_overlaps")
    return st, int(nc.value), float(mo.value)


def overlap_stats(state: np.ndarray):
    """(particles overlapping a higher-indexed particle, largest overlap)."""
    st = np.ascontiguousarray(state, dtype=np.float64)
    nc = C.c_int64()
    mo = C.c_double()
    _check(lib().ps_overlap_stats(_ptr(st), st.shape[0], C.byref(nc), C.byref(mo)), "ps_overlap_stats")
    return int(nc.value), float(mo.value)


def write_obj_spheres(path: str, state: np.ndarray) -> None:
    """ObjData::write: every particle as a triangulated sphere."""
    st = np.ascontiguousarray(state, dtype=np.float64)
    _check(lib().ps_write_obj_spheres(path.encode(), _ptr(st), st.shape[0]), "ps_write_obj_spheres")
