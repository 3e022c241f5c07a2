// ps_engine.cu — host engine and C ABI of libparticle_stabilizer_cuda.so.
//
// Owns the device state of one or many scenes, sizes their grids
// (ParticleModelCUDA::initBuckets, src/ParticleStabilizerCUDA/ParticleModelCUDA.cpp:62-113),
// bins container triangles, and issues blocks of steps as CUDA graphs on a
// private stream.  The step sequence replaces the host loop of
// PhysicsEngineCUDA::startSimulationLoop (PhysicsEngineCUDA.cpp:33-76), which
// synchronises the device after every one of its 7+ launches per step.
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "particle_stabilizer_b200.h"
#include "ps_adjoint.cuh"
#include "ps_lists.cuh"
#include "ps_scan.cuh"
#include "ps_stats.cuh"
#include "ps_step_kernels.cuh"

using namespace psb;

// ---- error reporting ---------------------------------------------------------
// The per-thread message behind ps_last_error() lives in host/ps_errors.cpp.
extern "C" int ps_internal_fail(int code, const char* msg);

// A runtime call that failed (an allocation the device cannot serve, say)
// also leaves its error as this thread's "last error", which the next
// cudaGetLastError returns: a later, unrelated call would report it again.
// Reporting a CUDA failure therefore clears it (errors that break the
// context stay sticky and keep being reported by the runtime itself).
static int fail(int code, const std::string& msg) {
  if (code == PS_ERR_CUDA || code == PS_ERR_NOMEM) (void)cudaGetLastError();
  return ps_internal_fail(code, msg.c_str());
}

#define PS_CUDA(expr)                                                                        \
  do {                                                                                       \
    cudaError_t e_ = (expr);                                                                 \
    if (e_ != cudaSuccess)                                                                   \
      return fail(e_ == cudaErrorMemoryAllocation ? PS_ERR_NOMEM : PS_ERR_CUDA,             \
                  std::string(#expr) + ": " + cudaGetErrorString(e_));                      \
  } while (0)


extern "C" int32_t ps_bounds_checked(void) {
#ifdef PS_DEBUG_BOUNDS
  return 1;
#else
  return 0;
#endif
}

namespace {
// NVTX range around an entry point, so a profiler's timeline shows the
// library's calls (no cost without an attached tool: NVTX is header-only and
// loads its back end only when one is present).
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};
}  // namespace


namespace {

// Restores the caller's current device on scope exit.
struct DeviceGuard {
  int prev = -1;
  bool ok = false;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) == cudaSuccess && cudaSetDevice(dev) == cudaSuccess) ok = true;
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

struct GridHost {
  double min[3], max[3], interval;
  int32_t nb[3];
  int64_t n_cells, cbase;
  // triangle bins
  double mesh_lo[3], mesh_hi[3], mesh_iv;
  int32_t mesh_nb[3];
  int64_t n_bins, bin_base, tri_base, n_tri;
};

size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

}  // namespace

struct ps_sim {
  int precision = PS_FP32;
  int device = 0;
  cudaStream_t stream = nullptr;
  int n_scenes = 0;
  std::vector<ps_scene_desc> desc;
  std::vector<std::vector<double>> tris;  // owned copies of the triangle soups
  std::vector<int64_t> pbase;             // n_scenes + 1
  int64_t n_total = 0;
  bool multi = false, has_mesh = false;

  // grids (sized on the first ps_set_state)
  bool grid_sized = false, grid_valid = false, stepped = false;
  std::vector<GridHost> grids;
  int64_t c_total = 0, bins_total = 0, tri_total = 0;

  // device memory
  void* part_arena = nullptr;
  void* cell_arena = nullptr;
  void *P0 = nullptr, *V0 = nullptr, *P1 = nullptr, *V1 = nullptr;
  uint32_t *orig = nullptr, *cell = nullptr, *slot = nullptr, *tmp = nullptr, *scell = nullptr;
  uint32_t *count = nullptr, *offset = nullptr, *err = nullptr, *d_pbase = nullptr;
  double* d_interval = nullptr;  // cell edge of each scene, for the device-side upload check
  uint32_t* tile_sum = nullptr;  // per-tile totals of `count` for the step's scan
  void* d_bounds = nullptr;       // per-scene, per-axis cell boundaries in the state precision
  double* staging = nullptr;  // n_total x 8 doubles
  void* d_scenes = nullptr;
  StatsPartial* d_stats = nullptr;
  StatsPartial* d_stats_out = nullptr;
  // triangle data
  void *d_tri = nullptr, *d_nrm = nullptr, *d_aabb = nullptr;
  uint32_t *d_bin_offset = nullptr, *d_bin_tri = nullptr;
  MeshView* d_mesh_view = nullptr;

  std::vector<SceneParams<float>> sp32;
  std::vector<SceneParams<double>> sp64;

  std::map<int64_t, cudaGraphExec_t> graphs;
  int64_t graph_block = 200;  // steps per captured CUDA graph (ps_autotune may change it)
  int32_t walk = WALK_ADAPTIVE;  // neighbour walk of the contact kernel (WALK_LANE / WALK_WARP / WALK_ADAPTIVE)
  int32_t contact_block = 256;    // threads per CTA of the contact kernel (WALK_LANE: 128, 256, 512; others: 256)
  int64_t last_launches = 0;
  std::map<int32_t, void*> checkpoints;  // slot -> device copy of (P0, V1, orig)
  cudaAccessPolicyWindow l2_window{};     // count + offset arrays kept in L2
  bool l2_window_on = false;
  size_t l2_limit = 0;                    // persisting set-aside this simulation wants
  size_t l2_prev_limit = 0;               // the context's set-aside before this simulation changed it
  bool l2_limit_set = false;
  // differentiation
  int64_t fwd_steps = 0, fwd_every = 0;   // last ps_forward_checkpointed
  std::vector<void*> fwd_ckpt;            // state at the start of each block, + final state last
  void* adj_arena = nullptr;              // tape, adjoint arrays, partials
  size_t adj_bytes = 0;
  // neighbour-list mode (ps_set_neighbor_lists); off when list_skin <= 0
  double list_skin = 0.0;                 // skin as a fraction of the cell edge
  int32_t list_cap = 0;                   // list capacity per sphere
  void* list_arena = nullptr;
  size_t list_bytes = 0;
  void* list_ckpt = nullptr;              // state at the start of a list-mode call
  int64_t list_fallbacks = 0;             // calls repeated on the grid path after an overflow
  int64_t list_rebuilds = 0;              // grid + list rebuilds requested by the device
  int64_t list_grid_steps = 0;            // list-mode steps run on the grid path (backoff)
  // backoff: a window of list steps that rebuilt more than once per
  // LIST_BACKOFF_RATE steps sends the next `list_backoff` steps to the grid path
  int64_t list_win_steps = 0, list_win_rebuilds = 0, list_backoff = 0, list_backoff_len = 0;
  unsigned list_rebuild_grid = 0;         // CTAs of the cooperative rebuild (one wave)
  unsigned list_step_grid = 0;            // CTAs of the list step kernel (one wave)
};

namespace {


int64_t n_scan(const ps_sim* s) { return s->c_total + 1; }

// Launch with programmatic stream serialization: the kernel may start while
// its predecessor on the stream drains; it waits (griddepcontrol.wait, a
// no-op for a normal launch) before reading anything the predecessor wrote.
template <typename... KArgs, typename... Args>
void pdl_launch(void (*k)(KArgs...), unsigned g, unsigned blk, cudaStream_t st, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(g);
  cfg.blockDim = dim3(blk);
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, k, args...);
}

// The step scan for this simulation's grid size (tile of 2,048 or 8,192 cells).
using StepScanFn = void (*)(const uint32_t*, uint32_t*, int64_t, const uint32_t*);
StepScanFn step_scan_kernel(int64_t n) {
  return step_scan_items(n) == STEP_SCAN_ITEMS_LARGE ? k_scan_with_tile_sums<STEP_SCAN_ITEMS_LARGE>
                                                    : k_scan_with_tile_sums<STEP_SCAN_ITEMS_SMALL>;
}

template <class T>
StepBufs<T> bufs(ps_sim* s) {
  StepBufs<T> b;
  b.P0 = static_cast<vec4_t<T>*>(s->P0);
  b.V0 = static_cast<vec4_t<T>*>(s->V0);
  b.P1 = static_cast<vec4_t<T>*>(s->P1);
  b.V1 = static_cast<vec4_t<T>*>(s->V1);
  b.orig = s->orig;
  b.cell = s->cell;
  b.slot = s->slot;
  b.tmp = s->tmp;
  b.count = s->count;
  b.offset = s->offset;
  b.err = s->err;
  b.scenes = static_cast<const SceneParams<T>*>(s->d_scenes);
  b.pbase = s->d_pbase;
  b.n_scenes = s->n_scenes;
  b.n = (uint32_t)s->n_total;
  b.tile_sum = s->tile_sum;
  b.scell = s->scell;
  b.bounds = static_cast<const T*>(s->d_bounds);
  b.n_tiles = (uint32_t)step_scan_tiles(n_scan(s));
  b.tile_shift = step_scan_shift(n_scan(s));
  b.n_scan = (uint32_t)n_scan(s);
  b.tape_p = nullptr;
  b.tape_v = nullptr;
  b.tape_vpre = nullptr;
  b.tape_o = nullptr;
  b.tape_cell = nullptr;
  return b;
}

template <class T>
const std::vector<SceneParams<T>>& params(const ps_sim* s);
template <>
const std::vector<SceneParams<float>>& params<float>(const ps_sim* s) {
  return s->sp32;
}
template <>
const std::vector<SceneParams<double>>& params<double>(const ps_sim* s) {
  return s->sp64;
}

unsigned blocks_for(int64_t n) { return (unsigned)((n + STEP_THREADS - 1) / STEP_THREADS); }
// grid of k_scatter / k_rank_move: MOVE_PER_THREAD particles per thread, and
// at least one thread per scan-scratch word
unsigned move_blocks(int64_t n, uint32_t words) {
  const int64_t per = (int64_t)STEP_THREADS * MOVE_PER_THREAD;
  return (unsigned)std::max<int64_t>((n + per - 1) / per, (words + STEP_THREADS - 1) / STEP_THREADS);
}

static_assert(WALK_LANE == PS_WALK_LANE && WALK_WARP == PS_WALK_WARP && WALK_ADAPTIVE == PS_WALK_ADAPTIVE,
              "walk ids of the C ABI");

// Contact kernel variants the tuner times: {walk, threads per CTA}, in the
// order of ps_tune_result::contact_ms.
constexpr int kContactConfigs = 5;
constexpr int32_t kContactConfig[kContactConfigs][2] = {
    {WALK_LANE, 128}, {WALK_LANE, 256}, {WALK_LANE, 512}, {WALK_WARP, 256}, {WALK_ADAPTIVE, 256}};

// The contact kernel of the simulation's neighbour walk and CTA size
// (ps_set_contact_kernel, ps_autotune).
template <class T, bool MULTI, bool MESH, bool FUSED>
struct ContactLaunch {
  void (*fn)(StepBufs<T>, SceneParams<T>, const MeshView*);
  unsigned block;
  unsigned grid;
};

template <class T, bool MULTI, bool MESH, bool FUSED>
ContactLaunch<T, MULTI, MESH, FUSED> contacts_kernel(const ps_sim* s) {
  ContactLaunch<T, MULTI, MESH, FUSED> c;
  if (s->walk == WALK_WARP) {
    c = {k_contacts<T, MULTI, MESH, FUSED, WALK_WARP, 256>, 256u, 0u};
  } else if (s->walk == WALK_ADAPTIVE) {
    c = {k_contacts<T, MULTI, MESH, FUSED, WALK_ADAPTIVE, 256>, 256u, 0u};
  } else if (s->contact_block == 128) {
    c = {k_contacts<T, MULTI, MESH, FUSED, WALK_LANE, 128>, 128u, 0u};
  } else if (s->contact_block == 512) {
    c = {k_contacts<T, MULTI, MESH, FUSED, WALK_LANE, 512>, 512u, 0u};
  } else {
    c = {k_contacts<T, MULTI, MESH, FUSED, WALK_LANE, 256>, 256u, 0u};
  }
  c.grid = (unsigned)((s->n_total + c.block - 1) / c.block);
  return c;
}

// ---- the launch sequence -----------------------------------------------------
template <class T, bool MULTI, bool MESH>
int64_t enqueue_steps(ps_sim* s, int64_t steps) {
  const StepBufs<T> b = bufs<T>(s);
  const SceneParams<T> sp0 = params<T>(s)[0];
  const unsigned gb = blocks_for(s->n_total);
  const unsigned gp = blocks_for(s->n_total);
  const unsigned gs = (unsigned)step_scan_tiles(n_scan(s));
  cudaStream_t st = s->stream;
  int64_t launches = 0;
  const MeshView* mv = s->d_mesh_view;
  const int64_t nsc = n_scan(s);
  const uint32_t nt = (uint32_t)s->n_total;
  pdl_launch(k_begin<T, MULTI, MESH, true>, gb, STEP_THREADS, st, b, sp0, mv);
  ++launches;
  for (int64_t k = 0; k < steps; ++k) {
    pdl_launch(step_scan_kernel(n_scan(s)), gs, SCAN_THREADS, st, (const uint32_t*)s->count, s->offset, nsc,
               (const uint32_t*)s->tile_sum);
    pdl_launch(k_scatter, move_blocks(s->n_total, b.n_tiles), STEP_THREADS, st, (const uint32_t*)s->cell, s->slot,
               (const uint32_t*)s->orig, (const uint32_t*)s->offset, s->tmp, s->count, nt, s->tile_sum, b.n_tiles, s->err);
    pdl_launch(k_rank_move<T>, move_blocks(s->n_total, 0), STEP_THREADS, st, b);
    if (k + 1 < steps) {
      const auto c = contacts_kernel<T, MULTI, MESH, true>(s);
      pdl_launch(c.fn, c.grid, c.block, st, b, sp0, mv);
    } else {
      const auto c = contacts_kernel<T, MULTI, MESH, false>(s);
      pdl_launch(c.fn, c.grid, c.block, st, b, sp0, mv);
    }
    launches += 4;
  }
  return launches;
}

// Eager launch sequence with an event pair around every kernel (profiling).
struct LaunchRecord {
  int kind;
  cudaEvent_t a, b;
};

template <class T, bool MULTI, bool MESH>
void enqueue_steps_recorded(ps_sim* s, int64_t steps, std::vector<LaunchRecord>& rec) {
  const StepBufs<T> b = bufs<T>(s);
  const SceneParams<T> sp0 = params<T>(s)[0];
  const unsigned gb = blocks_for(s->n_total);
  const unsigned gp = blocks_for(s->n_total);
  const unsigned gs = (unsigned)step_scan_tiles(n_scan(s));
  cudaStream_t st = s->stream;
  size_t r = 0;
  auto pre = [&](int kind) {
    rec[r].kind = kind;
    cudaEventRecord(rec[r].a, st);
  };
  auto post = [&]() { cudaEventRecord(rec[r++].b, st); };
  pre(PS_K_BEGIN);
  k_begin<T, MULTI, MESH, true><<<gb, STEP_THREADS, 0, st>>>(b, sp0, s->d_mesh_view);
  post();
  for (int64_t k = 0; k < steps; ++k) {
    pre(PS_K_SCAN);
    step_scan_kernel(n_scan(s))<<<gs, SCAN_THREADS, 0, st>>>(s->count, s->offset, n_scan(s), s->tile_sum);
    post();
    pre(PS_K_SCATTER);
    k_scatter<<<move_blocks(s->n_total, b.n_tiles), STEP_THREADS, 0, st>>>(s->cell, s->slot, s->orig, s->offset, s->tmp,
                                                                         s->count, (uint32_t)s->n_total, s->tile_sum, b.n_tiles, s->err);
    post();
    pre(PS_K_RANK_MOVE);
    k_rank_move<T><<<move_blocks(s->n_total, 0), STEP_THREADS, 0, st>>>(b);
    post();
    pre(PS_K_CONTACTS);
    if (k + 1 < steps) {
      const auto c = contacts_kernel<T, MULTI, MESH, true>(s);
      c.fn<<<c.grid, c.block, 0, st>>>(b, sp0, s->d_mesh_view);
    } else {
      const auto c = contacts_kernel<T, MULTI, MESH, false>(s);
      c.fn<<<c.grid, c.block, 0, st>>>(b, sp0, s->d_mesh_view);
    }
    post();
  }
}

template <class T>
void enqueue_steps_recorded_dispatch(ps_sim* s, int64_t steps, std::vector<LaunchRecord>& rec) {
  if (s->multi) {
    if (s->has_mesh)
      enqueue_steps_recorded<T, true, true>(s, steps, rec);
    else
      enqueue_steps_recorded<T, true, false>(s, steps, rec);
  } else {
    if (s->has_mesh)
      enqueue_steps_recorded<T, false, true>(s, steps, rec);
    else
      enqueue_steps_recorded<T, false, false>(s, steps, rec);
  }
}

// ---- neighbour-list mode ---------------------------------------------------------
size_t list_arena_bytes(const ps_sim* s) {
  const size_t n = (size_t)std::max<int64_t>(s->n_total, 1), vb = s->precision == PS_FP32 ? 16 : 32;
  return 5 * align_up(vb * n, 256) + 3 * align_up(4 * n, 256) + align_up(4 * n * (size_t)s->list_cap, 256) +
         align_up(4 * LIST_FLAG_WORDS, 256);
}

template <class T>
ListBufs<T> list_bufs(ps_sim* s) {
  const size_t n = (size_t)std::max<int64_t>(s->n_total, 1);
  const size_t b4 = align_up(sizeof(vec4_t<T>) * n, 256), bu = align_up(4 * n, 256);
  char* p = static_cast<char*>(s->list_arena);
  ListBufs<T> L;
  L.P[0] = reinterpret_cast<vec4_t<T>*>(p); p += b4;
  L.P[1] = reinterpret_cast<vec4_t<T>*>(p); p += b4;
  L.V[0] = reinterpret_cast<vec4_t<T>*>(p); p += b4;
  L.V[1] = reinterpret_cast<vec4_t<T>*>(p); p += b4;
  L.ref = reinterpret_cast<vec4_t<T>*>(p); p += b4;
  L.cell[0] = reinterpret_cast<uint32_t*>(p); p += bu;
  L.cell[1] = reinterpret_cast<uint32_t*>(p); p += bu;
  L.cnt = reinterpret_cast<uint32_t*>(p); p += bu;
  L.list = reinterpret_cast<uint32_t*>(p); p += align_up(4 * n * (size_t)s->list_cap, 256);
  L.flag = reinterpret_cast<uint32_t*>(p);
  L.cap = (uint32_t)s->list_cap;
  L.skin_frac = (T)s->list_skin;
  return L;
}

// `steps` steps on neighbour lists: a full rebuild from the at-rest state,
// then per step the gated cooperative rebuild and the list step kernel.
// Every graph starts from zeroed counts, whatever an earlier rebuild left.
template <class T, bool MULTI, bool MESH>
cudaError_t enqueue_steps_list(ps_sim* s, int64_t steps) {
  const StepBufs<T> b = bufs<T>(s);
  const ListBufs<T> L = list_bufs<T>(s);
  const SceneParams<T> sp0 = params<T>(s)[0];
  const unsigned gp = blocks_for(s->n_total);
  const unsigned gs = (unsigned)step_scan_tiles(n_scan(s));
  const unsigned gm0 = move_blocks(s->n_total, b.n_tiles), gm1 = move_blocks(s->n_total, 0);
  cudaStream_t st = s->stream;
  const MeshView* mv = s->d_mesh_view;
  const int64_t nsc = n_scan(s);
  const uint32_t nt = (uint32_t)s->n_total;
  cudaMemsetAsync(L.flag, 0, LIST_RESET_WORDS * sizeof(uint32_t), st);
  cudaMemsetAsync(s->count, 0, sizeof(uint32_t) * (size_t)nsc, st);
  cudaMemsetAsync(s->tile_sum, 0, sizeof(uint32_t) * (size_t)b.n_tiles, st);
  pdl_launch(k_begin<T, MULTI, MESH, true>, gp, STEP_THREADS, st, b, sp0, mv);
  pdl_launch(step_scan_kernel(n_scan(s)), gs, SCAN_THREADS, st, (const uint32_t*)s->count, s->offset, nsc,
             (const uint32_t*)s->tile_sum);
  pdl_launch(k_scatter, gm0, STEP_THREADS, st, (const uint32_t*)s->cell, s->slot, (const uint32_t*)s->orig,
             (const uint32_t*)s->offset, s->tmp, s->count, nt, s->tile_sum, b.n_tiles, s->err);
  pdl_launch(k_rank_move<T>, gm1, STEP_THREADS, st, b);
  pdl_launch(k_list_build<T, MULTI>, gp, STEP_THREADS, st, b, sp0, L, 0);
  for (int64_t k = 0; k < steps; ++k) {
    const int par = (int)(k & 1);
    if (k > 0) {
      // the rebuild works on state buffer `par`, in the order of the previous build
      StepBufs<T> br = b;
      br.P1 = L.P[par];
      br.V1 = L.V[par];
      br.cell = L.cell[par];
      cudaLaunchConfig_t cfg{};
      cfg.gridDim = dim3(s->list_rebuild_grid);
      cfg.blockDim = dim3(STEP_THREADS);
      cfg.stream = st;
      cudaLaunchAttribute at[1];
      at[0].id = cudaLaunchAttributeCooperative;
      at[0].val.cooperative = 1;
      cfg.attrs = at;
      cfg.numAttrs = 1;
      const cudaError_t e = cudaLaunchKernelEx(&cfg, k_list_rebuild<T, MULTI>, br, sp0, L, par, nsc, (uint32_t)gs,
                                               (uint32_t)gm0, (uint32_t)gm1);
      if (e != cudaSuccess) return e;
    }
    const unsigned gl = std::min(gp, s->list_step_grid);
    if (k + 1 < steps)
      pdl_launch(k_contacts_list<T, MULTI, MESH, true>, gl, STEP_THREADS, st, b, sp0, mv, L, par);
    else
      pdl_launch(k_contacts_list<T, MULTI, MESH, false>, gl, STEP_THREADS, st, b, sp0, mv, L, par);
  }
  return cudaGetLastError();
}

// CTAs of one wave of k_list_rebuild, which its grid barriers need resident,
// and of one wave of the list step kernel, which loops over the spheres.
template <class T, bool MULTI, bool MESH>
int list_grids(ps_sim* s) {
  int per_sm = 0, step_per_sm = 0, sms = 0;
  PS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_list_rebuild<T, MULTI>, STEP_THREADS, 0));
  PS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&step_per_sm, k_contacts_list<T, MULTI, MESH, true>,
                                                        STEP_THREADS, 0));
  PS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device));
  if (per_sm < 1 || step_per_sm < 1 || sms < 1)
    return fail(PS_ERR_CUDA, "ps_step: the list kernels cannot be resident");
  s->list_rebuild_grid = (unsigned)(per_sm * sms);
  s->list_step_grid = (unsigned)(step_per_sm * sms);
  return PS_OK;
}

template <class T>
cudaError_t enqueue_steps_list_dispatch(ps_sim* s, int64_t steps) {
  if (s->multi) {
    return s->has_mesh ? enqueue_steps_list<T, true, true>(s, steps) : enqueue_steps_list<T, true, false>(s, steps);
  }
  return s->has_mesh ? enqueue_steps_list<T, false, true>(s, steps) : enqueue_steps_list<T, false, false>(s, steps);
}

template <class T>
int64_t enqueue_steps_dispatch(ps_sim* s, int64_t steps) {
  if (s->multi) {
    return s->has_mesh ? enqueue_steps<T, true, true>(s, steps) : enqueue_steps<T, true, false>(s, steps);
  }
  return s->has_mesh ? enqueue_steps<T, false, true>(s, steps) : enqueue_steps<T, false, false>(s, steps);
}

// Rebuild the grid of the at-rest state without moving it (statistics and
// bucket queries before the first step).
template <class T, bool MULTI>
void enqueue_regrid(ps_sim* s) {
  const StepBufs<T> b = bufs<T>(s);
  const SceneParams<T> sp0 = params<T>(s)[0];
  const unsigned gb = blocks_for(s->n_total);
  const unsigned gp = blocks_for(s->n_total);
  cudaStream_t st = s->stream;
  k_begin<T, MULTI, false, false><<<gb, STEP_THREADS, 0, st>>>(b, sp0, s->d_mesh_view);
  k_tile_sums<<<(unsigned)step_scan_tiles(n_scan(s)), STEP_THREADS, 0, st>>>(s->count, n_scan(s), s->tile_sum,
                                                                              step_scan_shift(n_scan(s)));
  step_scan_kernel(n_scan(s))<<<(unsigned)step_scan_tiles(n_scan(s)), SCAN_THREADS, 0, st>>>(s->count, s->offset, n_scan(s),
                                                                                     s->tile_sum);
  k_scatter<<<move_blocks(s->n_total, b.n_tiles), STEP_THREADS, 0, st>>>(s->cell, s->slot, s->orig, s->offset, s->tmp,
                                                                       s->count, (uint32_t)s->n_total, s->tile_sum, b.n_tiles, s->err);
  k_rank_move<T><<<move_blocks(s->n_total, 0), STEP_THREADS, 0, st>>>(b);
  k_copy_vel<T><<<gp, STEP_THREADS, 0, st>>>(b);
}

int regrid(ps_sim* s) {
  if (s->n_total == 0) {
    s->grid_valid = true;
    return PS_OK;
  }
  if (s->precision == PS_FP32)
    s->multi ? enqueue_regrid<float, true>(s) : enqueue_regrid<float, false>(s);
  else
    s->multi ? enqueue_regrid<double, true>(s) : enqueue_regrid<double, false>(s);
  PS_CUDA(cudaGetLastError());
  s->grid_valid = true;
  return PS_OK;
}

int check_device_error(ps_sim* s) {
  uint32_t e = 0;
  PS_CUDA(cudaMemcpyAsync(&e, s->err, sizeof(uint32_t), cudaMemcpyDeviceToHost, s->stream));
  PS_CUDA(cudaStreamSynchronize(s->stream));
  if (e != 0) {
    std::string m = "device error word 0x" + std::to_string(e) + ":";
    if (e & PS_DEVERR_SCAN_TIMEOUT) m += " scan look-back wait expired;";
    if (e & PS_DEVERR_BAD_CELL) m += " cell id outside its scene;";
    if (e & PS_DEVERR_BOUNDS) m += " index out of bounds (bounds-checked build; the access was skipped);";
    uint32_t zero = 0;
    cudaMemcpyAsync(s->err, &zero, sizeof(uint32_t), cudaMemcpyHostToDevice, s->stream);
    cudaStreamSynchronize(s->stream);
    return fail(PS_ERR_DEVICE, m);
  }
  return PS_OK;
}

// ---- conversion kernels between the host AoS and the device SoA ------------
// Upload check of a new state against the grid sized by the first upload:
// each particle must fit a cell (2 r <= cell edge of its scene) and have a
// positive mass; the lowest failing index is kept in *bad (NaN fails too).
__global__ void k_upload_check(const double* __restrict__ aos, const uint32_t* __restrict__ pbase, int n_scenes,
                               const double* __restrict__ interval, uint32_t* bad, uint32_t n) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  int lo = 0, hi = n_scenes - 1;  // largest scene s with pbase[s] <= p
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (pbase[mid] <= p)
      lo = mid;
    else
      hi = mid - 1;
  }
  const double r = aos[8 * (size_t)p + 6], m = aos[8 * (size_t)p + 7];
  if (!(2.0 * r <= interval[lo]) || !(m > 0.0)) atomicMin(bad, p);
}

template <class T>
__global__ void k_upload(const double* __restrict__ aos, vec4_t<T>* P0, vec4_t<T>* V1, uint32_t* orig, uint32_t n) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const double* q = aos + 8 * (size_t)p;
  vec4_t<T> P, V;
  P.x = (T)q[0];
  P.y = (T)q[1];
  P.z = (T)q[2];
  P.w = (T)q[6];
  V.x = (T)q[3];
  V.y = (T)q[4];
  V.z = (T)q[5];
  V.w = (T)q[7];
  P0[p] = P;
  V1[p] = V;
  orig[p] = p;
}

template <class T>
__global__ void k_download(double* __restrict__ aos, const vec4_t<T>* P0, const vec4_t<T>* V1, const uint32_t* orig,
                           uint32_t n) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const vec4_t<T> P = P0[p], V = V1[p];
  double* q = aos + 8 * (size_t)orig[p];
  q[0] = (double)P.x;
  q[1] = (double)P.y;
  q[2] = (double)P.z;
  q[3] = (double)V.x;
  q[4] = (double)V.y;
  q[5] = (double)V.z;
  q[6] = (double)P.w;
  q[7] = (double)V.w;
}

__global__ void k_counts_from_offsets(const uint32_t* offset, uint32_t* counts, int64_t n) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c < n) counts[c] = offset[c + 1] - offset[c];
}

// ---- set-up ------------------------------------------------------------------
template <class T>
SceneParams<T> make_params(const ps_scene_desc& d, const GridHost& g, int64_t pbase, int64_t pcount) {
  SceneParams<T> sp{};
  for (int a = 0; a < 3; ++a) {
    sp.grid_lo[a] = (T)g.min[a];
    sp.box_lo[a] = (T)d.box_min[a];
    sp.box_hi[a] = (T)d.box_max[a];
    sp.gravity[a] = (T)d.gravity[a];
    sp.nb[a] = g.nb[a];
    sp.mesh_nb[a] = g.mesh_nb[a];
    sp.mesh_lo[a] = (T)g.mesh_lo[a];
    sp.mesh_hi[a] = (T)g.mesh_hi[a];
  }
  sp.interval = (T)g.interval;
  sp.e_lo[0] = (T)d.e_wall[PS_XMIN];
  sp.e_lo[1] = (T)d.e_wall[PS_YMIN];
  sp.e_lo[2] = (T)d.e_wall[PS_ZMIN];
  sp.e_hi[0] = (T)d.e_wall[PS_XMAX];
  sp.e_hi[1] = (T)d.e_wall[PS_YMAX];
  sp.e_hi[2] = (T)d.e_wall[PS_ZMAX];
  sp.dt = (T)d.dt;
  sp.k_spring = (T)d.k_spring;
  sp.e_sphere = (T)d.e_sphere;
  sp.e_poly = (T)d.e_wall[PS_ZMIN];  // polygon restitution = zMin (PhysicsEngineCUDA.cpp:112-114)
  sp.cbase = (uint32_t)g.cbase;
  sp.pbase = (uint32_t)pbase;
  sp.pcount = (uint32_t)pcount;
  sp.mesh_tri_base = (uint32_t)g.tri_base;
  sp.mesh_tris = (uint32_t)g.n_tri;
  sp.mesh_bin_base = (uint32_t)g.bin_base;
  sp.mesh_iv = (T)g.mesh_iv;
  sp.edge_quirk = d.edge_quirk;
  fast_udiv_magic((uint32_t)std::max(1, g.nb[2]), sp.div_nz_m, sp.div_nz_sh1, sp.div_nz_sh2);
  fast_udiv_magic((uint32_t)std::max(1, g.nb[1]), sp.div_ny_m, sp.div_ny_sh1, sp.div_ny_sh2);
  return sp;
}

// Host copy of the device bin function (same float/double operations).
template <class T>
int32_t host_mesh_axis(T x, T lo, T iv, int32_t nb) {
  const T q = (x - lo) / iv;
  if (!(q > T(0))) return 0;
  if (q >= (T)nb) return nb - 1;
  return (int32_t)q;
}

// Host copy of the device's axis_cell (same IEEE operations in T).
template <class T>
int32_t host_axis_cell(T x, T lo, T iv, int32_t nb) {
  const T q = (x - lo) / iv;
  if (!(q > T(0))) return 0;
  if (q >= (T)nb) return nb - 1;
  return (int32_t)q;
}

// Order-preserving map between finite/infinite T and unsigned integers.
inline uint64_t key_of(double x) {
  uint64_t u;
  std::memcpy(&u, &x, 8);
  return (u >> 63) ? ~u : (u | (1ull << 63));
}
inline double val_of(double, uint64_t k) {
  const uint64_t u = (k >> 63) ? (k & ~(1ull << 63)) : ~k;
  double x;
  std::memcpy(&x, &u, 8);
  return x;
}
inline uint32_t key_of(float x) {
  uint32_t u;
  std::memcpy(&u, &x, 4);
  return (u >> 31) ? ~u : (u | (1u << 31));
}
inline float val_of(float, uint32_t k) {
  const uint32_t u = (k >> 31) ? (k & ~(1u << 31)) : ~k;
  float x;
  std::memcpy(&x, &u, 4);
  return x;
}

// Boundaries B[0..nb] of one axis: B[k] is the smallest T with
// host_axis_cell(x) >= k (bisection over the ordered bit patterns, since the
// cell index is monotonic in x); B[0] = -inf, B[nb] = +inf.  Checked.
template <class T>
bool axis_bounds(T lo, T iv, int32_t nb, std::vector<T>& out) {
  using K = decltype(key_of(T(0)));
  const T inf = std::numeric_limits<T>::infinity();
  out.push_back(-inf);
  for (int32_t k = 1; k < nb; ++k) {
    K a = key_of(-inf), b = key_of(inf);  // f(val(a)) < k <= f(val(b))
    while (b - a > 1) {
      const K m = a + (b - a) / 2;
      if (host_axis_cell<T>(val_of(T(0), m), lo, iv, nb) >= k)
        b = m;
      else
        a = m;
    }
    const T x = val_of(T(0), b);
    if (host_axis_cell<T>(x, lo, iv, nb) != k || host_axis_cell<T>(val_of(T(0), b - 1), lo, iv, nb) != k - 1)
      return false;
    out.push_back(x);
  }
  out.push_back(inf);
  return true;
}

template <class T>
int upload_bounds(ps_sim* s) {
  std::vector<T> all;
  for (int sc = 0; sc < s->n_scenes; ++sc) {
    const GridHost& g = s->grids[sc];
    for (int a = 0; a < 3; ++a) {
      const uint32_t base = (uint32_t)all.size();
      if (!axis_bounds<T>((T)g.min[a], (T)g.interval, g.nb[a], all))
        return fail(PS_ERR_INVALID, "cell boundary table is not monotonic on axis " + std::to_string(a));
      if (s->precision == PS_FP32)
        s->sp32[sc].bnd_base[a] = base;
      else
        s->sp64[sc].bnd_base[a] = base;
    }
  }
  PS_CUDA(cudaMalloc(&s->d_bounds, sizeof(T) * all.size()));
  PS_CUDA(cudaMemcpy(s->d_bounds, all.data(), sizeof(T) * all.size(), cudaMemcpyHostToDevice));
  return PS_OK;
}

// Triangle data in precision T for every scene, binned by AABB.
template <class T>
int upload_mesh(ps_sim* s) {
  std::vector<T> tri, nrm, aabb;
  std::vector<uint32_t> bin_offset((size_t)s->bins_total + 1, 0), bin_tri;
  std::vector<std::vector<uint32_t>> per_bin_counts;
  tri.reserve((size_t)s->tri_total * 9);
  for (int sc = 0; sc < s->n_scenes; ++sc) {
    const GridHost& g = s->grids[sc];
    const std::vector<double>& soup = s->tris[sc];
    for (int64_t t = 0; t < g.n_tri; ++t) {
      const double* v = soup.data() + 9 * t;
      for (int k = 0; k < 9; ++k) tri.push_back((T)v[k]);
      // unit normal as PolygonContainerCUDA.cpp:73-88 (double, component / length)
      const double r0x = v[3] - v[0], r0y = v[4] - v[1], r0z = v[5] - v[2];
      const double r1x = v[6] - v[0], r1y = v[7] - v[1], r1z = v[8] - v[2];
      const double nx = r0y * r1z - r0z * r1y, ny = r0z * r1x - r0x * r1z, nz = r0x * r1y - r0y * r1x;
      const double len = std::sqrt(nx * nx + ny * ny + nz * nz);
      nrm.push_back((T)(nx / len));
      nrm.push_back((T)(ny / len));
      nrm.push_back((T)(nz / len));
      for (int a = 0; a < 3; ++a) aabb.push_back(std::min(std::min((T)v[a], (T)v[3 + a]), (T)v[6 + a]));
      for (int a = 0; a < 3; ++a) aabb.push_back(std::max(std::max((T)v[a], (T)v[3 + a]), (T)v[6 + a]));
    }
  }
  // two passes: count, then fill (ascending triangle id inside each bin)
  for (int pass = 0; pass < 2; ++pass) {
    std::vector<uint32_t> fill;
    if (pass == 1) {
      for (int64_t i = 0; i < s->bins_total; ++i) bin_offset[i + 1] += bin_offset[i];
      bin_tri.resize(bin_offset[s->bins_total]);
      fill.assign(bin_offset.begin(), bin_offset.end() - 1);
    }
    for (int sc = 0; sc < s->n_scenes; ++sc) {
      const GridHost& g = s->grids[sc];
      const T lo[3] = {(T)g.mesh_lo[0], (T)g.mesh_lo[1], (T)g.mesh_lo[2]};
      const T iv = (T)g.mesh_iv;
      for (int64_t t = 0; t < g.n_tri; ++t) {
        const int64_t gt = g.tri_base + t;
        int32_t b0[3], b1[3];
        for (int a = 0; a < 3; ++a) {
          b0[a] = host_mesh_axis<T>(aabb[6 * gt + a], lo[a], iv, g.mesh_nb[a]);
          b1[a] = host_mesh_axis<T>(aabb[6 * gt + 3 + a], lo[a], iv, g.mesh_nb[a]);
        }
        for (int32_t x = b0[0]; x <= b1[0]; ++x)
          for (int32_t y = b0[1]; y <= b1[1]; ++y)
            for (int32_t z = b0[2]; z <= b1[2]; ++z) {
              const int64_t bin = g.bin_base + ((int64_t)x * g.mesh_nb[1] + y) * g.mesh_nb[2] + z;
              if (pass == 0)
                bin_offset[bin + 1] += 1;
              else
                bin_tri[fill[bin]++] = (uint32_t)gt;
            }
      }
    }
  }
  const size_t bt = tri.size() * sizeof(T), bn = nrm.size() * sizeof(T), ba = aabb.size() * sizeof(T);
  PS_CUDA(cudaMalloc(&s->d_tri, std::max<size_t>(bt, 16)));
  PS_CUDA(cudaMalloc(&s->d_nrm, std::max<size_t>(bn, 16)));
  PS_CUDA(cudaMalloc(&s->d_aabb, std::max<size_t>(ba, 16)));
  PS_CUDA(cudaMalloc(&s->d_bin_offset, bin_offset.size() * sizeof(uint32_t)));
  PS_CUDA(cudaMalloc(&s->d_bin_tri, std::max<size_t>(bin_tri.size(), 1) * sizeof(uint32_t)));
  PS_CUDA(cudaMalloc(&s->d_mesh_view, sizeof(MeshView)));
  PS_CUDA(cudaMemcpy(s->d_tri, tri.data(), bt, cudaMemcpyHostToDevice));
  PS_CUDA(cudaMemcpy(s->d_nrm, nrm.data(), bn, cudaMemcpyHostToDevice));
  PS_CUDA(cudaMemcpy(s->d_aabb, aabb.data(), ba, cudaMemcpyHostToDevice));
  PS_CUDA(cudaMemcpy(s->d_bin_offset, bin_offset.data(), bin_offset.size() * sizeof(uint32_t), cudaMemcpyHostToDevice));
  if (!bin_tri.empty())
    PS_CUDA(cudaMemcpy(s->d_bin_tri, bin_tri.data(), bin_tri.size() * sizeof(uint32_t), cudaMemcpyHostToDevice));
  const MeshView mv{s->d_tri,
                    s->d_nrm,
                    s->d_aabb,
                    s->d_bin_offset,
                    s->d_bin_tri,
                    (uint32_t)s->tri_total,
                    (uint32_t)s->bins_total,
                    (uint32_t)bin_tri.size()};
  PS_CUDA(cudaMemcpy(s->d_mesh_view, &mv, sizeof(MeshView), cudaMemcpyHostToDevice));
  return PS_OK;
}

// Keep the per-cell count and offset arrays resident in L2: they take
// scattered atomics, scattered clears and random offset reads every step,
// while the particle arrays stream through.  The persisting carve-out is a
// limit of this process's CUDA context only.
void setup_l2_window(ps_sim* s, size_t bytes) {
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, s->device) != cudaSuccess) return;
  if (prop.persistingL2CacheMaxSize <= 0 || prop.accessPolicyMaxWindowSize <= 0) return;
  if (std::getenv("PSB200_NO_L2_WINDOW") != nullptr) return;
  const size_t win = std::min<size_t>(bytes, (size_t)prop.accessPolicyMaxWindowSize);
  size_t cur = 0;
  cudaDeviceGetLimit(&cur, cudaLimitPersistingL2CacheSize);
  if (!s->l2_limit_set) s->l2_prev_limit = cur;
  const size_t want = std::min<size_t>((size_t)prop.persistingL2CacheMaxSize, win);
  if (cur != want && cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, want) != cudaSuccess) {
    cudaGetLastError();
    return;
  }
  s->l2_limit = want;
  s->l2_limit_set = true;
  cudaDeviceGetLimit(&cur, cudaLimitPersistingL2CacheSize);
  s->l2_window.base_ptr = s->cell_arena;
  s->l2_window.num_bytes = win;
  s->l2_window.hitRatio = (float)std::min(1.0, (double)cur / (double)win);
  s->l2_window.hitProp = cudaAccessPropertyPersisting;
  s->l2_window.missProp = cudaAccessPropertyStreaming;
  cudaStreamAttrValue v{};
  v.accessPolicyWindow = s->l2_window;
  if (cudaStreamSetAttribute(s->stream, cudaStreamAttributeAccessPolicyWindow, &v) == cudaSuccess)
    s->l2_window_on = true;
  else
    cudaGetLastError();
}

// The set-aside is a limit of the whole context, and a larger one than the
// running simulation's window takes L2 from its ordinary accesses (a 1M-sphere
// step ran 20 % slower after a batch of large grids had raised it); each
// call sets it back to this simulation's own size.
void ensure_l2_limit(ps_sim* s) {
  if (!s->l2_window_on) return;
  size_t cur = 0;
  if (cudaDeviceGetLimit(&cur, cudaLimitPersistingL2CacheSize) == cudaSuccess && cur != s->l2_limit)
    cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, s->l2_limit);
  cudaGetLastError();
}

// Captured kernel nodes carry the window explicitly.
// `clear` gives the nodes an empty window instead (neighbour-list graphs:
// their steps do not touch the cell arrays, which only a rebuild reads).
void apply_l2_window(ps_sim* s, cudaGraph_t g, bool clear = false) {
  if (!s->l2_window_on) return;
  size_t n = 0;
  if (cudaGraphGetNodes(g, nullptr, &n) != cudaSuccess || n == 0) return;
  std::vector<cudaGraphNode_t> nodes(n);
  cudaGraphGetNodes(g, nodes.data(), &n);
  cudaKernelNodeAttrValue v{};
  v.accessPolicyWindow = s->l2_window;
  if (clear) v.accessPolicyWindow.num_bytes = 0;
  for (auto nd : nodes) {
    cudaGraphNodeType t;
    if (cudaGraphNodeGetType(nd, &t) == cudaSuccess && t == cudaGraphNodeTypeKernel)
      cudaGraphKernelNodeSetAttribute(nd, cudaKernelNodeAttributeAccessPolicyWindow, &v);
  }
  cudaGetLastError();
}

// Size every scene's grid from its radii and allocate the per-cell arrays.
int size_grids(ps_sim* s, const double* aos) {
  s->grids.assign(s->n_scenes, GridHost{});
  int64_t cbase = 0, bin_base = 0, tri_base = 0;
  for (int sc = 0; sc < s->n_scenes; ++sc) {
    const ps_scene_desc& d = s->desc[sc];
    GridHost& g = s->grids[sc];
    double r_max = 0.0;
    double plo[3] = {INFINITY, INFINITY, INFINITY}, phi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int64_t i = s->pbase[sc]; i < s->pbase[sc + 1]; ++i) {
      const double* q = aos + 8 * i;
      if (!(q[6] >= 0.0) || !std::isfinite(q[6]) || !(q[7] > 0.0))
        return fail(PS_ERR_INVALID, "scene " + std::to_string(sc) + ": particle " + std::to_string(i) +
                                        " has a negative/non-finite radius or a non-positive mass");
      r_max = std::max(r_max, q[6]);
      for (int a = 0; a < 3; ++a) {
        plo[a] = std::min(plo[a], q[a]);
        phi[a] = std::max(phi[a], q[a]);
      }
    }
    if (!s->tris[sc].empty()) {  // ps_create keeps the soup in s->tris (desc.tri is cleared)
      const std::vector<double>& soup = s->tris[sc];
      for (int a = 0; a < 3; ++a) {
        g.min[a] = INFINITY;
        g.max[a] = -INFINITY;
      }
      for (int64_t k = 0; k < 3 * d.n_tri; ++k)
        for (int a = 0; a < 3; ++a) {
          g.min[a] = std::min(g.min[a], soup[3 * k + a]);
          g.max[a] = std::max(g.max[a], soup[3 * k + a]);
        }
      for (int a = 0; a < 3; ++a) {
        g.mesh_lo[a] = g.min[a];
        g.mesh_hi[a] = g.max[a];
      }
      double ext = 0.0;
      for (int a = 0; a < 3; ++a) ext = std::max(ext, g.max[a] - g.min[a]);
      if (d.widen_domain && s->pbase[sc + 1] > s->pbase[sc]) {
        for (int a = 0; a < 3; ++a) {
          g.min[a] = std::min(g.min[a], plo[a] - r_max);
          g.max[a] = std::max(g.max[a], phi[a] + r_max);
        }
      }
      g.n_tri = d.n_tri;
      g.tri_base = tri_base;
      tri_base += d.n_tri;
      // bin edge: at least one particle cell, at most 128 bins along the longest side
      g.mesh_iv = std::max(r_max * 2.0 * 1.05, ext / 128.0);
      if (!(g.mesh_iv > 0.0)) g.mesh_iv = 1.0;
      for (int a = 0; a < 3; ++a) {
        double span = 0.0;
        for (int64_t k = 0; k < 3 * d.n_tri; ++k) span = std::max(span, soup[3 * k + a] - g.mesh_lo[a]);
        g.mesh_nb[a] = (int32_t)(span / g.mesh_iv) + 1;
      }
      g.n_bins = (int64_t)g.mesh_nb[0] * g.mesh_nb[1] * g.mesh_nb[2];
      g.bin_base = bin_base;
      bin_base += g.n_bins;
    } else {
      for (int a = 0; a < 3; ++a) {
        g.min[a] = d.box_min[a];
        g.max[a] = d.box_max[a];
        g.mesh_nb[a] = 1;
        g.mesh_lo[a] = 0.0;
        g.mesh_hi[a] = 0.0;
      }
      g.mesh_iv = 1.0;
    }
    if (!(r_max > 0.0) && s->pbase[sc + 1] > s->pbase[sc])
      return fail(PS_ERR_INVALID, "scene " + std::to_string(sc) + ": the largest radius must be positive");
    g.interval = d.cell_size > 0.0 ? d.cell_size : r_max * 2.0 * 1.05;  // ParticleModelCUDA.cpp:84
    if (!(g.interval > 0.0)) g.interval = 1.0;  // empty scene
    if (g.interval < 2.0 * r_max)
      return fail(PS_ERR_INVALID, "scene " + std::to_string(sc) + ": cell_size " + std::to_string(g.interval) +
                                      " is smaller than 2*r_max = " + std::to_string(2.0 * r_max));
    int64_t nc = 1;
    for (int a = 0; a < 3; ++a) {
      const double ncells = (g.max[a] - g.min[a]) / g.interval;
      if (!(ncells >= 0.0) || ncells > 2.0e9)
        return fail(PS_ERR_INVALID, "scene " + std::to_string(sc) + ": bad grid extent on axis " + std::to_string(a));
      g.nb[a] = (int32_t)ncells + 1;  // ParticleModelCUDA.cpp:89-91
      nc *= g.nb[a];
    }
    g.n_cells = nc;
    g.cbase = cbase;
    cbase += nc;
    if (cbase >= (int64_t)UINT32_MAX - 1)
      return fail(PS_ERR_INVALID, "too many grid cells over all scenes: " + std::to_string(cbase));
  }
  s->c_total = cbase;
  s->bins_total = bin_base;
  s->tri_total = tri_base;

  // per-cell arrays and scan scratch
  const size_t cells_b = align_up(sizeof(uint32_t) * (size_t)(s->c_total + 1), 256);
  const size_t tiles_b = align_up(sizeof(uint32_t) * (size_t)step_scan_tiles(n_scan(s)), 256);
  PS_CUDA(cudaMalloc(&s->cell_arena, 2 * cells_b + tiles_b));
  char* c = static_cast<char*>(s->cell_arena);
  s->count = reinterpret_cast<uint32_t*>(c);
  s->offset = reinterpret_cast<uint32_t*>(c + cells_b);
  s->tile_sum = reinterpret_cast<uint32_t*>(c + 2 * cells_b);
  PS_CUDA(cudaMemset(s->cell_arena, 0, 2 * cells_b + tiles_b));
  setup_l2_window(s, 2 * cells_b + tiles_b);

  {
    std::vector<double> iv((size_t)s->n_scenes);
    for (int sc = 0; sc < s->n_scenes; ++sc) iv[(size_t)sc] = s->grids[sc].interval;
    PS_CUDA(cudaMemcpy(s->d_interval, iv.data(), 8 * iv.size(), cudaMemcpyHostToDevice));
  }

  // scene parameter tables
  s->sp32.clear();
  s->sp64.clear();
  for (int sc = 0; sc < s->n_scenes; ++sc) {
    const int64_t pc = s->pbase[sc + 1] - s->pbase[sc];
    s->sp32.push_back(make_params<float>(s->desc[sc], s->grids[sc], s->pbase[sc], pc));
    s->sp64.push_back(make_params<double>(s->desc[sc], s->grids[sc], s->pbase[sc], pc));
  }
  {
    const int rc = s->precision == PS_FP32 ? upload_bounds<float>(s) : upload_bounds<double>(s);
    if (rc != PS_OK) return rc;
  }
  const size_t spb = s->precision == PS_FP32 ? sizeof(SceneParams<float>) : sizeof(SceneParams<double>);
  PS_CUDA(cudaMalloc(&s->d_scenes, spb * s->n_scenes));
  if (s->precision == PS_FP32)
    PS_CUDA(cudaMemcpy(s->d_scenes, s->sp32.data(), spb * s->n_scenes, cudaMemcpyHostToDevice));
  else
    PS_CUDA(cudaMemcpy(s->d_scenes, s->sp64.data(), spb * s->n_scenes, cudaMemcpyHostToDevice));
  if (s->has_mesh) {
    const int rc = s->precision == PS_FP32 ? upload_mesh<float>(s) : upload_mesh<double>(s);
    if (rc != PS_OK) return rc;
  }
  s->grid_sized = true;
  return PS_OK;
}

void free_sim(ps_sim* s) {
  for (void* p : s->fwd_ckpt) cudaFree(p);
  s->fwd_ckpt.clear();
  cudaFree(s->adj_arena);
  cudaFree(s->list_arena);
  cudaFree(s->list_ckpt);
  if (s->l2_window_on) {
    cudaStreamAttrValue v{};
    v.accessPolicyWindow.num_bytes = 0;
    cudaStreamSetAttribute(s->stream, cudaStreamAttributeAccessPolicyWindow, &v);
    cudaCtxResetPersistingL2Cache();
    cudaGetLastError();
  }
  if (s->l2_limit_set) {  // give the context back the set-aside it had
    cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, s->l2_prev_limit);
    cudaGetLastError();
  }
  for (auto& kv : s->checkpoints) cudaFree(kv.second);
  s->checkpoints.clear();
  for (auto& kv : s->graphs) cudaGraphExecDestroy(kv.second);
  s->graphs.clear();
  cudaFree(s->part_arena);
  cudaFree(s->cell_arena);
  cudaFree(s->d_scenes);
  cudaFree(s->d_bounds);
  cudaFree(s->d_tri);
  cudaFree(s->d_nrm);
  cudaFree(s->d_aabb);
  cudaFree(s->d_bin_offset);
  cudaFree(s->d_bin_tri);
  cudaFree(s->d_mesh_view);
  if (s->stream) cudaStreamDestroy(s->stream);
}

// ---- differentiation -----------------------------------------------------------
size_t state_bytes(const ps_sim* s) { return (size_t)(s->precision == PS_FP32 ? 16 : 32) * (size_t)s->n_total; }

int save_state(ps_sim* s, void*& buf) {
  const size_t vb = state_bytes(s), ob = 4 * (size_t)s->n_total;
  if (buf == nullptr) PS_CUDA(cudaMalloc(&buf, std::max<size_t>(2 * vb + ob, 16)));
  char* p = static_cast<char*>(buf);
  PS_CUDA(cudaMemcpyAsync(p, s->P0, vb, cudaMemcpyDeviceToDevice, s->stream));
  PS_CUDA(cudaMemcpyAsync(p + vb, s->V1, vb, cudaMemcpyDeviceToDevice, s->stream));
  PS_CUDA(cudaMemcpyAsync(p + 2 * vb, s->orig, ob, cudaMemcpyDeviceToDevice, s->stream));
  return PS_OK;
}

int load_state(ps_sim* s, const void* buf) {
  const size_t vb = state_bytes(s), ob = 4 * (size_t)s->n_total;
  const char* p = static_cast<const char*>(buf);
  PS_CUDA(cudaMemcpyAsync(s->P0, p, vb, cudaMemcpyDeviceToDevice, s->stream));
  PS_CUDA(cudaMemcpyAsync(s->V1, p + vb, vb, cudaMemcpyDeviceToDevice, s->stream));
  PS_CUDA(cudaMemcpyAsync(s->orig, p + 2 * vb, ob, cudaMemcpyDeviceToDevice, s->stream));
  s->grid_valid = false;
  return PS_OK;
}

// dL/d(final state), original order, gathered into the final state's sorted order.
template <class T>
__global__ void k_adj_upload(const double* __restrict__ g, const uint32_t* __restrict__ orig, vec4_t<T>* ax,
                             vec4_t<T>* av, uint32_t n) {
  const uint32_t o = blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= n) return;
  const double* q = g + 6 * (size_t)orig[o];
  vec4_t<T> x, v;
  x.x = (T)q[0]; x.y = (T)q[1]; x.z = (T)q[2]; x.w = T(0);
  v.x = (T)q[3]; v.y = (T)q[4]; v.z = (T)q[5]; v.w = T(0);
  ax[o] = x;
  av[o] = v;
}

// dL/d(initial state) from the initial state's sorted order back to original order.
template <class T>
__global__ void k_adj_download(const vec4_t<T>* ax, const vec4_t<T>* av, const uint32_t* __restrict__ orig,
                               double* __restrict__ g, uint32_t n) {
  const uint32_t o = blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= n) return;
  const vec4_t<T> x = ax[o], v = av[o];
  double* q = g + 6 * (size_t)orig[o];
  q[0] = (double)x.x; q[1] = (double)x.y; q[2] = (double)x.z;
  q[3] = (double)v.x; q[4] = (double)v.y; q[5] = (double)v.z;
}

// Tape row t of a block: the at-rest state after t steps in sorted order;
// rows t >= 1 also hold step t-1's grid (pre-contact velocities, cell ids).
template <class T>
TapeRow<T> tape_row(char* base, size_t row_bytes, int64_t n, int64_t t) {
  TapeRow<T> r;
  char* p = base + row_bytes * (size_t)t;
  r.p = reinterpret_cast<vec4_t<T>*>(p);
  r.v = r.p + n;
  r.vpre = r.v + n;
  r.o = reinterpret_cast<uint32_t*>(r.vpre + n);
  r.cell = r.o + n;
  return r;
}

size_t tape_row_bytes(size_t vec_bytes, int64_t n) {
  return align_up((3 * vec_bytes + 2 * sizeof(uint32_t)) * (size_t)n, 256);
}

// Recompute `steps` steps of a block eagerly (box containers): step k's
// contact kernel writes tape row k + 1, and its scan writes the cell offsets
// straight into offsets slot k, which its scatter, rank/move and contacts
// then read (no copy of the offsets per step).
template <class T, bool MULTI>
int enqueue_steps_taped(ps_sim* s, int64_t steps, char* tape, size_t row_bytes, uint32_t* offs, size_t offs_stride) {
  StepBufs<T> b = bufs<T>(s);
  const SceneParams<T> sp0 = params<T>(s)[0];
  const unsigned gp = blocks_for(s->n_total);
  const unsigned gs = (unsigned)step_scan_tiles(n_scan(s));
  cudaStream_t st = s->stream;
  k_begin<T, MULTI, false, true><<<gp, STEP_THREADS, 0, st>>>(b, sp0, s->d_mesh_view);
  for (int64_t k = 0; k < steps; ++k) {
    const TapeRow<T> row = tape_row<T>(tape, row_bytes, s->n_total, k + 1);
    b.tape_p = row.p;
    b.tape_v = row.v;
    b.tape_o = row.o;
    uint32_t* off_k = offs + offs_stride * (size_t)k;
    b.offset = off_k;
    pdl_launch(step_scan_kernel(n_scan(s)), gs, SCAN_THREADS, st, (const uint32_t*)s->count, off_k, n_scan(s),
               (const uint32_t*)s->tile_sum);
    pdl_launch(k_scatter, move_blocks(s->n_total, b.n_tiles), STEP_THREADS, st, (const uint32_t*)s->cell, s->slot,
               (const uint32_t*)s->orig, (const uint32_t*)off_k, s->tmp, s->count, (uint32_t)s->n_total,
               s->tile_sum, b.n_tiles, s->err);
    pdl_launch(k_rank_move<T>, move_blocks(s->n_total, 0), STEP_THREADS, st, b);
    b.tape_vpre = row.vpre;
    b.tape_cell = row.cell;
    const MeshView* mv = s->d_mesh_view;
    if (k + 1 < steps) {
      const auto c = contacts_kernel<T, MULTI, false, true>(s);
      pdl_launch(c.fn, c.grid, c.block, st, b, sp0, mv);
    } else {
      const auto c = contacts_kernel<T, MULTI, false, false>(s);
      pdl_launch(c.fn, c.grid, c.block, st, b, sp0, mv);
    }
  }
  return PS_OK;
}

template <class T, bool MULTI>
int backward_impl(ps_sim* s, const double* dl_dstate, ps_grad* grads, double* dl_dstate0) {
  const int64_t n = s->n_total, K = s->fwd_every;
  const size_t row_b = tape_row_bytes(sizeof(vec4_t<T>), n);
  const size_t tape_b = row_b * (size_t)(K + 1);                 // rows 0..K
  const size_t offs_stride = align_up(sizeof(uint32_t) * (size_t)n_scan(s), 256) / sizeof(uint32_t);
  const size_t offs_b = sizeof(uint32_t) * offs_stride * (size_t)K;  // cell offsets of each step's grid
  const size_t adj_b = align_up(sizeof(vec4_t<T>) * (size_t)n, 256);
  const size_t acc_b = align_up(ADJ_NACC * sizeof(double) * (size_t)n, 256);
  const size_t io_b = align_up(6 * sizeof(double) * (size_t)n, 256);
  const size_t red_b = align_up(ADJ_NACC * sizeof(double) * (size_t)s->n_scenes, 256);
  const size_t inv_b = align_up(sizeof(uint32_t) * (size_t)n, 256);
  const size_t need = tape_b + offs_b + 4 * adj_b + inv_b + acc_b + io_b + red_b;
  if (s->adj_bytes < need) {
    cudaFree(s->adj_arena);
    s->adj_arena = nullptr;
    s->adj_bytes = 0;
    PS_CUDA(cudaMalloc(&s->adj_arena, need));
    s->adj_bytes = need;
  }
  char* p = static_cast<char*>(s->adj_arena);
  char* tape = p;
  p += tape_b;
  uint32_t* offs = reinterpret_cast<uint32_t*>(p);
  p += offs_b;
  AdjBufs<T> a;
  a.tape = tape_row<T>(tape, row_b, n, 0);
  a.ax = reinterpret_cast<vec4_t<T>*>(p); p += adj_b;
  a.av = reinterpret_cast<vec4_t<T>*>(p); p += adj_b;
  a.ax2 = reinterpret_cast<vec4_t<T>*>(p); p += adj_b;
  a.av2 = reinterpret_cast<vec4_t<T>*>(p); p += adj_b;
  a.inv = reinterpret_cast<uint32_t*>(p); p += inv_b;
  a.acc = reinterpret_cast<double*>(p); p += acc_b;
  a.n = (uint32_t)n;
  double* io = reinterpret_cast<double*>(p); p += io_b;
  double* red = reinterpret_cast<double*>(p);
  cudaStream_t st = s->stream;
  const unsigned gp = blocks_for(n);
  unsigned adj_grid = 0;  // one wave of k_adj_contacts, which loops over the particles
  {
    int per_sm = 0, sms = 0;
    PS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_adj_contacts<T, MULTI>, STEP_THREADS, 0));
    PS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device));
    if (per_sm < 1 || sms < 1) return fail(PS_ERR_CUDA, "ps_backward: the adjoint contact kernel cannot be resident");
    adj_grid = (unsigned)(per_sm * sms);
  }
  // the final state's order (recomputing the last block reproduces it exactly)
  int rc0 = load_state(s, s->fwd_ckpt.back());
  if (rc0 != PS_OK) return rc0;
  PS_CUDA(cudaMemcpyAsync(io, dl_dstate, 6 * sizeof(double) * (size_t)n, cudaMemcpyHostToDevice, st));
  k_adj_upload<T><<<gp, STEP_THREADS, 0, st>>>(io, s->orig, a.ax, a.av, (uint32_t)n);
  PS_CUDA(cudaMemsetAsync(a.acc, 0, acc_b, st));
  const SceneParams<T> sp0 = params<T>(s)[0];
  const int64_t n_blocks = (s->fwd_steps + K - 1) / K;
  for (int64_t blk = n_blocks - 1; blk >= 0; --blk) {
    const int64_t kb = std::min(K, s->fwd_steps - blk * K);
    int rc = load_state(s, s->fwd_ckpt[(size_t)blk]);
    if (rc != PS_OK) return rc;
    // recompute the block, recording each step's input and grid (row 0 = block start)
    k_tape_write<T><<<gp, STEP_THREADS, 0, st>>>(bufs<T>(s), tape_row<T>(tape, row_b, n, 0));
    rc = enqueue_steps_taped<T, MULTI>(s, kb, tape, row_b, offs, offs_stride);
    if (rc != PS_OK) return rc;
    PS_CUDA(cudaGetLastError());
    for (int64_t t = kb - 1; t >= 0; --t) {
      // step t's sorted post-wall state and grid: row t + 1 and offsets t
      const TapeRow<T> g = tape_row<T>(tape, row_b, n, t + 1);
      StepBufs<T> b = bufs<T>(s);
      b.P0 = g.p;
      b.V0 = g.vpre;
      b.orig = g.o;
      b.scell = g.cell;
      b.offset = offs + offs_stride * (size_t)t;
      a.tape = tape_row<T>(tape, row_b, n, t);
      k_adj_contacts<T, MULTI><<<std::min(gp, adj_grid), STEP_THREADS, 0, st>>>(b, a, sp0);
      k_adj_walls_integrate<T, MULTI><<<gp, STEP_THREADS, 0, st>>>(b, a, sp0);
      PS_CUDA(cudaGetLastError());
    }
  }
  k_adj_reduce<<<s->n_scenes, 128, 0, st>>>(a.acc, s->d_pbase, s->n_scenes, (uint32_t)n, red);
  std::vector<double> h((size_t)ADJ_NACC * s->n_scenes);
  PS_CUDA(cudaMemcpyAsync(h.data(), red, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, st));
  if (dl_dstate0 != nullptr) {
    // block 0's row 0 is the initial state, in the order the adjoints now follow
    k_adj_download<T><<<gp, STEP_THREADS, 0, st>>>(a.ax, a.av, tape_row<T>(tape, row_b, n, 0).o, io, (uint32_t)n);
    PS_CUDA(cudaMemcpyAsync(dl_dstate0, io, 6 * sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost, st));
  }
  PS_CUDA(cudaStreamSynchronize(st));
  for (int sc = 0; sc < s->n_scenes; ++sc) {
    grads[sc].k_spring = h[ADJ_NACC * sc + ADJ_K];
    grads[sc].e_sphere = h[ADJ_NACC * sc + ADJ_E];
    for (int w = 0; w < 6; ++w) grads[sc].e_wall[w] = h[ADJ_NACC * sc + ADJ_WALL + w];
  }
  const int rc = load_state(s, s->fwd_ckpt.back());  // leave the final state in place
  if (rc != PS_OK) return rc;
  return check_device_error(s);
}

}  // namespace

// ---- C ABI -------------------------------------------------------------------
extern "C" int ps_create(const ps_scene_desc* scenes, int32_t n_scenes, int32_t precision, int32_t device,
                         ps_sim** out) {
  if (out == nullptr || scenes == nullptr || n_scenes <= 0)
    return fail(PS_ERR_INVALID, "ps_create: scenes, n_scenes > 0 and out are required");
  *out = nullptr;
  if (precision != PS_FP32 && precision != PS_FP64) return fail(PS_ERR_INVALID, "ps_create: precision must be PS_FP32 or PS_FP64");
  int ndev = 0;
  PS_CUDA(cudaGetDeviceCount(&ndev));
  if (device < 0 || device >= ndev) return fail(PS_ERR_INVALID, "ps_create: no CUDA device " + std::to_string(device));
  DeviceGuard guard(device);
  if (!guard.ok) return fail(PS_ERR_CUDA, "ps_create: cannot select device " + std::to_string(device));

  ps_sim* s = new ps_sim();
  s->precision = precision;
  s->device = device;
  s->n_scenes = n_scenes;
  s->desc.assign(scenes, scenes + n_scenes);
  s->tris.resize(n_scenes);
  s->pbase.assign(n_scenes + 1, 0);
  for (int sc = 0; sc < n_scenes; ++sc) {
    const ps_scene_desc& d = scenes[sc];
    if (d.n_particles < 0 || !(d.dt >= 0.0) || (d.tri == nullptr && d.n_tri != 0) || d.n_tri < 0) {
      delete s;
      return fail(PS_ERR_INVALID, "ps_create: scene " + std::to_string(sc) + " has a negative count, a bad dt or an inconsistent triangle list");
    }
    if (d.tri != nullptr && d.n_tri > 0) {
      s->tris[sc].assign(d.tri, d.tri + 9 * d.n_tri);
      s->has_mesh = true;
    }
    s->desc[sc].tri = nullptr;  // owned copy lives in s->tris
    s->pbase[sc + 1] = s->pbase[sc] + d.n_particles;
  }
  s->n_total = s->pbase[n_scenes];
  s->multi = n_scenes > 1;
  if (s->n_total >= (int64_t)SLOT_ALONE - 64) {  // slot tags and union walks stay below 2^31
    delete s;
    return fail(PS_ERR_INVALID, "ps_create: too many particles");
  }
  const size_t vb = s->precision == PS_FP32 ? 16 : 32;
  const size_t n = (size_t)std::max<int64_t>(s->n_total, 1);
  const size_t b4 = align_up(vb * n, 256), bu = align_up(4 * n, 256), bs = align_up(64 * n, 256);
  const size_t bp = align_up(4 * (size_t)(n_scenes + 1), 256), bi = align_up(8 * (size_t)n_scenes, 256);
  cudaError_t e = cudaMalloc(&s->part_arena,
                             4 * b4 + 5 * bu + bs + 256 + bp + bi + 2 * sizeof(StatsPartial) * kStatsBlocks + 256);
  if (e != cudaSuccess) {
    delete s;
    return fail(e == cudaErrorMemoryAllocation ? PS_ERR_NOMEM : PS_ERR_CUDA, std::string("ps_create: ") + cudaGetErrorString(e));
  }
  char* p = static_cast<char*>(s->part_arena);
  s->P0 = p; p += b4;
  s->V0 = p; p += b4;
  s->P1 = p; p += b4;
  s->V1 = p; p += b4;
  s->orig = reinterpret_cast<uint32_t*>(p); p += bu;
  s->cell = reinterpret_cast<uint32_t*>(p); p += bu;
  s->slot = reinterpret_cast<uint32_t*>(p); p += bu;
  s->tmp = reinterpret_cast<uint32_t*>(p); p += bu;
  s->scell = reinterpret_cast<uint32_t*>(p); p += bu;
  s->staging = reinterpret_cast<double*>(p); p += bs;
  s->err = reinterpret_cast<uint32_t*>(p); p += 256;
  s->d_pbase = reinterpret_cast<uint32_t*>(p); p += bp;
  s->d_interval = reinterpret_cast<double*>(p); p += bi;
  s->d_stats = reinterpret_cast<StatsPartial*>(p); p += sizeof(StatsPartial) * kStatsBlocks;
  s->d_stats_out = reinterpret_cast<StatsPartial*>(p);
  std::vector<uint32_t> pb(n_scenes + 1);
  for (int sc = 0; sc <= n_scenes; ++sc) pb[sc] = (uint32_t)s->pbase[sc];
  e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMemcpy(s->d_pbase, pb.data(), 4 * pb.size(), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(s->err, 0, 256);
  if (e != cudaSuccess) {
    free_sim(s);
    delete s;
    return fail(PS_ERR_CUDA, std::string("ps_create: ") + cudaGetErrorString(e));
  }
  *out = s;
  return PS_OK;
}

extern "C" int ps_set_state(ps_sim* s, const double* aos, int64_t n_total) {
  const NvtxRange nvtx_range("ps_set_state");
  if (s == nullptr || (aos == nullptr && n_total > 0)) return fail(PS_ERR_INVALID, "ps_set_state: null argument");
  if (n_total != s->n_total)
    return fail(PS_ERR_INVALID, "ps_set_state: expected " + std::to_string(s->n_total) + " particles, got " + std::to_string(n_total));
  DeviceGuard guard(s->device);
  const bool first = !s->grid_sized;
  if (first) {
    const int rc = size_grids(s, aos);
    if (rc != PS_OK) return rc;
  }
  if (n_total == 0) return PS_OK;
  PS_CUDA(cudaMemcpyAsync(s->staging, aos, 64 * (size_t)n_total, cudaMemcpyHostToDevice, s->stream));
  const unsigned g = blocks_for(n_total);
  if (!first) {
    // a later state must fit the grid the first one sized; checked on the
    // device (a host loop over the records cost milliseconds per upload at
    // 1M particles), before the state is replaced
    uint32_t* bad = s->err + 8;
    uint32_t h_bad = 0;
    PS_CUDA(cudaMemsetAsync(bad, 0xff, sizeof(uint32_t), s->stream));
    k_upload_check<<<g, STEP_THREADS, 0, s->stream>>>(s->staging, s->d_pbase, s->n_scenes, s->d_interval, bad,
                                                        (uint32_t)n_total);
    PS_CUDA(cudaGetLastError());
    PS_CUDA(cudaMemcpyAsync(&h_bad, bad, sizeof(uint32_t), cudaMemcpyDeviceToHost, s->stream));
    PS_CUDA(cudaStreamSynchronize(s->stream));
    if (h_bad != 0xffffffffu)
      return fail(PS_ERR_INVALID,
                  "ps_set_state: particle " + std::to_string(h_bad) + " does not fit the grid sized by the first upload");
  }
  if (s->precision == PS_FP32)
    k_upload<float><<<g, STEP_THREADS, 0, s->stream>>>(s->staging, static_cast<float4*>(s->P0),
                                                       static_cast<float4*>(s->V1), s->orig, (uint32_t)n_total);
  else
    k_upload<double><<<g, STEP_THREADS, 0, s->stream>>>(s->staging, static_cast<vec4_t<double>*>(s->P0),
                                                        static_cast<vec4_t<double>*>(s->V1), s->orig, (uint32_t)n_total);
  PS_CUDA(cudaGetLastError());
  // Keep the state at rest in grid order, as every step leaves it: the
  // first step after an upload (or after restoring a checkpoint saved now)
  // then counts its cells in sorted order, one tile-total atomic per warp,
  // instead of scattering them over every tile.
  const int rc = regrid(s);
  if (rc != PS_OK) return rc;
  PS_CUDA(cudaStreamSynchronize(s->stream));
  return PS_OK;
}

extern "C" int ps_get_state(ps_sim* s, double* out, int64_t n_total) {
  const NvtxRange nvtx_range("ps_get_state");
  if (s == nullptr || (out == nullptr && n_total > 0)) return fail(PS_ERR_INVALID, "ps_get_state: null argument");
  if (n_total != s->n_total) return fail(PS_ERR_INVALID, "ps_get_state: size mismatch");
  if (!s->grid_sized) return fail(PS_ERR_INVALID, "ps_get_state: no state uploaded");
  if (n_total == 0) return PS_OK;
  DeviceGuard guard(s->device);
  const unsigned g = blocks_for(n_total);
  if (s->precision == PS_FP32)
    k_download<float><<<g, STEP_THREADS, 0, s->stream>>>(s->staging, static_cast<float4*>(s->P0),
                                                         static_cast<float4*>(s->V1), s->orig, (uint32_t)n_total);
  else
    k_download<double><<<g, STEP_THREADS, 0, s->stream>>>(s->staging, static_cast<vec4_t<double>*>(s->P0),
                                                          static_cast<vec4_t<double>*>(s->V1), s->orig, (uint32_t)n_total);
  PS_CUDA(cudaGetLastError());
  PS_CUDA(cudaMemcpyAsync(out, s->staging, 64 * (size_t)n_total, cudaMemcpyDeviceToHost, s->stream));
  PS_CUDA(cudaStreamSynchronize(s->stream));
  return check_device_error(s);
}

namespace {

// Run n_steps as CUDA graphs of up to graph_block steps (grid path, or the
// neighbour-list path when `lists`), asynchronously.
int step_graphs(ps_sim* s, int64_t n_steps, bool lists) {
  int64_t left = n_steps;
  while (left > 0) {
    const int64_t L = std::min(left, s->graph_block);
    const int64_t key = lists ? (L | (int64_t(1) << 62)) : L;
    auto it = s->graphs.find(key);
    if (it == s->graphs.end()) {
      cudaGraph_t graph = nullptr;
      PS_CUDA(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
      cudaError_t ce = cudaSuccess;
      if (lists)
        ce = s->precision == PS_FP32 ? enqueue_steps_list_dispatch<float>(s, L) : enqueue_steps_list_dispatch<double>(s, L);
      else
        s->precision == PS_FP32 ? enqueue_steps_dispatch<float>(s, L) : enqueue_steps_dispatch<double>(s, L);
      if (ce == cudaSuccess) ce = cudaGetLastError();
      const cudaError_t ee = cudaStreamEndCapture(s->stream, &graph);
      if (ce != cudaSuccess || ee != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        return fail(PS_ERR_CUDA, std::string("ps_step: capture failed: ") + cudaGetErrorString(ce != cudaSuccess ? ce : ee));
      }
      apply_l2_window(s, graph, lists);
      cudaGraphExec_t exec = nullptr;
      const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
      cudaGraphDestroy(graph);
      if (ie != cudaSuccess) return fail(PS_ERR_CUDA, std::string("ps_step: instantiate failed: ") + cudaGetErrorString(ie));
      it = s->graphs.emplace(key, exec).first;
    }
    PS_CUDA(cudaGraphLaunch(it->second, s->stream));
    s->last_launches += lists ? 5 + 2 * L - 1 : 1 + 4 * L;
    left -= L;
  }
  return PS_OK;
}

// A rebuild costs a few list steps; when a window of at least
// LIST_BACKOFF_WINDOW list steps rebuilt more often than once per
// LIST_BACKOFF_RATE steps (a scene moving fast against its skin, or
// diverging), the following steps run on the grid path, for a stretch that
// doubles while this repeats.
constexpr int64_t LIST_BACKOFF_WINDOW = 256, LIST_BACKOFF_RATE = 4, LIST_BACKOFF_MIN = 1024,
                  LIST_BACKOFF_MAX = 65536;

// Neighbour-list path: exact as long as no list or overlap buffer overflows
// (checked after the call); otherwise the call is repeated on the grid path
// from the state it started from.
int step_lists(ps_sim* s, int64_t n_steps) {
  const size_t need = list_arena_bytes(s);
  if (s->list_arena == nullptr || s->list_bytes < need) {
    cudaFree(s->list_arena);
    s->list_arena = nullptr;
    s->list_bytes = 0;
    for (auto it = s->graphs.begin(); it != s->graphs.end();) {  // list graphs hold the old buffers
      if (it->first & (int64_t(1) << 62)) {
        cudaGraphExecDestroy(it->second);
        it = s->graphs.erase(it);
      } else {
        ++it;
      }
    }
    PS_CUDA(cudaMalloc(&s->list_arena, need));
    s->list_bytes = need;
  }
  if (s->list_rebuild_grid == 0) {
    int g;
    if (s->precision == PS_FP32)
      g = s->multi ? (s->has_mesh ? list_grids<float, true, true>(s) : list_grids<float, true, false>(s))
                   : (s->has_mesh ? list_grids<float, false, true>(s) : list_grids<float, false, false>(s));
    else
      g = s->multi ? (s->has_mesh ? list_grids<double, true, true>(s) : list_grids<double, true, false>(s))
                   : (s->has_mesh ? list_grids<double, false, true>(s) : list_grids<double, false, false>(s));
    if (g != PS_OK) return g;
  }
  uint32_t* rebuilds = s->precision == PS_FP32 ? list_bufs<float>(s).flag + LIST_REBUILDS
                                               : list_bufs<double>(s).flag + LIST_REBUILDS;
  PS_CUDA(cudaMemsetAsync(rebuilds, 0, sizeof(uint32_t), s->stream));
  // the grid path's persisting lines (cell counts and offsets) would hold
  // L2 that the list steps stream through
  if (s->l2_window_on) {
    PS_CUDA(cudaStreamSynchronize(s->stream));
    cudaCtxResetPersistingL2Cache();
    cudaGetLastError();
  }
  int rc = save_state(s, s->list_ckpt);
  if (rc == PS_OK) rc = step_graphs(s, n_steps, true);
  if (rc != PS_OK) return rc;
  uint32_t e = 0, nr = 0;
  PS_CUDA(cudaMemcpyAsync(&e, s->err, sizeof(uint32_t), cudaMemcpyDeviceToHost, s->stream));
  PS_CUDA(cudaMemcpyAsync(&nr, rebuilds, sizeof(uint32_t), cudaMemcpyDeviceToHost, s->stream));
  PS_CUDA(cudaStreamSynchronize(s->stream));
  s->list_rebuilds += nr;
  s->list_win_steps += n_steps;
  s->list_win_rebuilds += nr;
  if (s->list_win_steps >= LIST_BACKOFF_WINDOW) {
    if (s->list_win_rebuilds * LIST_BACKOFF_RATE > s->list_win_steps) {
      s->list_backoff_len = std::min<int64_t>(std::max<int64_t>(2 * s->list_backoff_len, LIST_BACKOFF_MIN),
                                              LIST_BACKOFF_MAX);
      s->list_backoff = s->list_backoff_len;
    } else {
      s->list_backoff_len = 0;
    }
    s->list_win_steps = s->list_win_rebuilds = 0;
  }
  constexpr uint32_t list_err = PS_DEVERR_LIST_OVERFLOW | PS_DEVERR_LIST_BARRIER;
  if (e & list_err) {
    // counts and tile totals may be left over from an interrupted rebuild
    const uint32_t rest = e & ~list_err;
    PS_CUDA(cudaMemcpyAsync(s->err, &rest, sizeof(uint32_t), cudaMemcpyHostToDevice, s->stream));
    PS_CUDA(cudaMemsetAsync(s->count, 0, sizeof(uint32_t) * (size_t)n_scan(s), s->stream));
    PS_CUDA(cudaMemsetAsync(s->tile_sum, 0, sizeof(uint32_t) * (size_t)step_scan_tiles(n_scan(s)), s->stream));
    PS_CUDA(cudaStreamSynchronize(s->stream));
    ++s->list_fallbacks;
    rc = load_state(s, s->list_ckpt);
    if (rc == PS_OK) rc = step_graphs(s, n_steps, false);
  }
  return rc;
}

}  // namespace

extern "C" int ps_set_neighbor_lists(ps_sim* s, double skin_fraction, int32_t max_neighbours) {
  if (s == nullptr || !(skin_fraction == 0.0 || (skin_fraction >= 0.01 && skin_fraction <= 1.0)) ||
      (skin_fraction > 0.0 && (max_neighbours < 1 || max_neighbours > 4096)))
    return fail(PS_ERR_INVALID,
                "ps_set_neighbor_lists: skin_fraction must be 0 or in [0.01, 1], and max_neighbours in [1, 4096]");
  DeviceGuard guard(s->device);
  if (max_neighbours != s->list_cap) {  // the arena and the list graphs are rebuilt on the next step
    cudaFree(s->list_arena);
    s->list_arena = nullptr;
    s->list_bytes = 0;
  }
  for (auto it = s->graphs.begin(); it != s->graphs.end();) {
    if (it->first & (int64_t(1) << 62)) {
      cudaGraphExecDestroy(it->second);
      it = s->graphs.erase(it);
    } else {
      ++it;
    }
  }
  s->list_skin = skin_fraction;
  s->list_cap = skin_fraction > 0.0 ? max_neighbours : 0;
  s->list_rebuilds = 0;
  s->list_fallbacks = 0;
  s->list_grid_steps = 0;
  s->list_win_steps = s->list_win_rebuilds = s->list_backoff = s->list_backoff_len = 0;
  return PS_OK;
}

extern "C" int ps_list_stats(ps_sim* s, int64_t* rebuilds, int64_t* fallbacks, int64_t* grid_steps) {
  if (s == nullptr) return fail(PS_ERR_INVALID, "ps_list_stats: null simulation");
  if (rebuilds != nullptr) *rebuilds = s->list_rebuilds;
  if (fallbacks != nullptr) *fallbacks = s->list_fallbacks;
  if (grid_steps != nullptr) *grid_steps = s->list_grid_steps;
  return PS_OK;
}

extern "C" int ps_step(ps_sim* s, int64_t n_steps) {
  const NvtxRange nvtx_range("ps_step");
  if (s == nullptr || n_steps < 0) return fail(PS_ERR_INVALID, "ps_step: bad argument");
  if (!s->grid_sized) return fail(PS_ERR_INVALID, "ps_step: call ps_set_state first");
  s->last_launches = 0;
  if (n_steps == 0 || s->n_total == 0) return PS_OK;
  DeviceGuard guard(s->device);
  ensure_l2_limit(s);
  const bool lists = s->list_skin > 0.0;
  int rc = PS_OK;
  int64_t left = n_steps;
  if (lists && s->list_backoff > 0) {
    const int64_t g = std::min(left, s->list_backoff);
    rc = step_graphs(s, g, false);
    s->list_backoff -= g;
    s->list_grid_steps += g;
    left -= g;
  }
  if (rc == PS_OK && left > 0) rc = lists ? step_lists(s, left) : step_graphs(s, left, false);
  if (rc != PS_OK) return rc;
  s->grid_valid = !lists;  // after the list path the grid arrays do not describe the at-rest state
  s->stepped = true;
  return PS_OK;
}

extern "C" int ps_checkpoint_save(ps_sim* s, int32_t slot) {
  if (s == nullptr || slot < 0) return fail(PS_ERR_INVALID, "ps_checkpoint_save: bad argument");
  if (!s->grid_sized) return fail(PS_ERR_INVALID, "ps_checkpoint_save: no state uploaded");
  DeviceGuard guard(s->device);
  const size_t vb = (s->precision == PS_FP32 ? 16 : 32) * (size_t)s->n_total, ob = 4 * (size_t)s->n_total;
  void*& buf = s->checkpoints[slot];
  if (buf == nullptr) PS_CUDA(cudaMalloc(&buf, std::max<size_t>(2 * vb + ob, 16)));
  char* p = static_cast<char*>(buf);
  PS_CUDA(cudaMemcpyAsync(p, s->P0, vb, cudaMemcpyDeviceToDevice, s->stream));
  PS_CUDA(cudaMemcpyAsync(p + vb, s->V1, vb, cudaMemcpyDeviceToDevice, s->stream));
  PS_CUDA(cudaMemcpyAsync(p + 2 * vb, s->orig, ob, cudaMemcpyDeviceToDevice, s->stream));
  return PS_OK;
}

extern "C" int ps_checkpoint_load(ps_sim* s, int32_t slot) {
  if (s == nullptr) return fail(PS_ERR_INVALID, "ps_checkpoint_load: null simulation");
  auto it = s->checkpoints.find(slot);
  if (it == s->checkpoints.end()) return fail(PS_ERR_INVALID, "ps_checkpoint_load: empty slot " + std::to_string(slot));
  DeviceGuard guard(s->device);
  const size_t vb = (s->precision == PS_FP32 ? 16 : 32) * (size_t)s->n_total, ob = 4 * (size_t)s->n_total;
  const char* p = static_cast<const char*>(it->second);
  PS_CUDA(cudaMemcpyAsync(s->P0, p, vb, cudaMemcpyDeviceToDevice, s->stream));
  PS_CUDA(cudaMemcpyAsync(s->V1, p + vb, vb, cudaMemcpyDeviceToDevice, s->stream));
  PS_CUDA(cudaMemcpyAsync(s->orig, p + 2 * vb, ob, cudaMemcpyDeviceToDevice, s->stream));
  s->grid_valid = false;
  return PS_OK;
}

extern "C" int ps_time_steps(ps_sim* s, int64_t n_steps, double* device_ms) {
  if (s == nullptr || device_ms == nullptr) return fail(PS_ERR_INVALID, "ps_time_steps: bad argument");
  DeviceGuard guard(s->device);
  cudaEvent_t a, b;
  PS_CUDA(cudaEventCreate(&a));
  PS_CUDA(cudaEventCreate(&b));
  PS_CUDA(cudaEventRecord(a, s->stream));
  int rc = ps_step(s, n_steps);
  cudaEventRecord(b, s->stream);
  cudaEventSynchronize(b);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (rc != PS_OK) return rc;
  *device_ms = (double)ms;
  return check_device_error(s);
}

namespace {

// Rebuild every grid-dependent buffer after the scenes' cell sizes changed.
// The particle arrays, the state and the checkpoints are kept; the captured
// step graphs, the adjoint arena and the recorded forward pass are dropped.
int resize_grids(ps_sim* s, const std::vector<double>& host_state) {
  for (auto& kv : s->graphs) cudaGraphExecDestroy(kv.second);
  s->graphs.clear();
  void** bufs_to_free[] = {&s->cell_arena, &s->d_scenes, &s->d_bounds, &s->d_tri, &s->d_nrm, &s->d_aabb,
                           &s->adj_arena};
  for (void** b : bufs_to_free) {
    cudaFree(*b);
    *b = nullptr;
  }
  cudaFree(s->d_bin_offset);
  cudaFree(s->d_bin_tri);
  cudaFree(s->d_mesh_view);
  s->d_bin_offset = s->d_bin_tri = nullptr;
  s->d_mesh_view = nullptr;
  s->adj_bytes = 0;
  s->fwd_steps = 0;
  s->l2_window_on = false;
  s->grid_sized = false;
  s->grid_valid = false;
  return size_grids(s, host_state.data());
}

}  // namespace

extern "C" int ps_autotune(ps_sim* s, int64_t trial_steps, const double* cell_factors, int32_t n_factors,
                           const int64_t* graph_blocks, int32_t n_blocks, double* ms_table, ps_tune_result* out) {
  const NvtxRange nvtx_range("ps_autotune");
  if (s == nullptr || out == nullptr || trial_steps < 1 || cell_factors == nullptr || n_factors < 1 ||
      graph_blocks == nullptr || n_blocks < 1)
    return fail(PS_ERR_INVALID, "ps_autotune: bad argument");
  if (!s->grid_sized) return fail(PS_ERR_INVALID, "ps_autotune: call ps_set_state first");
  for (int32_t f = 0; f < n_factors; ++f)
    if (!(cell_factors[f] >= 1.0) || !std::isfinite(cell_factors[f]))
      return fail(PS_ERR_INVALID, "ps_autotune: cell factors must be finite and >= 1");
  for (int32_t l = 0; l < n_blocks; ++l)
    if (graph_blocks[l] < 1) return fail(PS_ERR_INVALID, "ps_autotune: graph blocks must be >= 1");
  DeviceGuard guard(s->device);
  // the starting state, on the host (radii for the cell sizes) and on the device
  std::vector<double> host((size_t)8 * (size_t)std::max<int64_t>(s->n_total, 1));
  int rc = ps_get_state(s, host.data(), s->n_total);
  if (rc != PS_OK) return rc;
  std::vector<double> r_max(s->n_scenes, 0.0);
  for (int sc = 0; sc < s->n_scenes; ++sc)
    for (int64_t i = s->pbase[sc]; i < s->pbase[sc + 1]; ++i) r_max[sc] = std::max(r_max[sc], host[8 * i + 6]);
  void* saved = nullptr;
  rc = save_state(s, saved);
  if (rc != PS_OK) return rc;
  cudaEvent_t ea, eb;
  PS_CUDA(cudaEventCreate(&ea));
  PS_CUDA(cudaEventCreate(&eb));
  // one trial: warm-up (captures the graphs), restore, timed steps, restore
  auto trial = [&](double& ms_per_step) -> int {
    int r = load_state(s, saved);
    if (r == PS_OK) r = ps_step(s, std::min(trial_steps, s->graph_block));
    if (r == PS_OK) r = load_state(s, saved);
    if (r != PS_OK) return r;
    cudaEventRecord(ea, s->stream);
    r = ps_step(s, trial_steps);
    cudaEventRecord(eb, s->stream);
    if (cudaEventSynchronize(eb) != cudaSuccess) return fail(PS_ERR_CUDA, "ps_autotune: timing failed");
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ea, eb);
    ms_per_step = (double)ms / (double)trial_steps;
    if (r == PS_OK) r = check_device_error(s);
    return r;
  };
  auto apply_factor = [&](double f) -> int {
    for (int sc = 0; sc < s->n_scenes; ++sc)
      if (r_max[sc] > 0.0) s->desc[sc].cell_size = f * 2.0 * r_max[sc];
    return resize_grids(s, host);
  };
  double before = 0.0;
  rc = trial(before);
  double best = INFINITY, best_f = cell_factors[0];
  int64_t best_l = graph_blocks[0];
  for (int32_t f = 0; f < n_factors && rc == PS_OK; ++f) {
    rc = apply_factor(cell_factors[f]);
    for (int32_t l = 0; l < n_blocks && rc == PS_OK; ++l) {
      for (auto& kv : s->graphs) cudaGraphExecDestroy(kv.second);
      s->graphs.clear();
      s->graph_block = graph_blocks[l];
      double ms = 0.0;
      rc = trial(ms);
      if (ms_table != nullptr) ms_table[(size_t)f * (size_t)n_blocks + (size_t)l] = ms;
      if (rc == PS_OK && ms < best) {
        best = ms;
        best_f = cell_factors[f];
        best_l = graph_blocks[l];
      }
    }
  }
  if (rc == PS_OK) rc = apply_factor(best_f);
  for (auto& kv : s->graphs) cudaGraphExecDestroy(kv.second);
  s->graphs.clear();
  s->graph_block = best_l;
  // then the contact kernel on the chosen grid and graph length: the walk
  // and its CTA size (the summation order depends on neither)
  int32_t best_walk = s->walk, best_cb = s->contact_block;
  double best_k = INFINITY;
  for (int32_t v = 0; v < kContactConfigs && rc == PS_OK; ++v) {
    s->walk = kContactConfig[v][0];
    s->contact_block = kContactConfig[v][1];
    for (auto& kv : s->graphs) cudaGraphExecDestroy(kv.second);
    s->graphs.clear();
    double ms = 0.0;
    rc = trial(ms);
    out->contact_ms[v] = ms;
    if (rc == PS_OK && ms < best_k) {
      best_k = ms;
      best_walk = s->walk;
      best_cb = s->contact_block;
    }
  }
  s->walk = best_walk;
  s->contact_block = best_cb;
  for (auto& kv : s->graphs) cudaGraphExecDestroy(kv.second);
  s->graphs.clear();
  if (rc == PS_OK) rc = load_state(s, saved);
  if (rc == PS_OK) rc = ps_sync(s);
  cudaEventDestroy(ea);
  cudaEventDestroy(eb);
  cudaFree(saved);
  if (rc != PS_OK) return rc;
  out->cell_factor = best_f;
  out->graph_block = best_l;
  out->ms_per_step = std::min(best, best_k);
  out->before_ms_per_step = before;
  out->contact_walk = best_walk;
  out->contact_block = best_cb;
  return PS_OK;
}

extern "C" int ps_set_contact_kernel(ps_sim* s, int32_t walk, int32_t block) {
  if (s == nullptr) return fail(PS_ERR_INVALID, "ps_set_contact_kernel: null simulation");
  bool ok = false;
  for (int32_t v = 0; v < kContactConfigs; ++v) ok = ok || (kContactConfig[v][0] == walk && kContactConfig[v][1] == block);
  if (!ok)
    return fail(PS_ERR_INVALID, "ps_set_contact_kernel: walk/block must be PS_WALK_LANE/128, 256, 512, PS_WALK_WARP/256 or "
                "PS_WALK_ADAPTIVE/256");
  if (walk != s->walk || block != s->contact_block) {
    DeviceGuard guard(s->device);
    for (auto& kv : s->graphs) cudaGraphExecDestroy(kv.second);  // they hold the previous kernel
    s->graphs.clear();
    s->walk = walk;
    s->contact_block = block;
  }
  return PS_OK;
}

extern "C" int ps_get_contact_kernel(ps_sim* s, int32_t* walk, int32_t* block) {
  if (s == nullptr || walk == nullptr || block == nullptr) return fail(PS_ERR_INVALID, "ps_get_contact_kernel: bad argument");
  *walk = s->walk;
  *block = s->contact_block;
  return PS_OK;
}

extern "C" int ps_tune_neighbor_lists(ps_sim* s, int64_t trial_steps, const double* skins, int32_t n_skins,
                                      int32_t max_neighbours, double* ms_table, double* best_skin) {
  const NvtxRange nvtx_range("ps_tune_neighbor_lists");
  if (s == nullptr || best_skin == nullptr || trial_steps < 1 || skins == nullptr || n_skins < 1 ||
      max_neighbours < 1 || max_neighbours > 4096)
    return fail(PS_ERR_INVALID, "ps_tune_neighbor_lists: bad argument");
  for (int32_t k = 0; k < n_skins; ++k)
    if (!(skins[k] == 0.0 || (skins[k] >= 0.01 && skins[k] <= 1.0)))
      return fail(PS_ERR_INVALID, "ps_tune_neighbor_lists: each skin_fraction must be 0 or in [0.01, 1]");
  if (!s->grid_sized) return fail(PS_ERR_INVALID, "ps_tune_neighbor_lists: call ps_set_state first");
  DeviceGuard guard(s->device);
  void* saved = nullptr;
  int rc = save_state(s, saved);
  if (rc != PS_OK) return rc;
  cudaEvent_t ea, eb;
  PS_CUDA(cudaEventCreate(&ea));
  PS_CUDA(cudaEventCreate(&eb));
  // one trial: the same steps twice from the saved state, the second timed
  // (the first captures the graphs)
  auto trial = [&](double skin, double& ms_per_step) -> int {
    int r = ps_set_neighbor_lists(s, skin, max_neighbours);
    if (r == PS_OK) r = load_state(s, saved);
    if (r == PS_OK) r = ps_step(s, trial_steps);
    if (r == PS_OK) r = load_state(s, saved);
    if (r != PS_OK) return r;
    cudaEventRecord(ea, s->stream);
    r = ps_step(s, trial_steps);
    cudaEventRecord(eb, s->stream);
    if (cudaEventSynchronize(eb) != cudaSuccess) return fail(PS_ERR_CUDA, "ps_tune_neighbor_lists: timing failed");
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ea, eb);
    ms_per_step = (double)ms / (double)trial_steps;
    if (r == PS_OK) r = check_device_error(s);
    return r;
  };
  double best = INFINITY, best_k = skins[0];
  for (int32_t k = 0; k < n_skins && rc == PS_OK; ++k) {
    double ms = 0.0;
    rc = trial(skins[k], ms);
    if (ms_table != nullptr) ms_table[k] = ms;
    if (rc == PS_OK && ms < best) {
      best = ms;
      best_k = skins[k];
    }
  }
  if (rc == PS_OK) rc = ps_set_neighbor_lists(s, best_k, max_neighbours);
  if (rc == PS_OK) rc = load_state(s, saved);
  if (rc == PS_OK) rc = ps_sync(s);
  cudaEventDestroy(ea);
  cudaEventDestroy(eb);
  cudaFree(saved);
  if (rc != PS_OK) return rc;
  *best_skin = best_k;
  return PS_OK;
}

extern "C" int ps_profile_steps(ps_sim* s, int64_t n_steps, double* kernel_ms, int64_t* kernel_launches) {
  if (s == nullptr || kernel_ms == nullptr || kernel_launches == nullptr || n_steps < 1)
    return fail(PS_ERR_INVALID, "ps_profile_steps: bad argument");
  if (!s->grid_sized) return fail(PS_ERR_INVALID, "ps_profile_steps: call ps_set_state first");
  for (int k = 0; k < PS_K_COUNT; ++k) {
    kernel_ms[k] = 0.0;
    kernel_launches[k] = 0;
  }
  if (s->n_total == 0) return PS_OK;
  DeviceGuard guard(s->device);
  std::vector<LaunchRecord> rec((size_t)(1 + 4 * n_steps));
  for (auto& r : rec) {
    PS_CUDA(cudaEventCreate(&r.a));
    PS_CUDA(cudaEventCreate(&r.b));
  }
  if (s->precision == PS_FP32)
    enqueue_steps_recorded_dispatch<float>(s, n_steps, rec);
  else
    enqueue_steps_recorded_dispatch<double>(s, n_steps, rec);
  const cudaError_t le = cudaGetLastError();
  cudaStreamSynchronize(s->stream);
  for (auto& r : rec) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, r.a, r.b);
    kernel_ms[r.kind] += (double)ms;
    kernel_launches[r.kind] += 1;
    cudaEventDestroy(r.a);
    cudaEventDestroy(r.b);
  }
  if (le != cudaSuccess) return fail(PS_ERR_CUDA, std::string("ps_profile_steps: ") + cudaGetErrorString(le));
  s->grid_valid = true;
  return check_device_error(s);
}

extern "C" int ps_forward_checkpointed(ps_sim* s, int64_t n_steps, int64_t every) {
  const NvtxRange nvtx_range("ps_forward_checkpointed");
  if (s == nullptr || n_steps < 1 || every < 1) return fail(PS_ERR_INVALID, "ps_forward_checkpointed: bad argument");
  if (!s->grid_sized) return fail(PS_ERR_INVALID, "ps_forward_checkpointed: call ps_set_state first");
  if (s->has_mesh) return fail(PS_ERR_INVALID, "ps_forward_checkpointed: differentiation supports box containers only");
  DeviceGuard guard(s->device);
  const int64_t n_blocks = (n_steps + every - 1) / every;
  for (size_t k = (size_t)n_blocks + 1; k < s->fwd_ckpt.size(); ++k) cudaFree(s->fwd_ckpt[k]);
  s->fwd_ckpt.resize((size_t)n_blocks + 1, nullptr);
  for (int64_t blk = 0; blk < n_blocks; ++blk) {
    int rc = save_state(s, s->fwd_ckpt[(size_t)blk]);
    if (rc == PS_OK) rc = ps_step(s, std::min(every, n_steps - blk * every));
    if (rc != PS_OK) return rc;
  }
  int rc = save_state(s, s->fwd_ckpt.back());
  if (rc != PS_OK) return rc;
  s->fwd_steps = n_steps;
  s->fwd_every = every;
  return ps_sync(s);
}

extern "C" int ps_backward(ps_sim* s, const double* dl_dstate, ps_grad* grads, double* dl_dstate0) {
  const NvtxRange nvtx_range("ps_backward");
  if (s == nullptr || dl_dstate == nullptr || grads == nullptr) return fail(PS_ERR_INVALID, "ps_backward: null argument");
  if (s->fwd_steps < 1) return fail(PS_ERR_INVALID, "ps_backward: call ps_forward_checkpointed first");
  if (s->n_total == 0) {  // no particle: every gradient is zero
    for (int sc = 0; sc < s->n_scenes; ++sc) grads[sc] = ps_grad{};
    return PS_OK;
  }
  DeviceGuard guard(s->device);
  ensure_l2_limit(s);
  if (s->precision == PS_FP32)
    return s->multi ? backward_impl<float, true>(s, dl_dstate, grads, dl_dstate0)
                    : backward_impl<float, false>(s, dl_dstate, grads, dl_dstate0);
  return s->multi ? backward_impl<double, true>(s, dl_dstate, grads, dl_dstate0)
                  : backward_impl<double, false>(s, dl_dstate, grads, dl_dstate0);
}

extern "C" int ps_sync(ps_sim* s) {
  if (s == nullptr) return fail(PS_ERR_INVALID, "ps_sync: null simulation");
  DeviceGuard guard(s->device);
  PS_CUDA(cudaStreamSynchronize(s->stream));
  return check_device_error(s);
}

extern "C" int64_t ps_last_launch_count(ps_sim* s) { return s ? s->last_launches : -1; }

extern "C" int ps_grid_get(ps_sim* s, int32_t scene, ps_grid_info* out) {
  if (s == nullptr || out == nullptr || scene < 0 || scene >= s->n_scenes) return fail(PS_ERR_INVALID, "ps_grid_get: bad argument");
  if (!s->grid_sized) return fail(PS_ERR_INVALID, "ps_grid_get: no state uploaded");
  const GridHost& g = s->grids[scene];
  for (int a = 0; a < 3; ++a) {
    out->min[a] = g.min[a];
    out->nb[a] = g.nb[a];
  }
  out->interval = g.interval;
  out->n_cells = g.n_cells;
  out->cell_base = g.cbase;
  out->particle_base = s->pbase[scene];
  return PS_OK;
}

extern "C" int ps_buckets_get(ps_sim* s, uint32_t* counts, uint32_t* offsets, uint32_t* order) {
  if (s == nullptr) return fail(PS_ERR_INVALID, "ps_buckets_get: null simulation");
  if (!s->grid_sized) return fail(PS_ERR_INVALID, "ps_buckets_get: no state uploaded");
  DeviceGuard guard(s->device);
  if (!s->grid_valid) {
    const int rc = regrid(s);
    if (rc != PS_OK) return rc;
  }
  if (counts != nullptr && s->c_total > 0) {
    // the count array itself is cleared during the step; derive it from the offsets
    uint32_t* d = nullptr;
    PS_CUDA(cudaMallocAsync(&d, sizeof(uint32_t) * s->c_total, s->stream));
    k_counts_from_offsets<<<(unsigned)((s->c_total + 255) / 256), 256, 0, s->stream>>>(s->offset, d, s->c_total);
    cudaMemcpyAsync(counts, d, sizeof(uint32_t) * s->c_total, cudaMemcpyDeviceToHost, s->stream);
    cudaFreeAsync(d, s->stream);
    PS_CUDA(cudaGetLastError());
  }
  if (offsets != nullptr && s->c_total > 0)
    PS_CUDA(cudaMemcpyAsync(offsets, s->offset, sizeof(uint32_t) * s->c_total, cudaMemcpyDeviceToHost, s->stream));
  if (order != nullptr && s->n_total > 0)
    PS_CUDA(cudaMemcpyAsync(order, s->orig, sizeof(uint32_t) * s->n_total, cudaMemcpyDeviceToHost, s->stream));
  PS_CUDA(cudaStreamSynchronize(s->stream));
  return check_device_error(s);
}

extern "C" int ps_stats_get(ps_sim* s, int32_t scene, ps_stats* out) {
  if (s == nullptr || out == nullptr || scene < 0 || scene >= s->n_scenes) return fail(PS_ERR_INVALID, "ps_stats_get: bad argument");
  if (!s->grid_sized) return fail(PS_ERR_INVALID, "ps_stats_get: no state uploaded");
  DeviceGuard guard(s->device);
  std::memset(out, 0, sizeof(*out));
  const int64_t n = s->pbase[scene + 1] - s->pbase[scene];
  if (n == 0) return PS_OK;
  if (!s->grid_valid) {
    const int rc = regrid(s);
    if (rc != PS_OK) return rc;
  }
  const uint32_t first = (uint32_t)s->pbase[scene];
  if (s->precision == PS_FP32) {
    k_stats<float><<<kStatsBlocks, kStatsThreads, 0, s->stream>>>(bufs<float>(s), s->sp32[scene], first, (uint32_t)n, s->d_stats);
  } else {
    k_stats<double><<<kStatsBlocks, kStatsThreads, 0, s->stream>>>(bufs<double>(s), s->sp64[scene], first, (uint32_t)n, s->d_stats);
  }
  k_stats_final<<<1, 32, 0, s->stream>>>(s->d_stats, s->d_stats_out);
  PS_CUDA(cudaGetLastError());
  StatsPartial h{};
  PS_CUDA(cudaMemcpyAsync(&h, s->d_stats_out, sizeof(h), cudaMemcpyDeviceToHost, s->stream));
  PS_CUDA(cudaStreamSynchronize(s->stream));
  out->kinetic_energy = h.ke;
  for (int a = 0; a < 3; ++a) {
    out->min_pos[a] = h.mn[a];
    out->max_pos[a] = h.mx[a];
  }
  out->n_collided = (int64_t)h.collided;
  out->max_overlap = h.max_overlap;
  return check_device_error(s);
}

extern "C" int ps_destroy(ps_sim* s) {
  if (s == nullptr) return PS_OK;
  {
    DeviceGuard guard(s->device);
    if (s->stream) cudaStreamSynchronize(s->stream);
    free_sim(s);
  }
  delete s;
  return PS_OK;
}

extern "C" int ps_simulate(const ps_scene_desc* scene, const double* aos_in, double* aos_out, int64_t max_steps,
                           int32_t precision) {
  if (scene == nullptr || max_steps < 0) return fail(PS_ERR_INVALID, "ps_simulate: bad argument");
  ps_sim* s = nullptr;
  int rc = ps_create(scene, 1, precision, 0, &s);
  if (rc != PS_OK) return rc;
  rc = ps_set_state(s, aos_in, scene->n_particles);
  if (rc == PS_OK) rc = ps_step(s, max_steps);
  if (rc == PS_OK) rc = ps_get_state(s, aos_out, scene->n_particles);
  ps_destroy(s);
  return rc;
}

extern "C" size_t ps_exclusive_scan_scratch_bytes(int64_t n) { return n <= 0 ? 8 : scan_scratch_bytes(n); }

extern "C" int ps_exclusive_scan_u32(const uint32_t* d_in, uint32_t* d_out, int64_t n, void* d_scratch, void* stream) {
  if (n < 0 || (n > 0 && (d_in == nullptr || d_out == nullptr || d_scratch == nullptr)))
    return fail(PS_ERR_INVALID, "ps_exclusive_scan_u32: bad argument");
  if (n == 0) return PS_OK;
  if (n > (int64_t)1 << 40) return fail(PS_ERR_INVALID, "ps_exclusive_scan_u32: n too large");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // scratch: [uint32 ticket][uint32 error word][uint64 status per tile]
  uint32_t* err = static_cast<uint32_t*>(d_scratch) + 1;
  PS_CUDA(cudaMemsetAsync(d_scratch, 0, scan_scratch_bytes(n), st));
  k_exclusive_scan_u32<<<(unsigned)scan_num_tiles(n), SCAN_THREADS, 0, st>>>(d_in, d_out, n, static_cast<uint64_t*>(d_scratch),
                                                                             err);
  PS_CUDA(cudaGetLastError());
  return PS_OK;
}

// ---- exclusive scan that allocates nothing -------------------------------------
// Scratch for ps_exclusive_scan_u32_noalloc: the ticket word and one status
// word per tile, for at most PS_SCAN_NOALLOC_MAX_N elements.  Each GPU
// holds its own copy of this array from the moment the library is loaded on
// it until the process exits.
namespace {
constexpr int64_t kNoAllocMaxTiles = PS_SCAN_NOALLOC_MAX_N / SCAN_TILE;  // 16384
constexpr int kNoAllocMaxContexts = 64;
static_assert(PS_SCAN_NOALLOC_MAX_N % SCAN_TILE == 0, "whole tiles");
}  // namespace

static __device__ __align__(256) uint64_t g_noalloc_scan_scratch[1 + kNoAllocMaxTiles];
// Device error bits (PS_DEVERR_SCAN_TIMEOUT) of every call since the last
// ps_exclusive_scan_u32_noalloc_status on this GPU.  Kept apart from the
// scratch array, which each call clears.
static __device__ __align__(256) uint32_t g_noalloc_scan_error;

namespace {
// Device addresses of the two arrays per CUDA context, found on the first
// call made with that context current.  Host code must not pass the
// symbols themselves: on the host they name stand-ins, not device memory.
// Keyed by context rather than by device: a context of the caller's own, or
// the primary context made again after cudaDeviceReset, holds its own copies.
struct NoAllocAddrs {
  void* ctx;
  uint64_t* scratch;
  uint32_t* err;
};
NoAllocAddrs g_noalloc_addrs[kNoAllocMaxContexts];
int g_noalloc_n = 0;
std::mutex g_noalloc_mu;

using CtxGetCurrentFn = int (*)(void**);  // cuCtxGetCurrent, through the runtime's driver entry point

void* current_context() {
  static const CtxGetCurrentFn fn = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      f = nullptr;
    return reinterpret_cast<CtxGetCurrentFn>(f);
  }();
  void* ctx = nullptr;
  if (fn == nullptr || fn(&ctx) != 0) return nullptr;
  return ctx;
}

int noalloc_addrs(const char* who, uint64_t** scratch, uint32_t** err) {
  void* ctx = current_context();
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (ctx != nullptr) {
    for (int k = 0; k < g_noalloc_n; ++k)
      if (g_noalloc_addrs[k].ctx == ctx) {
        *scratch = g_noalloc_addrs[k].scratch;
        *err = g_noalloc_addrs[k].err;
        return PS_OK;
      }
  }
  void *ps = nullptr, *pe = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&ps, g_noalloc_scan_scratch);
  if (e == cudaSuccess) e = cudaGetSymbolAddress(&pe, g_noalloc_scan_error);
  if (e != cudaSuccess || ps == nullptr || pe == nullptr)
    return fail(PS_ERR_CUDA, std::string(who) + ": cudaGetSymbolAddress: " + cudaGetErrorString(e));
  *scratch = static_cast<uint64_t*>(ps);
  *err = static_cast<uint32_t*>(pe);
  if (ctx == nullptr) ctx = current_context();  // the lookup made the device's primary context current
  if (ctx != nullptr) {
    if (g_noalloc_n == kNoAllocMaxContexts) {  // the oldest entry makes room
      for (int m = 1; m < kNoAllocMaxContexts; ++m) g_noalloc_addrs[m - 1] = g_noalloc_addrs[m];
      --g_noalloc_n;
    }
    g_noalloc_addrs[g_noalloc_n++] = {ctx, *scratch, *err};
  }
  return PS_OK;
}
}  // namespace

extern "C" int ps_exclusive_scan_u32_noalloc(const uint32_t* d_in, uint32_t* d_out, int64_t n, void* stream) {
  if (n < 0 || (n > 0 && (d_in == nullptr || d_out == nullptr)))
    return fail(PS_ERR_INVALID, "ps_exclusive_scan_u32_noalloc: bad argument");
  if (n > PS_SCAN_NOALLOC_MAX_N)
    return fail(PS_ERR_INVALID, "ps_exclusive_scan_u32_noalloc: n = " + std::to_string(n) +
                                    " exceeds the fixed scratch capacity of " +
                                    std::to_string(PS_SCAN_NOALLOC_MAX_N) + " elements");
  if (n == 0) return PS_OK;
  uint64_t* scratch = nullptr;
  uint32_t* err = nullptr;
  const int rc = noalloc_addrs("ps_exclusive_scan_u32_noalloc", &scratch, &err);
  if (rc != PS_OK) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // the previous call left its ticket and tile flags behind: clear what this
  // call's tiles read
  PS_CUDA(cudaMemsetAsync(scratch, 0, scan_scratch_bytes(n), st));
  k_exclusive_scan_u32<<<(unsigned)scan_num_tiles(n), SCAN_THREADS, 0, st>>>(d_in, d_out, n, scratch, err);
  PS_CUDA(cudaGetLastError());
  return PS_OK;
}

extern "C" int ps_exclusive_scan_u32_noalloc_status(void* stream, uint32_t* device_error) {
  if (device_error == nullptr) return fail(PS_ERR_INVALID, "ps_exclusive_scan_u32_noalloc_status: null device_error");
  uint64_t* scratch = nullptr;
  uint32_t* err = nullptr;
  const int rc = noalloc_addrs("ps_exclusive_scan_u32_noalloc_status", &scratch, &err);
  if (rc != PS_OK) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  uint32_t word = 0;
  PS_CUDA(cudaMemcpyAsync(&word, err, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  PS_CUDA(cudaMemsetAsync(err, 0, sizeof(uint32_t), st));
  PS_CUDA(cudaStreamSynchronize(st));
  *device_error = word;
  return PS_OK;
}
