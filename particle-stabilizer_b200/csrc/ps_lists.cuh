// ps_lists.cuh — neighbour-list mode of the step (opt-in, ps_set_neighbor_lists).
//
// Between grid rebuilds the state stays in the sorted order of the last
// rebuild, in two alternating buffers; each step is one kernel that walks a
// per-sphere list of neighbours instead of the 27 grid cells.
//
// Exactness.  A pair changes a velocity only while it overlaps, i.e. while
// |x_i - x_j| < r_i + r_j.  A list built with the cut-off r_i + r_j + skin
// holds every such pair as long as no sphere has moved more than skin / 2
// since the build.  The step kernel applies the overlapping pairs of a
// sphere in ascending (cell id at this step, original id) order: the order
// in which the 27-cell walk of k_contacts meets them.  Overlap test and
// velocity update are contact_one itself, and a pair counts only when the
// cells of the two spheres at the step are adjacent (the 27-cell walk's own
// condition, which rounding in the hash can make stricter than the overlap),
// so every velocity is bit-identical to the grid step's.
//
// Rebuilds.  The step kernel also integrates the next step (as the fused
// k_contacts) and tests whether some sphere has moved more than about
// skin / 2 from where the lists were built; warps that see one set the flag
// word of the next step's parity.  Before each step a cooperative kernel,
// one wave of CTAs, reads the word of that step's parity: clear, it returns
// at once (about a microsecond; a conditional graph node costs ten); set, it
// runs count, scan, scatter, rank/move and list build as phases separated by
// grid barriers.  Each step kernel clears its own parity's word, which the
// rebuild before it has read, for the step after next.  A list longer than
// the capacity, or a sphere whose overlapping pairs change order and
// outnumber the sort buffer, sets PS_DEVERR_LIST_OVERFLOW, and a barrier
// that waits too long sets PS_DEVERR_LIST_BARRIER; the host then repeats
// the call on the grid path.
#pragma once

#include "ps_step_kernels.cuh"

namespace psb {

constexpr int LIST_CONTACTS_MAX = 32;  // sort buffer: overlapping pairs of a sphere whose order changed

// words of ListBufs::flag; the first LIST_RESET_WORDS are zeroed when a
// graph of steps starts
enum : int {
  LIST_MOVED = 0,     // [parity of a step]: rebuild before that step (2 words)
  LIST_BAR = 2,       // grid barrier: arrivals, generation (2 words)
  LIST_RESET_WORDS = 4,
  LIST_REBUILDS = 4,  // rebuilds in the running call
  LIST_FLAG_WORDS = 5
};

// List entries whose loads the step kernel issues together.  Measured on
// 1M-sphere scenes: FP32 single-scene runs gain most from 4; the batch
// variant (scene lookup) spills at 4 and is fastest at 2; FP64 spills at
// 2 and above and is fastest at 1.
template <class T, bool MULTI>
__host__ __device__ constexpr int list_batch() {
  return sizeof(T) == 4 ? (MULTI ? 2 : 4) : 1;
}

constexpr uint32_t LIST_BARRIER_SPIN_LIMIT = 1u << 22;  // x >= 64 ns sleeps: a wait of 0.25 s or more

template <class T>
struct ListBufs {
  vec4_t<T>* P[2];     // post-wall positions (x, r) of the step, list order; alternate by step
  vec4_t<T>* V[2];     // pre-contact velocities (v, m)
  uint32_t* cell[2];   // cell id of each slot at the step
  vec4_t<T>* ref;      // positions when the lists were built
  uint32_t* list;      // [k][slot]: neighbour slots, ascending (cell, original id) at the build
  uint32_t* cnt;       // list length per slot
  uint32_t* flag;      // LIST_FLAG_WORDS words (LIST_MOVED ...)
  uint32_t cap;        // list capacity per sphere
  T skin_frac;         // skin as a fraction of each scene's cell edge
};

// Cells [c0, c1] of one axis that can hold a point within `reach` of x.
// The hash is monotonic in x, so the cells of x - reach and x + reach bound
// them; the pad covers the rounding of x +- reach.
template <class T>
__device__ __forceinline__ void axis_span(T x, T reach, T lo, T iv, int32_t nb, int32_t& c0, int32_t& c1) {
  const T pad = reach + (fabs(x) + fabs(lo)) * T(1.0 / 1048576.0);
  c0 = axis_cell<T>(x - pad, lo, iv, nb);
  c1 = axis_cell<T>(x + pad, lo, iv, nb);
}

// List of slot i from the sorted post-wall state (P0, V0, scell) of a
// rebuild; the state is copied into the step buffer `dst` in the same order.
// Partners lie within r_i + r_max + skin <= r_i + cell / 2 + skin, which
// bounds the cells to visit on each axis.  Columns are visited in ascending
// cell id and slots in order, so each list is sorted by (cell, original id).
template <class T, bool MULTI, bool COH>
__device__ __forceinline__ void list_build_one(uint32_t i, const StepBufs<T>& b, const SceneParams<T>& sp0,
                                               const ListBufs<T>& L, int dst) {
  const SceneParams<T>& sp = scene_of<T, MULTI>(i, sp0, b.scenes, b.pbase, b.n_scenes);
  const vec4_t<T> P = b.P0[i];
  L.P[dst][i] = P;
  L.V[dst][i] = b.V0[i];
  L.cell[dst][i] = b.scell[i];
  L.ref[i] = P;
  const bool live = isfinite(P.x) && isfinite(P.y) && isfinite(P.z);
  const T skin = L.skin_frac * sp.interval;
  uint32_t k = 0;
  if (live) {
    const T reach = (P.w + T(0.5) * sp.interval + skin) * T(1.001);
    int32_t x0, x1, y0, y1, z0, z1;
    axis_span<T>(P.x, reach, sp.grid_lo[0], sp.interval, sp.nb[0], x0, x1);
    axis_span<T>(P.y, reach, sp.grid_lo[1], sp.interval, sp.nb[1], y0, y1);
    axis_span<T>(P.z, reach, sp.grid_lo[2], sp.interval, sp.nb[2], z0, z1);
    const uint32_t ny = (uint32_t)sp.nb[1], nz = (uint32_t)sp.nb[2];
    // candidates of one column's slot range [j0, j1)
    auto walk = [&](uint32_t j0, uint32_t j1) {
      if (!in_bounds(j1, (uint64_t)b.n + 1u, b.err)) return;
      for (uint32_t j = j0; j < j1; ++j) {
        if (j == i) continue;
        const vec4_t<T> Q = ld4c<T, COH>(b.P0 + j);
        const T dx = P.x - Q.x, dy = P.y - Q.y, dz = P.z - Q.z;
        // generous cut-off: the list may hold more than needed, never less
        const T cut = (P.w + Q.w + skin) * T(1.0001);
        if (dx * dx + dy * dy + dz * dz < cut * cut) {
          if (k < L.cap) L.list[(size_t)k * b.n + i] = j;
          ++k;
        }
      }
    };
    if (x1 - x0 < 3 && y1 - y0 < 3) {
      // the usual span of at most 3 x 3 columns: all range bounds are loaded
      // before the walk, which visits the columns in the same order
      uint32_t lo[9], hi[9];
#pragma unroll
      for (int q = 0; q < 9; ++q) {
        const int32_t bx = x0 + q / 3, by = y0 + q % 3;
        const bool ok = bx <= x1 && by <= y1;
        const uint32_t col = sp.cbase + ((uint32_t)(ok ? bx : x0) * ny + (uint32_t)(ok ? by : y0)) * nz;
        lo[q] = ok ? ld_ro<COH>(b.offset + col + (uint32_t)z0) : 0u;
        hi[q] = ok ? ld_ro<COH>(b.offset + col + (uint32_t)z1 + 1u) : 0u;
      }
#pragma unroll
      for (int q = 0; q < 9; ++q) walk(lo[q], hi[q]);
    } else {
      for (int32_t bx = x0; bx <= x1; ++bx) {
        for (int32_t by = y0; by <= y1; ++by) {
          const uint32_t col = sp.cbase + ((uint32_t)bx * ny + (uint32_t)by) * nz;
          walk(ld_ro<COH>(b.offset + col + (uint32_t)z0), ld_ro<COH>(b.offset + col + (uint32_t)z1 + 1u));
        }
      }
    }
  }
  L.cnt[i] = k < L.cap ? k : L.cap;
  if (k > L.cap) atomicOr(b.err, PS_DEVERR_LIST_OVERFLOW);
}

// The full rebuild that starts a call builds the lists with this kernel.
template <class T, bool MULTI>
__global__ void __launch_bounds__(STEP_THREADS) k_list_build(StepBufs<T> b, SceneParams<T> sp0, ListBufs<T> L,
                                                             int dst) {
  pdl_wait();
  const uint32_t i = blockIdx.x * STEP_THREADS + threadIdx.x;
  if (i < b.n) list_build_one<T, MULTI, false>(i, b, sp0, L, dst);
}

// Grid-wide barrier of a cooperative launch (every CTA resident): arrivals
// are counted in bar[0]; the last CTA to arrive resets the count and
// advances the generation bar[1], for which the others wait.  A CTA that
// waits past the limit records PS_DEVERR_LIST_BARRIER and returns false,
// and its caller leaves the kernel; no later barrier of the kernel can then
// complete, so at most one more phase runs, on data it indexes in bounds.
__device__ __forceinline__ bool grid_barrier(uint32_t* bar, uint32_t* err) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    volatile uint32_t* gen = bar + 1;
    const uint32_t g = *gen;
    __threadfence();
    if (atomicAdd(bar, 1u) == gridDim.x - 1u) {
      atomicExch(bar, 0u);
      __threadfence();
      atomicAdd(bar + 1, 1u);
    } else {
      uint32_t spins = 0;
      while (*gen == g) {
        if (++spins == LIST_BARRIER_SPIN_LIMIT) {
          atomicOr(err, PS_DEVERR_LIST_BARRIER);
          ok = 0;
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// Rebuild before step `par` when the gate is open: count the cells of the
// state in buffer `par` (b.P1 / b.V1 / b.cell point there), scan, scatter,
// rank and move into P0 / V0 / orig / scell, and build the lists, copying
// the sorted state back into buffer `par`.  One wave of CTAs loops over
// each phase's blocks or tiles; reads of data written earlier in the kernel
// go through L2 (COH).  A rebuild after a barrier failure is skipped: the
// counts may then be incomplete.
template <class T, bool MULTI>
__global__ void __launch_bounds__(STEP_THREADS) k_list_rebuild(StepBufs<T> b, SceneParams<T> sp0, ListBufs<T> L,
                                                               int par, int64_t n_cells, uint32_t scan_tiles,
                                                               uint32_t scatter_blocks, uint32_t move_blocks) {
  if (L.flag[LIST_MOVED + par] == 0u || (*b.err & PS_DEVERR_LIST_BARRIER) != 0u) return;
  if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(L.flag + LIST_REBUILDS, 1u);
  uint32_t* bar = L.flag + LIST_BAR;
  for (uint32_t base = blockIdx.x * STEP_THREADS; base < b.n; base += gridDim.x * STEP_THREADS) {
    const uint32_t p = base + threadIdx.x;
    const bool valid = p < b.n;
    count_cell(b.count, b.tile_sum, valid ? b.cell[p] : 0u, valid, b.tile_shift);
  }
  if (!grid_barrier(bar, b.err)) return;
  for (uint32_t t = blockIdx.x; t < scan_tiles; t += gridDim.x) {
    __syncthreads();  // the tile scan reuses its shared arrays
    if (b.tile_shift == 13u)
      scan_tile_with_sums<true, STEP_SCAN_ITEMS_LARGE>(t, b.count, b.offset, n_cells, b.tile_sum);
    else
      scan_tile_with_sums<true, STEP_SCAN_ITEMS_SMALL>(t, b.count, b.offset, n_cells, b.tile_sum);
  }
  if (!grid_barrier(bar, b.err)) return;
  for (uint32_t blk = blockIdx.x; blk < scatter_blocks; blk += gridDim.x)
    scatter_block<true>(blk, b.cell, b.slot, b.orig, b.offset, b.tmp, b.count, b.n, b.tile_sum, b.n_tiles, b.err);
  if (!grid_barrier(bar, b.err)) return;
  for (uint32_t blk = blockIdx.x; blk < move_blocks; blk += gridDim.x) rank_move_block<T, true>(blk, b);
  if (!grid_barrier(bar, b.err)) return;
  for (uint32_t i = blockIdx.x * STEP_THREADS + threadIdx.x; i < b.n; i += gridDim.x * STEP_THREADS)
    list_build_one<T, MULTI, true>(i, b, sp0, L, par);
}

// Overlap of a listed pair at this step, as contact_one decides it, plus
// the 27-cell walk's adjacency condition.  On success `key` orders the pair
// as the walk does: (cell at this step, original id).
template <class T>
__device__ __forceinline__ bool list_pair(const ListBufs<T>& L, const StepBufs<T>& b, const SceneParams<T>& sp,
                                          int src, const vec4_t<T>& P, const vec4_t<T>& Q, uint32_t j, int32_t cx,
                                          int32_t cy, int32_t cz, uint64_t& key) {
  using A = Ar<T>;
  const T margin = T(1) + T(1.0 / 1048576.0);
  const T dx = A::sub(P.x, Q.x), dy = A::sub(P.y, Q.y), dz = A::sub(P.z, Q.z);
  const T d2 = A::fma(dz, dz, A::fma(dy, dy, A::mul(dx, dx)));
  const T s = A::add(P.w, Q.w);
  if (d2 >= A::mul(A::mul(s, s), margin)) return false;
  if (!(A::sub(s, A::sqrt(d2)) > T(0))) return false;
  const uint32_t cj = L.cell[src][j];
  int32_t jx, jy, jz;
  cell_coords<T>(cj, sp, jx, jy, jz);
  if (abs(jx - cx) > 1 || abs(jy - cy) > 1 || abs(jz - cz) > 1) return false;
  key = ((uint64_t)cj << 32) | (uint64_t)__ldg(b.orig + j);
  return true;
}

// One step on the lists: contacts of the step held in buffer `src`, then
// (FUSED) the next step's integrate + container + cell id into buffer
// 1 - src and the displacement test, whose warps set the flag word of the
// next step; the last step of a call (not FUSED) writes the at-rest state
// (P0 positions, V1 velocities) instead.  Every load a sphere needs is
// issued up front, and list entries list_batch() at a time, so that each
// thread keeps several memory requests in flight.  One wave of CTAs loops
// over the spheres (no tail wave, no per-CTA launch cost): 1M spheres 37.2
// -> 34.5 us per step, 256 scenes 214 -> 155 us.
template <class T, bool MULTI, bool MESH, bool FUSED>
__global__ void __launch_bounds__(STEP_THREADS, sizeof(T) == 4 ? 4 : 3)
    k_contacts_list(StepBufs<T> b, SceneParams<T> sp0, const MeshView* mv, ListBufs<T> L, int src) {
  pdl_wait();
  const int dst = 1 - src;
  // this step's flag was read by the rebuild before it; clear it for the
  // step after next
  if (blockIdx.x == 0 && threadIdx.x == 0) L.flag[LIST_MOVED + src] = 0u;
  bool any_moved = false;
  // the loop bound is the same for the whole CTA, so every lane reaches the
  // warp vote after it
  for (uint32_t base = blockIdx.x * STEP_THREADS; base < b.n; base += gridDim.x * STEP_THREADS) {
  const uint32_t i = base + threadIdx.x;
  const bool valid = i < b.n;
  bool moved = false;
  if (valid) {
    const SceneParams<T>& sp = scene_of<T, MULTI>(i, sp0, b.scenes, b.pbase, b.n_scenes);
    const vec4_t<T>* __restrict__ Ps = L.P[src];
    vec4_t<T> P = Ps[i];
    const vec4_t<T> Vi = L.V[src][i];
    const uint32_t ci = L.cell[src][i];
    const uint32_t nl = L.cnt[i];
    vec4_t<T> R{};
    if (FUSED) R = L.ref[i];
    T vx = Vi.x, vy = Vi.y, vz = Vi.z;
    int32_t cx, cy, cz;
    cell_coords<T>(ci, sp, cx, cy, cz);
    const bool live = isfinite(P.x) && isfinite(P.y) && isfinite(P.z);
    if (live && nl > 0u) {
      const T ks = sp.k_spring, es = sp.e_sphere;
      // The list is in ascending (cell, original id) at the build; while
      // the overlapping pairs still come in ascending keys they are applied
      // in list order.
      uint64_t last = 0;
      bool ordered = true;
      constexpr int NB = list_batch<T, MULTI>();
      for (uint32_t k0 = 0; k0 < nl && ordered; k0 += NB) {
        uint32_t jj[NB];
        vec4_t<T> QQ[NB];
#pragma unroll
        for (int u = 0; u < NB; ++u) {
          jj[u] = k0 + u < nl ? L.list[(size_t)(k0 + u) * b.n + i] : i;
          if (!in_bounds(jj[u], b.n, b.err)) jj[u] = i;
        }
#pragma unroll
        for (int u = 0; u < NB; ++u) QQ[u] = ld4<T>(Ps + jj[u]);
#pragma unroll
        for (int u = 0; u < NB; ++u) {
          uint64_t kj;
          if (k0 + u < nl && ordered && list_pair<T>(L, b, sp, src, P, QQ[u], jj[u], cx, cy, cz, kj)) {
            if (kj < last) {
              ordered = false;
            } else {
              last = kj;
              contact_one<T>(L.V[src], jj[u], P, Vi, QQ[u], ks, es, vx, vy, vz);
            }
          }
        }
      }
      if (!ordered) {
        // some neighbour changed cells since the build: sort the
        // overlapping pairs and start over
        vx = Vi.x;
        vy = Vi.y;
        vz = Vi.z;
        uint64_t key[LIST_CONTACTS_MAX];
        uint32_t who[LIST_CONTACTS_MAX];
        int nc = 0;
        for (uint32_t k = 0; k < nl; ++k) {
          const uint32_t j = L.list[(size_t)k * b.n + i];
          if (!in_bounds(j, b.n, b.err)) continue;
          uint64_t kj;
          if (!list_pair<T>(L, b, sp, src, P, ld4<T>(Ps + j), j, cx, cy, cz, kj)) continue;
          if (nc == LIST_CONTACTS_MAX) {
            atomicOr(b.err, PS_DEVERR_LIST_OVERFLOW);
            break;
          }
          int m = nc++;
          while (m > 0 && key[m - 1] > kj) {
            key[m] = key[m - 1];
            who[m] = who[m - 1];
            --m;
          }
          key[m] = kj;
          who[m] = j;
        }
        for (int m = 0; m < nc; ++m) contact_one<T>(L.V[src], who[m], P, Vi, ld4<T>(Ps + who[m]), ks, es, vx, vy, vz);
      }
    }
    vec4_t<T> V = Vi;
    V.x = vx;
    V.y = vy;
    V.z = vz;
    if (FUSED) {
      integrate<T>(P, V, sp);
      if constexpr (MESH) {
        if (sp.mesh_tris > 0)
          mesh_contacts<T>(P, V, sp, *mv, b.err);
        else
          walls<T>(P, V, sp);
      } else {
        walls<T>(P, V, sp);
      }
      const uint32_t c = cell_near<T>(P.x, P.y, P.z, sp, b.bounds, cx, cy, cz);
      L.P[dst][i] = P;
      L.V[dst][i] = V;
      L.cell[dst][i] = c;
      // rebuild when the sphere is near half the skin from the build
      // position, or finite again after a non-finite build position; a
      // non-finite position takes part in no contact and asks for nothing
      const T ex = P.x - R.x, ey = P.y - R.y, ez = P.z - R.z;
      const T half = T(0.49) * L.skin_frac * sp.interval;
      const bool fin = isfinite(P.x) && isfinite(P.y) && isfinite(P.z);
      moved = fin && !(ex * ex + ey * ey + ez * ez <= half * half);
    } else {
      b.P0[i] = P;
      b.V1[i] = V;
    }
  }
  any_moved |= moved;
  }
  if (FUSED && __any_sync(0xffffffffu, any_moved) && (threadIdx.x & 31u) == 0u)
    atomicOr(L.flag + LIST_MOVED + dst, 1u);
}

}  // namespace psb
