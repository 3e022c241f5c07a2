// ps_step_kernels.cuh — the per-step kernels of the DEM hot path.
//
// Reference step (src/ParticleStabilizerCUDA/PhysicsEngineCUDA.cpp:38-42):
//   integrate -> container contacts -> grid rebuild -> sphere contacts (Jacobi)
// New pipeline, one launch per stage, all scenes of a batch in every launch:
//
//   k_begin     x += v dt, v += g dt, box walls / triangles, cell hash,
//               warp-aggregated count                    (first step of a call)
//   scan        exclusive scan of the cell counts        (ps_scan.cuh)
//   k_scatter   slot = --count[c] (atomic; leaves the counts at zero),
//               orig id -> tmp[offset[c] + slot]
//   k_rank_move canonical in-cell rank (ascending orig id), float4 state move
//   k_contacts  27-cell Jacobi contacts; FUSED also runs the next step's
//               integrate + container + hash + count in its epilogue
//
// Buffers (N particles, C cells over all scenes):
//   P0/V0  sorted state (pos_r, vel_m) read by k_contacts
//   P1/V1  integrated state written by k_begin / fused k_contacts
//   at rest between calls the state is (P0 positions, V1 velocities, orig)
//   orig   original particle index of each slot
//   cell, slot, tmp  per-particle uint32
//   count, offset    per-cell uint32, C+1 entries (count[C] stays 0)
#pragma once

#include "ps_device.cuh"
#include "ps_mesh.cuh"
#include "ps_scan.cuh"

namespace psb {

constexpr int STEP_THREADS = 256;

// ---- scene lookup ------------------------------------------------------------
template <class T, bool MULTI>
__device__ __forceinline__ const SceneParams<T>& scene_of(uint32_t p, const SceneParams<T>& sp0,
                                                          const SceneParams<T>* sps, const uint32_t* pbase,
                                                          int n_scenes) {
  if (!MULTI) return sp0;
  int lo = 0, hi = n_scenes - 1;  // largest s with pbase[s] <= p
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(pbase + mid) <= p)
      lo = mid;
    else
      hi = mid - 1;
  }
  return sps[lo];
}

// ---- cell hashing (ParticleModel_kernels.cu:42-73) ---------------------------
// Per-axis index (int)((x - lo) / interval), clamped to [0, nb-1]; NaN and
// negative quotients give 0.
template <class T>
__device__ __forceinline__ int32_t axis_cell(T x, T lo, T iv, int32_t nb) {
  using A = Ar<T>;
  const T q = A::div(A::sub(x, lo), iv);
  if (!(q > T(0))) return 0;
  if (q >= (T)nb) return nb - 1;
  return (int32_t)q;
}

template <class T>
__device__ __forceinline__ uint32_t cell_of(T x, T y, T z, const SceneParams<T>& sp, int32_t& cx, int32_t& cy,
                                            int32_t& cz) {
  cx = axis_cell<T>(x, sp.grid_lo[0], sp.interval, sp.nb[0]);
  cy = axis_cell<T>(y, sp.grid_lo[1], sp.interval, sp.nb[1]);
  cz = axis_cell<T>(z, sp.grid_lo[2], sp.interval, sp.nb[2]);
  // z fastest: (i*ny + j)*nz + k
  return sp.cbase + ((uint32_t)cx * (uint32_t)sp.nb[1] + (uint32_t)cy) * (uint32_t)sp.nb[2] + (uint32_t)cz;
}

// Cell index of x when the particle was in cell k before: the boundary test
// settles the usual case (no crossing) exactly; crossings and NaN take the
// division.  axis_cell is monotonic in x, so B[k] <= x < B[k+1] implies
// axis_cell(x) == k.
template <class T>
__device__ __forceinline__ int32_t axis_cell_near(T x, int32_t k, const T* B, T lo, T iv, int32_t nb) {
  if (__ldg(B + k) <= x && x < __ldg(B + k + 1)) return k;
  return axis_cell<T>(x, lo, iv, nb);
}

template <class T>
__device__ __forceinline__ uint32_t cell_near(T x, T y, T z, const SceneParams<T>& sp, const T* bounds, int32_t& cx,
                                              int32_t& cy, int32_t& cz) {
  cx = axis_cell_near<T>(x, cx, bounds + sp.bnd_base[0], sp.grid_lo[0], sp.interval, sp.nb[0]);
  cy = axis_cell_near<T>(y, cy, bounds + sp.bnd_base[1], sp.grid_lo[1], sp.interval, sp.nb[1]);
  cz = axis_cell_near<T>(z, cz, bounds + sp.bnd_base[2], sp.grid_lo[2], sp.interval, sp.nb[2]);
  return sp.cbase + ((uint32_t)cx * (uint32_t)sp.nb[1] + (uint32_t)cy) * (uint32_t)sp.nb[2] + (uint32_t)cz;
}

// ---- integrate (PhysicsEngine_kernels.cu:10-16) ------------------------------
template <class T>
__device__ __forceinline__ void integrate(vec4_t<T>& P, vec4_t<T>& V, const SceneParams<T>& sp) {
  using A = Ar<T>;
  P.x = A::fma(V.x, sp.dt, P.x);
  P.y = A::fma(V.y, sp.dt, P.y);
  P.z = A::fma(V.z, sp.dt, P.z);
  V.x = A::fma(sp.gravity[0], sp.dt, V.x);
  V.y = A::fma(sp.gravity[1], sp.dt, V.y);
  V.z = A::fma(sp.gravity[2], sp.dt, V.z);
}

// ---- box walls (BoxContainer_kernels.cu:17-52) --------------------------------
// Order xmin, ymin, zmin, xmax, ymax, zmax; the extents are taken before any
// clamp; the reflected component is -v*e whatever its sign.
template <class T>
__device__ __forceinline__ void walls(vec4_t<T>& P, vec4_t<T>& V, const SceneParams<T>& sp) {
  using A = Ar<T>;
  const T r = P.w;
  const T mnx = A::sub(P.x, r), mny = A::sub(P.y, r), mnz = A::sub(P.z, r);
  const T mxx = A::add(P.x, r), mxy = A::add(P.y, r), mxz = A::add(P.z, r);
  if (mnx < sp.box_lo[0]) { P.x = A::add(sp.box_lo[0], r); V.x = A::mul(-V.x, sp.e_lo[0]); }
  if (mny < sp.box_lo[1]) { P.y = A::add(sp.box_lo[1], r); V.y = A::mul(-V.y, sp.e_lo[1]); }
  if (mnz < sp.box_lo[2]) { P.z = A::add(sp.box_lo[2], r); V.z = A::mul(-V.z, sp.e_lo[2]); }
  if (mxx > sp.box_hi[0]) { P.x = A::sub(sp.box_hi[0], r); V.x = A::mul(-V.x, sp.e_hi[0]); }
  if (mxy > sp.box_hi[1]) { P.y = A::sub(sp.box_hi[1], r); V.y = A::mul(-V.y, sp.e_hi[1]); }
  if (mxz > sp.box_hi[2]) { P.z = A::sub(sp.box_hi[2], r); V.z = A::mul(-V.z, sp.e_hi[2]); }
}

// ---- cell count ---------------------------------------------------------------
// One atomic reduction per particle, whose result is not used (the warp
// does not wait for it; at a few particles per cell lanes rarely share a
// cell, so aggregating them first costs more than it saves); the slot
// inside the cell is taken later by k_scatter.  The same pass accumulates,
// warp-aggregated, the per-tile totals of the count array (1 << tile_shift
// cells per tile) that the step's scan uses in place of a look-back.
// With tile_sum null only the cell counts are taken (k_tile_sums forms the
// totals afterwards).
__device__ __forceinline__ void count_cell(uint32_t* count, uint32_t* tile_sum, uint32_t c, bool valid,
                                           uint32_t tile_shift) {
  const unsigned lane = threadIdx.x & 31u;
  const unsigned active = __ballot_sync(0xffffffffu, valid);
  if (valid && tile_sum == nullptr) {
    atomicAdd(count + c, 1u);
    return;
  }
  if (valid) {
    atomicAdd(count + c, 1u);
    const uint32_t t = c >> tile_shift;
    const int first = __ffs(active) - 1;
    if (__all_sync(active, t == __shfl_sync(active, t, first))) {
      // the usual case in sorted order: the whole warp counts into one tile
      if ((int)lane == first) atomicAdd(tile_sum + t, (uint32_t)__popc(active));
    } else {
      const unsigned tpeers = __match_any_sync(active, t);
      if ((int)lane == __ffs(tpeers) - 1) atomicAdd(tile_sum + t, (uint32_t)__popc(tpeers));
    }
  }
}

template <class T>
struct StepBufs {
  vec4_t<T>* P0;
  vec4_t<T>* V0;
  vec4_t<T>* P1;
  vec4_t<T>* V1;
  uint32_t* orig;
  uint32_t* cell;
  uint32_t* slot;
  uint32_t* tmp;
  uint32_t* count;
  uint32_t* offset;
  uint32_t* err;
  const SceneParams<T>* scenes;
  const uint32_t* pbase;  // n_scenes entries
  int32_t n_scenes;
  uint32_t n;             // particles over all scenes
  uint32_t* tile_sum;     // per-tile totals of `count`, cleared by k_scatter
  uint32_t n_tiles;       // tiles of the step scan
  uint32_t tile_shift;    // log2 of a step-scan tile's cells
  uint32_t n_scan;        // entries of count and offset (cells over all scenes + 1)
  uint32_t* scell;        // global cell id of each sorted slot (written by k_rank_move)
  const T* bounds;        // per-scene, per-axis cell boundaries (see SceneParams::bnd_base)
  // Optional tape row (null outside the adjoint's recompute): k_contacts
  // writes the at-rest state after its step in sorted order, and the
  // pre-contact velocity and sorted cell id of the step's grid.
  vec4_t<T>* tape_p;
  vec4_t<T>* tape_v;
  vec4_t<T>* tape_vpre;
  uint32_t* tape_o;
  uint32_t* tape_cell;
};

// Container step + hash + count on an integrated state, shared by k_begin and
// the fused epilogue of k_contacts.
template <class T, bool MESH>
__device__ __forceinline__ void finish_integrated(vec4_t<T>& P, vec4_t<T>& V, const SceneParams<T>& sp,
                                                  const MeshView* mv, uint32_t* err, uint32_t& c) {
  if constexpr (MESH) {
    if (sp.mesh_tris > 0)
      mesh_contacts<T>(P, V, sp, *mv, err);
    else
      walls<T>(P, V, sp);
  } else {
    walls<T>(P, V, sp);
  }
  int32_t cx, cy, cz;
  c = cell_of<T>(P.x, P.y, P.z, sp, cx, cy, cz);
}

// First kernel of a call: integrate + container + hash + count from the
// at-rest state (P0, V1).  With INTEGRATE false it only hashes (regrid).
template <class T, bool MULTI, bool MESH, bool INTEGRATE>
__global__ void __launch_bounds__(STEP_THREADS) k_begin(StepBufs<T> b, SceneParams<T> sp0, const MeshView* mv) {
  const uint32_t p = blockIdx.x * STEP_THREADS + threadIdx.x;
  const bool valid = p < b.n;
  uint32_t c = 0;
  pdl_wait();
  if (valid) {
    const SceneParams<T>& sp = scene_of<T, MULTI>(p, sp0, b.scenes, b.pbase, b.n_scenes);
    vec4_t<T> P = b.P0[p];
    vec4_t<T> V = b.V1[p];
    if (INTEGRATE) {
      integrate<T>(P, V, sp);
      finish_integrated<T, MESH>(P, V, sp, mv, b.err, c);
    } else {
      int32_t cx, cy, cz;
      c = cell_of<T>(P.x, P.y, P.z, sp, cx, cy, cz);
    }
    b.P1[p] = P;
    b.V1[p] = V;
    b.cell[p] = c;
  }
  // A regrid (INTEGRATE false) hashes a state in any order, often the
  // upload's: per-tile totals would take one contended atomic per sphere, so
  // it counts cells only and k_tile_sums forms the totals.
  count_cell(b.count, INTEGRATE ? b.tile_sum : nullptr, c, valid && in_bounds(c, b.n_scan - 1u, b.err), b.tile_shift);
}

// tile_sum[t] = sum of count over step-scan tile t (1 << tile_shift cells),
// one CTA per tile.
__global__ void __launch_bounds__(STEP_THREADS) k_tile_sums(const uint32_t* __restrict__ count, int64_t n,
                                                           uint32_t* __restrict__ tile_sum, uint32_t tile_shift) {
  __shared__ uint32_t s_red[STEP_THREADS / 32];
  const int64_t base = (int64_t)blockIdx.x << tile_shift;
  const int64_t end = base + (int64_t(1) << tile_shift);
  uint32_t sum = 0;
  for (int64_t e = base + threadIdx.x; e < end && e < n; e += STEP_THREADS) sum += count[e];
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, d);
  if ((threadIdx.x & 31u) == 0) s_red[threadIdx.x >> 5] = sum;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t t = 0;
    for (int w = 0; w < STEP_THREADS / 32; ++w) t += s_red[w];
    tile_sum[blockIdx.x] = t;
  }
}

constexpr int MOVE_PER_THREAD = 4;

// slot[p] of a sphere alone in its cell: its final position, tagged.  (The
// scan's offsets and positions are below 2^31: ps_create caps the particle
// count there.)
constexpr uint32_t SLOT_ALONE = 0x80000000u;

// slot = --count[c], a distinct slot of the cell for every member (the
// decrements bring every count back to zero for the next step);
// tmp[offset[c] + slot] = orig, and the slot is kept for k_rank_move.  A
// sphere alone in its cell (offset[c + 1] == offset[c] + 1, most cells at a
// few tenths of a sphere per cell) keeps its final position offset[c]
// instead, tagged SLOT_ALONE, so k_rank_move moves it without reading the
// offsets again or ranking.  The tile totals are cleared for the next count.
// MOVE_PER_THREAD particles per thread, strided by the block so that every
// load instruction stays coalesced; all loads are issued before the stores.
// Block `blk` of the scatter (COH: see ld_ro).
template <bool COH>
__device__ __forceinline__ void scatter_block(uint32_t blk, const uint32_t* __restrict__ cell,
                                              uint32_t* __restrict__ slot, const uint32_t* __restrict__ orig,
                                              const uint32_t* __restrict__ offset, uint32_t* tmp, uint32_t* count,
                                              uint32_t n, uint32_t* tile_sum, uint32_t n_tiles, uint32_t* err) {
  const uint32_t t = blk * STEP_THREADS + threadIdx.x;
  if (t < n_tiles) tile_sum[t] = 0u;
  const uint32_t base = blk * (STEP_THREADS * MOVE_PER_THREAD) + threadIdx.x;
  uint32_t c[MOVE_PER_THREAD], sl[MOVE_PER_THREAD], o[MOVE_PER_THREAD], off[MOVE_PER_THREAD],
      nxt[MOVE_PER_THREAD];
#pragma unroll
  for (int k = 0; k < MOVE_PER_THREAD; ++k) {
    const uint32_t p = base + k * STEP_THREADS;
    c[k] = p < n ? ld_pl<COH>(cell + p) : 0u;
    o[k] = p < n ? ld_pl<COH>(orig + p) : 0u;
  }
#pragma unroll
  for (int k = 0; k < MOVE_PER_THREAD; ++k) {
    const bool in = (base + k * STEP_THREADS) < n;
    off[k] = in ? ld_ro<COH>(offset + c[k]) : 0u;
    nxt[k] = in ? ld_ro<COH>(offset + c[k] + 1) : 0u;
    sl[k] = in ? atomicSub(count + c[k], 1u) - 1u : 0u;
  }
#pragma unroll
  for (int k = 0; k < MOVE_PER_THREAD; ++k) {
    if (base + k * STEP_THREADS < n && in_bounds(off[k] + sl[k], n, err)) {
      tmp[off[k] + sl[k]] = o[k];
      slot[base + k * STEP_THREADS] = nxt[k] - off[k] == 1u ? (off[k] | SLOT_ALONE) : sl[k];
    }
  }
}

__global__ void __launch_bounds__(STEP_THREADS) k_scatter(const uint32_t* __restrict__ cell,
                                                          uint32_t* __restrict__ slot,
                                                          const uint32_t* __restrict__ orig,
                                                          const uint32_t* __restrict__ offset, uint32_t* tmp,
                                                          uint32_t* count, uint32_t n, uint32_t* tile_sum,
                                                          uint32_t n_tiles, uint32_t* err) {
  pdl_wait();
  scatter_block<false>(blockIdx.x, cell, slot, orig, offset, tmp, count, n, tile_sum, n_tiles, err);
}

// Canonical position = offset[c] + #{members of c with a smaller orig id};
// moves the integrated state (P1, V1) there as (P0, V0) with its orig id.
// A sphere alone in its cell has its position from k_scatter (SLOT_ALONE).
template <class T, bool COH>
__device__ __forceinline__ void rank_move_block(uint32_t blk, const StepBufs<T>& b) {
  const uint32_t base = blk * (STEP_THREADS * MOVE_PER_THREAD) + threadIdx.x;
  // Loads in dependent rounds, each issued for all MOVE_PER_THREAD
  // particles before any store (the stores could alias them as far as the
  // compiler knows, which would otherwise serialise the rounds per particle):
  // cell, slot and the moved state; the cell's range (shared cells only);
  // the member's orig id.
  uint32_t c[MOVE_PER_THREAD], sl[MOVE_PER_THREAD], start[MOVE_PER_THREAD], end[MOVE_PER_THREAD],
      o[MOVE_PER_THREAD];
  vec4_t<T> P[MOVE_PER_THREAD], V[MOVE_PER_THREAD];
#pragma unroll
  for (int k = 0; k < MOVE_PER_THREAD; ++k) {
    const uint32_t p = base + k * STEP_THREADS;
    const bool in = p < b.n;
    c[k] = in ? b.cell[p] : 0u;
    sl[k] = in ? b.slot[p] : 0u;
    if (in) {
      P[k] = b.P1[p];
      V[k] = b.V1[p];
    }
  }
#pragma unroll
  for (int k = 0; k < MOVE_PER_THREAD; ++k) {
    const bool shared = base + k * STEP_THREADS < b.n && !(sl[k] & SLOT_ALONE);
    start[k] = shared ? ld_ro<COH>(b.offset + c[k]) : (sl[k] & ~SLOT_ALONE);
    end[k] = shared ? ld_ro<COH>(b.offset + c[k] + 1) : start[k] + 1u;
    if (!shared) sl[k] = 0u;
  }
#pragma unroll
  for (int k = 0; k < MOVE_PER_THREAD; ++k)
    o[k] = (base + k * STEP_THREADS < b.n && in_bounds(start[k] + sl[k], b.n, b.err)) ? b.tmp[start[k] + sl[k]] : 0u;
#pragma unroll
  for (int k = 0; k < MOVE_PER_THREAD; ++k) {
    if (base + k * STEP_THREADS >= b.n) continue;
    if (!in_bounds(end[k], b.n + 1u, b.err)) continue;
    uint32_t rank = 0;
    if (end[k] - start[k] > 1u)
      for (uint32_t s = start[k]; s < end[k]; ++s) rank += (b.tmp[s] < o[k]) ? 1u : 0u;
    const uint32_t d = start[k] + rank;
    if (!in_bounds(d, b.n, b.err)) continue;
    b.P0[d] = P[k];
    b.V0[d] = V[k];
    b.orig[d] = o[k];
    b.scell[d] = c[k];
  }
}

template <class T>
__global__ void __launch_bounds__(STEP_THREADS) k_rank_move(StepBufs<T> b) {
  pdl_wait();
  rank_move_block<T, false>(blockIdx.x, b);
}

// ---- sphere-sphere contacts (ParticleModel_kernels.cu:136-201) --------------
// One thread per sorted particle; the neighbours are read from the sorted
// arrays.  For each (dx, dy) column the three z-cells are contiguous in the
// sorted order, so 9 slot ranges cover the 27 cells, visited x-outer, y,
// z-inner, members in canonical order.  The 18 range bounds are loaded
// together before the candidate loop.
//
// Candidates far enough apart skip the square root: overlap > 0 holds exactly
// when sqrt_rn(d2) < s with s = r_i + r_j (rounded); if d2 >= fl(s*s)*(1+2^-20)
// then d2 > s*s, so sqrt(d2) > s and, rounding being monotonic,
// sqrt_rn(d2) >= s.  The filter therefore rejects only pairs the exact test
// rejects, and the result stays bit-identical.
// Contribution of neighbour j (position Pj) to particle i's velocity.
template <class T>
__device__ __forceinline__ void contact_one(const vec4_t<T>* __restrict__ V0, uint32_t j, const vec4_t<T>& P,
                                            const vec4_t<T>& Vi, const vec4_t<T>& Pj, T k, T e, T& vx, T& vy,
                                            T& vz) {
  using A = Ar<T>;
  const T margin = T(1) + T(1.0 / 1048576.0);
  const T dx = A::sub(P.x, Pj.x), dy = A::sub(P.y, Pj.y), dz = A::sub(P.z, Pj.z);
  const T d2 = A::fma(dz, dz, A::fma(dy, dy, A::mul(dx, dx)));
  const T s = A::add(P.w, Pj.w);
  if (d2 >= A::mul(A::mul(s, s), margin)) return;
  const T dist = A::sqrt(d2);
  const T overlap = A::sub(s, dist);
  if (overlap > T(0)) {
    const vec4_t<T> Vj = ld4<T>(V0 + j);
    const T rvx = A::sub(Vi.x, Vj.x), rvy = A::sub(Vi.y, Vj.y), rvz = A::sub(Vi.z, Vj.z);
    const T rvd = A::fma(rvz, dz, A::fma(rvy, dy, A::mul(rvx, dx)));
    const T cr = A::div(A::mul(A::mul(A::mul(T(2), Vj.w), rvd), e), A::mul(A::add(Vi.w, Vj.w), d2));
    const T cs = A::div(A::mul(k, overlap), A::mul(dist, Vi.w));
    const T f = A::sub(cs, cr);
    vx = A::fma(f, dx, vx);
    vy = A::fma(f, dy, vy);
    vz = A::fma(f, dz, vz);
  }
}

// Cell coordinates of a sorted slot from its global cell id.
template <class T>
__device__ __forceinline__ void cell_coords(uint32_t c, const SceneParams<T>& sp, int32_t& cx, int32_t& cy,
                                            int32_t& cz) {
  const uint32_t local = c - sp.cbase;
  const uint32_t col = fast_udiv(local, sp.div_nz_m, sp.div_nz_sh1, sp.div_nz_sh2);
  cz = (int32_t)(local - col * (uint32_t)sp.nb[2]);
  cx = (int32_t)fast_udiv(col, sp.div_ny_m, sp.div_ny_sh1, sp.div_ny_sh2);
  cy = (int32_t)(col - (uint32_t)cx * (uint32_t)sp.nb[1]);
}

// Register shuffle of a whole state vector from lane `src`.
template <class T>
__device__ __forceinline__ vec4_t<T> shfl4(const vec4_t<T>& v, int src) {
  vec4_t<T> r;
  r.x = __shfl_sync(0xffffffffu, v.x, src);
  r.y = __shfl_sync(0xffffffffu, v.y, src);
  r.z = __shfl_sync(0xffffffffu, v.z, src);
  r.w = __shfl_sync(0xffffffffu, v.w, src);
  return r;
}

// Walk of the neighbour columns by the whole warp (WALK_WARP).
//
// Every lane's range [mylo, myhi) in a neighbour column lies inside the
// warp's union [ulo, uhi) of that column: the 32 lanes hold consecutive
// sorted slots, so their ranges in the same neighbour column overlap or
// abut, and the union is about a warp's worth of candidates (28.8 on
// average, at most 67, on the 1M-sphere scene).  The union is read in
// windows of 32 * walk_window() slots, walk_window() coalesced loads per
// lane, lane l holding slots base + l + 32 k; each lane takes its own
// candidates from the holders by register shuffle, in ascending slot order.
// That is the per-lane order of the nine-loop walk, so every sum is
// bit-identical to it.
//
// Loads per lane and window, and columns whose first window is in flight
// while the current column is walked.
// Measured on the 1M-sphere scenes (FP32 contact kernel, 256 threads): one
// window of 32 and one column ahead 76.5 us; two windows and two ahead
// 102.7 us; one window three ahead 82.5 us; the lane walk 57.7 us.
template <class T>
__host__ __device__ constexpr int walk_window() {
  return 1;
}
template <class T>
__host__ __device__ constexpr int walk_ahead() {
  return 1;
}

template <class T>
struct Window {
  vec4_t<T> c[walk_window<T>()];
};

// Slots [base, base + 32 walk_window()) of a union ending at `end` (zeros
// past it; an empty union has base >= end).
template <class T>
__device__ __forceinline__ Window<T> load_window(const vec4_t<T>* __restrict__ P0, uint32_t base, uint32_t end,
                                                 unsigned lane) {
  Window<T> w;
#pragma unroll
  for (int k = 0; k < walk_window<T>(); ++k) {
    const uint32_t j = base + lane + 32u * k;
    if (base < end && j < end) {
      w.c[k] = ld4<T>(P0 + j);
    } else {
      w.c[k].x = w.c[k].y = w.c[k].z = w.c[k].w = T(0);
    }
  }
  return w;
}

template <class T>
__device__ __forceinline__ void walk_column(const vec4_t<T>* __restrict__ P0, const vec4_t<T>* __restrict__ V0,
                                            uint32_t i, unsigned lane, uint32_t mylo, uint32_t myhi, uint32_t ulo,
                                            uint32_t uhi, Window<T> win, const vec4_t<T>& P, const vec4_t<T>& Vi,
                                            T ks, T es, T& vx, T& vy, T& vz) {
  for (uint32_t wbase = ulo; wbase < uhi; wbase += 32u * walk_window<T>()) {  // warp-uniform
    if (wbase != ulo) win = load_window<T>(P0, wbase, uhi, lane);
#pragma unroll
    for (int k = 0; k < walk_window<T>(); ++k) {
      const uint32_t base = wbase + 32u * k;
      const uint32_t a = mylo > base ? mylo : base;
      const uint32_t e = myhi < base + 32u ? myhi : base + 32u;
      const uint32_t cnt = e > a ? e - a : 0u;
      const uint32_t mx = __reduce_max_sync(0xffffffffu, cnt);
      for (uint32_t t = 0; t < mx; ++t) {
        // for t < cnt the holder of slot a + t is lane a - base + t < 32
        const vec4_t<T> Pj = shfl4<T>(win.c[k], (int)((a - base + t) & 31u));
        const uint32_t j = a + t;
        if (t < cnt && j != i) contact_one<T>(V0, j, P, Vi, Pj, ks, es, vx, vy, vz);
      }
    }
  }
}

// Neighbour walk of k_contacts.
//   WALK_LANE: each thread loops over its own nine slot ranges.
//   WALK_WARP: the warp walks each column's union range together
//              (walk_column), with the first windows of the next
//              walk_ahead() columns loaded ahead, so a warp waits for a few
//              rounds of coalesced loads instead of one per candidate.
//   WALK_ADAPTIVE: each warp takes the per-lane walk or the flattened walk
//              (walk_flat), whichever its candidate counts predict to be
//              cheaper (adaptive_flat).
// All apply the same candidates in the same order.
enum : int { WALK_LANE = 0, WALK_WARP = 1, WALK_ADAPTIVE = 2 };

// a[q] for a run-time q in [0, 9), by a select tree on the bits of q (the
// array stays in registers).
__device__ __forceinline__ uint32_t pick9(const uint32_t (&a)[9], uint32_t q) {
  const bool b0 = (q & 1u) != 0u, b1 = (q & 2u) != 0u, b2 = (q & 4u) != 0u;
  const uint32_t a01 = b0 ? a[1] : a[0], a23 = b0 ? a[3] : a[2];
  const uint32_t a45 = b0 ? a[5] : a[4], a67 = b0 ? a[7] : a[6];
  const uint32_t a03 = b1 ? a23 : a01, a47 = b1 ? a67 : a45;
  const uint32_t a07 = b2 ? a47 : a03;
  return q == 8u ? a[8] : a07;
}

// Per-lane walk: the nine ranges in canonical order, one loop each; only
// the own column (q = 4) holds the sphere itself.  A warp takes, per
// column, as many trips as its busiest lane has candidates there.
template <class T>
__device__ __forceinline__ void walk_lanes(const vec4_t<T>* __restrict__ P0, const vec4_t<T>* __restrict__ V0,
                                           uint32_t i, const uint32_t (&lo)[9], const uint32_t (&hi)[9],
                                           const vec4_t<T>& P, const vec4_t<T>& Vi, T ks, T es, T& vx, T& vy,
                                           T& vz) {
#pragma unroll
  for (int q = 0; q < 9; ++q)
    for (uint32_t j = lo[q]; j < hi[q]; ++j) {
      if (q == 4 && j == i) continue;
      contact_one<T>(V0, j, P, Vi, ld4<T>(P0 + j), ks, es, vx, vy, vz);
    }
}

// Flattened walk: one loop over the concatenation of the non-empty ranges
// (ascending q, slots ascending within each: the same order), the next
// range's bounds picked from registers.  A warp takes as many trips as its
// busiest lane has candidates in all, but its lanes read from different
// columns in one trip.
template <class T>
__device__ __forceinline__ void walk_flat(const vec4_t<T>* __restrict__ P0, const vec4_t<T>* __restrict__ V0,
                                          uint32_t i, const uint32_t (&lo)[9], const uint32_t (&hi)[9],
                                          const vec4_t<T>& P, const vec4_t<T>& Vi, T ks, T es, T& vx, T& vy,
                                          T& vz) {
  uint32_t m = 0u;  // bit q: range q not started yet and not empty
#pragma unroll
  for (int q = 0; q < 9; ++q) m |= (lo[q] < hi[q] ? 1u : 0u) << q;
  uint32_t j = 0u, e = 0u;
  while (true) {
    if (j >= e) {
      if (m == 0u) break;
      const uint32_t q = (uint32_t)(__ffs(m) - 1);
      m &= m - 1u;
      j = pick9(lo, q);
      e = pick9(hi, q);
    }
    if (j != i) contact_one<T>(V0, j, P, Vi, ld4<T>(P0 + j), ks, es, vx, vy, vz);
    ++j;
  }
}

// The warp's choice of walk (every lane must call it): the per-lane walk
// takes sum_q max_lanes len_q trips, the flattened one max_lanes sum_q len_q
// trips at about 1.7 times the cost of a trip (measured on the 1M-sphere
// box scene: 17.0 against 8.3 trips, neighbour walk 35.5 against 29.6 us),
// so the flattened walk is taken when it saves at least that factor
// (4 col >= 7 flat).  Sparse grids (a few tenths of a sphere per cell) pass;
// dense piles, where both counts are equal, keep the per-lane walk.
__device__ __forceinline__ bool adaptive_flat(const uint32_t (&lo)[9], const uint32_t (&hi)[9]) {
  uint32_t total = 0u;  // distinct slots, below 2^31
  uint64_t col_trips = 0u;
#pragma unroll
  for (int q = 0; q < 9; ++q) {
    const uint32_t len = hi[q] - lo[q];
    total += len;
    col_trips += __reduce_max_sync(0xffffffffu, len);
  }
  const uint64_t flat_trips = __reduce_max_sync(0xffffffffu, total);
  return 4u * col_trips >= 7u * flat_trips;
}

// Resident CTAs per SM the contact kernel is compiled for: 1,024 threads
// per SM in FP32 (64 registers) and 768 in FP64 (85 registers), whatever
// the CTA size.
template <class T, int BLOCK>
__host__ __device__ constexpr int contact_min_blocks() {
  return (sizeof(T) == 4 ? 1024 : 768) / BLOCK > 0 ? (sizeof(T) == 4 ? 1024 : 768) / BLOCK : 1;
}

template <class T, bool MULTI, bool MESH, bool FUSED, int WALK, int BLOCK>
__global__ void __launch_bounds__(BLOCK, contact_min_blocks<T, BLOCK>()) k_contacts(StepBufs<T> b, SceneParams<T> sp0,
                                                                                    const MeshView* mv) {
  const uint32_t i = blockIdx.x * BLOCK + threadIdx.x;
  const bool valid = i < b.n;
  uint32_t c = 0;
  pdl_wait();
  // Lanes past the end walk empty ranges: the warp's shuffles and the
  // count's ballot need every lane.
  const SceneParams<T>& sp = scene_of<T, MULTI>(valid ? i : 0u, sp0, b.scenes, b.pbase, b.n_scenes);
  vec4_t<T> P, Vi;
  uint32_t my_cell = sp.cbase;
  if (valid) {
    P = b.P0[i];
    Vi = b.V0[i];
    my_cell = b.scell[i];
  } else {
    P.x = P.y = P.z = P.w = T(0);
    Vi = P;
  }
  T vx = Vi.x, vy = Vi.y, vz = Vi.z;
  int32_t cx, cy, cz;
  cell_coords<T>(my_cell, sp, cx, cy, cz);
  const int32_t nx = sp.nb[0], ny = sp.nb[1], nz = sp.nb[2];
  const uint32_t z0 = (uint32_t)(cz > 0 ? cz - 1 : 0);
  const uint32_t z1 = (uint32_t)(cz + 1 < nz ? cz + 1 : nz - 1) + 1u;
  // A particle whose own position is not finite has no contact: every
  // pair gives d2 = inf (rejected by the filter) or NaN (overlap NaN), so
  // its candidate loop is skipped.  Diverged particles all hash to a few
  // cells, where the loop would otherwise be quadratic.
  const bool live = valid && isfinite(P.x) && isfinite(P.y) && isfinite(P.z);
  uint32_t lo[9], hi[9];
#pragma unroll
  for (int q = 0; q < 9; ++q) {
    const int32_t bx = cx - 1 + q / 3, by = cy - 1 + q % 3;
    const bool ok = live && bx >= 0 && bx < nx && by >= 0 && by < ny;
    // in-range address even where the column does not exist
    const uint32_t col = ok ? sp.cbase + ((uint32_t)bx * (uint32_t)ny + (uint32_t)by) * (uint32_t)nz : sp.cbase;
    const bool inb = ok && in_bounds(col + z1, b.n_scan, b.err);
    lo[q] = inb ? __ldg(b.offset + col + z0) : 0u;
    hi[q] = inb ? __ldg(b.offset + col + z1) : 0u;
    if (!in_bounds(hi[q], b.n + 1u, b.err)) hi[q] = lo[q] = 0u;
  }
  const T ks = sp.k_spring, es = sp.e_sphere;
  if constexpr (WALK == WALK_LANE) {
    walk_lanes<T>(b.P0, b.V0, i, lo, hi, P, Vi, ks, es, vx, vy, vz);
  } else if constexpr (WALK == WALK_ADAPTIVE) {
    if (adaptive_flat(lo, hi))
      walk_flat<T>(b.P0, b.V0, i, lo, hi, P, Vi, ks, es, vx, vy, vz);
    else
      walk_lanes<T>(b.P0, b.V0, i, lo, hi, P, Vi, ks, es, vx, vy, vz);
  } else {
    const unsigned lane = threadIdx.x & 31u;
    // union bounds of each column, taken when its first window is loaded
    uint32_t ulo[9], uhi[9];
    Window<T> win[9];
    constexpr int AHEAD = walk_ahead<T>();
#pragma unroll
    for (int q = 0; q < 9 + AHEAD; ++q) {
      if (q < 9) {
        const bool has = lo[q] < hi[q];
        ulo[q] = __reduce_min_sync(0xffffffffu, has ? lo[q] : 0xffffffffu);
        uhi[q] = __reduce_max_sync(0xffffffffu, has ? hi[q] : 0u);
        win[q] = load_window<T>(b.P0, ulo[q], uhi[q], lane);
      }
      if (q >= AHEAD) {
        const int w = q - AHEAD;
        walk_column<T>(b.P0, b.V0, i, lane, lo[w], hi[w], ulo[w], uhi[w], win[w], P, Vi, ks, es, vx, vy, vz);
      }
    }
  }
  if (valid) {
    vec4_t<T> V = Vi;
    V.x = vx;
    V.y = vy;
    V.z = vz;
    if (b.tape_p != nullptr) {  // the at-rest state after this step, and this step's grid
      b.tape_p[i] = P;
      b.tape_v[i] = V;
      b.tape_vpre[i] = Vi;
      b.tape_o[i] = b.orig[i];
      b.tape_cell[i] = b.scell[i];
    }
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
      c = cell_near<T>(P.x, P.y, P.z, sp, b.bounds, cx, cy, cz);
      b.P1[i] = P;
      b.V1[i] = V;
      b.cell[i] = c;
    } else {
      b.V1[i] = V;
    }
  }
  if (FUSED) {
    count_cell(b.count, b.tile_sum, c, valid && in_bounds(c, b.n_scan - 1u, b.err), b.tile_shift);
  }
}

// Copy V0 -> V1 (restores the at-rest layout after a regrid).
template <class T>
__global__ void __launch_bounds__(STEP_THREADS) k_copy_vel(StepBufs<T> b) {
  const uint32_t p = blockIdx.x * STEP_THREADS + threadIdx.x;
  if (p < b.n) b.V1[p] = b.V0[p];
}

}  // namespace psb
