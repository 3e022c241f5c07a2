// ps_scan.cuh — single-pass exclusive prefix sum of uint32 with decoupled
// look-back.  It replaces the reference's multi-launch, recursive Blelloch
// scan (src/ParticleStabilizerCUDA/PrefixScan.cu:113-268), which allocates
// and frees block-sum arrays every step once the grid passes 2^20 cells.
//
// One launch, one read and one write per element.  Each CTA takes a tile of
// SCAN_TILE elements in ticket order (an atomic counter, so every
// predecessor tile is already running), publishes its aggregate, then all
// its threads look back over 256 predecessor status words per round until
// one holds an inclusive prefix.  A status word packs (value << 32 | flag)
// so value and flag travel in one 64-bit store.  Every wait on a predecessor
// is bounded: after SCAN_SPIN_LIMIT polls the thread records
// PS_DEVERR_SCAN_TIMEOUT in the error word and takes the missing value as 0,
// so the kernel always returns.
#pragma once

#include <cuda/atomic>

#include "ps_device.cuh"

namespace psb {

constexpr int SCAN_THREADS = 256;
constexpr int SCAN_ITEMS = 32;  // per thread: 128 contiguous bytes
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;
constexpr uint32_t SCAN_SPIN_LIMIT = 1u << 20;

enum : uint32_t { SCAN_FLAG_NONE = 0, SCAN_FLAG_AGG = 1, SCAN_FLAG_PREFIX = 2 };

// Tiles of the step scan (counts -> offsets with per-tile totals): 8,192
// cells, or 2,048 for grids below STEP_SCAN_SMALL_BELOW cells, whose large
// tiles would leave most SMs idle (the 110,592-cell lattice: scan 7.7 ->
// 6.6 us; the 1.45 M-cell pile 10.4 -> 8.5 us; the 4.02 M-cell funnel and the
// 7.95 M-cell box scene are as fast or faster with the large tile).
constexpr int STEP_SCAN_ITEMS_LARGE = 32;
constexpr int STEP_SCAN_ITEMS_SMALL = 8;
constexpr int64_t STEP_SCAN_SMALL_BELOW = 2500000;
__host__ __device__ inline int step_scan_items(int64_t n) {
  return n < STEP_SCAN_SMALL_BELOW ? STEP_SCAN_ITEMS_SMALL : STEP_SCAN_ITEMS_LARGE;
}
__host__ __device__ inline uint32_t step_scan_shift(int64_t n) {  // log2 of the tile's cells
  return step_scan_items(n) == STEP_SCAN_ITEMS_LARGE ? 13u : 11u;
}
__host__ __device__ inline int64_t step_scan_tiles(int64_t n) {
  return (n + (int64_t(1) << step_scan_shift(n)) - 1) >> step_scan_shift(n);
}
static_assert(SCAN_THREADS * STEP_SCAN_ITEMS_LARGE == (1 << 13), "large step tile");
static_assert(SCAN_THREADS * STEP_SCAN_ITEMS_SMALL == (1 << 11), "small step tile");

// Scratch layout: [ticket (uint32) | spare uint32] [status words: one uint64 per tile].
__host__ __device__ inline int64_t scan_num_tiles(int64_t n) { return (n + SCAN_TILE - 1) / SCAN_TILE; }
__host__ __device__ inline size_t scan_scratch_bytes(int64_t n) { return 8 + 8 * (size_t)scan_num_tiles(n); }

__device__ __forceinline__ uint64_t scan_ld(uint64_t* p) {
  return cuda::atomic_ref<uint64_t, cuda::thread_scope_device>(*p).load(cuda::memory_order_relaxed);
}
__device__ __forceinline__ void scan_st(uint64_t* p, uint64_t v) {
  cuda::atomic_ref<uint64_t, cuda::thread_scope_device>(*p).store(v, cuda::memory_order_relaxed);
}

// in and out may alias.  `scratch` must be zeroed before the launch.
__global__ void __launch_bounds__(SCAN_THREADS, 8) k_exclusive_scan_u32(const uint32_t* in, uint32_t* out, int64_t n,
                                                                     uint64_t* scratch, uint32_t* err) {
  __shared__ uint32_t s_warp[SCAN_THREADS / 32];
  __shared__ uint32_t s_tile;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  uint64_t* status = scratch + 1;

  if (tid == 0) s_tile = atomicAdd(reinterpret_cast<unsigned int*>(scratch), 1u);
  __syncthreads();
  const int64_t tile = s_tile;
  const int64_t base = tile * SCAN_TILE + (int64_t)tid * SCAN_ITEMS;

  // pass 1: per-thread sum only (values are re-read after the look-back, from
  // L1/L2, so a CTA holds few registers and every tile is resident at once)
  const bool vec = base + SCAN_ITEMS <= n && (((uintptr_t)(in + base)) & 15) == 0;
  uint32_t local = 0;
  if (vec) {
    const uint4* q = reinterpret_cast<const uint4*>(in + base);
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS / 4; ++k) {
      const uint4 w = q[k];
      local += w.x + w.y + w.z + w.w;
    }
  } else {
    for (int k = 0; k < SCAN_ITEMS; ++k) local += (base + k < n) ? in[base + k] : 0u;
  }

  // warp-inclusive scan of the per-thread sums
  uint32_t inc = local;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t t = __shfl_up_sync(0xffffffffu, inc, d);
    if (lane >= d) inc += t;
  }
  if (lane == 31) s_warp[warp] = inc;
  __syncthreads();
  uint32_t warp_excl = 0, tile_sum = 0;
#pragma unroll
  for (int w = 0; w < SCAN_THREADS / 32; ++w) {
    const uint32_t t = s_warp[w];
    warp_excl += (w < warp) ? t : 0u;
    tile_sum += t;
  }

  // publish the aggregate, then warp 0 looks back 32 predecessors per round
  __shared__ uint32_t s_prefix;
  if (warp == 0) {
    uint32_t prefix = 0;
    if (tile == 0) {
      if (lane == 0) scan_st(&status[0], ((uint64_t)tile_sum << 32) | SCAN_FLAG_PREFIX);
    } else {
      if (lane == 0) scan_st(&status[tile], ((uint64_t)tile_sum << 32) | SCAN_FLAG_AGG);
      int64_t pred = tile - 1;  // predecessor read by lane 0 this round
      uint32_t spins = 0;
      bool timed_out = false;
      while (true) {
        const int64_t idx = pred - lane;
        uint64_t s = (idx >= 0) ? scan_ld(&status[idx]) : (uint64_t)SCAN_FLAG_PREFIX;
        unsigned ns = 32;
        while (__any_sync(0xffffffffu, (s & 3u) == SCAN_FLAG_NONE)) {
          if (++spins > SCAN_SPIN_LIMIT) {
            timed_out = true;
            if ((s & 3u) == SCAN_FLAG_NONE) s = (uint64_t)SCAN_FLAG_PREFIX;  // give up: value 0
            break;
          }
          __nanosleep(ns);
          ns = ns < 512 ? 2 * ns : 512;
          if ((s & 3u) == SCAN_FLAG_NONE) s = scan_ld(&status[idx]);
        }
        const unsigned pm = __ballot_sync(0xffffffffu, (s & 3u) == SCAN_FLAG_PREFIX);
        const int stop = pm ? (__ffs(pm) - 1) : 31;
        uint32_t contrib = (lane <= stop) ? (uint32_t)(s >> 32) : 0u;
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) contrib += __shfl_xor_sync(0xffffffffu, contrib, d);
        prefix += contrib;
        if (pm) break;
        pred -= 32;
      }
      if (timed_out && lane == 0) atomicOr(err, PS_DEVERR_SCAN_TIMEOUT);
      if (lane == 0) scan_st(&status[tile], ((uint64_t)(prefix + tile_sum) << 32) | SCAN_FLAG_PREFIX);
    }
    if (lane == 0) s_prefix = prefix;
  }
  __syncthreads();
  const uint32_t prefix = s_prefix;

  // pass 2: re-read (in may alias out: each thread reads its own elements
  // before writing them) and write the exclusive prefixes
  asm volatile("" ::: "memory");
  uint32_t run = prefix + warp_excl + (inc - local);
  if (vec) {
    const uint4* q = reinterpret_cast<const uint4*>(in + base);
    uint4* w = reinterpret_cast<uint4*>(out + base);
    const bool vec_out = (((uintptr_t)(out + base)) & 15) == 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS / 4; ++k) {
      const uint4 x = q[k];
      uint4 y;
      y.x = run;
      run += x.x;
      y.y = run;
      run += x.y;
      y.z = run;
      run += x.z;
      y.w = run;
      run += x.w;
      if (vec_out) {
        w[k] = y;
      } else {
        out[base + 4 * k + 0] = y.x;
        out[base + 4 * k + 1] = y.y;
        out[base + 4 * k + 2] = y.z;
        out[base + 4 * k + 3] = y.w;
      }
    }
  } else {
    for (int k = 0; k < SCAN_ITEMS; ++k)
      if (base + k < n) {
        const uint32_t x = in[base + k];
        out[base + k] = run;
        run += x;
      }
  }
}

// Exclusive scan whose per-tile totals are already known: tile_sum[t] holds
// the sum of in[t*SCAN_TILE .. (t+1)*SCAN_TILE).  The step's counting kernels
// accumulate those totals while they count, so each CTA forms its tile's
// prefix from the totals before it and scans its own tile: one read and one
// write per element, and no CTA waits on another.
//
// Layout: warp w of the CTA owns the contiguous 1024 elements
// [w*1024, (w+1)*1024) of the tile as 8 rows of 32 uint4; in row k lane l
// holds elements 4*(32k + l) .. +3, so every load and store instruction of a
// warp covers 512 contiguous bytes.  Rows are scanned with warp shuffles and
// carried from row to row; warps are combined through shared memory.
// One CTA scans tile `tile`; a CTA that scans several tiles in turn
// synchronises its threads between them.
// ITEMS elements per thread: STEP_SCAN_ITEMS_LARGE (8,192-cell tiles) for
// large grids, STEP_SCAN_ITEMS_SMALL (2,048) where a grid would fill too few
// CTAs with the large tile.
template <bool COH, int ITEMS>
__device__ __forceinline__ void scan_tile_with_sums(int64_t tile, const uint32_t* __restrict__ in,
                                                    uint32_t* __restrict__ out, int64_t n,
                                                    const uint32_t* __restrict__ tile_sum) {
  constexpr int ROWS = ITEMS / 4;  // uint4 per lane
  __shared__ uint32_t s_warp[SCAN_THREADS / 32];
  __shared__ uint32_t s_pre[SCAN_THREADS / 32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

  const int64_t wbase = tile * (int64_t)(SCAN_THREADS * ITEMS) + (int64_t)warp * (32 * ITEMS);

  uint32_t pre = 0;
  for (int64_t t = tid; t < tile; t += SCAN_THREADS) pre += ld_ro<COH>(tile_sum + t);
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) pre += __shfl_xor_sync(0xffffffffu, pre, d);
  if (lane == 0) s_pre[warp] = pre;

  const bool full = wbase + 32 * ITEMS <= n;
  uint4 v[ROWS];
#pragma unroll
  for (int k = 0; k < ROWS; ++k) {
    const int64_t e = wbase + 4 * (32 * k + lane);
    if (full) {
      v[k] = __ldcs(reinterpret_cast<const uint4*>(in + e));
    } else {
      v[k].x = e + 0 < n ? ld_pl<COH>(in + e + 0) : 0u;
      v[k].y = e + 1 < n ? ld_pl<COH>(in + e + 1) : 0u;
      v[k].z = e + 2 < n ? ld_pl<COH>(in + e + 2) : 0u;
      v[k].w = e + 3 < n ? ld_pl<COH>(in + e + 3) : 0u;
    }
  }
  // scan row by row inside the warp; `carry` is the warp's running total
  uint32_t excl[ROWS];
  uint32_t carry = 0;
#pragma unroll
  for (int k = 0; k < ROWS; ++k) {
    const uint32_t sum = v[k].x + v[k].y + v[k].z + v[k].w;
    uint32_t inc = sum;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, inc, d);
      if (lane >= d) inc += t;
    }
    excl[k] = carry + inc - sum;
    carry += __shfl_sync(0xffffffffu, inc, 31);
  }
  if (lane == 0) s_warp[warp] = carry;
  __syncthreads();
  uint32_t off = 0;
#pragma unroll
  for (int w = 0; w < SCAN_THREADS / 32; ++w) off += s_pre[w] + ((w < warp) ? s_warp[w] : 0u);
#pragma unroll
  for (int k = 0; k < ROWS; ++k) {
    const int64_t e = wbase + 4 * (32 * k + lane);
    uint4 y;
    y.x = off + excl[k];
    y.y = y.x + v[k].x;
    y.z = y.y + v[k].y;
    y.w = y.z + v[k].z;
    if (full) {
      *reinterpret_cast<uint4*>(out + e) = y;
    } else {
      if (e + 0 < n) out[e + 0] = y.x;
      if (e + 1 < n) out[e + 1] = y.y;
      if (e + 2 < n) out[e + 2] = y.z;
      if (e + 3 < n) out[e + 3] = y.w;
    }
  }
}

template <int ITEMS>
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_with_tile_sums(const uint32_t* __restrict__ in,
                                                                     uint32_t* __restrict__ out, int64_t n,
                                                                     const uint32_t* __restrict__ tile_sum) {
  pdl_wait();
  scan_tile_with_sums<false, ITEMS>(blockIdx.x, in, out, n, tile_sum);
}

}  // namespace psb
