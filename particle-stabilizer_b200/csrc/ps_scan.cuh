// ps_scan.cuh — single-pass exclusive prefix sum of uint32 with decoupled
// look-back.  It replaces the reference's multi-launch, recursive Blelloch
// scan (src/ParticleStabilizerCUDA/PrefixScan.cu:113-268), which allocates
// and frees block-sum arrays every step once the grid passes 2^20 cells.
//
// One launch, one read and one write per element: each CTA takes a tile of
// SCAN_TILE elements in ticket order (an atomic counter, so every
// predecessor tile is already running), publishes its aggregate, then warp 0
// walks back over the predecessors' status words 32 at a time until it meets
// an inclusive prefix.  A status word packs (value << 32 | flag) so value and
// flag travel in one 64-bit store.  The wait on a predecessor is bounded:
// after SCAN_SPIN_LIMIT polls the tile records PS_DEVERR_SCAN_TIMEOUT in the
// error word, takes the missing value as 0 and finishes, so the kernel always
// returns.
#pragma once

#include <cuda/atomic>

#include "ps_device.cuh"

namespace psb {

constexpr int SCAN_THREADS = 256;
constexpr int SCAN_ITEMS = 16;  // per thread: 64 contiguous bytes
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;
constexpr uint32_t SCAN_SPIN_LIMIT = 1u << 20;

enum : uint32_t { SCAN_FLAG_NONE = 0, SCAN_FLAG_AGG = 1, SCAN_FLAG_PREFIX = 2 };

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
__global__ void __launch_bounds__(SCAN_THREADS) k_exclusive_scan_u32(const uint32_t* in, uint32_t* out, int64_t n,
                                                                     uint64_t* scratch, uint32_t* err) {
  __shared__ uint32_t s_warp[SCAN_THREADS / 32];
  __shared__ uint32_t s_tile;
  __shared__ uint32_t s_prefix;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  uint64_t* status = scratch + 1;

  if (tid == 0) s_tile = atomicAdd(reinterpret_cast<unsigned int*>(scratch), 1u);
  __syncthreads();
  const int64_t tile = s_tile;
  const int64_t base = tile * SCAN_TILE + (int64_t)tid * SCAN_ITEMS;

  uint32_t v[SCAN_ITEMS];
  if (base + SCAN_ITEMS <= n && (((uintptr_t)(in + base)) & 15) == 0) {
    const uint4* q = reinterpret_cast<const uint4*>(in + base);
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS / 4; ++k) {
      const uint4 w = q[k];
      v[4 * k + 0] = w.x;
      v[4 * k + 1] = w.y;
      v[4 * k + 2] = w.z;
      v[4 * k + 3] = w.w;
    }
  } else {
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) v[k] = (base + k < n) ? in[base + k] : 0u;
  }
  uint32_t local = 0;
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; ++k) local += v[k];

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

  // publish and look back
  if (warp == 0) {
    uint32_t prefix = 0;
    if (tile == 0) {
      if (lane == 0) scan_st(&status[0], ((uint64_t)tile_sum << 32) | SCAN_FLAG_PREFIX);
    } else {
      if (lane == 0) scan_st(&status[tile], ((uint64_t)tile_sum << 32) | SCAN_FLAG_AGG);
      int64_t pred = tile - 1;  // nearest predecessor handled by lane 0
      bool done = false;
      uint32_t spins = 0;
      while (!done) {
        const int64_t idx = pred - lane;
        uint64_t s = (idx >= 0) ? scan_ld(&status[idx]) : (uint64_t)SCAN_FLAG_PREFIX;
        while (__any_sync(0xffffffffu, (s & 3u) == SCAN_FLAG_NONE)) {
          if (++spins > SCAN_SPIN_LIMIT) {
            if (lane == 0) atomicOr(err, PS_DEVERR_SCAN_TIMEOUT);
            if ((s & 3u) == SCAN_FLAG_NONE) s = (uint64_t)SCAN_FLAG_PREFIX;  // give up: value 0
            break;
          }
          if ((s & 3u) == SCAN_FLAG_NONE) s = scan_ld(&status[idx]);
        }
        const uint32_t flag = (uint32_t)(s & 3u);
        const uint32_t val = (uint32_t)(s >> 32);
        const unsigned pmask = __ballot_sync(0xffffffffu, flag == SCAN_FLAG_PREFIX);
        // lanes up to and including the first inclusive prefix contribute
        const int stop = pmask ? (__ffs(pmask) - 1) : 31;
        uint32_t contrib = (lane <= stop) ? val : 0u;
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) contrib += __shfl_xor_sync(0xffffffffu, contrib, d);
        prefix += contrib;
        done = (pmask != 0);
        pred -= 32;
      }
      if (lane == 0) scan_st(&status[tile], ((uint64_t)(prefix + tile_sum) << 32) | SCAN_FLAG_PREFIX);
    }
    if (lane == 0) s_prefix = prefix;
  }
  __syncthreads();

  uint32_t run = s_prefix + warp_excl + (inc - local);
  uint32_t o[SCAN_ITEMS];
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; ++k) {
    o[k] = run;
    run += v[k];
  }
  if (base + SCAN_ITEMS <= n && (((uintptr_t)(out + base)) & 15) == 0) {
    uint4* q = reinterpret_cast<uint4*>(out + base);
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS / 4; ++k) q[k] = make_uint4(o[4 * k], o[4 * k + 1], o[4 * k + 2], o[4 * k + 3]);
  } else {
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k)
      if (base + k < n) out[base + k] = o[k];
  }
}

}  // namespace psb
