// ps_stats.cuh — per-scene statistics on the grid.
//
// Same quantities as ParticleStatisticsCUDA::calculateStatistics
// (src/ParticleStabilizerCUDA/ParticleStatisticsCUDA.cpp:11-62), whose host
// loop is O(N^2): kinetic energy sum 0.5 m |v|^2 and extents in FP64, the
// number of particles overlapping a higher-indexed particle and the largest
// overlap.  Overlapping pairs are found through the 27 neighbour cells of the
// current grid (exact, since cells are at least 2 r_max wide).  Partial sums
// go per block in a fixed order, then one block adds the partials in order,
// so the result is deterministic.
#pragma once

#include "ps_step_kernels.cuh"

namespace psb {

constexpr int kStatsBlocks = 592;  // 4 x 148 SMs
constexpr int kStatsThreads = 256;

struct StatsPartial {
  double ke;
  double mn[3];
  double mx[3];
  double max_overlap;
  unsigned long long collided;
  unsigned long long pad_;
};

template <class T>
__global__ void __launch_bounds__(kStatsThreads) k_stats(StepBufs<T> b, SceneParams<T> sp, uint32_t first, uint32_t n,
                                                         StatsPartial* part) {
  __shared__ StatsPartial red[kStatsThreads];
  StatsPartial a;
  a.ke = 0.0;
  for (int k = 0; k < 3; ++k) {
    a.mn[k] = INFINITY;
    a.mx[k] = -INFINITY;
  }
  a.max_overlap = 0.0;
  a.collided = 0;
  const uint32_t stride = kStatsBlocks * kStatsThreads;
  for (uint32_t t = blockIdx.x * kStatsThreads + threadIdx.x; t < n; t += stride) {
    const uint32_t i = first + t;
    const vec4_t<T> P = b.P0[i];
    const vec4_t<T> V = b.V1[i];
    const double vx = (double)V.x, vy = (double)V.y, vz = (double)V.z, m = (double)V.w;
    // 0.5 * m * (vx*vx + vy*vy + vz*vz)
    const double v2 = __dadd_rn(__dadd_rn(__dmul_rn(vx, vx), __dmul_rn(vy, vy)), __dmul_rn(vz, vz));
    a.ke = __dadd_rn(a.ke, __dmul_rn(__dmul_rn(0.5, m), v2));
    const double x[3] = {(double)P.x, (double)P.y, (double)P.z}, r = (double)P.w;
    for (int k = 0; k < 3; ++k) {
      a.mn[k] = fmin(a.mn[k], __dsub_rn(x[k], r));
      a.mx[k] = fmax(a.mx[k], __dadd_rn(x[k], r));
    }
    const uint32_t oi = b.orig[i];
    int32_t cx, cy, cz;
    (void)cell_of<T>(P.x, P.y, P.z, sp, cx, cy, cz);
    const int32_t nx = sp.nb[0], ny = sp.nb[1], nz = sp.nb[2];
    const int32_t z0 = cz > 0 ? cz - 1 : 0, z1 = cz + 1 < nz ? cz + 1 : nz - 1;
    bool hit = false;
    for (int32_t bx = cx - 1; bx <= cx + 1; ++bx) {
      if (bx < 0 || bx >= nx) continue;
      for (int32_t by = cy - 1; by <= cy + 1; ++by) {
        if (by < 0 || by >= ny) continue;
        const uint32_t col = sp.cbase + ((uint32_t)bx * (uint32_t)ny + (uint32_t)by) * (uint32_t)nz;
        const uint32_t s0 = b.offset[col + (uint32_t)z0], s1 = b.offset[col + (uint32_t)z1 + 1u];
        for (uint32_t j = s0; j < s1; ++j) {
          if (b.orig[j] <= oi) continue;
          const vec4_t<T> Q = b.P0[j];
          const double dx = __dsub_rn(x[0], (double)Q.x), dy = __dsub_rn(x[1], (double)Q.y),
                       dz = __dsub_rn(x[2], (double)Q.z);
          const double d = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)));
          const double ov = __dsub_rn(__dadd_rn(r, (double)Q.w), d);
          if (ov > 0.0) {
            hit = true;
            a.max_overlap = fmax(a.max_overlap, ov);
          }
        }
      }
    }
    a.collided += hit ? 1ull : 0ull;
  }
  red[threadIdx.x] = a;
  __syncthreads();
  for (int w = kStatsThreads / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) {
      StatsPartial& x = red[threadIdx.x];
      const StatsPartial& y = red[threadIdx.x + w];
      x.ke = __dadd_rn(x.ke, y.ke);
      for (int k = 0; k < 3; ++k) {
        x.mn[k] = fmin(x.mn[k], y.mn[k]);
        x.mx[k] = fmax(x.mx[k], y.mx[k]);
      }
      x.max_overlap = fmax(x.max_overlap, y.max_overlap);
      x.collided += y.collided;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

__global__ void k_stats_final(const StatsPartial* part, StatsPartial* out) {
  if (threadIdx.x != 0) return;
  StatsPartial a = part[0];
  for (int bI = 1; bI < kStatsBlocks; ++bI) {
    const StatsPartial& y = part[bI];
    a.ke = __dadd_rn(a.ke, y.ke);
    for (int k = 0; k < 3; ++k) {
      a.mn[k] = fmin(a.mn[k], y.mn[k]);
      a.mx[k] = fmax(a.mx[k], y.mx[k]);
    }
    a.max_overlap = fmax(a.max_overlap, y.max_overlap);
    a.collided += y.collided;
  }
  *out = a;
}

}  // namespace psb
