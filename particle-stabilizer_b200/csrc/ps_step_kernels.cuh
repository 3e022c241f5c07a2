// ps_step_kernels.cuh — the per-step kernels of the DEM hot path.
//
// Reference step (src/ParticleStabilizerCUDA/PhysicsEngineCUDA.cpp:38-42):
//   integrate -> container contacts -> grid rebuild -> sphere contacts (Jacobi)
// New pipeline, one launch per stage, all scenes of a batch in every launch:
//
//   k_begin     x += v dt, v += g dt, box walls / triangles, cell hash,
//               warp-aggregated count                    (first step of a call)
//   scan        exclusive scan of the cell counts        (ps_scan.cuh)
//   k_scatter   orig id -> tmp[offset[c] + slot]; clears count[c]
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

// ---- warp-aggregated cell count --------------------------------------------
// Lanes hashing to the same cell share one atomicAdd; each receives a
// distinct slot in [count_before, count_before + peers).
__device__ __forceinline__ uint32_t count_slot(uint32_t* count, uint32_t c, bool valid) {
  const unsigned lane = threadIdx.x & 31u;
  const unsigned active = __ballot_sync(0xffffffffu, valid);
  uint32_t slot = 0;
  if (valid) {
    const unsigned peers = __match_any_sync(active, c);
    const int leader = __ffs(peers) - 1;
    uint32_t base = 0;
    if ((int)lane == leader) base = atomicAdd(count + c, (uint32_t)__popc(peers));
    base = __shfl_sync(peers, base, leader);
    slot = base + (uint32_t)__popc(peers & ((1u << lane) - 1u));
  }
  return slot;
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
  uint64_t* scan_scratch; // zeroed by k_begin / k_scatter for the next scan
  uint32_t scan_words;
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
  if (p < b.scan_words) b.scan_scratch[p] = 0ull;
  const bool valid = p < b.n;
  uint32_t c = 0;
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
  const uint32_t s = count_slot(b.count, c, valid);
  if (valid) b.slot[p] = s;
}

// tmp[offset[c] + slot] = orig; count[c] = 0 (every non-zero count belongs
// to a cell some particle hashed to, so this restores an all-zero array).
__global__ void __launch_bounds__(STEP_THREADS) k_scatter(const uint32_t* __restrict__ cell,
                                                          const uint32_t* __restrict__ slot,
                                                          const uint32_t* __restrict__ orig,
                                                          const uint32_t* __restrict__ offset, uint32_t* tmp,
                                                          uint32_t* count, uint32_t n, uint64_t* scan_scratch,
                                                          uint32_t scan_words) {
  const uint32_t p = blockIdx.x * STEP_THREADS + threadIdx.x;
  if (p < scan_words) scan_scratch[p] = 0ull;
  if (p >= n) return;
  const uint32_t c = cell[p];
  tmp[offset[c] + slot[p]] = orig[p];
  count[c] = 0u;
}

// Canonical position = offset[c] + #{members of c with a smaller orig id};
// moves the integrated state (P1, V1) there as (P0, V0) with its orig id.
template <class T>
__global__ void __launch_bounds__(STEP_THREADS) k_rank_move(StepBufs<T> b) {
  const uint32_t p = blockIdx.x * STEP_THREADS + threadIdx.x;
  if (p >= b.n) return;
  const uint32_t c = b.cell[p];
  const uint32_t start = b.offset[c], end = b.offset[c + 1];
  const uint32_t o = b.tmp[start + b.slot[p]];
  uint32_t rank = 0;
  for (uint32_t s = start; s < end; ++s) rank += (b.tmp[s] < o) ? 1u : 0u;
  const uint32_t d = start + rank;
  b.P0[d] = b.P1[p];
  b.V0[d] = b.V1[p];
  b.orig[d] = o;
}

// ---- sphere-sphere contacts (ParticleModel_kernels.cu:136-201) --------------
// One thread per sorted particle; the neighbours are read from the sorted
// arrays.  For each (dx, dy) column the three z-cells are contiguous in the
// sorted order, so 9 slot ranges cover the 27 cells, visited x-outer, y,
// z-inner, members in canonical order.
template <class T, bool MULTI, bool MESH, bool FUSED>
__global__ void __launch_bounds__(STEP_THREADS) k_contacts(StepBufs<T> b, SceneParams<T> sp0, const MeshView* mv) {
  using A = Ar<T>;
  const uint32_t i = blockIdx.x * STEP_THREADS + threadIdx.x;
  const bool valid = i < b.n;
  uint32_t c = 0;
  if (valid) {
    const SceneParams<T>& sp = scene_of<T, MULTI>(i, sp0, b.scenes, b.pbase, b.n_scenes);
    vec4_t<T> P = b.P0[i];
    const vec4_t<T> Vi = b.V0[i];
    T vx = Vi.x, vy = Vi.y, vz = Vi.z;
    const T ri = P.w, mi = Vi.w;
    const T k = sp.k_spring, e = sp.e_sphere;
    int32_t cx, cy, cz;
    (void)cell_of<T>(P.x, P.y, P.z, sp, cx, cy, cz);
    const int32_t nx = sp.nb[0], ny = sp.nb[1], nz = sp.nb[2];
    const int32_t z0 = cz > 0 ? cz - 1 : 0;
    const int32_t z1 = cz + 1 < nz ? cz + 1 : nz - 1;
    for (int32_t bx = cx - 1; bx <= cx + 1; ++bx) {
      if (bx < 0 || bx >= nx) continue;
      for (int32_t by = cy - 1; by <= cy + 1; ++by) {
        if (by < 0 || by >= ny) continue;
        const uint32_t col = sp.cbase + ((uint32_t)bx * (uint32_t)ny + (uint32_t)by) * (uint32_t)nz;
        const uint32_t s0 = __ldg(b.offset + col + (uint32_t)z0);
        const uint32_t s1 = __ldg(b.offset + col + (uint32_t)z1 + 1u);
        for (uint32_t j = s0; j < s1; ++j) {
          if (j == i) continue;
          const vec4_t<T> Pj = ld4<T>(b.P0 + j);
          const T dx = A::sub(P.x, Pj.x), dy = A::sub(P.y, Pj.y), dz = A::sub(P.z, Pj.z);
          const T d2 = A::fma(dz, dz, A::fma(dy, dy, A::mul(dx, dx)));
          const T dist = A::sqrt(d2);
          const T overlap = A::sub(A::add(ri, Pj.w), dist);
          if (overlap > T(0)) {
            const vec4_t<T> Vj = ld4<T>(b.V0 + j);
            const T rvx = A::sub(Vi.x, Vj.x), rvy = A::sub(Vi.y, Vj.y), rvz = A::sub(Vi.z, Vj.z);
            const T rvd = A::fma(rvz, dz, A::fma(rvy, dy, A::mul(rvx, dx)));
            const T cr = A::div(A::mul(A::mul(A::mul(T(2), Vj.w), rvd), e), A::mul(A::add(mi, Vj.w), d2));
            const T cs = A::div(A::mul(k, overlap), A::mul(dist, mi));
            const T f = A::sub(cs, cr);
            vx = A::fma(f, dx, vx);
            vy = A::fma(f, dy, vy);
            vz = A::fma(f, dz, vz);
          }
        }
      }
    }
    vec4_t<T> V = Vi;
    V.x = vx;
    V.y = vy;
    V.z = vz;
    if (FUSED) {
      integrate<T>(P, V, sp);
      finish_integrated<T, MESH>(P, V, sp, mv, b.err, c);
      b.P1[i] = P;
      b.V1[i] = V;
      b.cell[i] = c;
    } else {
      b.V1[i] = V;
    }
  }
  if (FUSED) {
    const uint32_t s = count_slot(b.count, c, valid);
    if (valid) b.slot[i] = s;
  }
}

// Copy V0 -> V1 (restores the at-rest layout after a regrid).
template <class T>
__global__ void __launch_bounds__(STEP_THREADS) k_copy_vel(StepBufs<T> b) {
  const uint32_t p = blockIdx.x * STEP_THREADS + threadIdx.x;
  if (p < b.n) b.V1[p] = b.V0[p];
}

}  // namespace psb
