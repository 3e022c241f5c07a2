// ps_device.cuh — device-side types and arithmetic shared by the step kernels.
//
// Every floating-point operation of the step is issued as one explicitly
// rounded intrinsic (__fadd_rn, __fmaf_rn, ... / __dadd_rn, __fma_rn, ...),
// which the compiler never contracts or reorders.  The operation sequence is
// the one the CPU oracle (oracle/ps_oracle_impl.inc) performs, so results are
// reproducible bit for bit in FP32 and in FP64.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace psb {

// ---- explicit-rounding arithmetic -----------------------------------------
template <class T>
struct Ar;

template <>
struct Ar<float> {
  static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
  static __device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
  static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
  static __device__ __forceinline__ float div(float a, float b) { return __fdiv_rn(a, b); }
  static __device__ __forceinline__ float fma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
  static __device__ __forceinline__ float sqrt(float a) { return __fsqrt_rn(a); }
};

template <>
struct Ar<double> {
  static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
  static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
  static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
  static __device__ __forceinline__ double div(double a, double b) { return __ddiv_rn(a, b); }
  static __device__ __forceinline__ double fma(double a, double b, double c) { return __fma_rn(a, b, c); }
  static __device__ __forceinline__ double sqrt(double a) { return __dsqrt_rn(a); }
};

// ---- per-particle vector types ---------------------------------------------
// pos_r = (x, y, z, radius), vel_m = (vx, vy, vz, mass): 32 B per particle in
// FP32 (two float4), 64 B in FP64 (two double4, 32-byte aligned).
template <class T>
struct Vec4;
template <>
struct Vec4<float> {
  using type = float4;
};
template <>
struct Vec4<double> {
  struct __align__(32) type {
    double x, y, z, w;
  };
};
template <class T>
using vec4_t = typename Vec4<T>::type;

template <class T>
__device__ __forceinline__ vec4_t<T> ld4(const vec4_t<T>* p) {
  return *p;
}
template <>
__device__ __forceinline__ float4 ld4<float>(const float4* p) {
  return __ldg(p);
}

// Loads of data that the same kernel may have written earlier in its run (a
// persistent kernel with grid barriers, COH = true) go through L2
// (ld.global.cg); otherwise through the read-only path (ld_ro) or a plain
// load (ld_pl), as the kernels launched once per phase use them.
template <bool COH>
__device__ __forceinline__ uint32_t ld_ro(const uint32_t* p) {
  if constexpr (COH)
    return __ldcg(p);
  else
    return __ldg(p);
}
template <bool COH>
__device__ __forceinline__ uint32_t ld_pl(const uint32_t* p) {
  if constexpr (COH)
    return __ldcg(p);
  else
    return *p;
}
template <class T, bool COH>
__device__ __forceinline__ vec4_t<T> ld4c(const vec4_t<T>* p) {
  if constexpr (!COH) {
    return ld4<T>(p);
  } else if constexpr (sizeof(T) == 4) {
    return __ldcg(p);
  } else {
    const double2 a = __ldcg(reinterpret_cast<const double2*>(p));
    const double2 b = __ldcg(reinterpret_cast<const double2*>(p) + 1);
    vec4_t<T> v;
    v.x = a.x;
    v.y = a.y;
    v.z = b.x;
    v.w = b.y;
    return v;
  }
}

// Wait until the grid this kernel depends on has completed and its writes
// are visible, when it was launched with programmatic stream serialization
// (it may then start while that grid drains); a no-op for a normal launch.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// ---- per-scene parameters (device copy) -----------------------------------
// Scenes are concatenated: scene s owns particle slots [pbase, pbase+pcount)
// and cells [cbase, cbase + nb.x*nb.y*nb.z) of the global arrays.  The
// canonical order sorts by global cell id, so a scene's particles never leave
// its slot range.
template <class T>
struct SceneParams {
  T grid_lo[3];   // grid domain minimum
  T interval;     // cell edge
  T box_lo[3];    // box walls
  T box_hi[3];
  T e_lo[3];      // restitution of the x/y/z min walls
  T e_hi[3];      // restitution of the x/y/z max walls
  T gravity[3];
  T dt;
  T k_spring;
  T e_sphere;
  T e_poly;       // triangle-container restitution
  int32_t nb[3];  // cells per axis
  uint32_t cbase; // first global cell id
  uint32_t pbase; // first particle slot
  uint32_t pcount;
  // triangle container (mesh_tris == 0: box walls)
  uint32_t mesh_tri_base;  // first triangle in the global soup
  uint32_t mesh_tris;
  uint32_t mesh_bin_base;  // first bin of this scene's triangle bins
  int32_t mesh_nb[3];      // triangle-bin grid
  T mesh_lo[3];            // triangle-bin grid origin = lower corner of the mesh AABB
  T mesh_hi[3];            // upper corner of the mesh AABB
  T mesh_iv;               // triangle-bin edge
  int32_t edge_quirk;
  // unsigned division by nz and by ny with a multiply-high (Granlund &
  // Montgomery): q = (t + ((x - t) >> sh1)) >> sh2, t = umulhi(x, m)
  uint32_t div_nz_m, div_nz_sh1, div_nz_sh2;
  uint32_t div_ny_m, div_ny_sh1, div_ny_sh2;
  // cell boundaries: axis a of this scene uses bounds[bnd_base[a] + k] for
  // k = 0..nb[a]; the clamped cell index of x is k exactly when
  // bounds[k] <= x < bounds[k+1] (bounds[0] = -inf, bounds[nb] = +inf)
  uint32_t bnd_base[3];
};

__host__ __device__ inline uint32_t fast_udiv(uint32_t x, uint32_t m, uint32_t sh1, uint32_t sh2) {
#ifdef __CUDA_ARCH__
  const uint32_t t = __umulhi(x, m);
#else
  const uint32_t t = (uint32_t)(((uint64_t)x * m) >> 32);
#endif
  return (t + ((x - t) >> sh1)) >> sh2;
}

// Magic numbers of fast_udiv for a divisor d >= 1: l = ceil(log2 d),
// m = floor(2^32 (2^l - d) / d) + 1, sh1 = min(l, 1), sh2 = max(l - 1, 0).
inline void fast_udiv_magic(uint32_t d, uint32_t& m, uint32_t& sh1, uint32_t& sh2) {
  uint32_t l = 0;
  while (l < 32 && (1ull << l) < d) ++l;
  m = (uint32_t)((((uint64_t)1 << 32) * (((uint64_t)1 << l) - d)) / d + 1);
  sh1 = l < 1 ? l : 1;
  sh2 = l > 1 ? l - 1 : 0;
}

// Device error word bits (read by the host after a step block).
enum : uint32_t {
  PS_DEVERR_SCAN_TIMEOUT = 1u << 0,   // decoupled look-back gave up waiting
  PS_DEVERR_MESH_OVERFLOW = 1u << 1,  // reserved: hits beyond the buffer now take further passes
  PS_DEVERR_BAD_CELL = 1u << 2,       // a cell id fell outside its scene (never expected)
  PS_DEVERR_LIST_OVERFLOW = 1u << 3,  // neighbour-list mode: a list or a sphere's overlap buffer was full
  PS_DEVERR_LIST_BARRIER = 1u << 4,   // neighbour-list mode: a grid barrier of the rebuild gave up waiting
  PS_DEVERR_BOUNDS = 1u << 5,         // bounds-checked build: an index fell outside its array
};

// Bounds-checked build (compiled with -DPS_DEBUG_BOUNDS, `make debug`):
// in_bounds(i, n, err) is false when i >= n, records PS_DEVERR_BOUNDS, and
// the caller skips the access, so a wrong index shows up as an error status
// instead of a memory fault.  In the product build it is the constant true
// and costs nothing.
__device__ __forceinline__ bool in_bounds(uint64_t i, uint64_t n, uint32_t* err) {
#ifdef PS_DEBUG_BOUNDS
  if (i < n) return true;
  atomicOr(err, PS_DEVERR_BOUNDS);
  return false;
#else
  (void)i;
  (void)n;
  (void)err;
  return true;
#endif
}

}  // namespace psb
