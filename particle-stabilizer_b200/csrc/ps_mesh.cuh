// ps_mesh.cuh — triangle container on a binned mesh.
//
// Replaces the reference's dense N x P container
// (src/ParticleStabilizerCUDA/PolygonContainerCUDA.cpp:130-226 and
// PolygonContainerCUDA_kernels.cu:155-294: a bool[N*P] intersection matrix
// and five launches per step).  Triangles are binned once, at set-up, into a
// uniform grid by their AABB; a particle tests only the triangles binned in
// the cells its own AABB touches.  A triangle reachable from several cells is
// tested once: in the cell holding the minimum corner of the intersection of
// the two AABBs.  Hits are summed in ascending triangle index (the order of
// the oracle), with the same operations as the reference:
//   v <- mean over hits of e * (v - 2 (v.n) n)
//   x <- x + sum over hits of -(r - dot(-n, x - v0)) n
// all evaluated on the pre-container state.  A sphere may touch any number
// of triangles: hits are kept MESH_MAX_HITS at a time, in passes over the
// sphere's bins that each continue above the previous pass's largest id.
#pragma once

#include "ps_device.cuh"

namespace psb {

constexpr int MESH_MAX_HITS = 64;  // hits held per pass (more take further passes)

// Device view of every scene's binned triangles.
template <class T>
struct MeshViewT {
  const T* tri;          // 9 reals per triangle: v0, v1, v2
  const T* nrm;          // 3 reals per triangle: unit normal
  const T* aabb;         // 6 reals per triangle: min xyz, max xyz
  const uint32_t* bin_offset;  // CSR offsets per bin (+1)
  const uint32_t* bin_tri;     // triangle ids (global)
};

struct MeshView {
  const void* tri;
  const void* nrm;
  const void* aabb;
  const uint32_t* bin_offset;
  const uint32_t* bin_tri;
  uint32_t n_tri;      // triangles over all scenes
  uint32_t n_bins;     // bins over all scenes (bin_offset holds n_bins + 1)
  uint32_t n_bin_tri;  // entries of bin_tri
};

template <class T>
__device__ __forceinline__ T dot3(T ax, T ay, T az, T bx, T by, T bz) {
  using A = Ar<T>;
  return A::fma(az, bz, A::fma(ay, by, A::mul(ax, bx)));
}

template <class T>
struct V3 {
  T x, y, z;
};

template <class T>
__device__ __forceinline__ V3<T> v3sub(V3<T> a, V3<T> b) {
  using A = Ar<T>;
  return {A::sub(a.x, b.x), A::sub(a.y, b.y), A::sub(a.z, b.z)};
}
template <class T>
__device__ __forceinline__ T v3dot(V3<T> a, V3<T> b) {
  return dot3<T>(a.x, a.y, a.z, b.x, b.y, b.z);
}

// closest point on segment ab (PolygonContainerCUDA_kernels.cu:101-112)
template <class T>
__device__ __forceinline__ V3<T> seg_closest(V3<T> p, V3<T> a, V3<T> b) {
  using A = Ar<T>;
  const V3<T> ab = v3sub(b, a), ap = v3sub(p, a);
  T t = A::div(v3dot(ap, ab), v3dot(ab, ab));
  t = t < T(1) ? t : T(1);
  t = t > T(0) ? t : T(0);
  return {A::fma(ab.x, t, a.x), A::fma(ab.y, t, a.y), A::fma(ab.z, t, a.z)};
}

// getClosestPointOnPolygonKernelFunc (PolygonContainerCUDA_kernels.cu:114-153)
template <class T>
__device__ __forceinline__ V3<T> tri_closest(V3<T> a, V3<T> b, V3<T> c, V3<T> n, V3<T> p, int edge_quirk) {
  using A = Ar<T>;
  const T ip = v3dot(v3sub(p, a), n);
  const V3<T> q = {A::fma(-n.x, ip, p.x), A::fma(-n.y, ip, p.y), A::fma(-n.z, ip, p.z)};
  {
    const V3<T> v0 = v3sub(c, a), v1 = v3sub(b, a), v2 = v3sub(q, a);
    const T d00 = v3dot(v0, v0), d01 = v3dot(v0, v1), d02 = v3dot(v0, v2);
    const T d11 = v3dot(v1, v1), d12 = v3dot(v1, v2);
    const T inv = A::div(T(1), A::fma(d00, d11, -A::mul(d01, d01)));
    const T u = A::mul(A::fma(d11, d02, -A::mul(d01, d12)), inv);
    const T v = A::mul(A::fma(d00, d12, -A::mul(d01, d02)), inv);
    if ((u >= T(0)) && (v >= T(0)) && (A::add(u, v) <= T(1))) return q;
  }
  const V3<T> e0 = seg_closest(p, a, b), e1 = seg_closest(p, b, c), e2 = seg_closest(p, c, a);
  T s0, s1, s2;
  if (edge_quirk) {
    s0 = v3dot(p, e0);
    s1 = v3dot(p, e1);
    s2 = v3dot(p, e2);
  } else {
    const V3<T> d0 = v3sub(p, e0), d1 = v3sub(p, e1), d2 = v3sub(p, e2);
    s0 = v3dot(d0, d0);
    s1 = v3dot(d1, d1);
    s2 = v3dot(d2, d2);
  }
  V3<T> r = e0;
  T best = s0;
  if (s1 < best) { best = s1; r = e1; }
  if (s2 < best) { best = s2; r = e2; }
  return r;
}

template <class T>
__device__ __forceinline__ int32_t mesh_axis(T x, T lo, T iv, int32_t nb) {
  using A = Ar<T>;
  const T q = A::div(A::sub(x, lo), iv);
  if (!(q > T(0))) return 0;
  if (q >= (T)nb) return nb - 1;
  return (int32_t)q;
}

// Hits of one pass: walks the bins the sphere's AABB covers and keeps, in
// ascending order, the MESH_MAX_HITS smallest ids of the triangles it hits
// (above `after` unless `first`); true if a hit was left for a later pass.
template <class T>
__device__ __forceinline__ bool mesh_collect(const V3<T>& c, T r, const SceneParams<T>& sp, const MeshView& mvv,
                                             uint32_t* err, bool first, uint32_t after,
                                             uint32_t (&hits)[MESH_MAX_HITS], int& nh) {
  using A = Ar<T>;
  const MeshViewT<T> mv{static_cast<const T*>(mvv.tri), static_cast<const T*>(mvv.nrm),
                        static_cast<const T*>(mvv.aabb), mvv.bin_offset, mvv.bin_tri};
  const T lox = A::sub(c.x, r), loy = A::sub(c.y, r), loz = A::sub(c.z, r);
  const T hix = A::add(c.x, r), hiy = A::add(c.y, r), hiz = A::add(c.z, r);
  const int32_t bx0 = mesh_axis<T>(lox, sp.mesh_lo[0], sp.mesh_iv, sp.mesh_nb[0]);
  const int32_t by0 = mesh_axis<T>(loy, sp.mesh_lo[1], sp.mesh_iv, sp.mesh_nb[1]);
  const int32_t bz0 = mesh_axis<T>(loz, sp.mesh_lo[2], sp.mesh_iv, sp.mesh_nb[2]);
  const int32_t by1 = mesh_axis<T>(hiy, sp.mesh_lo[1], sp.mesh_iv, sp.mesh_nb[1]);
  // A sphere whose AABB misses the mesh AABB hits nothing: every triangle's
  // AABB lies inside the mesh AABB (both from the same rounded vertices), so
  // each closed AABB test would fail.  Such a sphere (above or beside the
  // container) walks no bins.
  const bool near = !(lox > sp.mesh_hi[0] || hix < sp.mesh_lo[0] || loy > sp.mesh_hi[1] || hiy < sp.mesh_lo[1] ||
                      loz > sp.mesh_hi[2] || hiz < sp.mesh_lo[2]);
  const int32_t bx1 = near ? mesh_axis<T>(hix, sp.mesh_lo[0], sp.mesh_iv, sp.mesh_nb[0]) : bx0 - 1;
  const int32_t bz1 = mesh_axis<T>(hiz, sp.mesh_lo[2], sp.mesh_iv, sp.mesh_nb[2]);
  nh = 0;
  bool more = false;
  for (int32_t bx = bx0; bx <= bx1; ++bx)
    for (int32_t by = by0; by <= by1; ++by)
      for (int32_t bz = bz0; bz <= bz1; ++bz) {
        const uint32_t bin = sp.mesh_bin_base +
                             ((uint32_t)bx * (uint32_t)sp.mesh_nb[1] + (uint32_t)by) * (uint32_t)sp.mesh_nb[2] +
                             (uint32_t)bz;
        if (!in_bounds(bin, mvv.n_bins, err)) continue;
        const uint32_t t0 = __ldg(mv.bin_offset + bin), t1 = __ldg(mv.bin_offset + bin + 1);
        if (!in_bounds(t1, (uint64_t)mvv.n_bin_tri + 1u, err)) continue;
        for (uint32_t s = t0; s < t1; ++s) {
          const uint32_t t = __ldg(mv.bin_tri + s);
          if (!in_bounds(t, mvv.n_tri, err)) continue;
          if (!first && t <= after) continue;  // applied by an earlier pass
          const T* bb = mv.aabb + 6 * (size_t)t;
          // closed AABB test (isIntersectedKernel :191-197)
          if (!(lox <= bb[3] && hix >= bb[0] && loy <= bb[4] && hiy >= bb[1] && loz <= bb[5] && hiz >= bb[2]))
            continue;
          // test each triangle once: in the bin of the intersection's minimum corner
          const T ix = lox > bb[0] ? lox : bb[0];
          const T iy = loy > bb[1] ? loy : bb[1];
          const T iz = loz > bb[2] ? loz : bb[2];
          if (mesh_axis<T>(ix, sp.mesh_lo[0], sp.mesh_iv, sp.mesh_nb[0]) != bx ||
              mesh_axis<T>(iy, sp.mesh_lo[1], sp.mesh_iv, sp.mesh_nb[1]) != by ||
              mesh_axis<T>(iz, sp.mesh_lo[2], sp.mesh_iv, sp.mesh_nb[2]) != bz)
            continue;
          if (nh == MESH_MAX_HITS && t > hits[nh - 1]) {  // a later pass takes it
            more = true;
            continue;
          }
          const T* tv = mv.tri + 9 * (size_t)t;
          const T* tn = mv.nrm + 3 * (size_t)t;
          const V3<T> a = {tv[0], tv[1], tv[2]}, b = {tv[3], tv[4], tv[5]}, cc = {tv[6], tv[7], tv[8]};
          const V3<T> n = {tn[0], tn[1], tn[2]};
          const V3<T> cp = tri_closest<T>(a, b, cc, n, c, sp.edge_quirk);
          const V3<T> rel = v3sub(cp, c);
          if (!(v3dot(rel, rel) < A::mul(r, r))) continue;
          if (nh == MESH_MAX_HITS) {  // full: the largest kept id moves to a later pass
            more = true;
            --nh;
          }
          // insert keeping ascending triangle order
          int k = nh++;
          while (k > 0 && hits[k - 1] > t) {
            hits[k] = hits[k - 1];
            --k;
          }
          hits[k] = t;
        }
      }
  return more;
}

// Adds the reflected velocities (calcModifiedVelocitySumKernel :235) and the
// position corrections (calcPosModificationAmountKernel :276-281) of hits
// [0, nh), in that order, all from the pre-container state (c, V).
template <class T>
__device__ __forceinline__ void mesh_accumulate(const uint32_t (&hits)[MESH_MAX_HITS], int nh, const V3<T>& c, T r,
                                                const vec4_t<T>& V, T e, const MeshView& mvv, T& svx, T& svy, T& svz,
                                                T& mx, T& my, T& mz) {
  using A = Ar<T>;
  const T* tri = static_cast<const T*>(mvv.tri);
  const T* nrm = static_cast<const T*>(mvv.nrm);
  for (int h = 0; h < nh; ++h) {
    const uint32_t t = hits[h];
    const T* tv = tri + 9 * (size_t)t;
    const T* tn = nrm + 3 * (size_t)t;
    const V3<T> n = {tn[0], tn[1], tn[2]};
    const T vn2 = A::mul(T(2), dot3<T>(V.x, V.y, V.z, n.x, n.y, n.z));
    svx = A::fma(e, A::fma(-vn2, n.x, V.x), svx);
    svy = A::fma(e, A::fma(-vn2, n.y, V.y), svy);
    svz = A::fma(e, A::fma(-vn2, n.z, V.z), svz);
    const T dtp = dot3<T>(-n.x, -n.y, -n.z, A::sub(c.x, tv[0]), A::sub(c.y, tv[1]), A::sub(c.z, tv[2]));
    const T sc = A::sub(r, dtp);
    mx = A::fma(-sc, n.x, mx);
    my = A::fma(-sc, n.y, my);
    mz = A::fma(-sc, n.z, mz);
  }
}

// Triangle container of one particle, CUDA semantics
// (PolygonContainerCUDA.cpp:130-226): every hit triangle in ascending index.
template <class T>
__device__ void mesh_contacts(vec4_t<T>& P, vec4_t<T>& V, const SceneParams<T>& sp, const MeshView& mvv,
                              uint32_t* err) {
  using A = Ar<T>;
  const T r = P.w;
  const V3<T> c = {P.x, P.y, P.z};
  // MESH_MAX_HITS hits per pass, in ascending triangle index: a sphere that
  // touches more triangles takes further passes, each starting above the
  // previous pass's largest id, so the sums come out as one ascending pass
  // over every hit would give them.  The ids rise from pass to pass, so the
  // passes end.
  T svx = 0, svy = 0, svz = 0, mx = 0, my = 0, mz = 0;
  uint32_t n_hits = 0;
  uint32_t after = 0;  // ids <= after were applied by earlier passes
  bool first = true;
  for (;;) {
    uint32_t hits[MESH_MAX_HITS];
    int nh = 0;
    const bool more = mesh_collect<T>(c, r, sp, mvv, err, first, after, hits, nh);
    mesh_accumulate<T>(hits, nh, c, r, V, sp.e_poly, mvv, svx, svy, svz, mx, my, mz);
    n_hits += (uint32_t)nh;
    if (__builtin_expect(!more || nh == 0, 1)) break;
    after = hits[nh - 1];
    first = false;
  }
  if (n_hits > 0) {  // calcAveragedVelocityKernel: only particles with a hit
    const T hc = (T)n_hits;
    V.x = A::div(svx, hc);
    V.y = A::div(svy, hc);
    V.z = A::div(svz, hc);
  }
  // modifyPositionKernel adds the (possibly zero) correction to every particle
  P.x = A::add(c.x, mx);
  P.y = A::add(c.y, my);
  P.z = A::add(c.z, mz);
}

}  // namespace psb
