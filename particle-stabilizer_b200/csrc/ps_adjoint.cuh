// ps_adjoint.cuh — reverse-mode adjoint of the DEM step (box container).
//
// Forward step (per particle i, the CUDA scheme of PhysicsEngineCUDA.cpp:38-42):
//   x' = x + v dt,  v' = v + g dt                       (integrate)
//   per axis: clamp to the walls, v <- -v e              (walls, events)
//   v''' = v'' + sum_j f_ij d_ij,  x''' = x''            (Jacobi contacts)
//   d = x_i - x_j, L = |d|, ov = r_i + r_j - L > 0,
//   f = k ov / (L m_i) - B (u.d) / L^2,  B = 2 m_j e / (m_i + m_j),  u = v_i - v_j
//
// Reverse sweep of one step, given the adjoints (xbar, vbar) of its output:
//   k_adj_contacts   (sorted order, gather): for each particle, the terms of
//                    the pairs where it receives and the pairs where it is the
//                    source (pairs are symmetric), so no atomics; partials of
//                    dL/dk and dL/de_sphere accumulated per sorted slot (a
//                    scene owns a fixed slot range, so per-scene sums are
//                    unchanged and the order is fixed by the canonical sort).
//   k_adj_walls_integrate (the tape row's sorted order): through the walls
//                    (clamp events recomputed from the recorded step input)
//                    and the integrate; partials of dL/de_wall by slot.
// The block recompute records, per step, the at-rest state after it in
// sorted order (positions, velocities, original ids) together with the
// step's grid (pre-contact velocities, sorted cell ids, and a copy of the
// cell offsets).  Row t + 1 plus offsets t are then exactly the sorted
// post-wall state and grid that step t's contacts read, so the reverse sweep
// runs the contact adjoint on them directly, without rebuilding the grid,
// and row t is the step's input for the walls/integrate adjoint.
// Wall clamps and contact activation are piecewise events taken from the
// forward values; radii and masses are constants.
#pragma once

#include "ps_step_kernels.cuh"

namespace psb {

enum : int { ADJ_K = 0, ADJ_E = 1, ADJ_WALL = 2 };  // acc rows: k, e_sphere, e_wall[6] (zMin..yMax)
constexpr int ADJ_NACC = 8;

template <class T>
struct TapeRow {
  vec4_t<T>* p;     // (x, r) per sorted slot
  vec4_t<T>* v;     // (v, m)
  vec4_t<T>* vpre;  // (v, m) before the contacts of the step that wrote the row
  uint32_t* o;      // original id
  uint32_t* cell;   // sorted cell id of that step's grid
};

template <class T>
struct AdjBufs {
  TapeRow<T> tape;        // input of the step being reversed
  vec4_t<T>* ax;          // adjoint of positions, original order (w unused): one 16/32-B access
  vec4_t<T>* av;          // adjoint of velocities
  vec4_t<T>* ax2;         // output of k_adj_contacts
  vec4_t<T>* av2;
  double* acc;            // ADJ_NACC rows of n, accumulated over steps: rows k, e by sorted
                          // slot, wall rows by original index
  uint32_t n;             // row length of acc
};

// Terms of one active pair for the receiver r and the source s:
// c_r = f d; g = adjoint of v_r's output.  Returns the adjoint of d (dd),
// of u (du) and the parameter partials.
template <class T>
__device__ __forceinline__ void pair_adjoint(T dx, T dy, T dz, T ux, T uy, T uz, T R, T mr, T ms, T k, T e, T gx,
                                             T gy, T gz, T& ddx, T& ddy, T& ddz, T& dux, T& duy, T& duz,
                                             double& dk, double& de) {
  const T L2 = dx * dx + dy * dy + dz * dz;
  const T L = sqrt(L2);
  const T ov = R - L;
  const T Bc = T(2) * ms * e / (mr + ms);
  const T ud = ux * dx + uy * dy + uz * dz;
  const T f = k * ov / (L * mr) - Bc * ud / L2;
  const T fbar = gx * dx + gy * dy + gz * dz;
  dk += (double)(fbar * ov / (L * mr));
  de += (double)(fbar * (-(T(2) * ms * ud) / ((mr + ms) * L2)));
  const T fL = -k * R / (L2 * mr) + T(2) * Bc * ud / (L2 * L);
  const T Lb = fbar * fL / L;
  const T udb = -fbar * Bc / L2;
  ddx = f * gx + Lb * dx + udb * ux;
  ddy = f * gy + Lb * dy + udb * uy;
  ddz = f * gz + Lb * dz + udb * uz;
  dux = udb * dx;
  duy = udb * dy;
  duz = udb * dz;
}

// Same activation test as the forward contact kernel (contact_one).
template <class T>
__device__ __forceinline__ bool pair_active(const vec4_t<T>& P, const vec4_t<T>& Pj) {
  using A = Ar<T>;
  const T margin = T(1) + T(1.0 / 1048576.0);
  const T dx = A::sub(P.x, Pj.x), dy = A::sub(P.y, Pj.y), dz = A::sub(P.z, Pj.z);
  const T d2 = A::fma(dz, dz, A::fma(dy, dy, A::mul(dx, dx)));
  const T s = A::add(P.w, Pj.w);
  if (d2 >= A::mul(A::mul(s, s), margin)) return false;
  return A::sub(s, A::sqrt(d2)) > T(0);
}

template <class T, bool MULTI>
__global__ void __launch_bounds__(STEP_THREADS) k_adj_contacts(StepBufs<T> b, AdjBufs<T> a, SceneParams<T> sp0) {
  const uint32_t i = blockIdx.x * STEP_THREADS + threadIdx.x;
  if (i >= b.n) return;
  const SceneParams<T>& sp = scene_of<T, MULTI>(i, sp0, b.scenes, b.pbase, b.n_scenes);
  const vec4_t<T> P = b.P0[i];
  const vec4_t<T> V = b.V0[i];
  const uint32_t oi = b.orig[i];
  const vec4_t<T> G = a.av[oi], X = a.ax[oi];
  const T gx = G.x, gy = G.y, gz = G.z;
  T xb0 = X.x, xb1 = X.y, xb2 = X.z;
  T vb0 = gx, vb1 = gy, vb2 = gz;
  double dk = 0.0, de = 0.0;
  int32_t cx, cy, cz;
  cell_coords<T>(b.scell[i], sp, cx, cy, cz);
  const int32_t nx = sp.nb[0], ny = sp.nb[1], nz = sp.nb[2];
  const uint32_t z0 = (uint32_t)(cz > 0 ? cz - 1 : 0);
  const uint32_t z1 = (uint32_t)(cz + 1 < nz ? cz + 1 : nz - 1) + 1u;
  const T k = sp.k_spring, e = sp.e_sphere;
  const bool live = isfinite(P.x) && isfinite(P.y) && isfinite(P.z);  // no active pair otherwise
  for (int q = 0; q < 9; ++q) {
    const int32_t bx = cx - 1 + q / 3, by = cy - 1 + q % 3;
    if (!live || bx < 0 || bx >= nx || by < 0 || by >= ny) continue;
    const uint32_t col = sp.cbase + ((uint32_t)bx * (uint32_t)ny + (uint32_t)by) * (uint32_t)nz;
    const uint32_t j0 = b.offset[col + z0], j1 = b.offset[col + z1];
    for (uint32_t j = j0; j < j1; ++j) {
      if (j == i) continue;
      const vec4_t<T> Pj = b.P0[j];
      if (!pair_active<T>(P, Pj)) continue;
      const vec4_t<T> Vj = b.V0[j];
      const uint32_t oj = b.orig[j];
      const T dx = P.x - Pj.x, dy = P.y - Pj.y, dz = P.z - Pj.z;
      const T ux = V.x - Vj.x, uy = V.y - Vj.y, uz = V.z - Vj.z;
      const T R = P.w + Pj.w;
      T ddx, ddy, ddz, dux, duy, duz;
      // i receives from j
      pair_adjoint<T>(dx, dy, dz, ux, uy, uz, R, V.w, Vj.w, k, e, gx, gy, gz, ddx, ddy, ddz, dux, duy, duz, dk, de);
      xb0 += ddx;
      xb1 += ddy;
      xb2 += ddz;
      vb0 += dux;
      vb1 += duy;
      vb2 += duz;
      // j receives from i: i enters as the source (d and u change sign)
      double dk2 = 0.0, de2 = 0.0;
      const vec4_t<T> H = a.av[oj];
      const T hx = H.x, hy = H.y, hz = H.z;
      pair_adjoint<T>(-dx, -dy, -dz, -ux, -uy, -uz, R, Vj.w, V.w, k, e, hx, hy, hz, ddx, ddy, ddz, dux, duy, duz, dk2,
                      de2);
      xb0 -= ddx;
      xb1 -= ddy;
      xb2 -= ddz;
      vb0 -= dux;
      vb1 -= duy;
      vb2 -= duz;
    }
  }
  vec4_t<T> xo = X, vo = G;
  xo.x = xb0;
  xo.y = xb1;
  xo.z = xb2;
  vo.x = vb0;
  vo.y = vb1;
  vo.z = vb2;
  a.ax2[oi] = xo;
  a.av2[oi] = vo;
  a.acc[(size_t)ADJ_K * a.n + i] += dk;
  a.acc[(size_t)ADJ_E * a.n + i] += de;
}

// Walls + integrate adjoint over the tape row's sorted slots.  The step
// input (x, v) comes from the tape; x' and v' and the clamp events are
// recomputed from it with the forward's operations.
template <class T, bool MULTI>
__global__ void __launch_bounds__(STEP_THREADS) k_adj_walls_integrate(StepBufs<T> b, AdjBufs<T> a,
                                                                      SceneParams<T> sp0) {
  const uint32_t p = blockIdx.x * STEP_THREADS + threadIdx.x;
  if (p >= b.n) return;
  const SceneParams<T>& sp = scene_of<T, MULTI>(p, sp0, b.scenes, b.pbase, b.n_scenes);
  const uint32_t o = a.tape.o[p];
  vec4_t<T> P = a.tape.p[p];
  vec4_t<T> V = a.tape.v[p];
  integrate<T>(P, V, sp);  // x', v'
  using A = Ar<T>;
  const T r = P.w;
  const T xs[3] = {P.x, P.y, P.z}, vs[3] = {V.x, V.y, V.z};
  const int lo_idx[3] = {PS_XMIN, PS_YMIN, PS_ZMIN}, hi_idx[3] = {PS_XMAX, PS_YMAX, PS_ZMAX};
  double* acc = a.acc + p;  // row c at acc[c * n]
  const vec4_t<T> X2 = a.ax2[o], V2 = a.av2[o];
  const T xb2[3] = {X2.x, X2.y, X2.z}, vb2[3] = {V2.x, V2.y, V2.z};
  T xo[3], vo[3];
#pragma unroll
  for (int ax = 0; ax < 3; ++ax) {
    const bool lo_hit = A::sub(xs[ax], r) < sp.box_lo[ax];
    const bool hi_hit = A::add(xs[ax], r) > sp.box_hi[ax];
    T xb = xb2[ax], vb = vb2[ax];
    const T v1 = lo_hit ? A::mul(-vs[ax], sp.e_lo[ax]) : vs[ax];  // velocity after the min clamp
    if (hi_hit) {
      acc[(size_t)(ADJ_WALL + hi_idx[ax]) * a.n] += (double)(-v1 * vb);
      vb = -sp.e_hi[ax] * vb;
      xb = T(0);
    }
    if (lo_hit) {
      acc[(size_t)(ADJ_WALL + lo_idx[ax]) * a.n] += (double)(-vs[ax] * vb);
      vb = -sp.e_lo[ax] * vb;
      xb = T(0);
    }
    // integrate: x' = x + v dt, v' = v + g dt
    xo[ax] = xb;
    vo[ax] = vb + sp.dt * xb;
  }
  vec4_t<T> xw = X2, vw = V2;
  xw.x = xo[0];
  xw.y = xo[1];
  xw.z = xo[2];
  vw.x = vo[0];
  vw.y = vo[1];
  vw.z = vo[2];
  a.ax[o] = xw;
  a.av[o] = vw;
}

// Copy the at-rest state (P0, V1, orig) into a tape row.
template <class T>
__global__ void k_tape_write(StepBufs<T> b, TapeRow<T> row) {
  const uint32_t p = blockIdx.x * STEP_THREADS + threadIdx.x;
  if (p >= b.n) return;
  row.p[p] = b.P0[p];
  row.v[p] = b.V1[p];
  row.o[p] = b.orig[p];
}


// Per-scene sums of the parameter partials (acc: ADJ_NACC rows of n), in a
// fixed order.
__global__ void k_adj_reduce(const double* acc, const uint32_t* pbase, int n_scenes, uint32_t n, double* out) {
  const int s = blockIdx.x;
  if (s >= n_scenes) return;
  const uint32_t p0 = pbase[s], p1 = s + 1 < n_scenes ? pbase[s + 1] : n;
  __shared__ double red[ADJ_NACC][128];
  double loc[ADJ_NACC];
  for (int c = 0; c < ADJ_NACC; ++c) loc[c] = 0.0;
  for (uint32_t p = p0 + threadIdx.x; p < p1; p += blockDim.x)
    for (int c = 0; c < ADJ_NACC; ++c) loc[c] += acc[(size_t)c * n + p];
  for (int c = 0; c < ADJ_NACC; ++c) red[c][threadIdx.x] = loc[c];
  __syncthreads();
  for (int w = 64; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w)
      for (int c = 0; c < ADJ_NACC; ++c) red[c][threadIdx.x] += red[c][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int c = 0; c < ADJ_NACC; ++c) out[ADJ_NACC * s + c] = red[c][0];
}

}  // namespace psb
