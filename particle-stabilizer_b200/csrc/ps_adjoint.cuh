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
  // Adjoints of positions and velocities (w unused), one 16/32-B record per
  // particle, kept in the sorted order of the at-rest state they belong to:
  // before step t's reverse they follow the order after step t (its grid's
  // order), after it the order of step t's input (the previous grid's), so
  // every kernel reads and writes them by slot.
  vec4_t<T>* ax;
  vec4_t<T>* av;
  vec4_t<T>* ax2;         // output of k_adj_contacts, in the order of step t's grid
  vec4_t<T>* av2;
  uint32_t* inv;          // slot in step t's grid of each original id (written by k_adj_contacts)
  double* acc;            // ADJ_NACC rows of n, accumulated over steps: rows k, e by sorted
                          // slot, wall rows by original index
  uint32_t n;             // row length of acc
};

// Geometry of one active pair, shared by its two directions: d = x_i - x_j,
// u = v_i - v_j, L = |d|, ov = R - L, ud = u.d, and the reciprocals.
template <class T>
struct PairGeom {
  T dx, dy, dz, ux, uy, uz, L, iL, iL2, ov, ud, R;
};

// Terms of one direction of an active pair for the receiver r and the
// source s: c_r = f d with f = k ov / (L m_r) - B ud / L^2,
// B = 2 m_s e / (m_r + m_s); g = adjoint of v_r's output; sgn = +1 when r is
// the pair's first sphere (d as stored) and -1 when it is the second (d and
// u negated, ud and L unchanged).  Returns the adjoint of d and of u with
// respect to the pair's stored d and u, and adds the parameter partials.
template <class T>
__device__ __forceinline__ void pair_adjoint(const PairGeom<T>& q, T sgn, T mr, T ms, T inv_msum, T k, T e, T gx,
                                             T gy, T gz, T& ddx, T& ddy, T& ddz, T& dux, T& duy, T& duz,
                                             double& dk, double& de) {
  const T imr = T(1) / mr;
  const T Bc = T(2) * ms * e * inv_msum;
  const T f = k * q.ov * q.iL * imr - Bc * q.ud * q.iL2;
  const T fbar = sgn * (gx * q.dx + gy * q.dy + gz * q.dz);
  dk += (double)(fbar * q.ov * q.iL * imr);
  de += (double)(fbar * (-(T(2) * ms * q.ud) * inv_msum * q.iL2));
  const T fL = -k * q.R * q.iL2 * imr + T(2) * Bc * q.ud * q.iL2 * q.iL;
  const T Lb = fbar * fL * q.iL;
  const T udb = -fbar * Bc * q.iL2;
  // adjoint of the direction's own d (= sgn d) and u (= sgn u), mapped back
  ddx = sgn * (f * gx) + Lb * q.dx + udb * q.ux;
  ddy = sgn * (f * gy) + Lb * q.dy + udb * q.uy;
  ddz = sgn * (f * gz) + Lb * q.dz + udb * q.uz;
  dux = udb * q.dx;
  duy = udb * q.dy;
  duz = udb * q.dz;
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
  // one wave of CTAs (occupancy x SMs, the host's choice) loops over the particles
  for (uint32_t i = blockIdx.x * STEP_THREADS + threadIdx.x; i < b.n; i += gridDim.x * STEP_THREADS) {
    const SceneParams<T>& sp = scene_of<T, MULTI>(i, sp0, b.scenes, b.pbase, b.n_scenes);
    const vec4_t<T> P = b.P0[i];
    const vec4_t<T> V = b.V0[i];
    const uint32_t oi = b.orig[i];
    a.inv[oi] = i;
    const vec4_t<T> G = a.av[i], X = a.ax[i];
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
    uint32_t lo[9], hi[9];
  #pragma unroll
    for (int q = 0; q < 9; ++q) {  // the 18 range bounds, loaded together
      const int32_t bx = cx - 1 + q / 3, by = cy - 1 + q % 3;
      const bool ok = live && bx >= 0 && bx < nx && by >= 0 && by < ny;
      const uint32_t col = ok ? sp.cbase + ((uint32_t)bx * (uint32_t)ny + (uint32_t)by) * (uint32_t)nz : sp.cbase;
      lo[q] = ok ? __ldg(b.offset + col + z0) : 0u;
      hi[q] = ok ? __ldg(b.offset + col + z1) : 0u;
    }
  #pragma unroll
    for (int q = 0; q < 9; ++q)
      for (uint32_t j = lo[q]; j < hi[q]; ++j) {
        if (q == 4 && j == i) continue;  // only the own column holds the sphere itself
        const vec4_t<T> Pj = ld4<T>(b.P0 + j);
        if (!pair_active<T>(P, Pj)) continue;
        const vec4_t<T> Vj = b.V0[j];
        const vec4_t<T> H = a.av[j];
        PairGeom<T> g;
        g.dx = P.x - Pj.x;
        g.dy = P.y - Pj.y;
        g.dz = P.z - Pj.z;
        g.ux = V.x - Vj.x;
        g.uy = V.y - Vj.y;
        g.uz = V.z - Vj.z;
        g.R = P.w + Pj.w;
        const T L2 = g.dx * g.dx + g.dy * g.dy + g.dz * g.dz;
        g.L = sqrt(L2);
        g.iL = T(1) / g.L;
        g.iL2 = T(1) / L2;
        g.ov = g.R - g.L;
        g.ud = g.ux * g.dx + g.uy * g.dy + g.uz * g.dz;
        const T inv_msum = T(1) / (V.w + Vj.w);
        T ddx, ddy, ddz, dux, duy, duz;
        // i receives from j
        pair_adjoint<T>(g, T(1), V.w, Vj.w, inv_msum, k, e, gx, gy, gz, ddx, ddy, ddz, dux, duy, duz, dk, de);
        xb0 += ddx;
        xb1 += ddy;
        xb2 += ddz;
        vb0 += dux;
        vb1 += duy;
        vb2 += duz;
        // j receives from i: that direction's d and u are -d and -u, so its
        // adjoints with respect to the stored d and u come back sign-mapped;
        // its parameter partials belong to j's own thread
        double dk2 = 0.0, de2 = 0.0;
        pair_adjoint<T>(g, T(-1), Vj.w, V.w, inv_msum, k, e, H.x, H.y, H.z, ddx, ddy, ddz, dux, duy, duz, dk2, de2);
        xb0 += ddx;
        xb1 += ddy;
        xb2 += ddz;
        vb0 += dux;
        vb1 += duy;
        vb2 += duz;
      }
    vec4_t<T> xo = X, vo = G;
    xo.x = xb0;
    xo.y = xb1;
    xo.z = xb2;
    vo.x = vb0;
    vo.y = vb1;
    vo.z = vb2;
    a.ax2[i] = xo;
    a.av2[i] = vo;
    a.acc[(size_t)ADJ_K * a.n + i] += dk;
    a.acc[(size_t)ADJ_E * a.n + i] += de;
  }
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
  const uint32_t i = a.inv[o];  // this particle's slot in step t's grid
  const vec4_t<T> X2 = a.ax2[i], V2 = a.av2[i];
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
  a.ax[p] = xw;
  a.av[p] = vw;
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
