/*
 * ps_oracle_dual.c — forward-mode (dual-number) FP64 reference gradients of
 * the CUDA-semantics DEM step.  TEST INFRASTRUCTURE (see ps_oracle.h).
 *
 * Values follow or_run_f64 operation for operation (box container only), so
 * they are bit-identical to it; alongside each state value the routine
 * carries its derivatives along `nd` directions.  A direction is a tangent
 * of the parameters (k_spring, e_sphere, the six wall restitutions in the
 * reference's order zMin, zMax, xMin, xMax, yMin, yMax) and of the initial
 * state.  Wall contacts and sphere-contact activation are treated as
 * piecewise events decided by the values, as in the reverse-mode device
 * adjoint.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "ps_oracle.h"

static inline int32_t cell_axis(double x, double lo, double iv, int32_t nb) {
  const double q = (x - lo) / iv;
  if (!(q > 0.0)) return 0;
  if (q >= (double)nb) return nb - 1;
  return (int32_t)q;
}

/* p: n x 8 state (values, updated in place).
 * dparam: nd x 8 parameter tangents (k, e_sphere, e_wall[6]).
 * dstate: nd x n x 6 state tangents (dx, dy, dz, dvx, dvy, dvz), updated. */
int32_t or_run_dual_f64(double* p, int64_t n, const or_params* prm, int64_t steps, int32_t nd,
                        const double* dparam, double* dstate) {
  if (n < 0 || steps < 0 || nd < 0 || prm == NULL || prm->tri != NULL) return -1;
  if (n == 0 || steps == 0) return 0;
  const or_grid* g = &prm->grid;
  int64_t* cell = (int64_t*)malloc(sizeof(int64_t) * (size_t)n);
  uint32_t* count = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)(g->n_cells + 1));
  uint32_t* offset = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)(g->n_cells + 1));
  uint32_t* order = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)n);
  double* snap = (double*)malloc(sizeof(double) * 8 * (size_t)n);
  double* dsnap = (double*)malloc(sizeof(double) * 6 * (size_t)n * (size_t)(nd > 0 ? nd : 1));
  double* acc = (double*)malloc(sizeof(double) * 3 * (size_t)(nd > 0 ? nd : 1));
  if (!cell || !count || !offset || !order || !snap || !dsnap || !acc) {
    free(cell); free(count); free(offset); free(order); free(snap); free(dsnap); free(acc);
    return -3;
  }
  const double dt = prm->dt, k = prm->k_spring, e = prm->e_sphere;
  const double lo[3] = {prm->box_min[0], prm->box_min[1], prm->box_min[2]};
  const double hi[3] = {prm->box_max[0], prm->box_max[1], prm->box_max[2]};
  const int elo_idx[3] = {OR_XMIN, OR_YMIN, OR_ZMIN}, ehi_idx[3] = {OR_XMAX, OR_YMAX, OR_ZMAX};
#define DS(d, i, c) dstate[((size_t)(d) * (size_t)n + (size_t)(i)) * 6 + (c)]
#define DP(d, c) dparam[(size_t)(d) * 8 + (c)]
  for (int64_t s = 0; s < steps; ++s) {
    /* integrate: x = fma(v, dt, x); v = fma(g, dt, v) */
    for (int64_t i = 0; i < n; ++i) {
      double* q = p + 8 * i;
      for (int a = 0; a < 3; ++a) {
        q[a] = fma(q[3 + a], dt, q[a]);
        q[3 + a] = fma(prm->gravity[a], dt, q[3 + a]);
        for (int32_t d = 0; d < nd; ++d) DS(d, i, a) += dt * DS(d, i, 3 + a);
      }
    }
    /* walls (BoxContainer_kernels.cu:17-52), events from the values */
    for (int64_t i = 0; i < n; ++i) {
      double* q = p + 8 * i;
      const double r = q[6];
      const double mn[3] = {q[0] - r, q[1] - r, q[2] - r}, mx[3] = {q[0] + r, q[1] + r, q[2] + r};
      for (int a = 0; a < 3; ++a) {
        if (mn[a] < lo[a]) {
          const double el = prm->e_wall[elo_idx[a]], v = q[3 + a];
          q[a] = lo[a] + r;
          q[3 + a] = -v * el;
          for (int32_t d = 0; d < nd; ++d) {
            DS(d, i, a) = 0.0;
            DS(d, i, 3 + a) = -(DS(d, i, 3 + a) * el + v * DP(d, 2 + elo_idx[a]));
          }
        }
      }
      for (int a = 0; a < 3; ++a) {
        if (mx[a] > hi[a]) {
          const double eh = prm->e_wall[ehi_idx[a]], v = q[3 + a];
          q[a] = hi[a] - r;
          q[3 + a] = -v * eh;
          for (int32_t d = 0; d < nd; ++d) {
            DS(d, i, a) = 0.0;
            DS(d, i, 3 + a) = -(DS(d, i, 3 + a) * eh + v * DP(d, 2 + ehi_idx[a]));
          }
        }
      }
    }
    /* grid */
    for (int64_t i = 0; i < n; ++i) {
      const double* q = p + 8 * i;
      cell[i] = ((int64_t)cell_axis(q[0], g->min[0], g->interval, g->nb[0]) * g->nb[1] +
                 cell_axis(q[1], g->min[1], g->interval, g->nb[1])) * (int64_t)g->nb[2] +
                cell_axis(q[2], g->min[2], g->interval, g->nb[2]);
    }
    or_count(cell, n, g->n_cells, count);
    count[g->n_cells] = 0;
    or_exclusive_scan(count, g->n_cells + 1, offset);
    or_stable_order(cell, n, offset, g->n_cells, order);
    memcpy(snap, p, sizeof(double) * 8 * (size_t)n);
    if (nd > 0) memcpy(dsnap, dstate, sizeof(double) * 6 * (size_t)n * (size_t)nd);
    /* Jacobi contacts, same values as or_contacts_f64, with tangents */
    for (int64_t i = 0; i < n; ++i) {
      const double* pi = snap + 8 * i;
      const double xi = pi[0], yi = pi[1], zi = pi[2], ri = pi[6], mi = pi[7];
      double vx = pi[3], vy = pi[4], vz = pi[5];
      for (int32_t d = 0; d < nd; ++d) acc[3 * d] = acc[3 * d + 1] = acc[3 * d + 2] = 0.0;
      const int32_t cx = cell_axis(xi, g->min[0], g->interval, g->nb[0]) - 1;
      const int32_t cy = cell_axis(yi, g->min[1], g->interval, g->nb[1]) - 1;
      const int32_t cz = cell_axis(zi, g->min[2], g->interval, g->nb[2]) - 1;
      for (int ox = 0; ox < 3; ++ox) {
        const int32_t bx = cx + ox;
        if (bx < 0 || bx >= g->nb[0]) continue;
        for (int oy = 0; oy < 3; ++oy) {
          const int32_t by = cy + oy;
          if (by < 0 || by >= g->nb[1]) continue;
          for (int oz = 0; oz < 3; ++oz) {
            const int32_t bz = cz + oz;
            if (bz < 0 || bz >= g->nb[2]) continue;
            const int64_t c = ((int64_t)bx * g->nb[1] + by) * (int64_t)g->nb[2] + bz;
            for (uint32_t sl = offset[c]; sl < offset[c + 1]; ++sl) {
              const int64_t j = order[sl];
              if (j == i) continue;
              const double* pj = snap + 8 * j;
              const double dx = xi - pj[0], dy = yi - pj[1], dz = zi - pj[2];
              const double d2 = fma(dz, dz, fma(dy, dy, dx * dx));
              const double dist = sqrt(d2);
              const double mj = pj[7];
              const double overlap = (ri + pj[6]) - dist;
              if (!(overlap > 0.0)) continue;
              const double rvx = pi[3] - pj[3], rvy = pi[4] - pj[4], rvz = pi[5] - pj[5];
              const double rvd = fma(rvz, dz, fma(rvy, dy, rvx * dx));
              const double cr = ((2.0 * mj) * rvd * e) / ((mi + mj) * d2);
              const double cs = (k * overlap) / (dist * mi);
              const double f = cs - cr;
              vx = fma(f, dx, vx);
              vy = fma(f, dy, vy);
              vz = fma(f, dz, vz);
              const double B = 2.0 * mj / (mi + mj);
              for (int32_t dd = 0; dd < nd; ++dd) {
                const double* ti = dsnap + ((size_t)dd * (size_t)n + (size_t)i) * 6;
                const double* tj = dsnap + ((size_t)dd * (size_t)n + (size_t)j) * 6;
                const double ddx = ti[0] - tj[0], ddy = ti[1] - tj[1], ddz = ti[2] - tj[2];
                const double dux = ti[3] - tj[3], duy = ti[4] - tj[4], duz = ti[5] - tj[5];
                const double dd2 = 2.0 * (dx * ddx + dy * ddy + dz * ddz);
                const double ddist = dd2 / (2.0 * dist);
                const double drvd = dux * dx + duy * dy + duz * dz + rvx * ddx + rvy * ddy + rvz * ddz;
                const double dk = DP(dd, 0), de = DP(dd, 1);
                const double dcs = (dk * overlap - k * ddist) / (dist * mi) - (k * overlap) * ddist / (dist * dist * mi);
                const double dcr = B * (de * rvd / d2 + e * drvd / d2 - e * rvd * dd2 / (d2 * d2));
                const double df = dcs - dcr;
                acc[3 * dd + 0] += df * dx + f * ddx;
                acc[3 * dd + 1] += df * dy + f * ddy;
                acc[3 * dd + 2] += df * dz + f * ddz;
              }
            }
          }
        }
      }
      double* oi = p + 8 * i;
      oi[3] = vx;
      oi[4] = vy;
      oi[5] = vz;
      for (int32_t d = 0; d < nd; ++d) {
        DS(d, i, 3) += acc[3 * d];
        DS(d, i, 4) += acc[3 * d + 1];
        DS(d, i, 5) += acc[3 * d + 2];
      }
    }
  }
#undef DS
#undef DP
  free(cell); free(count); free(offset); free(order); free(snap); free(dsnap); free(acc);
  return 0;
}
