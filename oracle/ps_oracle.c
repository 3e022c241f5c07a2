/*
 * ps_oracle.c — CPU oracle for the particle-stabilizer DEM step.
 *
 * TEST INFRASTRUCTURE ONLY (see ps_oracle.h).  Build with
 * -ffp-contract=off so the compiler adds no fused operations of its own:
 * the only fused multiply-adds are the explicit fma()/fmaf() calls.
 */
#define _DEFAULT_SOURCE /* sysconf */
#include "ps_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

/* host threads for the triangle pass of large calls */
#define OR_MAX_THREADS 64

/* ---- grid (ParticleModelCUDA.cpp:62-113, ParticleBucket.cpp:17-27) ---- */
double or_interval_cuda(double r_max) { return r_max * 2.0 * 1.05; }

double or_interval_cpu(double r_max) { return r_max * 2.0 * (double)1.05f; }

void or_grid_init(const double dmin[3], const double dmax[3], double interval, or_grid* g) {
  for (int a = 0; a < 3; ++a) {
    g->min[a] = dmin[a];
    g->max[a] = dmax[a];
    g->nb[a] = (int32_t)((dmax[a] - dmin[a]) / interval) + 1;
  }
  g->interval = interval;
  g->n_cells = (int64_t)g->nb[0] * g->nb[1] * g->nb[2];
}

/* ---- integer stages --------------------------------------------------- */
void or_count(const int64_t* cell, int64_t n, int64_t n_cells, uint32_t* count) {
  memset(count, 0, sizeof(uint32_t) * (size_t)n_cells);
  for (int64_t i = 0; i < n; ++i) count[cell[i]] += 1u;
}

void or_exclusive_scan(const uint32_t* in, int64_t len, uint32_t* out) {
  uint32_t run = 0;
  for (int64_t i = 0; i < len; ++i) {
    const uint32_t v = in[i];
    out[i] = run;
    run += v;
  }
}

void or_stable_order(const int64_t* cell, int64_t n, const uint32_t* offset, int64_t n_cells,
                     uint32_t* order) {
  uint32_t* fill = (uint32_t*)calloc((size_t)n_cells, sizeof(uint32_t));
  if (!fill) return;
  for (int64_t i = 0; i < n; ++i) {
    const int64_t c = cell[i];
    order[offset[c] + fill[c]] = (uint32_t)i;
    fill[c] += 1u;
  }
  free(fill);
}

/* ---- precision-generic scheme ----------------------------------------- */
#define REAL double
#define SFX(name) name##_f64
#define FMA_ fma
#define SQRT_ sqrt
#define OR_IS_F64 1
#include "ps_oracle_impl.inc"
#undef REAL
#undef SFX
#undef FMA_
#undef SQRT_
#undef OR_IS_F64

#define REAL float
#define SFX(name) name##_f32
#define FMA_ fmaf
#define SQRT_ sqrtf
#define OR_IS_F64 0
#include "ps_oracle_impl.inc"
#undef REAL
#undef SFX
#undef FMA_
#undef SQRT_
#undef OR_IS_F64

/* ---- CPU simulator's triangle container (FP64 only) ------------------- */
/* glm's definitions: dot = (x*x' + y*y') + z*z'; length = sqrt(dot(v,v));
 * distance(a,b) = length(b-a); normalize(v) = v * (1/sqrt(dot(v,v)));
 * cross as the usual determinant expansion.                               */
typedef struct { double x, y, z; } gv3;
static inline gv3 g_mk(double x, double y, double z) { gv3 v = {x, y, z}; return v; }
static inline gv3 g_sub(gv3 a, gv3 b) { return g_mk(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline double g_dot(gv3 a, gv3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
static inline double g_len(gv3 a) { return sqrt(g_dot(a, a)); }

static gv3 g_project(gv3 p, gv3 a, gv3 n) {
  const double ip = g_dot(g_sub(p, a), n);
  return g_mk(p.x - n.x * ip, p.y - n.y * ip, p.z - n.z * ip);
}

static int g_inside(gv3 p, gv3 a, gv3 b, gv3 c) {
  const gv3 v0 = g_sub(c, a), v1 = g_sub(b, a), v2 = g_sub(p, a);
  const double d00 = g_dot(v0, v0), d01 = g_dot(v0, v1), d02 = g_dot(v0, v2);
  const double d11 = g_dot(v1, v1), d12 = g_dot(v1, v2);
  const double inv = 1.0 / (d00 * d11 - d01 * d01);
  const double u = (d11 * d02 - d01 * d12) * inv;
  const double v = (d00 * d12 - d01 * d02) * inv;
  return (u >= 0.0) && (v >= 0.0) && (u + v <= 1.0);
}

static gv3 g_seg(gv3 p, gv3 a, gv3 b) {
  const gv3 ab = g_sub(b, a), ap = g_sub(p, a);
  double t = g_dot(ap, ab) / g_dot(ab, ab);
  t = (t < 1.0) ? t : 1.0;  /* std::min(1.0, t) */
  t = (0.0 < t) ? t : 0.0;  /* std::max(0.0, .) */
  return g_mk(a.x + ab.x * t, a.y + ab.y * t, a.z + ab.z * t);
}

/* PolygonContainer::getClosestPointOnPolygon (PolygonContainer.cpp:136-173) */
static gv3 g_closest(gv3 a, gv3 b, gv3 c, gv3 n, gv3 p) {
  gv3 q = g_project(p, a, n);
  if (g_inside(q, a, b, c)) return q;
  const gv3 e0 = g_seg(p, a, b);
  double best = g_len(g_sub(e0, p));
  q = e0;
  const gv3 e1 = g_seg(p, b, c);
  const double d1 = g_len(g_sub(e1, p));
  if (d1 < best) { best = d1; q = e1; }
  const gv3 e2 = g_seg(p, c, a);
  const double d2 = g_len(g_sub(e2, p));
  if (d2 < best) { best = d2; q = e2; }
  return q;
}

/* PolygonContainer::resolveCollisions (PolygonContainer.cpp:237-286): the
 * position correction is applied sequentially to the buffer position.     */
static void mesh_cpu_f64(double* p, int64_t n, const double* tri, int64_t n_tri, double e) {
  for (int64_t i = 0; i < n; ++i) {
    double* q = p + 8 * i;
    const gv3 c = g_mk(q[0], q[1], q[2]);
    const gv3 v = g_mk(q[3], q[4], q[5]);
    const double r = q[6];
    const gv3 lo = g_mk(c.x - r, c.y - r, c.z - r), hi = g_mk(c.x + r, c.y + r, c.z + r);
    gv3 bp = c, bv = g_mk(0.0, 0.0, 0.0);
    int64_t hits = 0;
    for (int64_t t = 0; t < n_tri; ++t) {
      const double* T = tri + 9 * t;
      const gv3 a = g_mk(T[0], T[1], T[2]), b = g_mk(T[3], T[4], T[5]), cc = g_mk(T[6], T[7], T[8]);
      const gv3 tmin = g_mk(fmin(fmin(a.x, b.x), cc.x), fmin(fmin(a.y, b.y), cc.y), fmin(fmin(a.z, b.z), cc.z));
      const gv3 tmax = g_mk(fmax(fmax(a.x, b.x), cc.x), fmax(fmax(a.y, b.y), cc.y), fmax(fmax(a.z, b.z), cc.z));
      if (lo.x > tmax.x || hi.x < tmin.x || lo.y > tmax.y || hi.y < tmin.y || lo.z > tmax.z ||
          hi.z < tmin.z)
        continue;
      const gv3 r0 = g_sub(b, a), r1 = g_sub(cc, a);
      const gv3 cr = g_mk(r0.y * r1.z - r1.y * r0.z, r0.z * r1.x - r1.z * r0.x, r0.x * r1.y - r1.x * r0.y);
      const double inv = 1.0 / sqrt(g_dot(cr, cr));
      const gv3 nrm = g_mk(cr.x * inv, cr.y * inv, cr.z * inv);
      const gv3 cp = g_closest(a, b, cc, nrm, c);
      if (!(g_len(g_sub(cp, c)) < r)) continue;
      const double vn2 = 2.0 * g_dot(v, nrm);
      bv.x += e * (v.x - vn2 * nrm.x);
      bv.y += e * (v.y - vn2 * nrm.y);
      bv.z += e * (v.z - vn2 * nrm.z);
      const double dtp = g_dot(g_mk(-nrm.x, -nrm.y, -nrm.z), g_sub(bp, a));
      const double mod = r - dtp;
      bp = g_mk(bp.x - mod * nrm.x, bp.y - mod * nrm.y, bp.z - mod * nrm.z);
      ++hits;
    }
    if (hits > 0) {
      const double h = (double)hits;
      q[0] = bp.x; q[1] = bp.y; q[2] = bp.z;
      q[3] = bv.x / h; q[4] = bv.y / h; q[5] = bv.z / h;
    }
  }
}

void or_mesh_f64(double* p, int64_t n, const double* tri, int64_t n_tri, double e_poly,
                 int32_t edge_quirk, int32_t cpu_semantics) {
  if (cpu_semantics)
    mesh_cpu_f64(p, n, tri, n_tri, e_poly);
  else
    mesh_cuda_f64(p, n, tri, n_tri, e_poly, edge_quirk);
}

/* ---- statistics (ParticleStatisticsCUDA.cpp:11-62) -------------------- */
void or_stats_f64(const double* p, int64_t n, or_stats* s) {
  memset(s, 0, sizeof(*s));
  if (n <= 0) return;
  for (int a = 0; a < 3; ++a) {
    s->min_pos[a] = p[a] - p[6];
    s->max_pos[a] = p[a] + p[6];
  }
  for (int64_t i = 0; i < n; ++i) {
    const double* q = p + 8 * i;
    s->kinetic_energy += 0.5 * q[7] * (q[3] * q[3] + q[4] * q[4] + q[5] * q[5]);
    for (int a = 0; a < 3; ++a) {
      s->min_pos[a] = fmin(s->min_pos[a], q[a] - q[6]);
      s->max_pos[a] = fmax(s->max_pos[a], q[a] + q[6]);
    }
  }
  for (int64_t i = 0; i < n; ++i) {
    const double* q = p + 8 * i;
    int hit = 0;
    for (int64_t j = i + 1; j < n; ++j) {
      const double* w = p + 8 * j;
      const double dx = q[0] - w[0], dy = q[1] - w[1], dz = q[2] - w[2];
      const double dist = sqrt(dx * dx + dy * dy + dz * dz);
      const double ov = q[6] + w[6] - dist;
      if (ov > 0.0) {
        hit = 1;
        if (ov > s->max_overlap) s->max_overlap = ov;
      }
    }
    s->n_collided += hit;
  }
}
