/*
 * ps_oracle.h — CPU oracle for the particle-stabilizer DEM step.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/,
 * __graft_entry__.smoke() and the cpu_baseline leg of bench.py may load it.
 * The product library (libparticle_stabilizer_cuda.so) never links it.
 *
 * It restates, in plain C, the per-step scheme of the reference's CUDA
 * simulator (src/ParticleStabilizerCUDA/), one function per reference stage:
 *
 *   integrate           PhysicsEngine_kernels.cu:3-18
 *   box walls           BoxContainer_kernels.cu:3-56
 *   triangle container  PolygonContainerCUDA_kernels.cu:69-294
 *   grid set-up         ParticleModelCUDA.cpp:62-113
 *   cell ids / counts   ParticleModel_kernels.cu:42-85
 *   exclusive scan      PrefixScan.cu:232-268 (exclusive-sum semantics)
 *   bucket register     ParticleModel_kernels.cu:105-125 (canonical order)
 *   sphere contacts     ParticleModel_kernels.cu:127-201
 *   step order          PhysicsEngineCUDA.cpp:38-42
 *
 * and, behind `cpu_semantics`, the reference's CPU simulator
 * (src/ParticleStabilizer/PhysicsEngine.cpp:19-47, ParticleModel.cpp:81-144,
 * ParticleBucket.cpp:17-106, BoxContainer.cpp:22-65), which differs in the
 * spring formula, the grid interval and the step order.
 *
 * Determinism: the reference CUDA path orders particles inside a cell by
 * atomicAdd and accumulates velocity with FP64 atomics, so it is not
 * reproducible run to run.  The oracle fixes one canonical order: cells in
 * ascending id, particles inside a cell in ascending original index, and the
 * 27 neighbour cells visited x-outer, y, z-inner.  Every floating-point
 * operation of the CUDA-semantics scheme is written as one explicitly
 * rounded operation (fma() where the device code fuses), so a device kernel
 * that performs the same operations in the same order reproduces the oracle
 * bit for bit, in FP32 and in FP64.
 *
 * State layout (host interchange, identical to the reference's
 * ParticlePrimitive<double3>, include/ParticleStabilizer/ParticleModel.hpp:7-25):
 *   8 reals per particle: x, y, z, vx, vy, vz, radius, mass.
 */
#ifndef PS_ORACLE_H
#define PS_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Wall restitution order used by the reference everywhere
 * (include/ParticleStabilizer/ContainerBase.hpp:10-34). */
enum { OR_ZMIN = 0, OR_ZMAX = 1, OR_XMIN = 2, OR_XMAX = 3, OR_YMIN = 4, OR_YMAX = 5 };

typedef struct {
  double min[3];      /* grid domain minimum (container AABB minimum)      */
  double max[3];      /* grid domain maximum                               */
  double interval;    /* cell edge                                         */
  int32_t nb[3];      /* cells per axis: (int)((max-min)/interval) + 1     */
  int64_t n_cells;    /* nb[0]*nb[1]*nb[2]                                 */
} or_grid;

typedef struct {
  /* box container (also the grid domain when there is no mesh) */
  double box_min[3];
  double box_max[3];
  double gravity[3];
  double e_wall[6];        /* zMin, zMax, xMin, xMax, yMin, yMax           */
  double k_spring;
  double e_sphere;
  double dt;
  /* triangle container: de-indexed soup, 9 reals per triangle; NULL = box */
  const double* tri;
  int64_t n_tri;
  double e_poly;           /* the reference passes e_wall[zMin] here        */
  int32_t edge_quirk;      /* 1: reference edge pick by dot(center, point)  */
  int32_t cpu_semantics;   /* 1: reference CPU simulator formulas/order     */
  or_grid grid;            /* filled by or_grid_init                        */
} or_params;

/* ---- grid ------------------------------------------------------------ */
/* interval = maxRadius * 2.0 * 1.05 (ParticleModelCUDA.cpp:84)            */
double or_interval_cuda(double r_max);
/* interval = maxRadius * 2.0 * (double)1.05f (ParticleBucket.cpp:20,
 * ParticleBucket.hpp:17)                                                  */
double or_interval_cpu(double r_max);
/* nb = (int)((max-min)/interval) + 1 per axis (ParticleModelCUDA.cpp:89-91) */
void or_grid_init(const double dmin[3], const double dmax[3], double interval, or_grid* g);

/* ---- integer stages (precision-independent once cell ids exist) ------- */
/* count[c] += 1 per particle (countParticlesInEachBucketKernel)           */
void or_count(const int64_t* cell, int64_t n, int64_t n_cells, uint32_t* count);
/* exclusive prefix sum of count (PrefixScan::sum_scan_blelloch)           */
void or_exclusive_scan(const uint32_t* in, int64_t len, uint32_t* out);
/* canonical register order: order[offset[c] + k] = k-th smallest particle
 * index in cell c (registerToBucketKernel with a deterministic slot)      */
void or_stable_order(const int64_t* cell, int64_t n, const uint32_t* offset,
                     int64_t n_cells, uint32_t* order);

/* ---- FP64 scheme ----------------------------------------------------- */
void or_cell_ids_f64(const double* p, int64_t n, const or_grid* g, int32_t clamp, int64_t* cell);
void or_integrate_f64(double* p, int64_t n, const double g[3], double dt, int32_t cpu_semantics);
void or_walls_f64(double* p, int64_t n, const double bmin[3], const double bmax[3],
                  const double e_wall[6]);
/* Jacobi sphere contacts: reads `snap`, writes velocities into `out`
 * (which must hold a copy of snap on entry).                              */
void or_contacts_f64(const double* snap, double* out, int64_t n, const or_grid* g,
                     const uint32_t* offset, const uint32_t* order,
                     double k_spring, double e_sphere, int32_t cpu_semantics);
void or_mesh_f64(double* p, int64_t n, const double* tri, int64_t n_tri, double e_poly,
                 int32_t edge_quirk, int32_t cpu_semantics);
/* full steps; returns 0, or a negative code on bad input                  */
int32_t or_run_f64(double* p, int64_t n, const or_params* prm, int64_t steps);

/* ---- FP32 scheme (same operations in float) --------------------------- */
void or_cell_ids_f32(const float* p, int64_t n, const or_grid* g, int32_t clamp, int64_t* cell);
void or_integrate_f32(float* p, int64_t n, const double g[3], double dt);
void or_walls_f32(float* p, int64_t n, const double bmin[3], const double bmax[3],
                  const double e_wall[6]);
void or_contacts_f32(const float* snap, float* out, int64_t n, const or_grid* g,
                     const uint32_t* offset, const uint32_t* order,
                     double k_spring, double e_sphere);
void or_mesh_f32(float* p, int64_t n, const double* tri, int64_t n_tri, double e_poly,
                 int32_t edge_quirk);
int32_t or_run_f32(float* p, int64_t n, const or_params* prm, int64_t steps);

/* ---- forward-mode reference gradients (FP64, box container) ----------- */
/* Values as or_run_f64; dparam: nd x 8 parameter tangents (k_spring,
 * e_sphere, e_wall[6]); dstate: nd x n x 6 state tangents (x, y, z, vx, vy,
 * vz), updated in place.  Returns 0, or negative on bad input.            */
int32_t or_run_dual_f64(double* p, int64_t n, const or_params* prm, int64_t steps, int32_t nd,
                        const double* dparam, double* dstate);

/* ---- statistics (ParticleStatisticsCUDA.cpp:11-62) -------------------- */
typedef struct {
  double kinetic_energy;
  double min_pos[3];
  double max_pos[3];
  int64_t n_collided;
  double max_overlap;
} or_stats;
/* O(N^2) exactly as the reference; small N only                           */
void or_stats_f64(const double* p, int64_t n, or_stats* s);

#ifdef __cplusplus
}
#endif
#endif /* PS_ORACLE_H */
