/*
 * particle_stabilizer_b200.h — C ABI of libparticle_stabilizer_cuda.so, the
 * B200 (sm_100a) implementation of particle-stabilizer's per-step DEM path.
 *
 * Plain C types only: pointers, sizes, int status codes.  Every function
 * returns PS_OK (0) or a negative PS_ERR_* code; ps_last_error() gives the
 * message of the calling thread's last failure.  Nothing here exits the
 * process (the reference's CUDA_CHECK_ERROR logs and calls exit(),
 * include/ParticleStabilizerCUDA/CudaCommon.cuh:18-28).
 *
 * Host state layout (AoS, 8 doubles per particle, the reference's
 * ParticlePrimitive<glm::dvec3>, include/ParticleStabilizer/ParticleModel.hpp:7-25):
 *   x, y, z, vx, vy, vz, radius, mass
 *
 * The library also exports the reference's own entry point
 *   extern "C" void runSimulateCUDA(...)
 * with the exact C++ signature of
 * include/ParticleStabilizerCUDA/PhysicsEngineCUDA.hpp:43-54; it is declared
 * in include/ps_runsimulate.hpp because its arguments are C++ types.
 */
#ifndef PARTICLE_STABILIZER_B200_H
#define PARTICLE_STABILIZER_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PS_OK 0
#define PS_ERR_INVALID (-1)      /* bad argument                                */
#define PS_ERR_CUDA (-2)         /* CUDA runtime error                          */
#define PS_ERR_NOMEM (-3)        /* device or host allocation failed            */
#define PS_ERR_DEVICE (-4)       /* a kernel raised its device error word       */
#define PS_ERR_IO (-5)           /* file could not be read or written           */

#define PS_FP32 0
#define PS_FP64 1

/* Wall restitution indices, in the reference's order
 * (include/ParticleStabilizer/ContainerBase.hpp:10-34). */
#define PS_ZMIN 0
#define PS_ZMAX 1
#define PS_XMIN 2
#define PS_XMAX 3
#define PS_YMIN 4
#define PS_YMAX 5

/* One scene: the arguments of runSimulateCUDA
 * (src/ParticleStabilizerCUDA/PhysicsEngineCUDA.cpp:86-97) minus the state. */
typedef struct ps_scene_desc {
  int64_t n_particles;
  double box_min[3];        /* box container (ignored when tri != NULL)        */
  double box_max[3];
  double gravity[3];
  double e_wall[6];         /* PS_ZMIN..PS_YMAX                                 */
  double k_spring;          /* coefficientOfSpring                              */
  double e_sphere;          /* coefficientOfRestitutionSphere                   */
  double dt;
  double cell_size;         /* grid cell edge; 0 = reference rule 2.0*1.05*r_max
                               (ParticleModelCUDA.cpp:84); must be >= 2*r_max   */
  const double* tri;        /* triangle container: 9 doubles per triangle
                               (de-indexed soup, PolygonContainerCUDA.cpp:35-53);
                               NULL = box                                        */
  int64_t n_tri;
  int32_t edge_quirk;       /* 1 = the reference's edge pick by dot(center, point)
                               (PolygonContainerCUDA_kernels.cu:130-150); 0 = true
                               nearest edge point                                */
  int32_t widen_domain;     /* triangle container: grid domain = mesh AABB union
                               initial particle AABB (the reference uses the mesh
                               AABB only, PhysicsEngineCUDA.cpp:117)             */
} ps_scene_desc;

typedef struct ps_stats {    /* ParticleStatisticsCUDA (ParticleStatisticsCUDA.hpp:9-24) */
  double kinetic_energy;     /* sum 0.5 m |v|^2, FP64 reduction                   */
  double min_pos[3];         /* min of centre - radius                            */
  double max_pos[3];         /* max of centre + radius                            */
  int64_t n_collided;        /* particles overlapping a higher-indexed particle   */
  double max_overlap;        /* max over pairs of r_i + r_j - |x_i - x_j|         */
} ps_stats;

typedef struct ps_grid_info {
  double min[3];             /* grid domain minimum                              */
  double interval;           /* cell edge                                        */
  int32_t nb[3];             /* cells per axis                                    */
  int64_t n_cells;
  int64_t cell_base;         /* first global cell id of this scene               */
  int64_t particle_base;     /* first particle slot of this scene                */
} ps_grid_info;

typedef struct ps_sim ps_sim;

/* Message of this thread's last failure ("" if none). */
const char* ps_last_error(void);

/* 1 when this library is the bounds-checked build (compiled with
 * -DPS_DEBUG_BOUNDS, lib_debug/): device indexes into the bucket, order and
 * state arrays are checked, an index out of range is skipped and the call
 * that syncs next fails with PS_ERR_DEVICE; 0 for the product build.  No
 * counterpart in the reference. */
int32_t ps_bounds_checked(void);

/* Create a simulation of n_scenes independent scenes on CUDA device
 * `device`, in PS_FP32 or PS_FP64.  One scene replaces the set-up half of
 * runSimulateCUDA: ParticleModelCUDA ctor + container ctor + initBuckets
 * (PhysicsEngineCUDA.cpp:98-117, ParticleModelCUDA.cpp:4-52,62-113).
 * Several scenes advance together in every launch (batched execution).
 * The grid's r_max is taken from the first ps_set_state.  At most
 * 2^31 - 65 particles over all scenes (PS_ERR_INVALID beyond). */
int ps_create(const ps_scene_desc* scenes, int32_t n_scenes, int32_t precision, int32_t device, ps_sim** out);

/* Upload host state, scenes concatenated in order (replaces the H2D copy
 * of ParticleModelCUDA.cpp:36-43).  Also sizes the grids on first call. */
int ps_set_state(ps_sim* sim, const double* aos, int64_t n_total);

/* Download state in original particle order (ParticleModelCUDA::getParticles,
 * ParticleModelCUDA.cpp:183-189, and the copy-back of PhysicsEngineCUDA.cpp:154-174). */
int ps_get_state(ps_sim* sim, double* aos_out, int64_t n_total);

/* Advance every scene by n_steps steps (the loop body of
 * PhysicsEngineCUDA::startSimulationLoop, PhysicsEngineCUDA.cpp:38-42).
 * Asynchronous on the simulation's stream; blocks of steps run as CUDA graphs. */
int ps_step(ps_sim* sim, int64_t n_steps);

/* Wait for the stream and check the device error word. */
int ps_sync(ps_sim* sim);

/* Statistics of one scene (ParticleStatisticsCUDA::calculateStatistics,
 * ParticleStatisticsCUDA.cpp:11-62), using the grid instead of O(N^2). */
int ps_stats_get(ps_sim* sim, int32_t scene, ps_stats* out);

/* Grid of one scene (BucketContext, ParticleModelCUDA.hpp:17-32). */
int ps_grid_get(ps_sim* sim, int32_t scene, ps_grid_info* out);

/* Bucket arrays of the last grid rebuild over all scenes: per-cell counts
 * and exclusive offsets (n_cells_total entries each; the reference's
 * _deviceBucketCounter and _deviceBucketCumsumCounter), and the particle
 * index list in canonical order (cells ascending, original index ascending
 * inside a cell; the reference's _deviceBucket, ParticleModelCUDA.cpp:115-155).
 * Any pointer may be NULL. */
int ps_buckets_get(ps_sim* sim, uint32_t* counts, uint32_t* offsets, uint32_t* order);

/* Number of kernel launches issued by the last ps_step. */
int64_t ps_last_launch_count(ps_sim* sim);

/* Device-side checkpoints of the at-rest state (positions, velocities,
 * particle order) in numbered slots, kept in device memory.  No counterpart
 * in the reference (it has no checkpointing); used for restarts, the
 * checkpointed backward pass and benchmarking from a fixed state.
 * Ordered on the simulation's stream. */
int ps_checkpoint_save(ps_sim* sim, int32_t slot);
int ps_checkpoint_load(ps_sim* sim, int32_t slot);

/* Measurement (no counterpart in the reference, whose host loop syncs after
 * every launch): ps_time_steps runs ps_step(n_steps) between two CUDA events
 * recorded on the simulation's stream and returns the device milliseconds.
 * ps_profile_steps runs n_steps with every kernel launched on its own
 * between events and returns, per kernel kind (PS_K_*), the summed device
 * milliseconds and the launch count. */
#define PS_K_BEGIN 0     /* integrate + container + hash + count (first step of a call) */
#define PS_K_SCAN 1      /* decoupled look-back scan of the cell counts                  */
#define PS_K_SCATTER 2   /* slot ids into cell order, count reset                        */
#define PS_K_RANK_MOVE 3 /* canonical in-cell rank + state move                          */
#define PS_K_CONTACTS 4  /* sphere contacts (+ next integrate/container/hash/count)      */
#define PS_K_COUNT 5
int ps_time_steps(ps_sim* sim, int64_t n_steps, double* device_ms);
int ps_profile_steps(ps_sim* sim, int64_t n_steps, double* kernel_ms, int64_t* kernel_launches);

int ps_destroy(ps_sim* sim);

/* ---- differentiation (no counterpart in the reference) -------------------
 * Gradients of a loss of the final state with respect to the spring
 * coefficient, the sphere restitution, the six wall restitutions and the
 * initial state, for box-container scenes.  Two calls:
 *   ps_forward_checkpointed  advances n_steps from the current state,
 *                            keeping a device checkpoint every
 *                            `checkpoint_every` steps;
 *   ps_backward              given dL/d(final state), re-runs each block of
 *                            steps from its checkpoint and sweeps the adjoint
 *                            of contacts, walls and integration backwards.
 * Wall clamps and contact activation are taken as fixed events of the
 * forward values.  dl_dstate and dl_dstate0 are n_total x 6 doubles
 * (dL/dx, dL/dy, dL/dz, dL/dvx, dL/dvy, dL/dvz) in original particle order;
 * grads has one entry per scene.  After ps_backward the state is the final
 * state again. */
typedef struct ps_grad {
  double k_spring;
  double e_sphere;
  double e_wall[6];          /* PS_ZMIN..PS_YMAX */
} ps_grad;
int ps_forward_checkpointed(ps_sim* sim, int64_t n_steps, int64_t checkpoint_every);
int ps_backward(ps_sim* sim, const double* dl_dstate, ps_grad* grads, double* dl_dstate0);

/* ---- autotuning (no counterpart in the reference, whose cell edge is fixed
 * at 2.1 r_max, ParticleModelCUDA.cpp:84, and which has no step graphs) ----
 * ps_autotune times `trial_steps` steps from the current state for every
 * pair of a cell-size factor f (each scene's cell edge becomes f * 2 * r_max
 * of that scene; f >= 1) and a graph block length L (steps per captured CUDA
 * graph), keeps the fastest pair, and restores the state.  ms_table (may be
 * NULL) receives n_factors x n_blocks milliseconds per step, factor-major.
 * The cell size changes the grid and with it the summation order of the
 * contacts, so later trajectories are those of the chosen grid: deterministic,
 * and equal to the oracle's with that cell size, but not bit-equal to runs
 * with the previous grid.  A recorded ps_forward_checkpointed is dropped.
 * Then, on the chosen grid and L, it times the five contact kernels
 * (PS_WALK_LANE with 128, 256 and 512 threads per CTA, PS_WALK_WARP and
 * PS_WALK_ADAPTIVE with 256) and keeps the fastest; they give identical
 * results.
 * Allocates device memory (grids, graphs, one state copy). */
/* ---- neighbour-list mode (no counterpart in the reference, which rebuilds
 * its grid every step, ParticleModelCUDA.cpp:115-155) ----
 * ps_set_neighbor_lists(sim, skin_fraction, max_neighbours): with
 * skin_fraction in [0.01, 1], ps_step keeps per-sphere lists of the spheres
 * within r_i + r_j + skin (skin = skin_fraction x the scene's cell edge) and
 * rebuilds grid and lists only when some sphere has moved about skin / 2
 * since the last build (the device decides, step by step, through
 * conditional graph nodes); 0 switches the mode off (the default).
 * Results are bit-identical to the grid path: the overlapping pairs of each
 * sphere are applied in the grid walk's order.  A list longer than
 * max_neighbours, or more than 32 overlapping pairs on one sphere whose
 * order changed since the build, makes ps_step repeat the whole call on the
 * grid path from its starting state.  When the device rebuilds more often
 * than once per 4 steps over 256 or more steps, the next 1,024 steps run on
 * the grid path (doubling, up to 65,536, while that repeats); both paths
 * give the same states.  In this mode ps_step returns after the device has
 * finished.
 * ps_list_stats: rebuilds requested by the device, calls repeated on the
 * grid path after an overflow, and steps run on the grid path by the
 * backoff, all counted from the last ps_set_neighbor_lists; null pointers
 * are skipped. */
int ps_set_neighbor_lists(ps_sim* sim, double skin_fraction, int32_t max_neighbours);
int ps_list_stats(ps_sim* sim, int64_t* rebuilds, int64_t* fallbacks, int64_t* grid_steps);
/* Times trial_steps steps from the current state for every skin fraction in
 * skins[n_skins] (0 = the grid path), writes ms per step to ms_table (may be
 * null), keeps the fastest (ps_set_neighbor_lists) and restores the state. */
int ps_tune_neighbor_lists(ps_sim* sim, int64_t trial_steps, const double* skins, int32_t n_skins,
                           int32_t max_neighbours, double* ms_table, double* best_skin);

typedef struct ps_tune_result {
  double cell_factor;        /* chosen f                                          */
  int64_t graph_block;       /* chosen L                                          */
  double ms_per_step;        /* trial time per step with the choice               */
  double before_ms_per_step; /* trial time per step with the grid, L and contact  */
                             /* kernel in effect when ps_autotune was called      */
  int32_t contact_walk;      /* chosen contact kernel: PS_WALK_LANE/_WARP/_ADAPTIVE */
  int32_t contact_block;     /* and its threads per CTA                           */
  double contact_ms[5];      /* ms per step, with the chosen f and L, of the      */
                             /* contact kernels LANE/128, LANE/256, LANE/512,     */
                             /* WARP/256, ADAPTIVE/256                            */
} ps_tune_result;
int ps_autotune(ps_sim* sim, int64_t trial_steps, const double* cell_factors, int32_t n_factors,
                const int64_t* graph_blocks, int32_t n_blocks, double* ms_table, ps_tune_result* out);

/* The contact kernel's neighbour walk.  The reference runs 27 threads per
 * particle, one per neighbour cell (ParticleModel_kernels.cu:136-201,
 * launch :342-372); there is nothing to choose there.  PS_WALK_LANE: each
 * thread loops over its own nine slot ranges (the 27 cells as nine
 * (x, y) columns of three z-cells), 128, 256 or 512 threads per CTA.
 * PS_WALK_WARP: each warp reads the union of its 32 spheres' candidates in
 * a neighbour column with coalesced loads and hands them to the lanes by
 * register shuffle; 256 threads per CTA (measured slower than the lane walk
 * on every scene tried; kept as a tuner candidate).  PS_WALK_ADAPTIVE:
 * each warp chooses, from its spheres' range lengths, between the per-lane
 * walk and a flattened one (one loop over the concatenation of a thread's
 * non-empty ranges, so the warp waits for as many candidate loads as its
 * busiest lane has in all, not for the busiest lane of every column in
 * turn); the flattened walk wins on sparse grids, the per-lane walk on
 * dense piles; 256 threads.  Every variant applies
 * the same candidates in the same order, so results are bit-identical;
 * only the speed differs.  The default is PS_WALK_ADAPTIVE with 256 threads.
 * Changing it drops the captured step graphs. */
#define PS_WALK_LANE 0
#define PS_WALK_WARP 1
#define PS_WALK_ADAPTIVE 2
int ps_set_contact_kernel(ps_sim* sim, int32_t walk, int32_t block);
int ps_get_contact_kernel(ps_sim* sim, int32_t* walk, int32_t* block);

/* runSimulateCUDA with POD arguments: create, upload, max_steps steps,
 * download, destroy.  aos_out may alias aos_in. */
int ps_simulate(const ps_scene_desc* scene, const double* aos_in, double* aos_out, int64_t max_steps,
                int32_t precision);

/* Exclusive prefix sum of n uint32 on the device (PrefixScan::sum_scan_blelloch,
 * src/ParticleStabilizerCUDA/PrefixScan.cu:232-268), single pass with
 * decoupled look-back.  d_in may equal d_out.  d_scratch must hold
 * ps_exclusive_scan_scratch_bytes(n) bytes; the call clears it.  Ordered on
 * `stream` (a cudaStream_t, NULL = legacy default stream). */
size_t ps_exclusive_scan_scratch_bytes(int64_t n);
int ps_exclusive_scan_u32(const uint32_t* d_in, uint32_t* d_out, int64_t n, void* d_scratch, void* stream);

/* The same exclusive scan for callers that cannot allocate device memory:
 * code that runs while its stream is being captured into a CUDA graph (where
 * cudaMalloc is not allowed), real-time loops that cannot afford the device-
 * wide synchronisation cudaMalloc/cudaFree imply, and hosts whose device
 * memory is fully handed out to their own pool allocator.  It has no
 * counterpart in the reference.  It allocates nothing: its scratch is a
 * fixed array inside this library (128 KB per GPU, held from the moment the
 * library is loaded on that GPU until the process exits), so n is limited to
 * PS_SCAN_NOALLOC_MAX_N elements; larger n returns PS_ERR_INVALID.  The first
 * call in each CUDA context (the device's primary context, or a context of
 * the caller's own) looks up the array's device address; make that first
 * call before any stream capture.  Every call on a device shares the one
 * array, so calls whose kernels may overlap on the GPU (different streams
 * without ordering) race and give wrong results: order them on one stream.
 * d_in may equal d_out.  A look-back wait that gives up (a bounded wait; it
 * never hangs) leaves a wrong prefix and records PS_DEVERR_SCAN_TIMEOUT in a
 * device word that ps_exclusive_scan_u32_noalloc_status reports. */
#define PS_SCAN_NOALLOC_MAX_N 134217728LL
int ps_exclusive_scan_u32_noalloc(const uint32_t* d_in, uint32_t* d_out, int64_t n, void* stream);

/* Device error bits recorded by ps_exclusive_scan_u32_noalloc calls in the
 * current CUDA context since the previous status query: 0 when every scan
 * was complete, PS_DEVERR_SCAN_TIMEOUT (1) when a look-back wait gave up
 * and that call's prefix is wrong.  Waits for the work queued on `stream`,
 * so query on the stream the scans ran on; clears the bits.  Allocates
 * nothing.  No counterpart in the reference. */
int ps_exclusive_scan_u32_noalloc_status(void* stream, uint32_t* device_error);

/* CSV particle file, the reference's format (src/ParticleStabilizer/ParticleIO.cpp:58-144):
 * header line skipped; rows x,y,z,r; mass = density*4/3*pi*r^3; velocity is
 * the given vector.  ps_read_csv returns the row count in *n_out and fills
 * at most `cap` rows.  ps_write_csv writes x,y,z,radius in fixed 10-char fields. */
int ps_read_csv(const char* path, const double velocity[3], double density, double* aos_out, int64_t cap,
                int64_t* n_out);
int ps_write_csv(const char* path, const double* aos, int64_t n);

/* Binary state file for checkpoint / resume.  No counterpart in the
 * reference: its CSV output keeps positions and radii only, so a run cannot
 * be continued from it.  This file keeps every particle record in full
 * (8 doubles: x, y, z, vx, vy, vz, radius, mass, original order) and the
 * number of steps taken, so a run resumed from it continues bit for bit.
 * Layout, little-endian: 8-byte magic "PSB2STAT", uint32 version (1),
 * uint32 0, int64 n, int64 steps, then 8*n doubles.
 * ps_read_state_bin returns the record count in *n_out and fills at most
 * `cap` records (aos_out may be NULL to query the count). */
int ps_write_state_bin(const char* path, const double* aos, int64_t n, int64_t steps);
int ps_read_state_bin(const char* path, double* aos_out, int64_t cap, int64_t* n_out, int64_t* steps_out);

/* OBJ container file (PolygonContainerCUDA::readFromFile,
 * PolygonContainerCUDA.cpp:314-350): triangles de-indexed to 9 doubles each,
 * vertices read in single precision as assimp's default ai_real. */
int ps_read_obj(const char* path, double* tri_out, int64_t cap, int64_t* n_tri_out);

/* ---- after the path: the CLI's post-processing of a result (host code) ----
 * ps_resolve_overlaps   ParticleModel::resolveOverlaps
 *                       (src/ParticleStabilizer/ParticleModel.cpp:154-259):
 *   walks the particles in ascending order of coordinate `axis` (0, 1, 2) and
 *   lifts each along that axis onto the first lower-ranked particle it
 *   overlaps, re-ranking as the reference does; positions in `aos` (n x 8
 *   reference records) are updated in place, with the reference's results.
 *   If n_collided and max_overlap are not NULL they receive the closing
 *   overlap check (as ps_overlap_stats).  Non-finite positions are rejected.
 * ps_overlap_stats      the reference's closing check (ParticleModel.cpp:232-256):
 *   particles overlapping a higher-indexed particle, and the largest
 *   r_i + r_j - |x_i - x_j|; grid-based instead of O(N^2).
 * ps_write_obj_spheres  ObjData::write (src/ParticleStabilizer/ObjData.cpp:8-140):
 *   every particle as a triangulated sphere; the same text, formatted in
 *   parallel. */
int ps_resolve_overlaps(double* aos, int64_t n, int32_t axis, int64_t* n_collided, double* max_overlap);
int ps_overlap_stats(const double* aos, int64_t n, int64_t* n_collided, double* max_overlap);
int ps_write_obj_spheres(const char* path, const double* aos, int64_t n);

#ifdef __cplusplus
}
#endif
#endif /* PARTICLE_STABILIZER_B200_H */
