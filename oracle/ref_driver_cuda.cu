// ref_driver_cuda.cu — harness around the reference's own CUDA simulator.
//
// TEST INFRASTRUCTURE.  Linked with the unmodified reference sources
// (src/ParticleStabilizerCUDA/{ParticleModelCUDA,BoxContainerCUDA,
// PolygonContainerCUDA}.cpp and the *_kernels.cu / PrefixScan.cu files),
// compiled for sm_100a into oracle/_ref/libref_cuda.so.  It drives the
// per-step body of PhysicsEngineCUDA::startSimulationLoop
// (src/ParticleStabilizerCUDA/PhysicsEngineCUDA.cpp:38-42) without the
// O(N^2) host statistics, and reads back the bucket arrays so tests can
// compare cell counts and scan offsets with the new kernels.
//
// Only box scenes whose particles start inside the box, and mesh scenes
// whose particles stay inside the mesh AABB, are safe to run: the
// reference's count/register kernels do not clamp cell ids
// (ParticleModel_kernels.cu:49-56).  refc_create rejects other inputs.

// Standard and CUDA headers first, so the access override below touches
// only the reference's own class declarations.
#include <assimp/Importer.hpp>
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <filesystem>
#include <fstream>
#include <iostream>
#include <limits>
#include <memory>
#include <set>
#include <sstream>
#include <string>
#include <vector>

#define private public
#include <ParticleStabilizerCUDA/BoxContainerCUDA.hpp>
#include <ParticleStabilizerCUDA/ParticleModelCUDA.hpp>
#include <ParticleStabilizerCUDA/PhysicsEngine_kernels.cuh>
#include <ParticleStabilizerCUDA/PolygonContainerCUDA.hpp>
#undef private

namespace {
struct RefCuda {
  std::vector<ParticlePtr> particles;
  std::shared_ptr<ParticleModelCUDA> model;
  std::shared_ptr<ContainerBaseCUDA> container;
  double3 gravity;
  double dt = 0.0;
};

void step_once(RefCuda* h) {
  lanchUpdatePositionAndVelocityKernel(h->model->getDeviceParticles(), h->model->getNumParticles(), h->gravity,
                                       h->dt);
  h->container->resolveCollisions(h->model->getDeviceParticles());
  h->model->resolveCollisions();
}
}  // namespace

extern "C" {

// Returns nullptr when a particle lies outside the grid domain.
void* refc_create(const double* aos, int64_t n, const double box_min[3], const double box_max[3],
                  const char* obj_path, const double gravity[3], const double e_wall[6], double k_spring,
                  double e_sphere, double dt) {
  auto* h = new RefCuda();
  for (int64_t i = 0; i < n; ++i) {
    const double* q = aos + 8 * i;
    h->particles.push_back(std::make_shared<Particle>(glm::dvec3(q[0], q[1], q[2]), glm::dvec3(q[3], q[4], q[5]),
                                                      q[6], q[7]));
  }
  const CoefficientOfRestitutionWall ew(e_wall[0], e_wall[1], e_wall[2], e_wall[3], e_wall[4], e_wall[5]);
  h->model = std::make_shared<ParticleModelCUDA>(h->particles, k_spring, e_sphere);
  if (obj_path != nullptr && obj_path[0] != '\0') {
    h->container = std::make_shared<PolygonContainerCUDA>(std::string(obj_path), ew.zMin, n);
  } else {
    h->container = std::make_shared<BoxContainerCUDA>(make_double3(box_min[0], box_min[1], box_min[2]),
                                                      make_double3(box_max[0], box_max[1], box_max[2]), ew, n);
  }
  const double3 lo = h->container->getMinCoords(), hi = h->container->getMaxCoords();
  const bool is_box = (obj_path == nullptr || obj_path[0] == '\0');
  for (int64_t i = 0; i < n; ++i) {
    const double* q = aos + 8 * i;
    // Box: the walls clamp every centre into [min+r, max-r] before the grid
    // is built, which stays in the domain when 2r fits the box.  Mesh: the
    // centre must already lie in the mesh AABB.
    const bool ok = is_box ? (2.0 * q[6] < hi.x - lo.x && 2.0 * q[6] < hi.y - lo.y && 2.0 * q[6] < hi.z - lo.z)
                           : (q[0] >= lo.x && q[0] <= hi.x && q[1] >= lo.y && q[1] <= hi.y && q[2] >= lo.z &&
                              q[2] <= hi.z);
    if (!ok) {
      delete h;
      return nullptr;
    }
  }
  h->model->initBuckets(lo, hi);
  h->gravity = make_double3(gravity[0], gravity[1], gravity[2]);
  h->dt = dt;
  return h;
}

void refc_step(void* hp, int64_t steps) {
  auto* h = static_cast<RefCuda*>(hp);
  for (int64_t s = 0; s < steps; ++s) step_once(h);
}

// Device seconds for `steps` steps, CUDA events on the default stream (every
// reference launcher synchronises the device after its kernel).
double refc_time_steps(void* hp, int64_t steps) {
  auto* h = static_cast<RefCuda*>(hp);
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  cudaDeviceSynchronize();
  cudaEventRecord(a);
  for (int64_t s = 0; s < steps; ++s) step_once(h);
  cudaEventRecord(b);
  cudaEventSynchronize(b);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return 1e-3 * (double)ms;
}

void refc_get_state(void* hp, double* out) {
  auto* h = static_cast<RefCuda*>(hp);
  ParticleCUDA* p = h->model->getParticles();
  for (int64_t i = 0; i < h->model->getNumParticles(); ++i) {
    double* q = out + 8 * i;
    q[0] = p[i].position.x;
    q[1] = p[i].position.y;
    q[2] = p[i].position.z;
    q[3] = p[i].velocity.x;
    q[4] = p[i].velocity.y;
    q[5] = p[i].velocity.z;
    q[6] = p[i].radius;
    q[7] = p[i].mass;
  }
  delete[] p;
}

// Grid chosen by ParticleModelCUDA::initBuckets: nb[3], interval, min[3].
void refc_get_grid(void* hp, int32_t nb[3], double* interval, double dmin[3]) {
  auto* h = static_cast<RefCuda*>(hp);
  const BucketContext& b = h->model->_bucketContext;
  nb[0] = b.nBuckets.x;
  nb[1] = b.nBuckets.y;
  nb[2] = b.nBuckets.z;
  *interval = b.interval;
  dmin[0] = b.minCoords.x;
  dmin[1] = b.minCoords.y;
  dmin[2] = b.minCoords.z;
}

// Bucket arrays left by the last step's updateBuckets
// (ParticleModelCUDA.cpp:115-155): per-cell counts, exclusive offsets and
// the particle index list.
void refc_get_buckets(void* hp, uint32_t* counts, uint32_t* offsets, int64_t* bucket) {
  auto* h = static_cast<RefCuda*>(hp);
  const BucketContext& b = h->model->_bucketContext;
  const int64_t c = (int64_t)b.nBuckets.x * b.nBuckets.y * b.nBuckets.z;
  cudaMemcpy(counts, h->model->_deviceBucketCounter, sizeof(uint32_t) * c, cudaMemcpyDeviceToHost);
  cudaMemcpy(offsets, h->model->_deviceBucketCumsumCounter, sizeof(uint32_t) * c, cudaMemcpyDeviceToHost);
  cudaMemcpy(bucket, h->model->_deviceBucket, sizeof(int64_t) * h->model->getNumParticles(),
             cudaMemcpyDeviceToHost);
}

void refc_destroy(void* hp) { delete static_cast<RefCuda*>(hp); }

}  // extern "C"
