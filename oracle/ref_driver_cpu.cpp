// ref_driver_cpu.cpp — harness around the reference's own CPU simulator.
//
// TEST INFRASTRUCTURE.  Linked with the unmodified reference sources
// (src/ParticleStabilizer/{ParticleModel,ParticleBucket,BoxContainer,
// PolygonContainer,ParticleIO}.cpp) into oracle/_ref/libref_cpu.so.  It
// drives the per-step body of PhysicsEngine::startSimulationLoop
// (src/ParticleStabilizer/PhysicsEngine.cpp:38-48) without the O(N^2)
// statistics block, and exposes the reference's CSV reader/writer and the
// CLI's post-processing (ParticleModel::resolveOverlaps, ObjData::write).
#include <ParticleStabilizer/BoxContainer.hpp>
#include <ParticleStabilizer/ObjData.hpp>
#include <ParticleStabilizer/ParticleIO.hpp>
#include <ParticleStabilizer/ParticleModel.hpp>
#include <ParticleStabilizer/PolygonContainer.hpp>

#include <chrono>
#include <cstdint>
#include <memory>
#include <string>
#include <vector>

namespace {
struct RefCpu {
  std::vector<ParticlePtr> particles;
  std::shared_ptr<ParticleModel> model;
  std::shared_ptr<ContainerBase> container;
  glm::dvec3 gravity;
  double dt = 0.0;
};

void step_once(RefCpu* h) {
  {
    // PhysicsEngine::updatePositionAndVelocity (PhysicsEngine.cpp:19-26)
    const auto& particles = h->model->getParticles();
    for (auto& particle : particles) {
      particle->position += particle->velocity * h->dt;
      particle->velocity += h->gravity * h->dt;
    }
  }
  h->model->updateBuckets();
  auto particles = h->model->getParticles();
  h->container->resolveCollisions(particles);
  h->model->resolveCollisions();
}
}  // namespace

extern "C" {

void* refh_create(const double* aos, int64_t n, const double box_min[3], const double box_max[3],
                  const char* obj_path, const double gravity[3], const double e_wall[6], double k_spring,
                  double e_sphere, double dt) {
  auto* h = new RefCpu();
  h->particles.reserve((size_t)n);
  for (int64_t i = 0; i < n; ++i) {
    const double* q = aos + 8 * i;
    h->particles.push_back(std::make_shared<Particle>(glm::dvec3(q[0], q[1], q[2]), glm::dvec3(q[3], q[4], q[5]),
                                                      q[6], q[7]));
  }
  const CoefficientOfRestitutionWall ew(e_wall[0], e_wall[1], e_wall[2], e_wall[3], e_wall[4], e_wall[5]);
  h->model = std::make_shared<ParticleModel>(h->particles, k_spring, e_sphere);
  if (obj_path != nullptr && obj_path[0] != '\0') {
    h->container = std::make_shared<PolygonContainer>(std::string(obj_path), ew.zMin, (size_t)n);
  } else {
    h->container = std::make_shared<BoxContainer>(glm::dvec3(box_min[0], box_min[1], box_min[2]),
                                                  glm::dvec3(box_max[0], box_max[1], box_max[2]), ew);
  }
  h->model->initBuckets(h->container->getMinCoords(), h->container->getMaxCoords());
  h->gravity = glm::dvec3(gravity[0], gravity[1], gravity[2]);
  h->dt = dt;
  return h;
}

void refh_step(void* hp, int64_t steps) {
  auto* h = static_cast<RefCpu*>(hp);
  for (int64_t s = 0; s < steps; ++s) step_once(h);
}

// Wall-clock seconds for `steps` steps (std::chrono::steady_clock).
double refh_time_steps(void* hp, int64_t steps) {
  auto* h = static_cast<RefCpu*>(hp);
  const auto t0 = std::chrono::steady_clock::now();
  for (int64_t s = 0; s < steps; ++s) step_once(h);
  const auto t1 = std::chrono::steady_clock::now();
  return std::chrono::duration<double>(t1 - t0).count();
}

void refh_get_state(void* hp, double* out) {
  auto* h = static_cast<RefCpu*>(hp);
  const auto particles = h->model->getParticles();
  for (size_t i = 0; i < particles.size(); ++i) {
    double* q = out + 8 * i;
    q[0] = particles[i]->position.x;
    q[1] = particles[i]->position.y;
    q[2] = particles[i]->position.z;
    q[3] = particles[i]->velocity.x;
    q[4] = particles[i]->velocity.y;
    q[5] = particles[i]->velocity.z;
    q[6] = particles[i]->radius;
    q[7] = particles[i]->mass;
  }
}

void refh_destroy(void* hp) { delete static_cast<RefCpu*>(hp); }

// ParticleData::readFromCSV (ParticleIO.cpp:90-144).  Returns the number of
// particles read; fills at most `cap` rows of `out`.
int64_t refh_read_csv(const char* path, const double vel[3], double density, double* out, int64_t cap) {
  ParticleData data = ParticleData::readFromCSV(std::string(path), glm::dvec3(vel[0], vel[1], vel[2]), density);
  const int64_t n = (int64_t)data.particles.size();
  for (int64_t i = 0; i < n && i < cap; ++i) {
    const auto& p = data.particles[(size_t)i];
    double* q = out + 8 * i;
    q[0] = p->position.x;
    q[1] = p->position.y;
    q[2] = p->position.z;
    q[3] = p->velocity.x;
    q[4] = p->velocity.y;
    q[5] = p->velocity.z;
    q[6] = p->radius;
    q[7] = p->mass;
  }
  return n;
}

// ParticleData::writeAsCSV (ParticleIO.cpp:58-88).
void refh_write_csv(const double* aos, int64_t n, const char* path) {
  std::vector<ParticlePtr> v;
  for (int64_t i = 0; i < n; ++i) {
    const double* q = aos + 8 * i;
    v.push_back(std::make_shared<Particle>(glm::dvec3(q[0], q[1], q[2]), glm::dvec3(q[3], q[4], q[5]), q[6], q[7]));
  }
  ParticleData data(v);
  data.writeAsCSV(std::string(path));
}

// PolygonContainer::readFromFile (PolygonContainer.cpp:381-417) followed by
// the de-indexing of the constructor: 9 doubles per triangle.
int64_t refh_read_obj(const char* path, double* tri_out, int64_t cap) {
  std::vector<glm::dvec3> vertices;
  std::vector<int64_t> indices;
  PolygonContainer::readFromFile(std::string(path), vertices, indices);
  const int64_t n_tri = (int64_t)(indices.size() / 3);
  for (int64_t t = 0; t < n_tri && t < cap; ++t) {
    for (int c = 0; c < 3; ++c) {
      const glm::dvec3& v = vertices[(size_t)indices[(size_t)(3 * t + c)]];
      tri_out[9 * t + 3 * c + 0] = v.x;
      tri_out[9 * t + 3 * c + 1] = v.y;
      tri_out[9 * t + 3 * c + 2] = v.z;
    }
  }
  return n_tri;
}

namespace {
std::vector<Particle> records_to_particles(const double* aos, int64_t n) {
  std::vector<Particle> v;
  v.reserve((size_t)n);
  for (int64_t i = 0; i < n; ++i) {
    const double* q = aos + 8 * i;
    v.emplace_back(glm::dvec3(q[0], q[1], q[2]), glm::dvec3(q[3], q[4], q[5]), q[6], q[7]);
  }
  return v;
}
}  // namespace

// ParticleModel::resolveOverlaps (ParticleModel.cpp:154-259); positions
// written back into aos.
void refh_resolve_overlaps(double* aos, int64_t n, int32_t axis) {
  std::vector<Particle> v = records_to_particles(aos, n);
  ParticleModel::resolveOverlaps(v, axis);
  for (int64_t i = 0; i < n; ++i) {
    aos[8 * i + 0] = v[(size_t)i].position.x;
    aos[8 * i + 1] = v[(size_t)i].position.y;
    aos[8 * i + 2] = v[(size_t)i].position.z;
  }
}

// ObjData::write (ObjData.cpp:8-140).
void refh_write_obj(const char* path, const double* aos, int64_t n) {
  ObjData::write(std::string(path), records_to_particles(aos, n));
}

}  // extern "C"
