// ps_runsimulate.hpp — the reference's own C++ entry point, exported by
// libparticle_stabilizer_cuda.so with the exact signature of
// include/ParticleStabilizerCUDA/PhysicsEngineCUDA.hpp:43-54 (defined in
// src/ParticleStabilizerCUDA/PhysicsEngineCUDA.cpp:86-175), so the
// reference's CLI can dlopen("./libparticle_stabilizer_cuda.so") and call
// dlsym("runSimulateCUDA") unchanged (src/App/ParticleStabilizerMain.cpp:24-35,235-256).
//
// The symbol has C linkage but C++ argument types.  The types below are
// layout-compatible with the reference's: glm::dvec3 is three doubles and
// trivially copyable; ParticlePrimitive<glm::dvec3> is {position, velocity,
// radius, mass} = 64 bytes; CoefficientOfRestitutionWall is six doubles in
// the order zMin, zMax, xMin, xMax, yMin, yMax.  Both sides must use the
// same C++ standard library ABI (libstdc++, _GLIBCXX_USE_CXX11_ABI=1).
#pragma once

#include <cstddef>
#include <memory>
#include <string>
#include <vector>

namespace psb_compat {

struct dvec3 {
  double x, y, z;
};

template <class Vector3>
struct ParticlePrimitive {
  Vector3 position;
  Vector3 velocity;
  double radius;
  double mass;
};

using Particle = ParticlePrimitive<dvec3>;
using ParticlePtr = std::shared_ptr<Particle>;

struct CoefficientOfRestitutionWall {
  double zMin, zMax, xMin, xMax, yMin, yMax;
};

static_assert(sizeof(dvec3) == 24, "glm::dvec3 layout");
static_assert(sizeof(Particle) == 64, "ParticlePrimitive<glm::dvec3> layout");
static_assert(sizeof(CoefficientOfRestitutionWall) == 48, "CoefficientOfRestitutionWall layout");

}  // namespace psb_compat

// Runs maxSteps steps of the scene and fills `resultParticles` (pre-sized by
// the caller) in input order.  Logs the reference's bucket, statistics and
// timing lines.  On any failure it logs a CRITICAL line and calls
// exit(EXIT_FAILURE), as the reference's CUDA_CHECK_ERROR does.
// Precision is FP64 (the reference's) unless the environment variable
// PSB200_PRECISION=fp32.  `toVisualize` is accepted and ignored with a
// warning: no graphics stack exists on the target machines.
extern "C" void runSimulateCUDA(const std::vector<psb_compat::ParticlePtr>& particles, const psb_compat::dvec3 boxMin,
                                const psb_compat::dvec3 boxMax, const std::string containerPath,
                                const psb_compat::dvec3 gravity,
                                const psb_compat::CoefficientOfRestitutionWall coefficientOfRestitutionWall,
                                const double coefficientOfSpring, const double coefficientOfRestitutionSphere,
                                const double dt, const size_t maxSteps, const bool toVisualize,
                                std::vector<psb_compat::Particle>& resultParticles);
