// ref_main_stubs.cpp — link stubs for the reference's own command line.
//
// TEST INFRASTRUCTURE.  oracle/Makefile links the unmodified
// src/App/ParticleStabilizerMain.cpp and src/ParticleStabilizer/
// DynamicLoader.cpp with the reference's CPU sources into oracle/_ref/
// ref_main, so a test can run the reference's `main` with --cuda against
// this repository's libparticle_stabilizer_cuda.so, loaded by the
// reference's own dlopen("./libparticle_stabilizer_cuda.so") and
// dlsym("runSimulateCUDA") (ParticleStabilizerMain.cpp:235-256,
// DynamicLoader.cpp:5-46).
//
// The CPU simulator runSimulate (src/ParticleStabilizer/PhysicsEngine.cpp)
// also drives the viewer, whose submodule is absent and which has no
// graphics stack to run on here; it is replaced by this stub, so the binary
// serves the --cuda path only.
#include <cstdio>
#include <cstdlib>

#include <ParticleStabilizer/PhysicsEngine.hpp>

void runSimulate(const std::vector<ParticlePtr>&, const glm::dvec3, const glm::dvec3, const std::string,
                 const glm::dvec3, const CoefficientOfRestitutionWall, const double, const double, const double,
                 const size_t, const bool, std::vector<Particle>&) {
  std::fprintf(stderr, "ref_main: built for the --cuda path only\n");
  std::exit(2);
}
