// ps_main.cpp — particle_stabilizer_main, the reference's command line
// (src/App/ParticleStabilizerMain.cpp:40-301) over the B200 library.
//
// Same flags, defaults and file formats.  Like the reference's --cuda path it
// loads ./libparticle_stabilizer_cuda.so with dlopen and calls its
// runSimulateCUDA symbol (ParticleStabilizerMain.cpp:19-21,235-256).  The
// reference's CPU simulator is not part of this program: the B200 path runs
// whether or not --cuda is given.  Extra flags: --fp32 (single precision),
// --cell-size S, --widen-domain, --lib PATH, and --dump-state /
// --resume-state (a binary file with every particle record and the step
// count, which the reference's CSV cannot give).  --visualize has no graphics
// stack to open and is reported and skipped.  After the run, as the
// reference (ParticleStabilizerMain.cpp:274-296): --resolve-overlap-axis
// (ps_resolve_overlaps), then the CSV, then --out-obj-path
// (ps_write_obj_spheres).
#include <dlfcn.h>

#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <string>
#include <vector>

#include "particle_stabilizer_b200.h"
#include "ps_runsimulate.hpp"

using namespace psb_compat;

using runSimulateCUDA_t = void (*)(const std::vector<ParticlePtr>&, const dvec3, const dvec3, const std::string,
                                   const dvec3, const CoefficientOfRestitutionWall, const double, const double,
                                   const double, const size_t, const bool, std::vector<Particle>&);
using read_csv_t = int (*)(const char*, const double*, double, double*, int64_t, int64_t*);
using write_csv_t = int (*)(const char*, const double*, int64_t);
using resolve_t = int (*)(double*, int64_t, int32_t, int64_t*, double*);
using write_obj_t = int (*)(const char*, const double*, int64_t);
using last_error_t = const char* (*)();
using write_state_t = int (*)(const char*, const double*, int64_t, int64_t);
using read_state_t = int (*)(const char*, double*, int64_t, int64_t*, int64_t*);

namespace {

struct Args {
  std::string particleFilePath, objOutPath, particleOutPath, containerPath, libPath = "./libparticle_stabilizer_cuda.so";
  std::string dumpStatePath, resumeStatePath;  // binary state files (checkpoint / resume)
  dvec3 initialVelocity{0.0, 0.0, -10.0};
  double density = 1.0;
  CoefficientOfRestitutionWall e_wall{0.5, 0.5, 0.5, 0.5, 0.5, 0.5};
  double k = 1.0, e_sphere = 0.1;
  dvec3 gravity{0.0, 0.0, -10.0}, boxMin{0.0, 0.0, 0.0}, boxMax{10.0, 20.0, 30.0};
  double dt = 0.00001, cellSize = 0.0;
  bool toVisualize = false, toUseCUDA = false, fp32 = false, widen = false;
  int64_t maxSteps = 100000;
  int resolveOverlapAxis = -1;
};

void usage() {
  std::cout << "particle_stabilizer_main (B200) — a simulator for particle dynamics in a container\n"
               "usage: ./particle_stabilizer_main [Options] particleFilePath\n"
               "  -h                                             show this help\n"
               "  --cuda                                         accepted (the B200 path always runs)\n"
               "  --initial-velocity X Y Z  --density MASS\n"
               "  --coeff-of-restitution-wall Z_MIN Z_MAX X_MIN X_MAX Y_MIN Y_MAX\n"
               "  --coeff-of-spring SPRING  --coeff-of-restitution-sphere E  --gravity X Y Z\n"
               "  --dt DT  --max-steps N  --box-min X Y Z  --box-max X Y Z  --container OBJ\n"
               "  --out-csv-path CSV  --out-obj-path OBJ  --resolve-overlap-axis AXIS  --visualize\n"
               "  --fp32  --cell-size S  --widen-domain  --lib PATH\n"
               "  --dump-state BIN    after the run, write every particle record and the step count\n"
               "  --resume-state BIN  start from a dumped state (the particle file is then optional)\n";
}

bool parse(int argc, char** argv, Args& a) {
  if (argc < 2) return false;
  auto need = [&](int& i, int k) {
    if (i + k >= argc) {
      std::cerr << "missing value for " << argv[i] << "\n";
      std::exit(EXIT_FAILURE);
    }
  };
  for (int i = 1; i < argc; ++i) {
    const std::string s = argv[i];
    if (s == "-h") return false;
    if (s == "--out-obj-path") { need(i, 1); a.objOutPath = argv[++i]; }
    else if (s == "--out-csv-path") { need(i, 1); a.particleOutPath = argv[++i]; }
    else if (s == "--initial-velocity") { need(i, 3); a.initialVelocity = {std::stod(argv[i + 1]), std::stod(argv[i + 2]), std::stod(argv[i + 3])}; i += 3; }
    else if (s == "--density") { need(i, 1); a.density = std::stod(argv[++i]); }
    else if (s == "--coeff-of-restitution-wall") {
      need(i, 6);
      a.e_wall = {std::stod(argv[i + 1]), std::stod(argv[i + 2]), std::stod(argv[i + 3]),
                  std::stod(argv[i + 4]), std::stod(argv[i + 5]), std::stod(argv[i + 6])};
      i += 6;
    }
    else if (s == "--coeff-of-spring") { need(i, 1); a.k = std::stod(argv[++i]); }
    else if (s == "--coeff-of-restitution-sphere") { need(i, 1); a.e_sphere = std::stod(argv[++i]); }
    else if (s == "--gravity") { need(i, 3); a.gravity = {std::stod(argv[i + 1]), std::stod(argv[i + 2]), std::stod(argv[i + 3])}; i += 3; }
    else if (s == "--box-min") { need(i, 3); a.boxMin = {std::stod(argv[i + 1]), std::stod(argv[i + 2]), std::stod(argv[i + 3])}; i += 3; }
    else if (s == "--box-max") { need(i, 3); a.boxMax = {std::stod(argv[i + 1]), std::stod(argv[i + 2]), std::stod(argv[i + 3])}; i += 3; }
    else if (s == "--container") { need(i, 1); a.containerPath = argv[++i]; }
    else if (s == "--dt") { need(i, 1); a.dt = std::stod(argv[++i]); }
    else if (s == "--visualize") a.toVisualize = true;
    else if (s == "--max-steps") { need(i, 1); a.maxSteps = std::stoll(argv[++i]); }
    else if (s == "--resolve-overlap-axis") { need(i, 1); a.resolveOverlapAxis = std::stoi(argv[++i]); }
    else if (s == "--cuda") a.toUseCUDA = true;
    else if (s == "--fp32") a.fp32 = true;
    else if (s == "--cell-size") { need(i, 1); a.cellSize = std::stod(argv[++i]); }
    else if (s == "--widen-domain") a.widen = true;
    else if (s == "--lib") { need(i, 1); a.libPath = argv[++i]; }
    else if (s == "--dump-state") { need(i, 1); a.dumpStatePath = argv[++i]; }
    else if (s == "--resume-state") { need(i, 1); a.resumeStatePath = argv[++i]; }
    else a.particleFilePath = s;
  }
  return !a.particleFilePath.empty() || !a.resumeStatePath.empty();
}

}  // namespace

int main(int argc, char** argv) {
  Args a;
  if (!parse(argc, argv, a)) {
    usage();
    return EXIT_SUCCESS;
  }
  if (a.fp32) setenv("PSB200_PRECISION", "fp32", 1);
  if (a.widen) setenv("PSB200_WIDEN_DOMAIN", "1", 1);
  if (a.cellSize > 0) {  // all 17 digits, so the library reads back the same double
    char buf[32];
    std::snprintf(buf, sizeof buf, "%.17g", a.cellSize);
    setenv("PSB200_CELL_SIZE", buf, 1);
  }

  void* h = dlopen(a.libPath.c_str(), RTLD_LAZY);
  if (h == nullptr) {
    std::cerr << "Cannot open library: " << dlerror() << "\n";
    return EXIT_FAILURE;
  }
  auto run = reinterpret_cast<runSimulateCUDA_t>(dlsym(h, "runSimulateCUDA"));
  auto read_csv = reinterpret_cast<read_csv_t>(dlsym(h, "ps_read_csv"));
  auto write_csv = reinterpret_cast<write_csv_t>(dlsym(h, "ps_write_csv"));
  auto last_error = reinterpret_cast<last_error_t>(dlsym(h, "ps_last_error"));
  auto resolve = reinterpret_cast<resolve_t>(dlsym(h, "ps_resolve_overlaps"));
  auto write_obj = reinterpret_cast<write_obj_t>(dlsym(h, "ps_write_obj_spheres"));
  if (!run || !read_csv || !write_csv || !last_error || !resolve || !write_obj) {
    std::cerr << "Cannot load symbol: 'runSimulateCUDA' from the shared library.\n";
    return EXIT_FAILURE;
  }
  if (!a.toUseCUDA) std::cout << "[info] this program runs the B200 path (--cuda implied)\n";

  auto write_state = reinterpret_cast<write_state_t>(dlsym(h, "ps_write_state_bin"));
  auto read_state = reinterpret_cast<read_state_t>(dlsym(h, "ps_read_state_bin"));
  if ((!a.dumpStatePath.empty() || !a.resumeStatePath.empty()) && (!write_state || !read_state)) {
    std::cerr << "Cannot load symbol: 'ps_write_state_bin' from the shared library.\n";
    return EXIT_FAILURE;
  }

  int64_t n = 0, steps_before = 0;
  std::vector<double> aos;
  if (!a.resumeStatePath.empty()) {
    // every record in full (velocities included) and the steps already taken
    if (read_state(a.resumeStatePath.c_str(), nullptr, 0, &n, &steps_before) != PS_OK) {
      std::cerr << "[critical] " << last_error() << "\n";
      return EXIT_FAILURE;
    }
    aos.resize((size_t)(8 * n));
    read_state(a.resumeStatePath.c_str(), aos.data(), n, &n, &steps_before);
    std::cout << "[info] Resumed " << n << " particles after " << steps_before << " steps from file: "
              << a.resumeStatePath << "\n";
  } else {
    // ParticleData::readFromCSV (ParticleIO.cpp:90-144)
    const double vel[3] = {a.initialVelocity.x, a.initialVelocity.y, a.initialVelocity.z};
    if (read_csv(a.particleFilePath.c_str(), vel, a.density, nullptr, 0, &n) != PS_OK) {
      std::cerr << "[critical] " << last_error() << "\n";
      return EXIT_FAILURE;
    }
    aos.resize((size_t)(8 * n));
    read_csv(a.particleFilePath.c_str(), vel, a.density, aos.data(), n, &n);
    std::cout << "[info] Read " << n << " particles from file: " << a.particleFilePath << "\n";
  }

  std::vector<ParticlePtr> particles;
  particles.reserve((size_t)n);
  for (int64_t i = 0; i < n; ++i) {
    const double* q = aos.data() + 8 * i;
    particles.push_back(std::make_shared<Particle>(Particle{{q[0], q[1], q[2]}, {q[3], q[4], q[5]}, q[6], q[7]}));
  }
  std::vector<Particle> result((size_t)n);
  run(particles, a.boxMin, a.boxMax, a.containerPath, a.gravity, a.e_wall, a.k, a.e_sphere, a.dt, (size_t)a.maxSteps,
      a.toVisualize, result);

  for (int64_t i = 0; i < n; ++i) {
    double* q = aos.data() + 8 * i;
    const Particle& p = result[(size_t)i];
    q[0] = p.position.x; q[1] = p.position.y; q[2] = p.position.z;
    q[3] = p.velocity.x; q[4] = p.velocity.y; q[5] = p.velocity.z;
    q[6] = p.radius; q[7] = p.mass;
  }
  if (!a.dumpStatePath.empty()) {  // before any post-processing: the state a resumed run continues from
    const int64_t steps = steps_before + (a.maxSteps == 0 ? 1 : a.maxSteps);  // the loop takes at least one step
    if (write_state(a.dumpStatePath.c_str(), aos.data(), n, steps) != PS_OK) {
      std::cerr << "[error] " << last_error() << "\n";
      return EXIT_FAILURE;
    }
    std::cout << "[info] Wrote the state after " << steps << " steps to file " << a.dumpStatePath << "\n";
  }
  if (a.resolveOverlapAxis >= 0) {  // ParticleModel::resolveOverlaps (ParticleModel.cpp:154-259)
    std::cout << "[info] ### Resolving overlaps\n";
    int64_t n_collided = 0;
    double max_overlap = 0.0;
    if (resolve(aos.data(), n, a.resolveOverlapAxis, &n_collided, &max_overlap) != PS_OK) {
      std::cerr << "[error] " << last_error() << "\n";
      return EXIT_FAILURE;
    }
    char line[128];
    std::snprintf(line, sizeof(line), "Max collision distance: %.15lf", max_overlap);
    std::cout << "[info] Number of collided particles: " << n_collided << " / " << n << "\n"
              << "[info] " << line << "\n[info] ### Finished resolving overlaps\n";
  }
  if (!a.particleOutPath.empty()) {
    if (write_csv(a.particleOutPath.c_str(), aos.data(), n) != PS_OK) {
      std::cerr << "[error] " << last_error() << "\n";
      return EXIT_FAILURE;
    }
    std::cout << "[info] Finished writing to file " << a.particleOutPath << "\n";
  }
  if (!a.objOutPath.empty()) {  // ObjData::write (ObjData.cpp:8-140)
    std::cout << "[info] Writing to file " << a.objOutPath << "\n";
    if (write_obj(a.objOutPath.c_str(), aos.data(), n) != PS_OK) {
      std::cerr << "[error] " << last_error() << "\n";
      return EXIT_FAILURE;
    }
    std::cout << "[info] Finished writing to file " << a.objOutPath << "\n";
  }
  std::cout << "[info] Simulation completed successfully.\n";
  return EXIT_SUCCESS;
}
