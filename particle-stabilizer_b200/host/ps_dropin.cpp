// ps_dropin.cpp — runSimulateCUDA, the reference's own entry point
// (src/ParticleStabilizerCUDA/PhysicsEngineCUDA.cpp:86-175), over the C ABI.
//
// Same arguments, same behaviour visible to the caller: builds the scene,
// logs the bucket grid, runs maxSteps steps with a statistics block every
// 10 s of wall time and at the last step (PhysicsEngineCUDA.cpp:45-71), then
// fills resultParticles in input order.  Failures are logged at CRITICAL and
// end the process with exit(EXIT_FAILURE), as CUDA_CHECK_ERROR does
// (include/ParticleStabilizerCUDA/CudaCommon.cuh:18-28).  Statistics come from
// the grid (ps_stats_get) instead of the reference's host O(N^2) loop.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <ctime>
#include <string>
#include <vector>

#include "particle_stabilizer_b200.h"
#include "ps_runsimulate.hpp"

// defined in ps_engine.cu: records the message returned by ps_last_error()
extern "C" int ps_internal_fail(int code, const char* msg);

namespace {

void log_line(const char* level, const std::string& msg) {
  const std::time_t t = std::time(nullptr);
  char ts[32];
  std::strftime(ts, sizeof(ts), "%Y-%m-%d %H:%M:%S", std::localtime(&t));
  std::printf("[%s] [%s] %s\n", ts, level, msg.c_str());
  std::fflush(stdout);
}

[[noreturn]] void die(const std::string& what) {
  log_line("critical", what + ": " + ps_last_error());
  std::exit(EXIT_FAILURE);
}

void check(int rc, const char* what) {
  if (rc != PS_OK) die(what);
}

std::string d2s(double v) { return std::to_string(v); }

void log_stats(ps_sim* sim, int64_t step, double elapsed, int64_t n) {
  ps_stats st;
  check(ps_stats_get(sim, 0, &st), "statistics");
  log_line("info", "######################## Step " + std::to_string(step) + ", Elapsed time: " + d2s(elapsed) +
                       " [sec] ########################");
  log_line("info", "Total kinetic energy         : " + d2s(st.kinetic_energy));
  log_line("info", "Max position                 : (" + d2s(st.max_pos[0]) + ", " + d2s(st.max_pos[1]) + ", " +
                       d2s(st.max_pos[2]) + ")");
  log_line("info", "Min position                 : (" + d2s(st.min_pos[0]) + ", " + d2s(st.min_pos[1]) + ", " +
                       d2s(st.min_pos[2]) + ")");
  log_line("info", "Number of collided particles : " + std::to_string(st.n_collided) + " / " + std::to_string(n));
  log_line("info", "Max collision distance       : " + d2s(st.max_overlap));
}

}  // namespace

extern "C" void runSimulateCUDA(const std::vector<psb_compat::ParticlePtr>& particles, const psb_compat::dvec3 boxMin,
                                const psb_compat::dvec3 boxMax, const std::string containerPath,
                                const psb_compat::dvec3 gravity,
                                const psb_compat::CoefficientOfRestitutionWall e_wall, const double coefficientOfSpring,
                                const double coefficientOfRestitutionSphere, const double dt, const size_t maxSteps,
                                const bool toVisualize, std::vector<psb_compat::Particle>& resultParticles) {
  const int64_t n = (int64_t)particles.size();
  const char* prec_env = std::getenv("PSB200_PRECISION");
  const int precision = (prec_env != nullptr && std::string(prec_env) == "fp32") ? PS_FP32 : PS_FP64;
  if (toVisualize) log_line("warning", "--visualize is not available (no graphics stack); running headless");

  ps_scene_desc d{};
  d.n_particles = n;
  d.box_min[0] = boxMin.x;
  d.box_min[1] = boxMin.y;
  d.box_min[2] = boxMin.z;
  d.box_max[0] = boxMax.x;
  d.box_max[1] = boxMax.y;
  d.box_max[2] = boxMax.z;
  d.gravity[0] = gravity.x;
  d.gravity[1] = gravity.y;
  d.gravity[2] = gravity.z;
  d.e_wall[PS_ZMIN] = e_wall.zMin;
  d.e_wall[PS_ZMAX] = e_wall.zMax;
  d.e_wall[PS_XMIN] = e_wall.xMin;
  d.e_wall[PS_XMAX] = e_wall.xMax;
  d.e_wall[PS_YMIN] = e_wall.yMin;
  d.e_wall[PS_YMAX] = e_wall.yMax;
  d.k_spring = coefficientOfSpring;
  d.e_sphere = coefficientOfRestitutionSphere;
  d.dt = dt;
  d.edge_quirk = 1;
  if (const char* w = std::getenv("PSB200_WIDEN_DOMAIN")) d.widen_domain = std::atoi(w) != 0;
  if (const char* c = std::getenv("PSB200_CELL_SIZE")) d.cell_size = std::atof(c);

  std::vector<double> tri;
  if (!containerPath.empty()) {
    int64_t nt = 0;
    check(ps_read_obj(containerPath.c_str(), nullptr, 0, &nt), "reading the container");
    if (nt == 0) {
      ps_internal_fail(PS_ERR_IO, ("no triangles in " + containerPath).c_str());
      die("reading the container");
    }
    tri.resize((size_t)(9 * nt));
    check(ps_read_obj(containerPath.c_str(), tri.data(), nt, &nt), "reading the container");
    d.tri = tri.data();
    d.n_tri = nt;
    log_line("info", "nPolygons = " + std::to_string(nt));
  }

  std::vector<double> aos((size_t)(8 * n));
  for (int64_t i = 0; i < n; ++i) {
    const psb_compat::Particle& p = *particles[(size_t)i];
    double* q = aos.data() + 8 * i;
    q[0] = p.position.x;
    q[1] = p.position.y;
    q[2] = p.position.z;
    q[3] = p.velocity.x;
    q[4] = p.velocity.y;
    q[5] = p.velocity.z;
    q[6] = p.radius;
    q[7] = p.mass;
  }

  ps_sim* sim = nullptr;
  check(ps_create(&d, 1, precision, 0, &sim), "creating the simulation");
  check(ps_set_state(sim, aos.data(), n), "uploading particles");
  ps_grid_info g;
  check(ps_grid_get(sim, 0, &g), "grid");
  log_line("info", "################################################ Bucket info #################################################");
  log_line("info", "# (minX, minY, minZ)                : (" + d2s(g.min[0]) + ", " + d2s(g.min[1]) + ", " + d2s(g.min[2]) + ")");
  log_line("info", "# (nBucketsX, nBucketsY, nBucketsZ) : (" + std::to_string(g.nb[0]) + ", " + std::to_string(g.nb[1]) + ", " +
                       std::to_string(g.nb[2]) + ")");
  log_line("info", "# interval                          : " + d2s(g.interval));
  log_line("info", "# precision                         : " + std::string(precision == PS_FP32 ? "fp32" : "fp64"));
  // neighbour lists (same results as the grid path): "auto" tunes the skin
  // (about 1,000 trial steps, so only for runs of 10,000 steps or more; a
  // shorter run keeps the grid path), a number sets it (0 keeps the grid path)
  if (const char* nl = std::getenv("PSB200_NEIGHBOR_LISTS")) {
    const std::string mode(nl);
    if (mode == "auto" && maxSteps < 10000) {
      log_line("info", "# neighbour lists (auto)            : off for runs under 10,000 steps");
    } else {
      double skin = 0.0;
      if (mode == "auto") {
        const double skins[] = {0.0, 0.02, 0.05, 0.1, 0.2};
        double ms[5];
        check(ps_tune_neighbor_lists(sim, 100, skins, 5, 64, ms, &skin), "tuning neighbour lists");
      } else {
        skin = std::atof(nl);
        check(ps_set_neighbor_lists(sim, skin, 64), "neighbour lists");
      }
      log_line("info", "# neighbour-list skin (x cell edge) : " + d2s(skin));
    }
  }
  log_line("info", "##############################################################################################################");

  const auto t0 = std::chrono::steady_clock::now();
  auto t_prev = t0;
  int64_t done = 0;
  // the reference's loop runs its body before testing nSteps >= maxSteps,
  // so maxSteps == 0 still takes one step (PhysicsEngineCUDA.cpp:33-76)
  const int64_t total = maxSteps == 0 ? 1 : (int64_t)maxSteps;
  while (done < total) {
    // chunks of steps between wall-clock checks of the 10 s cadence
    const int64_t chunk = std::min<int64_t>(total - done, 2000);
    check(ps_step(sim, chunk), "stepping");
    check(ps_sync(sim), "stepping");
    done += chunk;
    const auto now = std::chrono::steady_clock::now();
    const double since = std::chrono::duration<double>(now - t_prev).count();
    if (since > 10.0 || done == (int64_t)maxSteps) {
      log_stats(sim, done, std::chrono::duration<double>(now - t0).count(), n);
      t_prev = now;
    }
  }
  log_line("info", "Total elapsed time: " + d2s(std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count()) +
                       " [sec]");

  check(ps_get_state(sim, aos.data(), n), "downloading particles");
  ps_destroy(sim);
  resultParticles.resize((size_t)n);
  for (int64_t i = 0; i < n; ++i) {
    const double* q = aos.data() + 8 * i;
    resultParticles[(size_t)i] = psb_compat::Particle{{q[0], q[1], q[2]}, {q[3], q[4], q[5]}, q[6], q[7]};
  }
}
