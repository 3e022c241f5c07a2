/* The C ABI from plain C, as INTEGRATION.md shows it: read n particle
 * records (8 doubles each) from a binary file, advance them n_steps in one
 * box scene (box [0,1]^3, gravity -9.8 in z, walls 0.8, spring 1e4, sphere
 * restitution 0.5, dt 1e-5), write the records back in original order.
 *
 *   step_lattice IN.bin N_STEPS OUT.bin [fp64]
 *
 * Exit status 0 on success; otherwise the library's message on stderr. */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "particle_stabilizer_b200.h"

static int fail(const char* what) {
  fprintf(stderr, "%s: %s\n", what, ps_last_error());
  return 1;
}

int main(int argc, char** argv) {
  if (argc < 4) {
    fprintf(stderr, "usage: %s IN.bin N_STEPS OUT.bin [fp64]\n", argv[0]);
    return 2;
  }
  FILE* f = fopen(argv[1], "rb");
  if (!f) return 2;
  fseek(f, 0, SEEK_END);
  const long bytes = ftell(f);
  fseek(f, 0, SEEK_SET);
  const int64_t n = bytes / (8 * (long)sizeof(double));
  double* particles = malloc((size_t)(n > 0 ? n : 1) * 8 * sizeof(double));
  if (!particles || fread(particles, sizeof(double), (size_t)(8 * n), f) != (size_t)(8 * n)) return 2;
  fclose(f);

  ps_scene_desc d;
  memset(&d, 0, sizeof d);
  d.n_particles = n;
  d.box_max[0] = d.box_max[1] = d.box_max[2] = 1.0;
  d.gravity[2] = -9.8;
  for (int w = 0; w < 6; ++w) d.e_wall[w] = 0.8; /* PS_ZMIN..PS_YMAX */
  d.k_spring = 1e4;
  d.e_sphere = 0.5;
  d.dt = 1e-5;
  d.edge_quirk = 1;

  ps_sim* sim = NULL;
  const int32_t precision = (argc > 4 && strcmp(argv[4], "fp64") == 0) ? PS_FP64 : PS_FP32;
  if (ps_create(&d, 1, precision, /*device*/ 0, &sim) != PS_OK) return fail("ps_create");
  if (ps_set_state(sim, particles, n) != PS_OK) return fail("ps_set_state");
  if (ps_step(sim, atoll(argv[2])) != PS_OK) return fail("ps_step");
  if (ps_get_state(sim, particles, n) != PS_OK) return fail("ps_get_state");
  if (ps_destroy(sim) != PS_OK) return fail("ps_destroy");

  f = fopen(argv[3], "wb");
  if (!f || fwrite(particles, sizeof(double), (size_t)(8 * n), f) != (size_t)(8 * n)) return 2;
  fclose(f);
  free(particles);
  return 0;
}
