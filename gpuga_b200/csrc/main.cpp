// gpuga: command-line driver with the reference's interface (main.cu:25-80).
// stdin: the number of input directories, then the directories.  For each one
// it fits the potential with the GA of <dir>/ga.in and writes ga.out,
// force.out, energy.out and virial.out there.
//   gpuga [--seed S] [--path batched|plain64|plain32] [--device D] [--host-loop]
//         [--ri-self-energy] [--nn2b-consistent] [--nn2b-taper R1 R2] [--neighbor-cells 0|1|2] < input.txt
// The options map onto gpuga_options and gpuga_ga_set_device_loop; without them the run keeps
// the reference's semantics.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "../../include/gpuga.h"

int main(int argc, char** argv) {
  gpuga_options opt;
  gpuga_default_options(&opt);
  opt.verbose = 1;
  unsigned seed = 12345678u;  // the reference's -DDEBUG seed (ga.cu:47-48)
  int device_loop = 1;
  const char* usage =
      "usage: %s [--seed S] [--device D] [--path batched|plain64|plain32] [--host-loop] [--ri-self-energy]\n"
      "          [--nn2b-consistent] [--nn2b-taper R1 R2] [--neighbor-cells 0|1|2] < input.txt\n";
  for (int i = 1; i < argc; ++i) {
    if (!strcmp(argv[i], "--seed") && i + 1 < argc) {
      seed = (unsigned)strtoul(argv[++i], nullptr, 0);
    } else if (!strcmp(argv[i], "--device") && i + 1 < argc) {
      opt.device = atoi(argv[++i]);
    } else if (!strcmp(argv[i], "--path") && i + 1 < argc) {
      const char* p = argv[++i];
      opt.path = !strcmp(p, "plain64") ? GPUGA_PATH_PLAIN64 : (!strcmp(p, "plain32") ? GPUGA_PATH_PLAIN32 : GPUGA_PATH_BATCHED);
    } else if (!strcmp(argv[i], "--host-loop")) {
      device_loop = 0;
    } else if (!strcmp(argv[i], "--ri-self-energy")) {
      opt.ri_self_energy = 1;
    } else if (!strcmp(argv[i], "--nn2b-consistent")) {
      opt.nn2b_consistent = 1;
    } else if (!strcmp(argv[i], "--nn2b-taper") && i + 2 < argc) {
      opt.nn2b_r1 = (float)atof(argv[++i]);
      opt.nn2b_r2 = (float)atof(argv[++i]);
    } else if (!strcmp(argv[i], "--neighbor-cells") && i + 1 < argc) {
      opt.neighbor_cells = atoi(argv[++i]);
    } else {
      fprintf(stderr, usage, argv[0]);
      return 2;
    }
  }
  printf("\n***************************************************************\n");
  printf("*     GPUGA fitness engine for B200 (%s)                *\n", gpuga_version());
  printf("***************************************************************\n\n");
  int n_inputs = 0;
  if (scanf("%d", &n_inputs) != 1) {
    fprintf(stderr, "Error: reading error for number of inputs.\n");
    return 1;
  }
  for (int n = 0; n < n_inputs; ++n) {
    char dir[4096];
    if (scanf("%4095s", dir) != 1) {
      fprintf(stderr, "Error: reading error for input directory.\n");
      return 1;
    }
    printf("Run simulation for '%s'.\n", dir);
    auto t0 = std::chrono::steady_clock::now();
    gpuga_engine* e = nullptr;
    gpuga_ga* g = nullptr;
    int s = gpuga_engine_create(dir, &opt, &e);
    if (s == GPUGA_OK) s = gpuga_ga_create(e, dir, seed, &g);
    if (s == GPUGA_OK && !device_loop) s = gpuga_ga_set_device_loop(g, 0, 0);
    if (s == GPUGA_OK) s = gpuga_ga_run(g, dir);
    if (s != GPUGA_OK) {
      fprintf(stderr, "Error: %s\n", gpuga_last_error());
      gpuga_ga_destroy(g);
      gpuga_engine_destroy(e);
      return 1;
    }
    gpuga_ga_destroy(g);
    gpuga_engine_destroy(e);
    double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    printf("Time used for '%s' = %f s.\n", dir, secs);
  }
  printf("Finished running gpuga.\n");
  return 0;
}
