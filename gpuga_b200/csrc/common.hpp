// Shared host-side definitions: status handling, the training-set record the
// parsers fill, and CUDA error plumbing.  Errors never exit the process: every
// failure becomes a negative status plus a thread-local message.
#pragma once
#include <cuda_runtime.h>

#include <cstdio>
#include <string>
#include <vector>

#include "../../include/gpuga.h"

namespace gpuga {

void set_error(const char* fmt, ...);
const char* last_error();

// Turns a CUDA error into GPUGA_ERR_CUDA (or _OOM) with file:line in the message.
int cuda_status(cudaError_t e, const char* what, const char* file, int line);

#define GPUGA_CUDA(call)                                                   \
  do {                                                                     \
    cudaError_t e__ = (call);                                              \
    if (e__ != cudaSuccess) return ::gpuga::cuda_status(e__, #call, __FILE__, __LINE__); \
  } while (0)

#define GPUGA_TRY(call)        \
  do {                         \
    int s__ = (call);          \
    if (s__ != GPUGA_OK) return s__; \
  } while (0)

// potential.in (fitness.cu:220-314) plus the engine's NN2B options.
struct PotentialSpec {
  int type = -1;         // 0 RI, 1 Tersoff one-element, 2 Tersoff two-element, 3 NN2B,
                         // 4 RI with anion charge -q (charge-neutral 1:1 lattices; extension)
  int num_neurons = 0;   // NN2B only
  int num_vars = 0;
  float cutoff = 0.f;    // neighbor-list cutoff
  float w_force = 0.f, w_energy = 0.f, w_stress = 0.f;
  std::vector<float> pmin, pmax;
  float nn_r1 = 7.0f, nn_r2 = 8.0f;  // nn2b.cuh:36-37
  int nn_consistent = 0;              // 0 keeps nn2b.cu:147-148 order
  int ri_self = 0;                    // RI: subtract the damped-Coulomb self energy (off in ri.cu)
};

// RI and its charge-neutral variant share every kernel; only the anion charge differs.
__host__ __device__ inline bool is_ri_type(int t) { return t == 0 || t == 4; }
// anion charge / cation charge: -1/2 in ri.cu:40-43, -1 for potential type 4
__host__ __device__ inline double ri_charge_ratio(int t) { return t == 4 ? -1.0 : -0.5; }

// train.in after parsing (fitness.cu:59-182), in the reference's layouts.
struct TrainingSet {
  int Nc = 0, Nc_force = 0, N = 0, N_force = 0, max_Na = 0;
  std::vector<int> Na, Na_sum, type;
  std::vector<float> r;           // SoA [x(N) y(N) z(N)]
  std::vector<float> h;           // 18 floats per config: box (columns = cell vectors) + inverse
  std::vector<float> pe_ref;      // [Nc]
  std::vector<float> virial_ref;  // [c + Nc*k]
  std::vector<float> force_ref;   // SoA [3N]
  double norm_force = 0, norm_energy = 0, norm_virial = 0;  // FP64 normalisers
};

// ga.in (ga.cu:214-316)
struct GAParams {
  int maximum_generation = 1000;
  int population_size = 200;
  int parent_number = 100;
  float mutation_rate = 0.2f;
};

int num_vars_for(int potential_type, int num_neurons);
int read_potential_in(const std::string& dir, PotentialSpec* spec);
int read_train_in(const std::string& dir, TrainingSet* ts);
int read_ga_in(const std::string& dir, GAParams* ga);
// Validation + derived fields shared by the file and array constructors.
int finish_training_set(TrainingSet* ts);
void box_inverse(float* h);  // fitness.cu:40-57 (FP32)

// FP32 decode of x in [0,1] (fitness.cu:320-324): min + (max - min) * x without contraction.
void decode_params(const PotentialSpec& spec, const float* x01, float* params);

}  // namespace gpuga
