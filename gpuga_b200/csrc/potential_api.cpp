// The reference's Potential plug-in interface (potential.cuh:22-41) and
// Neighbor::compute (neighbor.cu:68-83) as C entry points over caller-owned
// device arrays in the reference's layouts.
#include <cstring>
#include <vector>

#include "engine.hpp"

using namespace gpuga;

struct gpuga_potential {
  int type = -1, num_neurons = 0, num_vars = 0;
  std::vector<float> params;
  bool have_params = false;
  int N = 0, max_Na = 0;
  void* scratch = nullptr;
  size_t bytes = 0;
  PotentialSpec opts;  // NN2B taper options (reference defaults)
};

namespace {
RefPotentialScratch carve(void* base, int potential_type, int num_neurons, int N, int max_Na) {
  const size_t slots = (size_t)N * (size_t)max_Na;
  auto up = [](size_t b) { return (b + 255) & ~(size_t)255; };
  char* p = static_cast<char*>(base);
  RefPotentialScratch s;
  s.g64 = reinterpret_cast<double4*>(p);
  p += up(slots * sizeof(double4));
  s.rev = reinterpret_cast<int*>(p);
  p += up(slots * sizeof(int));
  s.f5 = reinterpret_cast<float*>(p);
  p += up(5 * slots * sizeof(float));
  s.w = reinterpret_cast<float*>(p);
  (void)potential_type;
  (void)num_neurons;
  return s;
}
}  // namespace

extern "C" {

int gpuga_potential_create(int potential_type, int num_neurons, gpuga_potential** out) {
  if (!out) {
    set_error("gpuga_potential_create: null output");
    return GPUGA_ERR_ARG;
  }
  const int nv = num_vars_for(potential_type, num_neurons);
  if (nv < 0 || (potential_type == 3 && (num_neurons < 1 || num_neurons > 32))) {
    set_error("unsupported potential type %d (neurons %d).", potential_type, num_neurons);
    return GPUGA_ERR_UNSUPPORTED;
  }
  gpuga_potential* p = new gpuga_potential;
  p->type = potential_type;
  p->num_neurons = num_neurons;
  p->num_vars = nv;
  p->params.assign(nv, 0.f);
  *out = p;
  return GPUGA_OK;
}

// Potential::initialize(N, max_Na): scratch sized like the reference's
// N x max_Na per-bond buffers (minimal_tersoff.cu:30-37).
int gpuga_potential_initialize(gpuga_potential* p, int N, int max_Na) {
  if (!p || N < 1 || max_Na < 1) {
    set_error("gpuga_potential_initialize: invalid argument");
    return GPUGA_ERR_ARG;
  }
  if (p->scratch) cudaFree(p->scratch);
  p->scratch = nullptr;
  p->bytes = ref_potential_scratch_bytes(p->type, p->num_neurons, N, max_Na);
  GPUGA_CUDA(cudaMalloc(&p->scratch, p->bytes));
  p->N = N;
  p->max_Na = max_Na;
  return GPUGA_OK;
}

// Potential::update_potential (potential.cuh:26): parameters in potential.in order.
int gpuga_potential_update(gpuga_potential* p, const float* params, int num_params) {
  if (!p || !params || num_params != p->num_vars) {
    set_error("gpuga_potential_update: expected %d parameters", p ? p->num_vars : -1);
    return GPUGA_ERR_ARG;
  }
  memcpy(p->params.data(), params, sizeof(float) * num_params);
  p->have_params = true;
  return GPUGA_OK;
}

int gpuga_potential_find_force(gpuga_potential* p, int Nc, int N, const int* Na, const int* Na_sum, int max_Na,
                               const int* type, const float* h, const int* NN, const int* NL, const float* r,
                               float* f, float* virial, float* pe, void* stream) {
  if (!p || !Na || !Na_sum || !type || !h || !NN || !NL || !r || !f || !virial || !pe || Nc < 1) {
    set_error("gpuga_potential_find_force: invalid argument");
    return GPUGA_ERR_ARG;
  }
  if (!p->scratch || N > p->N || (size_t)N * max_Na > (size_t)p->N * p->max_Na || max_Na > p->max_Na) {
    set_error("gpuga_potential_find_force: call gpuga_potential_initialize(N >= %d, max_Na >= %d) first", N, max_Na);
    return GPUGA_ERR_ARG;
  }
  if (!p->have_params) {
    set_error("gpuga_potential_find_force: call gpuga_potential_update first");
    return GPUGA_ERR_ARG;
  }
  const RefPotentialScratch s = carve(p->scratch, p->type, p->num_neurons, N, max_Na);
  return ref_potential_find_force(p->type, p->num_neurons, p->params.data(), p->opts, Nc, N, Na, Na_sum, max_Na,
                                  type, h, NN, NL, r, f, virial, pe, s, (cudaStream_t)stream);
}

int gpuga_potential_destroy(gpuga_potential* p) {
  if (!p) return GPUGA_OK;
  if (p->scratch) cudaFree(p->scratch);
  delete p;
  return GPUGA_OK;
}

int gpuga_neighbor_compute(int Nc, int N, int max_Na, const int* Na, const int* Na_sum, const float* r,
                           const float* h, float cutoff, int* NN, int* NL, void* stream) {
  if (Nc < 1 || N < 1 || !Na || !Na_sum || !r || !h || !NN || !NL) {
    set_error("gpuga_neighbor_compute: invalid argument");
    return GPUGA_ERR_ARG;
  }
  return neighbor_reference_layout(Nc, N, max_Na, Na, Na_sum, r, h, cutoff, NN, NL, (cudaStream_t)stream);
}

}  // extern "C"
