// Engine life cycle and the generation driver: upload of the training set,
// geometry build, per-population plans, CUDA-graph capture of one generation
// (H2D population copy, decode, batched launches, fitness fold, D2H copy).
#include <algorithm>
#include <cmath>
#include <cstring>

#include "engine.hpp"

namespace gpuga {

Engine::~Engine() {
  if (device >= 0) cudaSetDevice(device);
  plans.clear();  // graphs, pinned staging and launch sets
  for (void* ptr : allocations) cudaFree(ptr);
  if (p_out) cudaFree(p_out);
  if (p_w) cudaFree(p_w);
  if (stream) cudaStreamDestroy(stream);
}

int Engine::dalloc(void** p, size_t bytes) {
  bytes = std::max<size_t>(bytes, 16);
  cudaError_t err = cudaMalloc(p, bytes);
  if (err != cudaSuccess) {
    *p = nullptr;
    return cuda_status(err, "cudaMalloc", __FILE__, __LINE__);
  }
  allocations.push_back(*p);
  allocation_bytes[*p] = bytes;
  device_bytes += bytes;
  return GPUGA_OK;
}

void Engine::dfree(void* p) {
  auto it = std::find(allocations.begin(), allocations.end(), p);
  if (it == allocations.end()) return;
  allocations.erase(it);
  device_bytes -= allocation_bytes[p];
  allocation_bytes.erase(p);
  cudaFree(p);
}

namespace {
template <class T>
int upload(Engine* e, T** dst, const T* src, size_t n) {
  GPUGA_TRY(e->alloc(dst, std::max<size_t>(n, 1)));
  if (n) GPUGA_CUDA(cudaMemcpy(*dst, src, sizeof(T) * n, cudaMemcpyHostToDevice));
  return GPUGA_OK;
}
}  // namespace

int engine_create(const PotentialSpec& spec, TrainingSet&& ts, const gpuga_options& opt, Engine** out) {
  std::unique_ptr<Engine> e(new Engine);
  e->opt = opt;
  e->spec = spec;
  e->ts = std::move(ts);
  e->device = opt.device;
  int ndev = 0;
  GPUGA_CUDA(cudaGetDeviceCount(&ndev));
  if (opt.device < 0 || opt.device >= ndev) {
    set_error("device %d not available (%d devices).", opt.device, ndev);
    return GPUGA_ERR_ARG;
  }
  GPUGA_CUDA(cudaSetDevice(opt.device));
  GPUGA_CUDA(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking));
  const TrainingSet& t = e->ts;
  DevSet& d = e->d;
  d.Nc = t.Nc;
  d.Nc_force = t.Nc_force;
  d.N = t.N;
  d.N_force = t.N_force;
  d.max_Na = t.max_Na;
  d.potential_type = spec.type;
  d.num_types = spec.type == 2 ? 2 : 1;
  d.num_neurons = spec.num_neurons;
  d.num_vars = spec.num_vars;
  d.norm_force = t.norm_force;
  d.norm_energy = t.norm_energy;
  d.norm_virial = t.norm_virial;
  d.w_force = spec.w_force;
  d.w_energy = spec.w_energy;
  d.w_stress = spec.w_stress;
  if (is_ri_type(spec.type)) {
    for (int v : t.type)
      if (v < 0 || v > 1) {
        set_error("the RI potential expects atom types 0 (cation) and 1 (anion); found %d.", v);
        return GPUGA_ERR_PARSE;
      }
    const double r2 = ri_charge_ratio(spec.type) * ri_charge_ratio(spec.type);
    std::vector<double> qsum(t.Nc, 0.0);
    for (int c = 0; c < t.Nc; ++c)
      for (int k = 0; k < t.Na[c]; ++k) qsum[c] += t.type[t.Na_sum[c] + k] == 0 ? 1.0 : r2;
    GPUGA_TRY(upload(e.get(), &d.ri_qsum, qsum.data(), qsum.size()));
  }
  if (spec.type == 2) {
    for (int v : t.type)
      if (v < 0) {
        set_error("negative atom type %d.", v);
        return GPUGA_ERR_PARSE;
      }
  }
  GPUGA_TRY(upload(e.get(), &d.Na, t.Na.data(), t.Na.size()));
  GPUGA_TRY(upload(e.get(), &d.Na_sum, t.Na_sum.data(), t.Na_sum.size()));
  GPUGA_TRY(upload(e.get(), &d.type, t.type.data(), t.type.size()));
  GPUGA_TRY(upload(e.get(), &d.r, t.r.data(), t.r.size()));
  GPUGA_TRY(upload(e.get(), &d.h, t.h.data(), t.h.size()));
  GPUGA_TRY(upload(e.get(), &d.force_ref, t.force_ref.data(), t.force_ref.size()));
  std::vector<double> Eref(t.pe_ref.begin(), t.pe_ref.end()), Wref(t.virial_ref.begin(), t.virial_ref.end());
  GPUGA_TRY(upload(e.get(), &d.E_ref, Eref.data(), Eref.size()));
  GPUGA_TRY(upload(e.get(), &d.W_ref, Wref.data(), Wref.size()));
  GPUGA_TRY(upload(e.get(), &e->d_pmin, spec.pmin.data(), spec.pmin.size()));
  GPUGA_TRY(upload(e.get(), &e->d_pmax, spec.pmax.data(), spec.pmax.size()));
  GPUGA_TRY(build_geometry(e.get()));
  if (opt.verbose) {
    printf("Number of configurations is %d:\n", t.Nc);
    printf("    %d force configurations;\n", t.Nc_force);
    printf("    %d energy-virial configurations.\n", t.Nc - t.Nc_force);
    printf("Total number of atoms is %d:\n", t.N);
    printf("    %d atoms in the largest configuration;\n", t.max_Na);
    printf("    %d atoms in force configurations;\n", t.N_force);
    printf("    %d atoms in energy-virial configurations.\n", t.N - t.N_force);
    for (int c = 0; c < t.Nc; ++c) {  // neighbor.cu:78-82
      printf("NN[%d]=%d,", c, e->h_NN[t.Na_sum[c]]);
      if (0 == (c + 1) % 8) printf("\n");
    }
    printf("\n");
  }
  *out = e.release();
  return GPUGA_OK;
}

int plan_get(Engine* e, int P, Plan** out) {
  auto it = e->plans.find(P);
  if (it != e->plans.end()) {
    *out = it->second.get();
    return GPUGA_OK;
  }
  Plan* p = nullptr;
  GPUGA_TRY(plan_build(e, P, &p));
  e->plans[P].reset(p);
  *out = p;
  return GPUGA_OK;
}

namespace {
int get_plan(Engine* e, int P, Plan** out) { return plan_get(e, P, out); }

// One generation from pinned host memory to pinned host memory.
int enqueue_generation(Engine* e, Plan* plan, cudaStream_t st) {
  const size_t nbytes = sizeof(float) * (size_t)plan->P * e->d.num_vars;
  GPUGA_CUDA(cudaMemcpyAsync(plan->d_pop, plan->h_pop, nbytes, cudaMemcpyHostToDevice, st));
  GPUGA_TRY(launchset_enqueue(plan->ls.get(), st));
  GPUGA_CUDA(cudaMemcpyAsync(plan->h_fit, plan->d_fitness, sizeof(double) * plan->P, cudaMemcpyDeviceToHost, st));
  GPUGA_CUDA(cudaMemcpyAsync(plan->h_fit + plan->P, plan->d_comps, sizeof(double) * 3 * plan->P,
                             cudaMemcpyDeviceToHost, st));
  return GPUGA_OK;
}

int run_batched(Engine* e, int P, const float* pop01, double* fitness, double* comps) {
  Plan* plan = nullptr;
  GPUGA_TRY(get_plan(e, P, &plan));
  cudaStream_t st = e->stream;
  // the staged path reads the plan's own population / fitness buffers
  GPUGA_TRY(launchset_retarget(plan->ls.get(), 0, plan->d_pop, plan->d_fitness,
                               plan->dump ? plan->d_fdump : nullptr, st));
  GPUGA_CUDA(cudaStreamSynchronize(st));
  memcpy(plan->h_pop, pop01, sizeof(float) * (size_t)P * e->d.num_vars);
  const bool use_graph = e->opt.use_graph && !plan->dump && !plan->ls->timing;
  if (use_graph) {
    if (!plan->graph) {
      cudaGraph_t g = nullptr;
      GPUGA_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
      int s = enqueue_generation(e, plan, st);
      cudaError_t ce = cudaStreamEndCapture(st, &g);
      if (s != GPUGA_OK) {
        if (g) cudaGraphDestroy(g);
        return s;
      }
      GPUGA_CUDA(ce);
      cudaError_t ie = cudaGraphInstantiate(&plan->graph, g, 0);
      cudaGraphDestroy(g);
      GPUGA_CUDA(ie);
    }
    GPUGA_CUDA(cudaGraphLaunch(plan->graph, st));
  } else {
    GPUGA_TRY(enqueue_generation(e, plan, st));
  }
  GPUGA_CUDA(cudaStreamSynchronize(st));
  memcpy(fitness, plan->h_fit, sizeof(double) * P);
  if (comps) {
    for (int p = 0; p < P; ++p)
      for (int k = 0; k < 3; ++k) comps[3 * (size_t)p + k] = plan->h_fit[P + 3 * (size_t)p + k];
  }
  return GPUGA_OK;
}

}  // namespace

int engine_fitness(Engine* e, int path, int P, const float* pop01, double* fitness, double* comps) {
  if (P <= 0 || !pop01 || !fitness) {
    set_error("gpuga_fitness: invalid arguments (P=%d).", P);
    return GPUGA_ERR_ARG;
  }
  GPUGA_CUDA(cudaSetDevice(e->device));
  switch (path) {
    case GPUGA_PATH_BATCHED: return run_batched(e, P, pop01, fitness, comps);
    case GPUGA_PATH_PLAIN64: return plain_fitness(e, true, P, pop01, fitness, comps);
    case GPUGA_PATH_PLAIN32: return plain_fitness(e, false, P, pop01, fitness, comps);
    default: set_error("unknown path %d.", path); return GPUGA_ERR_ARG;
  }
}

// Batched path on caller-owned device buffers, enqueued on the caller's stream.
int engine_fitness_device(Engine* e, int P, const float* d_pop, double* d_fitness, cudaStream_t st) {
  GPUGA_CUDA(cudaSetDevice(e->device));
  Plan* plan = nullptr;
  GPUGA_TRY(get_plan(e, P, &plan));
  GPUGA_TRY(launchset_retarget(plan->ls.get(), 0, d_pop, d_fitness, nullptr, st));
  return launchset_enqueue(plan->ls.get(), st);
}

int engine_last_results(Engine* e, int P, double* energy, double* virial, double* force_sq) {
  auto it = e->plans.find(P);
  if (it == e->plans.end()) {
    set_error("no batched evaluation with P=%d has run.", P);
    return GPUGA_ERR_ARG;
  }
  const int Nc = e->d.Nc;
  std::vector<double> res((size_t)P * Nc * kResK);
  GPUGA_CUDA(cudaMemcpy(res.data(), it->second->d_res, sizeof(double) * res.size(), cudaMemcpyDeviceToHost));
  for (size_t pc = 0; pc < (size_t)P * Nc; ++pc) {
    if (energy) energy[pc] = res[pc * kResK];
    if (virial)
      for (int k = 0; k < 6; ++k) virial[pc * 6 + k] = res[pc * kResK + 1 + k];
    if (force_sq) force_sq[pc] = res[pc * kResK + 7];
  }
  return GPUGA_OK;
}

int engine_batched_forces(Engine* e, int P, const float* pop01, float* forces_out) {
  GPUGA_CUDA(cudaSetDevice(e->device));
  Plan* plan = nullptr;
  GPUGA_TRY(get_plan(e, P, &plan));
  const size_t n = (size_t)P * 3 * e->d.N_force;
  if (!plan->d_fdump) GPUGA_TRY(e->alloc(&plan->d_fdump, n));
  std::vector<double> fit(P);
  plan->dump = true;
  int s = run_batched(e, P, pop01, fit.data(), nullptr);
  plan->dump = false;
  if (s == GPUGA_OK) {
    cudaError_t ce = cudaMemcpy(forces_out, plan->d_fdump, sizeof(float) * n, cudaMemcpyDeviceToHost);
    if (ce != cudaSuccess) s = cuda_status(ce, "cudaMemcpy", __FILE__, __LINE__);
  }
  return s;
}

}  // namespace gpuga
