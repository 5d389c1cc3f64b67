// Device-resident GA loop: the generation of ga.cu:73-212 with its selection,
// crossover and mutation on the GPU, behind the batched fitness launches.
//
// The random draws of a generation never depend on fitness values (parents are
// chosen by rank from fixed cumulative probabilities, ga.cu:41-46, 200-212), so
// the host draws them from the GA's own std::mt19937 stream, in the
// reference's order, a window of generations ahead (GA::draw_plan), while the
// device runs the previous window.  Per generation the device then runs, with
// no host round trip:
//
//   batched fitness  ->  ga_rank  ->  ga_breed  ->  ga_mutate  ->  ga_advance
//
// ga_rank reproduces the reference's stable insertion sort (ga.cu:105-119)
// exactly, NaN included: a NaN never moves and no value passes one, so the
// sort is a stable sort of every NaN-free run between NaNs; each individual's
// position is its segment start + the number of smaller values in its segment
// + the number of equal values before it.  One generation is captured in a CUDA
// graph (one per plan buffer) and replayed for every generation of a window;
// a device counter tells the kernels which generation of the window they run.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <memory>

#include "engine.hpp"
#include "ga.hpp"

namespace gpuga {

// Largest population whose FP32 fitness vector fits the rank kernel's shared memory.
constexpr int kMaxDevicePopulation = 49152;

__global__ void ga_rank(int P, int d, const double* __restrict__ fit64, const float* __restrict__ pop,
                        float* __restrict__ sorted, float* __restrict__ fit_sorted, float* __restrict__ hist,
                        const int* __restrict__ gen, int* __restrict__ order) {
  extern __shared__ float f[];
  for (int j = threadIdx.x; j < P; j += blockDim.x) f[j] = __double2float_rn(fit64[j]);  // the GA ranks FP32 values
  __syncthreads();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P) return;
  const float fi = f[i];
  int r = i;
  if (!isnan(fi)) {
    int s = i;
    while (s > 0 && !isnan(f[s - 1])) --s;
    int e = i + 1;
    while (e < P && !isnan(f[e])) ++e;
    r = s;
    for (int j = s; j < e; ++j) {
      const float fj = f[j];
      r += (fj < fi) || (fj == fi && j < i);
    }
  }
  fit_sorted[r] = fi;
  if (order) order[r] = i;
  if (!pop) return;
  const float* src = pop + (size_t)i * d;
  float* dst = sorted + (size_t)r * d;
  for (int m = 0; m < d; ++m) dst[m] = src[m];
  if (r == 0) {
    float* h = hist + (size_t)(*gen) * (d + 1);
    h[0] = fi;
    for (int m = 0; m < d; ++m) h[1 + m] = src[m];
  }
}

// ga.cu:161-186 on the sorted population: rows below parent_number are the
// parents, each pair of children takes genes [0, point) from one parent and
// [point, d) from the other.
__global__ void ga_breed(int P, int d, int parent_number, const int* __restrict__ pairs, int pairs_per_gen,
                         const float* __restrict__ sorted, float* __restrict__ pop, const int* __restrict__ gen) {
  const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= (long long)P * d) return;
  const int r = (int)(n / d), c = (int)(n - (long long)r * d);
  float v;
  if (r < parent_number) {
    v = sorted[n];
  } else {
    const int m = r - parent_number;
    const int* q = pairs + ((size_t)(*gen) * pairs_per_gen + m / 2) * 3;
    const int first = c < q[2] ? q[0] : q[1];
    const int second = c < q[2] ? q[1] : q[0];
    v = sorted[(size_t)((m & 1) ? second : first) * d + c];
  }
  pop[n] = v;
}

// ga.cu:188-198 with repeated genes already folded on the host.
__global__ void ga_mutate(const int* __restrict__ off, const int* __restrict__ idx, const float* __restrict__ val,
                          float* __restrict__ pop, const int* __restrict__ gen) {
  const int g = *gen;
  const int k = off[g] + blockIdx.x * blockDim.x + threadIdx.x;
  if (k < off[g + 1]) pop[idx[k]] = val[k];
}

__global__ void ga_advance(int* gen) { *gen += 1; }

struct DeviceGA {
  Engine* e = nullptr;
  int P = 0, d = 0, window = 0, pairs_per_gen = 0, mut_cap = 0;
  float* d_pop = nullptr;
  float* d_sorted = nullptr;
  float* d_fit32 = nullptr;
  double* d_fit64 = nullptr;
  int* d_gen = nullptr;
  // per plan buffer (two, so the host draws a window while the device runs the other)
  int* d_pairs[2] = {nullptr, nullptr};
  int* d_off[2] = {nullptr, nullptr};
  int* d_midx[2] = {nullptr, nullptr};
  float* d_mval[2] = {nullptr, nullptr};
  float* d_hist[2] = {nullptr, nullptr};
  int* h_pairs[2] = {nullptr, nullptr};
  int* h_off[2] = {nullptr, nullptr};
  int* h_midx[2] = {nullptr, nullptr};
  float* h_mval[2] = {nullptr, nullptr};
  float* h_hist[2] = {nullptr, nullptr};
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  cudaEvent_t done[2] = {nullptr, nullptr};
  std::vector<void*> dev, host;
  ~DeviceGA() {
    for (int b = 0; b < 2; ++b) {
      if (graph[b]) cudaGraphExecDestroy(graph[b]);
      if (done[b]) cudaEventDestroy(done[b]);
    }
    for (void* p : dev) cudaFree(p);
    for (void* p : host) cudaFreeHost(p);
  }
  template <class T>
  int dalloc(T** p, size_t n) {
    GPUGA_CUDA(cudaMalloc(reinterpret_cast<void**>(p), std::max<size_t>(n, 1) * sizeof(T)));
    dev.push_back(*p);
    return GPUGA_OK;
  }
  template <class T>
  int halloc(T** p, size_t n) {
    GPUGA_CUDA(cudaMallocHost(reinterpret_cast<void**>(p), std::max<size_t>(n, 1) * sizeof(T)));
    host.push_back(*p);
    return GPUGA_OK;
  }
};

void device_ga_free(DeviceGA* s) { delete s; }

int device_rank(int device, int P, const double* fitness, int* order, float* sorted) {
  if (P < 1 || P > kMaxDevicePopulation) {
    set_error("device ranking supports 1..%d values (got %d).", kMaxDevicePopulation, P);
    return GPUGA_ERR_ARG;
  }
  GPUGA_CUDA(cudaSetDevice(device));
  double* d_fit = nullptr;
  int* d_order = nullptr;
  float* d_sorted = nullptr;
  cudaError_t ce = cudaMalloc(&d_fit, sizeof(double) * P);
  if (ce == cudaSuccess) ce = cudaMalloc(&d_order, sizeof(int) * P);
  if (ce == cudaSuccess) ce = cudaMalloc(&d_sorted, sizeof(float) * P);
  if (ce == cudaSuccess) ce = cudaMemcpy(d_fit, fitness, sizeof(double) * P, cudaMemcpyHostToDevice);
  if (ce == cudaSuccess && sizeof(float) * P > 48 * 1024)
    ce = cudaFuncSetAttribute(ga_rank, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(sizeof(float) * P));
  if (ce == cudaSuccess) {
    ga_rank<<<(P + 255) / 256, 256, sizeof(float) * P>>>(P, 0, d_fit, nullptr, nullptr, d_sorted, nullptr, nullptr,
                                                         d_order);
    ce = cudaGetLastError();
  }
  if (ce == cudaSuccess) ce = cudaMemcpy(order, d_order, sizeof(int) * P, cudaMemcpyDeviceToHost);
  if (ce == cudaSuccess && sorted) ce = cudaMemcpy(sorted, d_sorted, sizeof(float) * P, cudaMemcpyDeviceToHost);
  cudaFree(d_fit);
  cudaFree(d_order);
  cudaFree(d_sorted);
  if (ce != cudaSuccess) return cuda_status(ce, "device_rank", __FILE__, __LINE__);
  return GPUGA_OK;
}

namespace {

int setup(Engine* e, const GA& ga, int window, DeviceGA** out) {
  std::unique_ptr<DeviceGA> s(new DeviceGA);
  s->e = e;
  s->P = ga.gp.population_size;
  s->d = ga.d;
  s->window = window;
  s->pairs_per_gen = ga.child_number / 2;
  s->mut_cap = std::max(ga.mutation_count(0), 1);  // counts never grow with the generation
  const size_t Pd = (size_t)s->P * s->d;
  GPUGA_TRY(s->dalloc(&s->d_pop, Pd));
  GPUGA_TRY(s->dalloc(&s->d_sorted, Pd));
  GPUGA_TRY(s->dalloc(&s->d_fit32, s->P));
  GPUGA_TRY(s->dalloc(&s->d_fit64, s->P));
  GPUGA_TRY(s->dalloc(&s->d_gen, 1));
  for (int b = 0; b < 2; ++b) {
    const size_t np = (size_t)window * s->pairs_per_gen * 3, nm = (size_t)window * s->mut_cap,
                 nh = (size_t)window * (s->d + 1);
    GPUGA_TRY(s->dalloc(&s->d_pairs[b], np));
    GPUGA_TRY(s->dalloc(&s->d_off[b], window + 1));
    GPUGA_TRY(s->dalloc(&s->d_midx[b], nm));
    GPUGA_TRY(s->dalloc(&s->d_mval[b], nm));
    GPUGA_TRY(s->dalloc(&s->d_hist[b], nh));
    GPUGA_TRY(s->halloc(&s->h_pairs[b], np));
    GPUGA_TRY(s->halloc(&s->h_off[b], window + 1));
    GPUGA_TRY(s->halloc(&s->h_midx[b], nm));
    GPUGA_TRY(s->halloc(&s->h_mval[b], nm));
    GPUGA_TRY(s->halloc(&s->h_hist[b], nh));
    GPUGA_CUDA(cudaEventCreateWithFlags(&s->done[b], cudaEventDisableTiming));
  }
  const size_t rank_smem = sizeof(float) * s->P;
  if (rank_smem > 48 * 1024)
    GPUGA_CUDA(cudaFuncSetAttribute(ga_rank, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rank_smem));
  *out = s.release();
  return GPUGA_OK;
}

// One generation on buffer b: fitness of d_pop, then rank, breed, mutate, advance.
int enqueue_one(DeviceGA* s, LaunchSet* ls, int b, cudaStream_t st) {
  GPUGA_TRY(launchset_enqueue(ls, st));
  const int P = s->P, d = s->d;
  ga_rank<<<(P + 255) / 256, 256, sizeof(float) * P, st>>>(P, d, s->d_fit64, s->d_pop, s->d_sorted, s->d_fit32,
                                                          s->d_hist[b], s->d_gen, nullptr);
  GPUGA_CUDA(cudaGetLastError());
  const long long Pd = (long long)P * d;
  ga_breed<<<(unsigned)((Pd + 255) / 256), 256, 0, st>>>(P, d, P - 2 * s->pairs_per_gen, s->d_pairs[b],
                                                         s->pairs_per_gen, s->d_sorted, s->d_pop, s->d_gen);
  GPUGA_CUDA(cudaGetLastError());
  ga_mutate<<<(s->mut_cap + 255) / 256, 256, 0, st>>>(s->d_off[b], s->d_midx[b], s->d_mval[b], s->d_pop, s->d_gen);
  GPUGA_CUDA(cudaGetLastError());
  ga_advance<<<1, 1, 0, st>>>(s->d_gen);
  GPUGA_CUDA(cudaGetLastError());
  return GPUGA_OK;
}

// Draws generations [g0, g0 + n) into host buffer b.
void draw_window(GA& ga, DeviceGA* s, int b, int g0, int n) {
  GenPlan plan;
  int moff = 0;
  s->h_off[b][0] = 0;
  for (int k = 0; k < n; ++k) {
    ga.draw_plan(g0 + k, &plan);
    memcpy(s->h_pairs[b] + (size_t)k * s->pairs_per_gen * 3, plan.pairs.data(), sizeof(int) * plan.pairs.size());
    const int m = (int)plan.mut_idx.size();
    memcpy(s->h_midx[b] + moff, plan.mut_idx.data(), sizeof(int) * m);
    memcpy(s->h_mval[b] + moff, plan.mut_val.data(), sizeof(float) * m);
    moff += m;
    s->h_off[b][k + 1] = moff;
  }
}

int upload_window(DeviceGA* s, int b, int n, cudaStream_t st) {
  GPUGA_CUDA(cudaMemcpyAsync(s->d_pairs[b], s->h_pairs[b], sizeof(int) * (size_t)n * s->pairs_per_gen * 3,
                             cudaMemcpyHostToDevice, st));
  GPUGA_CUDA(cudaMemcpyAsync(s->d_off[b], s->h_off[b], sizeof(int) * (n + 1), cudaMemcpyHostToDevice, st));
  const int m = s->h_off[b][n];
  if (m > 0) {
    GPUGA_CUDA(cudaMemcpyAsync(s->d_midx[b], s->h_midx[b], sizeof(int) * m, cudaMemcpyHostToDevice, st));
    GPUGA_CUDA(cudaMemcpyAsync(s->d_mval[b], s->h_mval[b], sizeof(float) * m, cudaMemcpyHostToDevice, st));
  }
  return GPUGA_OK;
}

int run_window(DeviceGA* s, LaunchSet* ls, int b, int n, bool use_graph, cudaStream_t st) {
  GPUGA_CUDA(cudaMemsetAsync(s->d_gen, 0, sizeof(int), st));
  if (use_graph && !s->graph[b]) {
    cudaGraph_t g = nullptr;
    GPUGA_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    int rc = enqueue_one(s, ls, b, st);
    cudaError_t ce = cudaStreamEndCapture(st, &g);
    if (rc != GPUGA_OK) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    GPUGA_CUDA(ce);
    cudaError_t ie = cudaGraphInstantiate(&s->graph[b], g, 0);
    cudaGraphDestroy(g);
    GPUGA_CUDA(ie);
  }
  for (int k = 0; k < n; ++k) {
    if (use_graph) {
      GPUGA_CUDA(cudaGraphLaunch(s->graph[b], st));
    } else {
      GPUGA_TRY(enqueue_one(s, ls, b, st));
    }
  }
  GPUGA_CUDA(cudaMemcpyAsync(s->h_hist[b], s->d_hist[b], sizeof(float) * (size_t)n * (s->d + 1),
                             cudaMemcpyDeviceToHost, st));
  GPUGA_CUDA(cudaEventRecord(s->done[b], st));
  return GPUGA_OK;
}

void emit_lines(const GA& ga, const DeviceGA* s, int b, int g0, int n, std::string* lines) {
  for (int k = 0; k < n; ++k) {
    const float* h = s->h_hist[b] + (size_t)k * (s->d + 1);
    *lines += ga_output_line(g0 + k, h[0], h + 1, ga.pmin.data(), ga.pmax.data(), s->d);
  }
}

}  // namespace

int device_ga_advance(Engine* e, GA* ga, DeviceGA** state, int generations, int window,
                      const std::function<void(const std::string&)>& sink) {
  if (e->opt.path != GPUGA_PATH_BATCHED) {
    set_error("the device GA loop runs on the batched path only (engine path %d).", e->opt.path);
    return GPUGA_ERR_ARG;
  }
  const int P = ga->gp.population_size;
  if (P > kMaxDevicePopulation) {
    set_error("the device GA loop supports populations up to %d (got %d).", kMaxDevicePopulation, P);
    return GPUGA_ERR_UNSUPPORTED;
  }
  if (window < 1) window = 32;
  generations = std::min(generations, ga->gp.maximum_generation - ga->generation);
  if (generations <= 0) return GPUGA_OK;
  GPUGA_CUDA(cudaSetDevice(e->device));
  DeviceGA* s = *state;
  if (s && (s->window < window || s->P != P || s->d != ga->d)) {
    delete s;
    s = *state = nullptr;
  }
  if (!s) {
    GPUGA_TRY(setup(e, *ga, window, &s));
    *state = s;
  }
  window = s->window;
  cudaStream_t st = e->stream;
  Plan* plan = nullptr;
  GPUGA_TRY(plan_get(e, P, &plan));
  LaunchSet* ls = plan->ls.get();
  GPUGA_TRY(launchset_retarget(ls, 0, s->d_pop, s->d_fit64, nullptr, st));
  const bool use_graph = e->opt.use_graph && !ls->timing;
  GPUGA_CUDA(cudaMemcpyAsync(s->d_pop, ga->population.data(), sizeof(float) * (size_t)P * s->d,
                             cudaMemcpyHostToDevice, st));

  // window k runs on buffer k % 2; the host draws window k + 1 while the device runs window k
  const int g_start = ga->generation;
  int nwin = (generations + window - 1) / window;
  auto wlen = [&](int k) { return std::min(window, generations - k * window); };
  draw_window(*ga, s, 0, g_start, wlen(0));
  GPUGA_TRY(upload_window(s, 0, wlen(0), st));
  GPUGA_TRY(run_window(s, ls, 0, wlen(0), use_graph, st));
  for (int k = 0; k < nwin; ++k) {
    const int b = k & 1;
    if (k + 1 < nwin) {
      // buffer b^1 was last read by window k - 1, which finished before window k started
      if (k >= 1) GPUGA_CUDA(cudaEventSynchronize(s->done[b ^ 1]));
      draw_window(*ga, s, b ^ 1, g_start + (k + 1) * window, wlen(k + 1));
      GPUGA_TRY(upload_window(s, b ^ 1, wlen(k + 1), st));
      GPUGA_TRY(run_window(s, ls, b ^ 1, wlen(k + 1), use_graph, st));
    }
    GPUGA_CUDA(cudaEventSynchronize(s->done[b]));
    std::string lines;
    emit_lines(*ga, s, b, g_start + k * window, wlen(k), &lines);
    if (sink) sink(lines);
  }
  GPUGA_CUDA(cudaMemcpyAsync(ga->population.data(), s->d_pop, sizeof(float) * (size_t)P * s->d,
                             cudaMemcpyDeviceToHost, st));
  GPUGA_CUDA(cudaMemcpyAsync(ga->fitness.data(), s->d_fit32, sizeof(float) * P, cudaMemcpyDeviceToHost, st));
  GPUGA_CUDA(cudaStreamSynchronize(st));
  ga->generation = g_start + generations;
  return GPUGA_OK;
}

}  // namespace gpuga
