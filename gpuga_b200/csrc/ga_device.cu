// Device-resident GA loop: the generation of ga.cu:73-212 with its selection,
// crossover and mutation on the GPU, behind the batched fitness launches, for
// one GA or for every job of the serving loop at once.
//
// The random draws of a generation never depend on fitness values (parents are
// chosen by rank from fixed cumulative probabilities, ga.cu:41-46, 200-212), so
// the host draws them from each GA's own std::mt19937 stream, in the
// reference's order, a window of generations ahead (GA::draw_plan).  Per
// generation the device then runs, with no host round trip:
//
//   batched fitness (all jobs) -> ga_rank -> ga_breed -> ga_mutate -> ga_advance
//
// The four GA kernels cover all jobs of a batch in one launch each: a job
// table holds every job's buffers and each block finds its job through a
// block -> job map, as the fitness launches do with their work items.
// ga_rank reproduces the reference's stable insertion sort (ga.cu:105-119)
// exactly, NaN included: a NaN never moves and no value passes one, so the
// sort is a stable sort of every NaN-free run between NaNs; each individual's
// position is its segment start + the number of smaller values in its segment
// + the number of equal values before it.  One generation is captured in a CUDA
// graph per plan buffer and replayed for every generation of a window; per-job
// device counters tell the kernels which generation of the window they run.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <memory>

#include "engine.hpp"
#include "ga.hpp"

namespace gpuga {

// Largest population whose FP32 fitness vector fits the rank kernel's shared memory.
constexpr int kMaxDevicePopulation = 49152;
constexpr int kGABlock = 256;

// One row of a batch's GA job table (plan buffers of one stage).
struct GAJob {
  int P, d, parent_number, pairs_per_gen;
  int rank_block0, breed_block0, mut_block0;
  float* pop;           // [P][d]: evaluated, then overwritten by the next generation
  float* sorted;        // [P][d]
  float* fit32;         // [P] sorted FP32 fitness
  const double* fit64;  // [P] from the fitness fold
  float* hist;          // [window][1 + d]: best fitness and elite genes per generation
  int* gen;             // generation within the window
  const int* pairs;     // [window][pairs_per_gen][3]
  const int* off;       // [window + 1] mutation offsets
  const int* midx;
  const float* mval;
};

// Ranks the FP32-rounded fitness values of one job (or of an explicit fitness
// vector, for gpuga_ga_rank_device) and writes the sorted population, the
// sorted fitness and the elite of the generation.
__device__ __forceinline__ void rank_block(int P, int d, const double* __restrict__ fit64,
                                           const float* __restrict__ pop, float* __restrict__ sorted,
                                           float* __restrict__ fit_sorted, float* __restrict__ hist, int gen,
                                           int* __restrict__ order, int i, float* f) {
  for (int j = threadIdx.x; j < P; j += blockDim.x) f[j] = __double2float_rn(fit64[j]);  // the GA ranks FP32 values
  __syncthreads();
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
    float* h = hist + (size_t)gen * (d + 1);
    h[0] = fi;
    for (int m = 0; m < d; ++m) h[1 + m] = src[m];
  }
}

__global__ void ga_rank_jobs(const GAJob* __restrict__ jobs, const int* __restrict__ block_job) {
  extern __shared__ float f[];
  const GAJob& J = jobs[block_job[blockIdx.x]];
  const int i = (blockIdx.x - J.rank_block0) * blockDim.x + threadIdx.x;
  rank_block(J.P, J.d, J.fit64, J.pop, J.sorted, J.fit32, J.hist, *J.gen, nullptr, i, f);
}

__global__ void ga_rank_values(int P, const double* __restrict__ fit64, float* __restrict__ fit_sorted,
                               int* __restrict__ order) {
  extern __shared__ float f[];
  rank_block(P, 0, fit64, nullptr, nullptr, fit_sorted, nullptr, 0, order, blockIdx.x * blockDim.x + threadIdx.x,
             f);
}

// ga.cu:161-186 on the sorted population: rows below parent_number are the
// parents, each pair of children takes genes [0, point) from one parent and
// [point, d) from the other.
__global__ void ga_breed_jobs(const GAJob* __restrict__ jobs, const int* __restrict__ block_job) {
  const GAJob& J = jobs[block_job[blockIdx.x]];
  const int P = J.P, d = J.d;
  const long long n = (long long)(blockIdx.x - J.breed_block0) * blockDim.x + threadIdx.x;
  if (n >= (long long)P * d) return;
  const int r = (int)(n / d), c = (int)(n - (long long)r * d);
  float v;
  if (r < J.parent_number) {
    v = J.sorted[n];
  } else {
    const int m = r - J.parent_number;
    const int* q = J.pairs + ((size_t)(*J.gen) * J.pairs_per_gen + m / 2) * 3;
    const int first = c < q[2] ? q[0] : q[1];
    const int second = c < q[2] ? q[1] : q[0];
    v = J.sorted[(size_t)((m & 1) ? second : first) * d + c];
  }
  J.pop[n] = v;
}

// ga.cu:188-198 with repeated genes already folded on the host.
__global__ void ga_mutate_jobs(const GAJob* __restrict__ jobs, const int* __restrict__ block_job) {
  const GAJob& J = jobs[block_job[blockIdx.x]];
  const int g = *J.gen;
  const int k = J.off[g] + (blockIdx.x - J.mut_block0) * blockDim.x + threadIdx.x;
  if (k < J.off[g + 1]) J.pop[J.midx[k]] = J.mval[k];
}

__global__ void ga_advance_jobs(const GAJob* __restrict__ jobs, int njobs) {
  for (int j = threadIdx.x; j < njobs; j += blockDim.x) *jobs[j].gen += 1;
}

// The GA kernels of several jobs, launched together behind one launch set.
struct GABatch {
  std::vector<DeviceGA*> jobs;
  LaunchSet* ls = nullptr;
  GAJob* d_table[2] = {nullptr, nullptr};
  int *d_rank_map = nullptr, *d_breed_map = nullptr, *d_mut_map = nullptr;
  int n_rank = 0, n_breed = 0, n_mut = 0;
  size_t rank_smem = 0;
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  cudaEvent_t done[2] = {nullptr, nullptr};
  std::vector<cudaEvent_t> gen_ev[2];  // per-generation timing events of the last window on buffer b
  ~GABatch() {
    for (int b = 0; b < 2; ++b) {
      if (graph[b]) cudaGraphExecDestroy(graph[b]);
      if (done[b]) cudaEventDestroy(done[b]);
      cudaFree(d_table[b]);
      for (cudaEvent_t e : gen_ev[b]) cudaEventDestroy(e);
    }
    cudaFree(d_rank_map);
    cudaFree(d_breed_map);
    cudaFree(d_mut_map);
  }
};

// Per-GA device state: population buffers and two plan stages (the host draws
// one while the device runs the other).
struct DeviceGA {
  int P = 0, d = 0, window = 0, pairs_per_gen = 0, mut_cap = 0;
  float* d_pop = nullptr;
  float* d_sorted = nullptr;
  float* d_fit32 = nullptr;
  double* d_fit64 = nullptr;
  int* d_gen = nullptr;
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
  std::unique_ptr<GABatch> solo;  // the one-job batch of device_ga_advance
  std::vector<void*> dev, host;
  ~DeviceGA() {
    solo.reset();
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
void ga_batch_free(GABatch* b) { delete b; }
float* device_ga_population(DeviceGA* s) { return s->d_pop; }
double* device_ga_fitness64(DeviceGA* s) { return s->d_fit64; }
const float* device_ga_history(const DeviceGA* s, int b) { return s->h_hist[b]; }

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
    ce = cudaFuncSetAttribute(ga_rank_values, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(sizeof(float) * P));
  if (ce == cudaSuccess) {
    ga_rank_values<<<(P + kGABlock - 1) / kGABlock, kGABlock, sizeof(float) * P>>>(P, d_fit, d_sorted, d_order);
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

int device_ga_setup(const GA& ga, int window, DeviceGA** out) {
  const int P = ga.gp.population_size;
  if (P > kMaxDevicePopulation) {
    set_error("the device GA loop supports populations up to %d (got %d).", kMaxDevicePopulation, P);
    return GPUGA_ERR_UNSUPPORTED;
  }
  std::unique_ptr<DeviceGA> s(new DeviceGA);
  s->P = P;
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
  }
  *out = s.release();
  return GPUGA_OK;
}

namespace {

int enqueue_generation(GABatch* B, int b, cudaStream_t st) {
  GPUGA_TRY(launchset_enqueue(B->ls, st));
  ga_rank_jobs<<<B->n_rank, kGABlock, B->rank_smem, st>>>(B->d_table[b], B->d_rank_map);
  GPUGA_CUDA(cudaGetLastError());
  ga_breed_jobs<<<B->n_breed, kGABlock, 0, st>>>(B->d_table[b], B->d_breed_map);
  GPUGA_CUDA(cudaGetLastError());
  ga_mutate_jobs<<<B->n_mut, kGABlock, 0, st>>>(B->d_table[b], B->d_mut_map);
  GPUGA_CUDA(cudaGetLastError());
  ga_advance_jobs<<<1, 128, 0, st>>>(B->d_table[b], (int)B->jobs.size());
  GPUGA_CUDA(cudaGetLastError());
  return GPUGA_OK;
}

}  // namespace

int ga_batch_build(const std::vector<DeviceGA*>& jobs, LaunchSet* ls, GABatch** out) {
  std::unique_ptr<GABatch> B(new GABatch);
  B->jobs = jobs;
  B->ls = ls;
  std::vector<int> rmap, bmap, mmap;
  std::vector<GAJob> rows[2];
  int maxP = 1;
  for (size_t j = 0; j < jobs.size(); ++j) {
    const DeviceGA* s = jobs[j];
    maxP = std::max(maxP, s->P);
    GAJob row{};
    row.P = s->P;
    row.d = s->d;
    row.parent_number = s->P - 2 * s->pairs_per_gen;
    row.pairs_per_gen = s->pairs_per_gen;
    row.rank_block0 = (int)rmap.size();
    row.breed_block0 = (int)bmap.size();
    row.mut_block0 = (int)mmap.size();
    const long long Pd = (long long)s->P * s->d;
    for (int k = 0; k < (s->P + kGABlock - 1) / kGABlock; ++k) rmap.push_back((int)j);
    for (long long k = 0; k < (Pd + kGABlock - 1) / kGABlock; ++k) bmap.push_back((int)j);
    for (int k = 0; k < (s->mut_cap + kGABlock - 1) / kGABlock; ++k) mmap.push_back((int)j);
    row.pop = s->d_pop;
    row.sorted = s->d_sorted;
    row.fit32 = s->d_fit32;
    row.fit64 = s->d_fit64;
    row.gen = s->d_gen;
    for (int b = 0; b < 2; ++b) {
      GAJob r = row;
      r.hist = s->d_hist[b];
      r.pairs = s->d_pairs[b];
      r.off = s->d_off[b];
      r.midx = s->d_midx[b];
      r.mval = s->d_mval[b];
      rows[b].push_back(r);
    }
  }
  B->n_rank = (int)rmap.size();
  B->n_breed = (int)bmap.size();
  B->n_mut = (int)mmap.size();
  B->rank_smem = sizeof(float) * maxP;
  GPUGA_CUDA(cudaMalloc(&B->d_rank_map, sizeof(int) * std::max<size_t>(rmap.size(), 1)));
  GPUGA_CUDA(cudaMalloc(&B->d_breed_map, sizeof(int) * std::max<size_t>(bmap.size(), 1)));
  GPUGA_CUDA(cudaMalloc(&B->d_mut_map, sizeof(int) * std::max<size_t>(mmap.size(), 1)));
  GPUGA_CUDA(cudaMemcpy(B->d_rank_map, rmap.data(), sizeof(int) * rmap.size(), cudaMemcpyHostToDevice));
  GPUGA_CUDA(cudaMemcpy(B->d_breed_map, bmap.data(), sizeof(int) * bmap.size(), cudaMemcpyHostToDevice));
  GPUGA_CUDA(cudaMemcpy(B->d_mut_map, mmap.data(), sizeof(int) * mmap.size(), cudaMemcpyHostToDevice));
  for (int b = 0; b < 2; ++b) {
    GPUGA_CUDA(cudaMalloc(&B->d_table[b], sizeof(GAJob) * std::max<size_t>(jobs.size(), 1)));
    GPUGA_CUDA(cudaMemcpy(B->d_table[b], rows[b].data(), sizeof(GAJob) * jobs.size(), cudaMemcpyHostToDevice));
    GPUGA_CUDA(cudaEventCreateWithFlags(&B->done[b], cudaEventDisableTiming));
  }
  if (B->rank_smem > 48 * 1024)
    GPUGA_CUDA(cudaFuncSetAttribute(ga_rank_jobs, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)B->rank_smem));
  *out = B.release();
  return GPUGA_OK;
}

// Draws generations [g0, g0 + n) of `ga` into its host plan buffer b.
void device_ga_draw(GA& ga, DeviceGA* s, int b, int g0, int n) {
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

int device_ga_upload(DeviceGA* s, int b, int n, cudaStream_t st) {
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

// n generations of every job of the batch on plan buffer b (uploaded before), then the
// generation histories back to the host; done[b] marks the end.  With `timed`, events
// bracket every generation (ga_batch_generation_ms).
int ga_batch_window(GABatch* B, int b, int n, bool use_graph, bool timed, cudaStream_t st) {
  for (DeviceGA* s : B->jobs) GPUGA_CUDA(cudaMemsetAsync(s->d_gen, 0, sizeof(int), st));
  if (use_graph && !B->graph[b]) {
    cudaGraph_t g = nullptr;
    GPUGA_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    int rc = enqueue_generation(B, b, st);
    cudaError_t ce = cudaStreamEndCapture(st, &g);
    if (rc != GPUGA_OK) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    GPUGA_CUDA(ce);
    cudaError_t ie = cudaGraphInstantiate(&B->graph[b], g, 0);
    cudaGraphDestroy(g);
    GPUGA_CUDA(ie);
  }
  std::vector<cudaEvent_t>& ev = B->gen_ev[b];
  while (timed && (int)ev.size() < n + 1) {
    cudaEvent_t e;
    GPUGA_CUDA(cudaEventCreate(&e));
    ev.push_back(e);
  }
  if (timed) GPUGA_CUDA(cudaEventRecord(ev[0], st));
  for (int k = 0; k < n; ++k) {
    if (use_graph) {
      GPUGA_CUDA(cudaGraphLaunch(B->graph[b], st));
    } else {
      GPUGA_TRY(enqueue_generation(B, b, st));
    }
    if (timed) GPUGA_CUDA(cudaEventRecord(ev[k + 1], st));
  }
  for (DeviceGA* s : B->jobs)
    GPUGA_CUDA(cudaMemcpyAsync(s->h_hist[b], s->d_hist[b], sizeof(float) * (size_t)n * (s->d + 1),
                               cudaMemcpyDeviceToHost, st));
  GPUGA_CUDA(cudaEventRecord(B->done[b], st));
  return GPUGA_OK;
}

int ga_batch_wait(GABatch* B, int b) {
  GPUGA_CUDA(cudaEventSynchronize(B->done[b]));
  return GPUGA_OK;
}

int ga_batch_generation_ms(GABatch* B, int b, int n, std::vector<double>* ms) {
  for (int k = 0; k < n; ++k) {
    float t = 0.f;
    GPUGA_CUDA(cudaEventElapsedTime(&t, B->gen_ev[b][k], B->gen_ev[b][k + 1]));
    ms->push_back(t);
  }
  return GPUGA_OK;
}

// Copies the device population and sorted fitness back into the host GA after
// `generations` device generations.
int device_ga_sync_host(GA* ga, DeviceGA* s, int generations, cudaStream_t st) {
  GPUGA_CUDA(cudaMemcpyAsync(ga->population.data(), s->d_pop, sizeof(float) * (size_t)s->P * s->d,
                             cudaMemcpyDeviceToHost, st));
  GPUGA_CUDA(cudaMemcpyAsync(ga->fitness.data(), s->d_fit32, sizeof(float) * s->P, cudaMemcpyDeviceToHost, st));
  GPUGA_CUDA(cudaStreamSynchronize(st));
  ga->generation += generations;
  return GPUGA_OK;
}

int device_ga_advance(Engine* e, GA* ga, DeviceGA** state, int generations, int window,
                      const std::function<void(const std::string&)>& sink) {
  if (e->opt.path != GPUGA_PATH_BATCHED) {
    set_error("the device GA loop runs on the batched path only (engine path %d).", e->opt.path);
    return GPUGA_ERR_ARG;
  }
  const int P = ga->gp.population_size;
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
    GPUGA_TRY(device_ga_setup(*ga, window, &s));
    *state = s;
  }
  window = s->window;
  cudaStream_t st = e->stream;
  Plan* plan = nullptr;
  GPUGA_TRY(plan_get(e, P, &plan));
  LaunchSet* ls = plan->ls.get();
  if (!s->solo || s->solo->ls != ls) {
    GABatch* B = nullptr;
    GPUGA_TRY(ga_batch_build({s}, ls, &B));
    s->solo.reset(B);
  }
  GABatch* B = s->solo.get();
  GPUGA_TRY(launchset_retarget(ls, 0, s->d_pop, s->d_fit64, nullptr, st));
  const bool use_graph = e->opt.use_graph && !ls->timing;
  GPUGA_CUDA(cudaMemcpyAsync(s->d_pop, ga->population.data(), sizeof(float) * (size_t)P * s->d,
                             cudaMemcpyHostToDevice, st));

  // window k runs on buffer k % 2; the host draws window k + 1 while the device runs window k
  const int g_start = ga->generation;
  const int nwin = (generations + window - 1) / window;
  auto wlen = [&](int k) { return std::min(window, generations - k * window); };
  device_ga_draw(*ga, s, 0, g_start, wlen(0));
  GPUGA_TRY(device_ga_upload(s, 0, wlen(0), st));
  GPUGA_TRY(ga_batch_window(B, 0, wlen(0), use_graph, false, st));
  for (int k = 0; k < nwin; ++k) {
    const int b = k & 1;
    if (k + 1 < nwin) {
      // buffer b^1 was last read by window k - 1, which finished before window k started
      if (k >= 1) GPUGA_TRY(ga_batch_wait(B, b ^ 1));
      device_ga_draw(*ga, s, b ^ 1, g_start + (k + 1) * window, wlen(k + 1));
      GPUGA_TRY(device_ga_upload(s, b ^ 1, wlen(k + 1), st));
      GPUGA_TRY(ga_batch_window(B, b ^ 1, wlen(k + 1), use_graph, false, st));
    }
    GPUGA_TRY(ga_batch_wait(B, b));
    std::string lines;
    for (int q = 0; q < wlen(k); ++q) {
      const float* h = s->h_hist[b] + (size_t)q * (s->d + 1);
      lines += ga_output_line(g_start + k * window + q, h[0], h + 1, ga->pmin.data(), ga->pmax.data(), s->d);
    }
    if (sink) sink(lines);
  }
  return device_ga_sync_host(ga, s, generations, st);
}

}  // namespace gpuga
