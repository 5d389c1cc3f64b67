// Serving loop: many fitting jobs on one GPU with continuous batching.
//
// A scheduler thread owns the device.  Jobs are admitted in arrival order as
// long as the sum of their device footprints stays within the HBM budget and
// the number of resident jobs is below max_jobs; every resident job keeps its
// training set, population and GA buffers and per-(individual, configuration)
// results on the GPU.  The scheduler advances all resident jobs together in
// windows of up to kWindow generations.  Each generation is one CUDA graph: a
// single launch set (one decode, the shared batched force launches whose work
// items come from all jobs, one fitness fold) evaluates every job's
// population, then the batched GA kernels (ga_device.cu) select, cross over
// and mutate every job's population from random choices the host drew for the
// window in advance -- no population or fitness crosses PCIe between
// generations.  Jobs that arrive while others run join at the next window
// boundary; finished or cancelled jobs leave and free their memory.  Work
// items of different jobs never share a CTA and all reductions are
// fixed-order, so a job's trajectory is identical alone and in any mix.
// There is no counterpart in the reference, which fits one potential per
// process (main.cu:25-55).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>

#include "engine.hpp"
#include "ga.hpp"

using namespace gpuga;

struct gpuga_engine {
  Engine* e;
};

namespace {

using Clock = std::chrono::steady_clock;

enum JobState { kQueued = 0, kRunning = 1, kDone = 2, kFailed = 3, kCancelled = 4 };

struct Job {
  int id = 0;
  int state = kQueued;
  int status = GPUGA_OK;
  std::string error;
  // inputs
  std::string dir;
  PotentialSpec spec;
  TrainingSet ts;
  GAParams gp;
  unsigned seed = 0;
  Engine* engine = nullptr;  // owned unless `shared`
  bool shared = false;
  size_t bytes = 0;          // admission estimate
  // run state
  Plan* plan = nullptr;             // the job's own buffers (owned by plan_owner)
  std::unique_ptr<Plan> plan_owner;
  GA ga;                            // host side: random stream and plan draws
  std::unique_ptr<DeviceGA, void (*)(DeviceGA*)> dga{nullptr, device_ga_free};
  int gens_total = 0;
  std::vector<float> best;
  std::vector<float> elite;
  bool cancel_requested = false;
  Clock::time_point t_submit, t_start, t_end;
};

// Admission estimate of a training set's device footprint: per atom ~64 B,
// per bond ~80 B (FP64 + FP32 geometry, indices, RI terms), per three-body
// term 4 B, with the neighbor count estimated from the cell density.
size_t estimate_bytes(const PotentialSpec& spec, const TrainingSet& ts, int P) {
  double bonds = 0, trip = 0;
  const double rc = spec.cutoff;
  for (int c = 0; c < ts.Nc; ++c) {
    const float* h = ts.h.data() + 18 * (size_t)c;
    const double vol = std::fabs((double)h[0] * (h[4] * h[8] - h[5] * h[7]) + (double)h[1] * (h[5] * h[6] - h[3] * h[8]) +
                                 (double)h[2] * (h[3] * h[7] - h[4] * h[6]));
    const double na = ts.Na[c];
    double z = vol > 0 ? na / vol * 4.18879 * rc * rc * rc : na - 1;
    z = std::min(z, na - 1.0);
    bonds += na * z;
    trip += na * z * z;
  }
  const bool tersoff = spec.type == 1 || spec.type == 2;
  double bytes = 64.0 * ts.N + 80.0 * bonds + (tersoff ? 4.0 * trip : 0.0);
  bytes += (double)P * ts.Nc * kResK * 8.0 + (double)P * (spec.num_vars + 40) * 8.0;
  return (size_t)(1.25 * bytes) + (8u << 20);
}

}  // namespace

// Generations per scheduling window (admission, retirement and cancellation
// happen at window boundaries).
constexpr int kWindow = 8;

struct gpuga_server {
  int device = 0;
  double budget = 0;
  int max_jobs = 0;
  std::mutex mu;
  std::condition_variable cv;       // wakes the scheduler
  std::condition_variable idle_cv;  // wakes drain()
  std::deque<Job*> queue;
  std::vector<Job*> running;
  std::map<int, std::unique_ptr<Job>> jobs;
  int next_id = 1;
  bool stop = false;
  size_t bytes_in_use = 0;
  std::thread worker;
  cudaStream_t st = nullptr;
  std::unique_ptr<LaunchSet> ls;
  std::unique_ptr<GABatch, void (*)(GABatch*)> gab{nullptr, ga_batch_free};
  std::vector<int> ls_ids;
  // statistics
  std::vector<double> tick_ms;  // device time of each generation (all resident jobs)
  long batches = 0, finished = 0;
  double evals = 0, busy_s = 0;
  int peak_resident = 0;
  int worker_status = GPUGA_OK;

  void run();
  bool admit_locked(std::unique_lock<std::mutex>& lock);
  int window();
  void finish(Job* j, int state, int status, const char* msg);
};

void gpuga_server::finish(Job* j, int state, int status, const char* msg) {
  j->state = state;
  j->status = status;
  if (msg) j->error = msg;
  j->t_end = Clock::now();
  j->dga.reset();
  j->plan_owner.reset();
  j->plan = nullptr;
  if (j->engine && !j->shared) delete j->engine;
  j->engine = nullptr;
  bytes_in_use -= std::min(bytes_in_use, j->bytes);
  if (state == kDone) ++finished;
}

// Moves queued jobs into the resident set while they fit (mu held).
bool gpuga_server::admit_locked(std::unique_lock<std::mutex>& lock) {
  bool changed = false;
  while (!queue.empty() && (int)running.size() < max_jobs) {
    Job* j = queue.front();
    if (j->cancel_requested) {
      queue.pop_front();
      finish(j, kCancelled, GPUGA_ERR_CANCELLED, "cancelled before it started");
      changed = true;
      continue;
    }
    if ((double)(bytes_in_use + j->bytes) > budget && !running.empty()) break;  // wait for memory
    queue.pop_front();
    bytes_in_use += j->bytes;
    j->state = kRunning;
    j->t_start = Clock::now();
    lock.unlock();
    int s = GPUGA_OK;
    if (!j->engine) {
      gpuga_options opt;
      gpuga_default_options(&opt);
      opt.device = device;
      Engine* e = nullptr;
      s = engine_create(j->spec, std::move(j->ts), opt, &e);
      if (s == GPUGA_OK) j->engine = e;
    }
    if (s == GPUGA_OK) {
      Plan* p = nullptr;
      s = plan_build(j->engine, j->gp.population_size, &p);
      j->plan_owner.reset(p);
      j->plan = p;
    }
    if (s == GPUGA_OK)
      s = j->ga.init(j->engine->spec.num_vars, j->engine->spec.pmin.data(), j->engine->spec.pmax.data(), j->gp,
                     j->seed);
    if (s == GPUGA_OK) {
      DeviceGA* g = nullptr;
      s = device_ga_setup(j->ga, kWindow, &g);
      j->dga.reset(g);
    }
    if (s == GPUGA_OK) {
      const cudaError_t ce = cudaMemcpy(device_ga_population(j->dga.get()), j->ga.population.data(),
                                        sizeof(float) * j->ga.population.size(), cudaMemcpyHostToDevice);
      if (ce != cudaSuccess) s = cuda_status(ce, "cudaMemcpy", __FILE__, __LINE__);
    }
    lock.lock();
    if (s != GPUGA_OK) {
      finish(j, kFailed, s, last_error());
    } else {
      running.push_back(j);
      peak_resident = std::max(peak_resident, (int)running.size());
    }
    changed = true;
  }
  return changed;
}

// Up to kWindow generations of every resident job: shared fitness launches and
// batched GA kernels per generation, one CUDA graph, no host round trip.
int gpuga_server::window() {
  std::vector<int> ids;
  for (Job* j : running) ids.push_back(j->id);
  if (!ls || ids != ls_ids) {
    gab.reset();
    std::vector<std::pair<Engine*, Plan*>> v;
    std::vector<DeviceGA*> g;
    for (Job* j : running) {
      v.push_back({j->engine, j->plan});
      g.push_back(j->dga.get());
    }
    ls.reset(new LaunchSet);
    GPUGA_TRY(launchset_build(v, ls.get()));
    for (size_t k = 0; k < running.size(); ++k)
      GPUGA_TRY(launchset_retarget(ls.get(), (int)k, device_ga_population(g[k]), device_ga_fitness64(g[k]), nullptr,
                                   st));
    GABatch* b = nullptr;
    GPUGA_TRY(ga_batch_build(g, ls.get(), &b));
    gab.reset(b);
    ls_ids = ids;
  }
  int n = kWindow;
  for (Job* j : running) n = std::min(n, j->gens_total - j->ga.generation);
  if (n <= 0) return GPUGA_OK;
  const auto t0 = Clock::now();
  for (Job* j : running) {
    device_ga_draw(j->ga, j->dga.get(), 0, j->ga.generation, n);
    GPUGA_TRY(device_ga_upload(j->dga.get(), 0, n, st));
  }
  GPUGA_TRY(ga_batch_window(gab.get(), 0, n, true, true, st));
  GPUGA_TRY(ga_batch_wait(gab.get(), 0));
  std::vector<double> ms;
  GPUGA_TRY(ga_batch_generation_ms(gab.get(), n, &ms));
  for (Job* j : running) {
    const float* h = device_ga_history(j->dga.get(), 0);
    for (int q = 0; q < n; ++q) j->best.push_back(h[(size_t)q * (j->ga.d + 1)]);
    j->ga.generation += n;
    evals += (double)j->plan->P * j->engine->d.N * n;
  }
  // latency: device time of each generation; throughput: wall time of the window (plan draws,
  // uploads and the history read-back included)
  for (double t : ms) tick_ms.push_back(t);
  busy_s += std::chrono::duration<double>(Clock::now() - t0).count();
  batches += n;
  return GPUGA_OK;
}

void gpuga_server::run() {
  cudaSetDevice(device);
  if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
    std::lock_guard<std::mutex> g(mu);
    worker_status = GPUGA_ERR_CUDA;
    idle_cv.notify_all();
    return;
  }
  std::unique_lock<std::mutex> lock(mu);
  while (true) {
    admit_locked(lock);
    if (running.empty()) {
      idle_cv.notify_all();
      if (stop) break;
      cv.wait(lock);
      continue;
    }
    lock.unlock();
    const int s = window();
    lock.lock();
    // retire finished, failed and cancelled jobs at the window boundary
    std::vector<Job*> keep;
    for (Job* j : running) {
      if (s != GPUGA_OK) {
        finish(j, kFailed, s, last_error());
      } else if (j->cancel_requested) {
        finish(j, kCancelled, GPUGA_ERR_CANCELLED, "cancelled");
      } else if (j->ga.generation >= j->gens_total) {
        // the final population (row 0 = the last generation's elite) comes back once
        const int ss = device_ga_sync_host(&j->ga, j->dga.get(), 0, st);
        if (ss != GPUGA_OK) {
          finish(j, kFailed, ss, last_error());
          continue;
        }
        j->elite.assign(j->ga.population.begin(), j->ga.population.begin() + j->ga.d);
        finish(j, kDone, GPUGA_OK, nullptr);
      } else {
        keep.push_back(j);
      }
    }
    running.swap(keep);
    if (s != GPUGA_OK) worker_status = s;
  }
  gab.reset();
  ls.reset();
  cudaStreamDestroy(st);
  st = nullptr;
}

extern "C" {

int gpuga_server_create(int device, double hbm_budget_bytes, int max_jobs, gpuga_server** out) {
  if (!out || hbm_budget_bytes <= 0 || max_jobs < 1) {
    set_error("gpuga_server_create: invalid argument");
    return GPUGA_ERR_ARG;
  }
  int ndev = 0;
  GPUGA_CUDA(cudaGetDeviceCount(&ndev));
  if (device < 0 || device >= ndev) {
    set_error("device %d not available.", device);
    return GPUGA_ERR_ARG;
  }
  gpuga_server* s = new gpuga_server;
  s->device = device;
  s->budget = hbm_budget_bytes;
  s->max_jobs = max_jobs;
  s->worker = std::thread([s] { s->run(); });
  *out = s;
  return GPUGA_OK;
}

static int enqueue_job(gpuga_server* s, std::unique_ptr<Job> j, int* job_id) {
  std::lock_guard<std::mutex> g(s->mu);
  if ((double)j->bytes > s->budget) {
    set_error("job needs about %zu bytes of device memory, above the server budget of %.0f bytes.", j->bytes,
              s->budget);
    return GPUGA_ERR_BUDGET;
  }
  j->id = s->next_id++;
  j->t_submit = Clock::now();
  Job* raw = j.get();
  s->jobs[raw->id] = std::move(j);
  s->queue.push_back(raw);
  if (job_id) *job_id = raw->id;
  s->cv.notify_all();
  return GPUGA_OK;
}

int gpuga_server_submit(gpuga_server* s, const char* dir, unsigned seed, int generations, int* job_id) {
  if (!s || !dir) {
    set_error("gpuga_server_submit: null argument");
    return GPUGA_ERR_ARG;
  }
  std::unique_ptr<Job> j(new Job);
  j->dir = dir;
  j->seed = seed;
  int st = read_potential_in(dir, &j->spec);
  if (st == GPUGA_OK) st = read_train_in(dir, &j->ts);
  if (st == GPUGA_OK) st = read_ga_in(dir, &j->gp);
  if (st != GPUGA_OK) return st;
  j->gens_total = generations > 0 ? generations : j->gp.maximum_generation;
  if (generations > 0 && j->gp.maximum_generation < generations) j->gp.maximum_generation = generations;
  j->bytes = estimate_bytes(j->spec, j->ts, j->gp.population_size);
  return enqueue_job(s, std::move(j), job_id);
}

int gpuga_server_submit_engine(gpuga_server* s, gpuga_engine* e, int population_size, int parent_number,
                               float mutation_rate, int generations, unsigned seed, int* job_id) {
  if (!s || !e || population_size < 2 || generations < 1) {
    set_error("gpuga_server_submit_engine: invalid argument");
    return GPUGA_ERR_ARG;
  }
  if (e->e->device != s->device) {
    set_error("the engine lives on device %d, the server on %d.", e->e->device, s->device);
    return GPUGA_ERR_ARG;
  }
  std::unique_ptr<Job> j(new Job);
  j->engine = e->e;
  j->shared = true;
  j->seed = seed;
  j->gp.population_size = population_size;
  j->gp.parent_number = parent_number;
  j->gp.mutation_rate = mutation_rate;
  j->gp.maximum_generation = generations;
  j->gens_total = generations;
  j->bytes = (size_t)((double)population_size * e->e->d.Nc * kResK * 8.0 +
                      (double)population_size * (e->e->d.num_vars + 40) * 8.0) + (1u << 20);
  return enqueue_job(s, std::move(j), job_id);
}

int gpuga_server_poll(gpuga_server* s, int job_id, int* progress) {
  if (!s) {
    set_error("gpuga_server_poll: null server");
    return GPUGA_ERR_ARG;
  }
  std::lock_guard<std::mutex> g(s->mu);
  auto it = s->jobs.find(job_id);
  if (it == s->jobs.end()) {
    set_error("unknown job %d.", job_id);
    return GPUGA_ERR_ARG;
  }
  Job* j = it->second.get();
  if (progress) {
    progress[0] = j->state == kRunning || j->state == kDone ? j->ga.generation : 0;
    progress[1] = j->gens_total;
    progress[2] = j->state;
  }
  if (j->state == kQueued || j->state == kRunning) return GPUGA_ERR_NOT_READY;
  if (j->status != GPUGA_OK) set_error("job %d: %s", job_id, j->error.c_str());
  return j->status;
}

int gpuga_server_result(gpuga_server* s, int job_id, float* best_out, float* elite01_out) {
  if (!s) {
    set_error("gpuga_server_result: null server");
    return GPUGA_ERR_ARG;
  }
  std::lock_guard<std::mutex> g(s->mu);
  auto it = s->jobs.find(job_id);
  if (it == s->jobs.end()) {
    set_error("unknown job %d.", job_id);
    return GPUGA_ERR_ARG;
  }
  Job* j = it->second.get();
  if (j->state != kDone) {
    set_error("job %d has not finished.", job_id);
    return j->state == kQueued || j->state == kRunning ? GPUGA_ERR_NOT_READY : j->status;
  }
  if (best_out) memcpy(best_out, j->best.data(), sizeof(float) * j->best.size());
  if (elite01_out) memcpy(elite01_out, j->elite.data(), sizeof(float) * j->elite.size());
  return GPUGA_OK;
}

int gpuga_server_cancel(gpuga_server* s, int job_id) {
  if (!s) {
    set_error("gpuga_server_cancel: null server");
    return GPUGA_ERR_ARG;
  }
  std::lock_guard<std::mutex> g(s->mu);
  auto it = s->jobs.find(job_id);
  if (it == s->jobs.end()) {
    set_error("unknown job %d.", job_id);
    return GPUGA_ERR_ARG;
  }
  it->second->cancel_requested = true;
  s->cv.notify_all();
  return GPUGA_OK;
}

int gpuga_server_drain(gpuga_server* s, double timeout_s) {
  if (!s) {
    set_error("gpuga_server_drain: null server");
    return GPUGA_ERR_ARG;
  }
  std::unique_lock<std::mutex> lock(s->mu);
  const auto deadline = Clock::now() + std::chrono::duration_cast<Clock::duration>(
                                           std::chrono::duration<double>(timeout_s > 0 ? timeout_s : 1e9));
  while (!(s->queue.empty() && s->running.empty()) && s->worker_status == GPUGA_OK) {
    if (s->idle_cv.wait_until(lock, deadline) == std::cv_status::timeout &&
        !(s->queue.empty() && s->running.empty())) {
      set_error("gpuga_server_drain: jobs still running after %.1f s", timeout_s);
      return GPUGA_ERR_TIMEOUT;
    }
  }
  if (s->worker_status != GPUGA_OK) {
    set_error("the scheduler stopped with status %d", s->worker_status);
    return s->worker_status;
  }
  return GPUGA_OK;
}

int gpuga_server_stats(gpuga_server* s, double* out) {
  if (!s || !out) {
    set_error("gpuga_server_stats: null argument");
    return GPUGA_ERR_ARG;
  }
  std::lock_guard<std::mutex> g(s->mu);
  std::vector<double> t = s->tick_ms;
  std::sort(t.begin(), t.end());
  auto pct = [&](double q) {
    if (t.empty()) return 0.0;
    const double pos = q * (t.size() - 1);
    const size_t lo = (size_t)std::floor(pos), hi = (size_t)std::ceil(pos);
    return t[lo] + (t[hi] - t[lo]) * (pos - lo);
  };
  out[0] = (double)s->batches;
  out[1] = (double)s->finished;
  out[2] = pct(0.50);
  out[3] = pct(0.99);
  out[4] = s->busy_s > 0 ? s->evals / s->busy_s : 0.0;
  out[5] = (double)s->bytes_in_use;
  out[6] = (double)s->peak_resident;
  out[7] = s->evals;
  return GPUGA_OK;
}

int gpuga_server_destroy(gpuga_server* s) {
  if (!s) return GPUGA_OK;
  {
    std::lock_guard<std::mutex> g(s->mu);
    s->stop = true;
    for (Job* j : s->queue) j->cancel_requested = true;
    for (Job* j : s->running) j->cancel_requested = true;
    s->cv.notify_all();
  }
  if (s->worker.joinable()) s->worker.join();
  for (auto& kv : s->jobs)
    if (kv.second->engine && !kv.second->shared) delete kv.second->engine;
  delete s;
  return GPUGA_OK;
}

}  // extern "C"
