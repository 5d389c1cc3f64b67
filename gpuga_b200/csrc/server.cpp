// Serving loop: many fitting jobs on one GPU with continuous batching.
//
// Three kinds of work, two host threads.
//
//   Loader thread.  Admits queued jobs in arrival order while the sum of their
//   device footprints stays within the HBM budget and fewer than max_jobs are
//   loading, ready or running: parses nothing (submit did), builds the engine
//   (training set upload, neighbor lists, geometry), the population plan, the
//   host GA (seeded RNG stream) and the device GA buffers, uploads the initial
//   population and hands the job to the scheduler as "ready".  It also frees
//   the device memory of finished jobs and (when nothing is resident, or 64 have
//   accumulated) of retired launch sets, so that no cudaFree (which waits for the
//   device) runs on the scheduler thread or between the windows of a busy period.
//
//   Scheduler thread.  Owns one stream and runs all resident jobs together in
//   windows of up to kWindow generations.  Each generation is one CUDA graph:
//   one launch set (one decode, the shared batched force launches whose work
//   items come from all jobs, one fitness fold) evaluates every job's
//   population, then the batched GA kernels (ga_device.cu) select, cross over
//   and mutate every job's population from random choices the host drew for
//   the window in advance -- no population or fitness crosses PCIe between
//   generations.  Windows are pipelined: while window k runs, the scheduler
//   decides window k + 1's members (jobs that still have generations left plus
//   every ready job), rebuilds the launch set and GA batch if they changed,
//   draws and uploads the next plans into the other plan buffer and enqueues
//   window k + 1 behind window k; only then does it wait for window k and
//   harvest its generation histories.
//
// Work items of different jobs never share a CTA and all reductions are
// fixed-order, so a job's trajectory is identical alone and in any mix.
// Latency is reported three ways: the device time of each generation of all
// resident jobs; per job and generation the wall-clock time between the job's
// successive window harvests divided by the window's generations (every stall
// of a running job -- rebuilds, admissions of others, frees -- included; a
// job's first window counts from its enqueue); and per job the time from
// submission to the harvest of its first window (queueing, setup, the wait for
// the window in flight and the first window itself).  There is no counterpart
// in the reference, which fits one potential per process (main.cu:25-55).
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
  int gens_queued = 0;              // generations enqueued on the device (>= ga.generation)
  std::vector<float> best;
  std::vector<float> elite;
  bool cancel_requested = false;
  Clock::time_point t_submit, t_start, t_end, t_mark;
};

// Admission estimate of a training set's device footprint: per atom ~64 B,
// per bond ~80 B (FP64 + FP32 geometry, indices, RI terms), per three-body
// term 4 B, with the neighbor count estimated from the cell density.
size_t estimate_bytes(const PotentialSpec& spec, const TrainingSet& ts, int P) {
  double bonds = 0, trip = 0, force_bonds = 0;
  const double rc = spec.cutoff;
  for (int c = 0; c < ts.Nc; ++c) {
    const float* h = ts.h.data() + 18 * (size_t)c;
    const double vol = std::fabs((double)h[0] * (h[4] * h[8] - h[5] * h[7]) + (double)h[1] * (h[5] * h[6] - h[3] * h[8]) +
                                 (double)h[2] * (h[3] * h[7] - h[4] * h[6]));
    const double na = ts.Na[c];
    double z = vol > 0 ? na / vol * 4.18879 * rc * rc * rc : na - 1;
    z = std::min(z, na - 1.0);
    bonds += na * z;
    if (c < ts.Nc_force) force_bonds += na * z;
    trip += na * z * z;
  }
  const bool tersoff = spec.type == 1 || spec.type == 2;
  double bytes = 64.0 * ts.N + 88.0 * bonds + (tersoff ? 4.0 * trip : 0.0);
  bytes += (double)P * ts.Nc * kResK * 8.0 + (double)P * (spec.num_vars + 40) * 8.0;
  if (spec.type == 3) bytes += 4.0 * P * force_bonds;  // NN2B force items' per-pair scratch
  return (size_t)(1.25 * bytes) + (8u << 20);
}

// A resident set's shared launches and GA batch.
struct Batch {
  std::vector<Job*> jobs;
  std::unique_ptr<LaunchSet> ls;
  std::unique_ptr<GABatch, void (*)(GABatch*)> gab{nullptr, ga_batch_free};
};

// A window enqueued on the scheduler's stream.
struct Window {
  Batch* batch = nullptr;
  int b = 0;   // plan buffer
  int n = 0;   // generations
};

double percentile(std::vector<double> t, double q) {
  if (t.empty()) return 0.0;
  std::sort(t.begin(), t.end());
  const double pos = q * (t.size() - 1);
  const size_t lo = (size_t)std::floor(pos), hi = (size_t)std::ceil(pos);
  return t[lo] + (t[hi] - t[lo]) * (pos - lo);
}

}  // namespace

// Generations per scheduling window (admission, retirement and cancellation
// happen at window boundaries).
constexpr int kWindow = 8;
constexpr size_t kRetiredBacklog = 64;  // retired launch sets kept before the loader frees them

struct gpuga_server {
  int device = 0;
  double budget = 0;
  int max_jobs = 0;
  std::mutex mu;
  std::condition_variable cv;         // wakes the scheduler
  std::condition_variable loader_cv;  // wakes the loader
  std::condition_variable idle_cv;    // wakes drain()
  std::deque<Job*> queue;             // submitted, not yet taken by the loader
  int loading = 0;                    // jobs the loader is setting up
  std::vector<Job*> ready;            // set up, joining at the next window boundary
  std::vector<Job*> running;          // members of the last enqueued window
  std::vector<Job*> retiring;         // left with the window in flight, retired after it
  std::vector<Job*> graveyard;        // finished jobs whose device memory the loader frees
  std::vector<std::unique_ptr<Batch>> retired;  // launch sets no window uses any more
  std::map<int, std::unique_ptr<Job>> jobs;
  int next_id = 1;
  bool stop = false;
  bool hold = false;                  // gpuga_server_hold: no new windows start
  size_t bytes_in_use = 0;
  std::thread worker, loader;
  cudaStream_t st = nullptr, st_copy = nullptr;
  // statistics
  std::vector<double> tick_ms;   // device time of each generation of all resident jobs
  std::vector<double> wall_ms;   // per job and generation: wall-clock time, stalls included
  std::vector<double> first_ms;  // per job: submission to the harvest of its first window (wall clock)
  long batches = 0, finished = 0;
  double evals = 0, busy_s = 0;
  int peak_resident = 0;
  int worker_status = GPUGA_OK;

  void run();
  void load();
  int setup(Job* j);
  int build_batch(const std::vector<Job*>& members, std::unique_ptr<Batch>* out);
  int harvest(const Window& w);
  void finish(Job* j, int state, int status, const char* msg);
  int resident() const { return loading + (int)ready.size() + (int)running.size(); }
};

// Marks a job finished (mu held); its device memory goes to the loader's graveyard.
void gpuga_server::finish(Job* j, int state, int status, const char* msg) {
  j->state = state;
  j->status = status;
  if (msg) j->error = msg;
  j->t_end = Clock::now();
  bytes_in_use -= std::min(bytes_in_use, j->bytes);
  if (state == kDone) ++finished;
  graveyard.push_back(j);
  loader_cv.notify_all();
  cv.notify_all();
  idle_cv.notify_all();
}

// Loader thread work for one admitted job (mu not held).
int gpuga_server::setup(Job* j) {
  if (!j->engine) {
    gpuga_options opt;
    gpuga_default_options(&opt);
    opt.device = device;
    // the fixed tile rule: trial launches timed on a GPU that runs other jobs' windows would
    // measure the contention, not the tiles (every tile gives the same results)
    opt.tiles = kTileDefault;
    Engine* e = nullptr;
    GPUGA_TRY(engine_create(j->spec, std::move(j->ts), opt, &e));
    j->engine = e;
  }
  Plan* p = nullptr;
  GPUGA_TRY(plan_build(j->engine, j->gp.population_size, &p));
  j->plan_owner.reset(p);
  j->plan = p;
  GPUGA_TRY(j->ga.init(j->engine->spec.num_vars, j->engine->spec.pmin.data(), j->engine->spec.pmax.data(), j->gp,
                       j->seed));
  DeviceGA* g = nullptr;
  GPUGA_TRY(device_ga_setup(j->ga, kWindow, &g));
  j->dga.reset(g);
  GPUGA_CUDA(cudaMemcpy(device_ga_population(g), j->ga.population.data(), sizeof(float) * j->ga.population.size(),
                        cudaMemcpyHostToDevice));
  return GPUGA_OK;
}

void gpuga_server::load() {
  cudaSetDevice(device);
  std::unique_lock<std::mutex> lock(mu);
  while (true) {
    // Retired launch sets (a few MB each) are freed only when the scheduler has nothing resident
    // or a backlog has built up: every cudaFree waits for the device to drain, and one per
    // admission would stall the windows in flight.  Finished jobs are freed at once (their
    // memory goes back to the admission budget).
    const bool idle = running.empty() && ready.empty() && loading == 0;
    const bool free_retired = !retired.empty() && (idle || stop || retired.size() >= kRetiredBacklog);
    if (!graveyard.empty() || free_retired) {
      std::vector<Job*> dead;
      dead.swap(graveyard);
      std::vector<std::unique_ptr<Batch>> old;
      if (free_retired) old.swap(retired);
      lock.unlock();
      old.clear();
      for (Job* j : dead) {
        j->dga.reset();
        j->plan_owner.reset();
        j->plan = nullptr;
        if (j->engine && !j->shared) delete j->engine;
        j->engine = nullptr;
      }
      lock.lock();
      continue;
    }
    if (!queue.empty() && resident() < max_jobs) {
      Job* j = queue.front();
      if (j->cancel_requested) {
        queue.pop_front();
        finish(j, kCancelled, GPUGA_ERR_CANCELLED, "cancelled before it started");
        continue;
      }
      if ((double)(bytes_in_use + j->bytes) <= budget || resident() == 0) {
        queue.pop_front();
        bytes_in_use += j->bytes;
        ++loading;
        lock.unlock();
        const int s = setup(j);
        lock.lock();
        --loading;
        if (s != GPUGA_OK) {
          finish(j, kFailed, s, last_error());
        } else if (j->cancel_requested) {
          finish(j, kCancelled, GPUGA_ERR_CANCELLED, "cancelled before it started");
        } else {
          j->state = kRunning;
          j->t_start = j->t_mark = Clock::now();
          ready.push_back(j);
          cv.notify_all();
        }
        continue;
      }
    }
    if (stop && queue.empty()) break;
    loader_cv.wait(lock);
  }
}

// Launch set and GA batch of a resident set (host work plus small uploads; no wait on the device).
int gpuga_server::build_batch(const std::vector<Job*>& members, std::unique_ptr<Batch>* out) {
  std::unique_ptr<Batch> B(new Batch);
  B->jobs = members;
  std::vector<std::pair<Engine*, Plan*>> v;
  std::vector<std::pair<const float*, double*>> targets;
  std::vector<DeviceGA*> g;
  for (Job* j : members) {
    v.push_back({j->engine, j->plan});
    targets.push_back({device_ga_population(j->dga.get()), device_ga_fitness64(j->dga.get())});
    g.push_back(j->dga.get());
  }
  B->ls.reset(new LaunchSet);
  GPUGA_TRY(launchset_build(v, B->ls.get(), &targets));
  GABatch* gb = nullptr;
  GPUGA_TRY(ga_batch_build(g, B->ls.get(), &gb));
  B->gab.reset(gb);
  *out = std::move(B);
  return GPUGA_OK;
}

// Waits for window w and records its results (mu not held; the jobs' run state is the
// scheduler's own).
int gpuga_server::harvest(const Window& w) {
  GPUGA_TRY(ga_batch_wait(w.batch->gab.get(), w.b));
  const auto now = Clock::now();
  std::vector<double> ms;
  GPUGA_TRY(ga_batch_generation_ms(w.batch->gab.get(), w.b, w.n, &ms));
  std::lock_guard<std::mutex> g(mu);
  for (Job* j : w.batch->jobs) {
    const float* h = device_ga_history(j->dga.get(), w.b);
    for (int q = 0; q < w.n; ++q) j->best.push_back(h[(size_t)q * (j->ga.d + 1)]);
    if (j->ga.generation == 0)
      first_ms.push_back(std::chrono::duration<double, std::milli>(now - j->t_submit).count());
    j->ga.generation += w.n;
    evals += (double)j->plan->P * j->engine->d.N * w.n;
    const double per_gen = std::chrono::duration<double, std::milli>(now - j->t_mark).count() / w.n;
    for (int q = 0; q < w.n; ++q) wall_ms.push_back(per_gen);
    j->t_mark = now;
  }
  for (double t : ms) tick_ms.push_back(t);
  batches += w.n;
  return GPUGA_OK;
}

void gpuga_server::run() {
  cudaSetDevice(device);
  if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&st_copy, cudaStreamNonBlocking) != cudaSuccess) {
    std::lock_guard<std::mutex> g(mu);
    worker_status = GPUGA_ERR_CUDA;
    idle_cv.notify_all();
    return;
  }
  std::unique_ptr<Batch> cur_batch;  // the launch set of the last enqueued window
  Window cur;                        // in flight (cur.batch == nullptr: none)
  Clock::time_point busy_since{};
  int status = GPUGA_OK;
  std::unique_lock<std::mutex> lock(mu);
  while (true) {
    // members of the next window: jobs with generations left after the one in flight, then
    // every ready job (as many as the slots allow; the loader respects max_jobs already)
    std::vector<Job*> next, leaving;
    for (Job* j : running) {
      if (status == GPUGA_OK && !j->cancel_requested && j->gens_queued < j->gens_total) next.push_back(j);
      else leaving.push_back(j);
    }
    if (status == GPUGA_OK) {
      for (Job* j : ready) next.push_back(j);
      ready.clear();
    }
    if ((next.empty() || hold) && !cur.batch && leaving.empty()) {
      running = next;  // held: loaded jobs wait here, no window starts
      if (next.empty() && cur_batch) retired.push_back(std::move(cur_batch));
      loader_cv.notify_all();
      idle_cv.notify_all();
      if (stop && queue.empty() && loading == 0 && ready.empty() && running.empty()) break;
      cv.wait(lock);
      continue;
    }
    const bool enqueue = !hold;
    running = next;  // visible to drain() and poll() while the lock is released
    retiring = leaving;
    peak_resident = std::max(peak_resident, (int)next.size());
    lock.unlock();
    if (busy_since == Clock::time_point{} && !next.empty() && enqueue) busy_since = Clock::now();
    // enqueue window k + 1 behind window k
    Window nxt;
    std::unique_ptr<Batch> next_batch;
    if (!next.empty() && enqueue) {
      int s = GPUGA_OK;
      Batch* use = cur_batch.get();
      if (!cur_batch || cur_batch->jobs != next) {
        s = build_batch(next, &next_batch);
        use = next_batch.get();
      }
      int n = kWindow;
      for (Job* j : next) n = std::min(n, j->gens_total - j->gens_queued);
      const int b = cur.batch ? cur.b ^ 1 : 0;
      for (Job* j : next) {
        if (s != GPUGA_OK) break;
        device_ga_draw(j->ga, j->dga.get(), b, j->gens_queued, n);
        s = device_ga_upload(j->dga.get(), b, n, st);
      }
      if (s == GPUGA_OK) s = ga_batch_window(use->gab.get(), b, n, true, true, st);
      if (s == GPUGA_OK) {
        nxt = Window{use, b, n};
        const auto t_enq = Clock::now();
        for (Job* j : next) {
          if (j->gens_queued == 0) j->t_mark = t_enq;  // its generations start behind window k
          j->gens_queued += n;
        }
      } else {
        status = s;
      }
    }
    // then wait for window k
    if (cur.batch && status == GPUGA_OK) status = harvest(cur);
    if ((!nxt.batch || status != GPUGA_OK) && busy_since != Clock::time_point{}) {
      // nothing follows: the busy period ends with window k
      busy_s += std::chrono::duration<double>(Clock::now() - busy_since).count();
      busy_since = Clock::time_point{};
    }
    lock.lock();
    // retire the jobs that left with window k (finished, cancelled or failed)
    for (Job* j : leaving) {
      if (status != GPUGA_OK) {
        finish(j, kFailed, status, last_error());
      } else if (j->ga.generation >= j->gens_total) {
        // the final population (row 0 = the last generation's elite) comes back on a second
        // stream: no later window touches this job's buffers
        lock.unlock();
        const int ss = device_ga_sync_host(&j->ga, j->dga.get(), 0, st_copy);
        lock.lock();
        if (ss != GPUGA_OK) {
          finish(j, kFailed, ss, last_error());
          continue;
        }
        j->elite.assign(j->ga.population.begin(), j->ga.population.begin() + j->ga.d);
        finish(j, kDone, GPUGA_OK, nullptr);
      } else {
        finish(j, kCancelled, GPUGA_ERR_CANCELLED, "cancelled");
      }
    }
    if (status != GPUGA_OK) {
      worker_status = status;
      for (Job* j : next) finish(j, kFailed, status, last_error());
      next.clear();
      nxt = Window{};
    }
    if (next_batch) {
      if (cur_batch) retired.push_back(std::move(cur_batch));
      cur_batch = std::move(next_batch);
      loader_cv.notify_all();
    }
    running = next;
    retiring.clear();
    cur = nxt;
  }
  lock.unlock();
  cur_batch.reset();
  cudaStreamDestroy(st);
  cudaStreamDestroy(st_copy);
  st = st_copy = nullptr;
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
  s->loader = std::thread([s] { s->load(); });
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
  s->loader_cv.notify_all();
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
    progress[0] = j->state == kQueued ? 0 : j->ga.generation;  // cancelled / failed: generations run
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
  s->loader_cv.notify_all();
  return GPUGA_OK;
}

int gpuga_server_hold(gpuga_server* s, int on) {
  if (!s) {
    set_error("gpuga_server_hold: null server");
    return GPUGA_ERR_ARG;
  }
  std::lock_guard<std::mutex> g(s->mu);
  s->hold = on != 0;
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
  auto idle = [&] {
    return s->queue.empty() && s->loading == 0 && s->ready.empty() && s->running.empty() && s->retiring.empty();
  };
  while (!idle() && s->worker_status == GPUGA_OK) {
    if (s->idle_cv.wait_until(lock, deadline) == std::cv_status::timeout && !idle()) {
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

int gpuga_server_stats(gpuga_server* s, double* out, int n) {
  if (!s || !out || n < 0) {
    set_error("gpuga_server_stats: invalid argument");
    return GPUGA_ERR_ARG;
  }
  std::lock_guard<std::mutex> g(s->mu);
  const double v[] = {(double)s->batches,
                      (double)s->finished,
                      percentile(s->tick_ms, 0.50),
                      percentile(s->tick_ms, 0.99),
                      s->busy_s > 0 ? s->evals / s->busy_s : 0.0,
                      (double)s->bytes_in_use,
                      (double)s->peak_resident,
                      s->evals,
                      percentile(s->wall_ms, 0.50),
                      percentile(s->wall_ms, 0.99),
                      s->busy_s,
                      percentile(s->first_ms, 0.50),
                      percentile(s->first_ms, 0.99)};
  const int m = std::min(n, (int)(sizeof(v) / sizeof(v[0])));
  for (int k = 0; k < m; ++k) out[k] = v[k];
  return GPUGA_OK;
}

int gpuga_server_destroy(gpuga_server* s) {
  if (!s) return GPUGA_OK;
  {
    std::lock_guard<std::mutex> g(s->mu);
    s->stop = true;
    s->hold = false;
    for (Job* j : s->queue) j->cancel_requested = true;
    for (Job* j : s->running) j->cancel_requested = true;
    for (Job* j : s->ready) j->cancel_requested = true;
    s->cv.notify_all();
    s->loader_cv.notify_all();
  }
  if (s->worker.joinable()) s->worker.join();
  {
    std::lock_guard<std::mutex> g(s->mu);
    s->loader_cv.notify_all();
  }
  if (s->loader.joinable()) s->loader.join();
  for (auto& kv : s->jobs)
    if (kv.second->engine && !kv.second->shared) delete kv.second->engine;
  delete s;
  return GPUGA_OK;
}

}  // extern "C"
