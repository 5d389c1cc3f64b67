// extern "C" entry points of libgpuga_b200.so (declared in include/gpuga.h).
#include <cmath>
#include <cstring>
#include <string>

#include "engine.hpp"
#include "ga.hpp"

using namespace gpuga;

struct gpuga_engine {
  Engine* e;
};
struct gpuga_ga {
  GA g;
  Engine* e = nullptr;
  gpuga_fitness_cb cb = nullptr;
  void* user = nullptr;
  std::vector<double> fit64;
  DeviceGA* dga = nullptr;  // device-resident loop state, built on first use
  int device_loop = 1;      // gpuga_ga_run on the device loop (engine GAs on the batched path)
  int window = 32;          // generations per device-loop window
  ~gpuga_ga() { device_ga_free(dga); }
};

namespace gpuga {
int engine_fitness_device(Engine* e, int P, const float* d_pop, double* d_fitness, cudaStream_t st);
int engine_last_results(Engine* e, int P, double* energy, double* virial, double* force_sq);
int engine_batched_forces(Engine* e, int P, const float* pop01, float* forces_out);
}  // namespace gpuga

#define CHECK_ARG(cond, msg)       \
  do {                             \
    if (!(cond)) {                 \
      set_error("%s", msg);        \
      return GPUGA_ERR_ARG;        \
    }                              \
  } while (0)

extern "C" {

void gpuga_default_options(gpuga_options* opt) {
  if (!opt) return;
  memset(opt, 0, sizeof *opt);
  opt->device = 0;
  opt->path = GPUGA_PATH_BATCHED;
  opt->use_graph = 1;
  opt->nn2b_consistent = 0;
  opt->nn2b_r1 = 7.0f;
  opt->nn2b_r2 = 8.0f;
  opt->verbose = 0;
  opt->tiles = 0;
  opt->fitness_fold = 0;
}

const char* gpuga_last_error(void) { return last_error(); }
const char* gpuga_version(void) { return "gpuga-b200 0.1"; }

static int finish_create(PotentialSpec& spec, TrainingSet&& ts, const gpuga_options* opt, gpuga_engine** out) {
  gpuga_options o;
  if (opt) o = *opt;
  else gpuga_default_options(&o);
  spec.nn_r1 = o.nn2b_r1;
  spec.nn_r2 = o.nn2b_r2;
  spec.nn_consistent = o.nn2b_consistent;
  spec.ri_self = o.ri_self_energy ? 1 : 0;
  if (spec.type == 3 && !(spec.nn_r2 > spec.nn_r1)) {
    set_error("NN2B taper needs r2 > r1 (got %g, %g).", spec.nn_r1, spec.nn_r2);
    return GPUGA_ERR_ARG;
  }
  Engine* e = nullptr;
  int s = engine_create(spec, std::move(ts), o, &e);
  if (s != GPUGA_OK) return s;
  *out = new gpuga_engine{e};
  return GPUGA_OK;
}

int gpuga_engine_create(const char* dir, const gpuga_options* opt, gpuga_engine** out) {
  CHECK_ARG(dir && out, "gpuga_engine_create: null argument");
  *out = nullptr;
  PotentialSpec spec;
  TrainingSet ts;
  int s = read_potential_in(dir, &spec);
  if (s != GPUGA_OK) return s;
  s = read_train_in(dir, &ts);
  if (s != GPUGA_OK) return s;
  return finish_create(spec, std::move(ts), opt, out);
}

int gpuga_engine_create_from_arrays(int potential_type, int num_neurons, float cutoff, const float* weights,
                                    const float* pmin, const float* pmax, int Nc, int Nc_force, const int* Na,
                                    const int* type, const float* r, const float* box9, const float* pe_ref,
                                    const float* virial_ref, const float* force_ref, const gpuga_options* opt,
                                    gpuga_engine** out) {
  CHECK_ARG(out && weights && pmin && pmax && Na && type && r && box9, "gpuga_engine_create_from_arrays: null argument");
  *out = nullptr;
  PotentialSpec spec;
  spec.type = potential_type;
  spec.num_neurons = num_neurons;
  spec.num_vars = num_vars_for(potential_type, num_neurons);
  if (spec.num_vars < 0 || (potential_type == 3 && num_neurons < 1)) {
    set_error("unsupported potential type.");
    return GPUGA_ERR_UNSUPPORTED;
  }
  spec.cutoff = cutoff;
  spec.w_force = weights[0];
  spec.w_energy = weights[1];
  spec.w_stress = weights[2];
  if (spec.w_force < 0 || spec.w_energy < 0 || spec.w_stress < 0) {
    set_error("weights should be >= 0");
    return GPUGA_ERR_PARSE;
  }
  spec.pmin.assign(pmin, pmin + spec.num_vars);
  spec.pmax.assign(pmax, pmax + spec.num_vars);
  TrainingSet ts;
  ts.Nc = Nc;
  ts.Nc_force = Nc_force;
  CHECK_ARG(Nc > 0, "Nc must be positive");
  ts.Na.assign(Na, Na + Nc);
  long long N = 0;
  for (int c = 0; c < Nc; ++c) N += std::max(Na[c], 0);
  CHECK_ARG(N < (1LL << 30), "too many atoms");
  ts.type.assign(type, type + N);
  ts.r.assign(r, r + 3 * N);
  ts.h.assign(18 * (size_t)Nc, 0.f);
  for (int c = 0; c < Nc; ++c) {
    const float* t = box9 + 9 * (size_t)c;
    float* h = ts.h.data() + 18 * (size_t)c;
    h[0] = t[0]; h[3] = t[1]; h[6] = t[2];
    h[1] = t[3]; h[4] = t[4]; h[7] = t[5];
    h[2] = t[6]; h[5] = t[7]; h[8] = t[8];
    box_inverse(h);
  }
  ts.pe_ref.assign(Nc, 0.f);
  ts.virial_ref.assign(6 * (size_t)Nc, 0.f);
  ts.force_ref.assign(3 * N, 0.f);
  if (pe_ref) ts.pe_ref.assign(pe_ref, pe_ref + Nc);
  if (virial_ref) ts.virial_ref.assign(virial_ref, virial_ref + 6 * (size_t)Nc);
  if (force_ref) ts.force_ref.assign(force_ref, force_ref + 3 * N);
  int s = finish_training_set(&ts);
  if (s != GPUGA_OK) return s;
  return finish_create(spec, std::move(ts), opt, out);
}

int gpuga_parse_inputs(const char* dir, int* sz) {
  CHECK_ARG(dir, "gpuga_parse_inputs: null directory");
  PotentialSpec spec;
  TrainingSet ts;
  GAParams gp;
  int s = read_potential_in(dir, &spec);
  if (s != GPUGA_OK) return s;
  s = read_train_in(dir, &ts);
  if (s != GPUGA_OK) return s;
  std::string ga_path = std::string(dir) + "/ga.in";
  if (FILE* f = fopen(ga_path.c_str(), "r")) {
    fclose(f);
    s = read_ga_in(dir, &gp);
    if (s != GPUGA_OK) return s;
  }
  if (sz) {
    const int v[11] = {spec.type, spec.num_vars, spec.num_neurons, ts.Nc, ts.Nc_force, ts.N, ts.N_force,
                       ts.max_Na, gp.population_size, gp.parent_number, gp.maximum_generation};
    memcpy(sz, v, sizeof v);
  }
  return GPUGA_OK;
}

int gpuga_engine_destroy(gpuga_engine* e) {
  if (!e) return GPUGA_OK;
  delete e->e;
  delete e;
  return GPUGA_OK;
}

int gpuga_engine_info(const gpuga_engine* h, int* s) {
  CHECK_ARG(h && s, "gpuga_engine_info: null argument");
  const Engine* e = h->e;
  s[0] = e->spec.type;
  s[1] = e->spec.num_vars;
  s[2] = e->spec.num_neurons;
  s[3] = e->ts.Nc;
  s[4] = e->ts.Nc_force;
  s[5] = e->ts.N;
  s[6] = e->ts.N_force;
  s[7] = e->ts.max_Na;
  s[8] = e->d.B;
  s[9] = e->d.max_Z;
  return GPUGA_OK;
}

int gpuga_engine_bounds(const gpuga_engine* h, float* pmin, float* pmax) {
  CHECK_ARG(h, "gpuga_engine_bounds: null engine");
  const Engine* e = h->e;
  if (pmin) memcpy(pmin, e->spec.pmin.data(), sizeof(float) * e->spec.num_vars);
  if (pmax) memcpy(pmax, e->spec.pmax.data(), sizeof(float) * e->spec.num_vars);
  return GPUGA_OK;
}

int gpuga_engine_norms(const gpuga_engine* h, double* n3) {
  CHECK_ARG(h && n3, "gpuga_engine_norms: null argument");
  n3[0] = h->e->ts.norm_force;
  n3[1] = h->e->ts.norm_energy;
  n3[2] = h->e->ts.norm_virial;
  return GPUGA_OK;
}

int gpuga_engine_neighbors(const gpuga_engine* h, int* NN, int* NL) {
  CHECK_ARG(h, "gpuga_engine_neighbors: null engine");
  const Engine* e = h->e;
  const int N = e->ts.N;
  if (NN) memcpy(NN, e->h_NN.data(), sizeof(int) * N);
  if (NL) {
    for (int i = 0; i < N; ++i)
      for (int k = 0; k < e->h_NN[i]; ++k) NL[(size_t)k * N + i] = e->h_nbr[e->h_off[i] + k];
  }
  return GPUGA_OK;
}

int gpuga_engine_neighbors_csr(const gpuga_engine* h, int* NN, int* nbr) {
  CHECK_ARG(h, "gpuga_engine_neighbors_csr: null engine");
  const Engine* e = h->e;
  if (NN) memcpy(NN, e->h_NN.data(), sizeof(int) * e->ts.N);
  if (nbr) memcpy(nbr, e->h_nbr.data(), sizeof(int) * (size_t)e->d.B);
  return GPUGA_OK;
}

int gpuga_fitness(gpuga_engine* h, int P, const float* pop01, double* fitness_out) {
  CHECK_ARG(h, "gpuga_fitness: null engine");
  return engine_fitness(h->e, h->e->opt.path, P, pop01, fitness_out, nullptr);
}

int gpuga_fitness_ex(gpuga_engine* h, int path, int P, const float* pop01, double* fitness_out,
                     double* components_out) {
  CHECK_ARG(h, "gpuga_fitness_ex: null engine");
  return engine_fitness(h->e, path, P, pop01, fitness_out, components_out);
}

int gpuga_fitness_device(gpuga_engine* h, int P, const float* d_pop01, double* d_fitness, void* stream) {
  CHECK_ARG(h && d_pop01 && d_fitness && P > 0, "gpuga_fitness_device: invalid argument");
  return engine_fitness_device(h->e, P, d_pop01, d_fitness, (cudaStream_t)stream);
}

int gpuga_last_config_results(gpuga_engine* h, int P, double* energy, double* virial, double* force_sq) {
  CHECK_ARG(h, "gpuga_last_config_results: null engine");
  return engine_last_results(h->e, P, energy, virial, force_sq);
}

int gpuga_batched_forces(gpuga_engine* h, int P, const float* pop01, float* forces_out) {
  CHECK_ARG(h && pop01 && forces_out && P > 0, "gpuga_batched_forces: invalid argument");
  return engine_batched_forces(h->e, P, pop01, forces_out);
}

int gpuga_plan_info(gpuga_engine* h, int P, int* n_launches, double* per_launch, int cap) {
  CHECK_ARG(h && P > 0, "gpuga_plan_info: invalid argument");
  Plan* plan = nullptr;
  GPUGA_CUDA(cudaSetDevice(h->e->device));
  int s = plan_get(h->e, P, &plan);
  if (s != GPUGA_OK) return s;
  LaunchSet* ls = plan->ls.get();
  s = launchset_collect_timing(ls);
  if (s != GPUGA_OK) return s;
  const int n = (int)ls->launches.size();
  if (n_launches) *n_launches = n;
  if (per_launch) {
    for (int k = 0; k < n && k < cap; ++k) {
      const Launch& L = ls->launches[k];
      double* o = per_launch + 8 * (size_t)k;
      o[0] = L.kind;
      o[1] = L.kind == 2 ? L.nmax : L.zclass;
      o[2] = L.force;
      o[3] = L.count;
      o[4] = L.units;
      o[5] = L.flops;
      o[6] = L.sfu;
      o[7] = ls->t_count ? ls->t_ms[k] / ls->t_count : 0.0;
    }
  }
  return GPUGA_OK;
}

int gpuga_plan_kernels(gpuga_engine* h, int P, int* kernels) {
  CHECK_ARG(h && P > 0 && kernels, "gpuga_plan_kernels: invalid argument");
  Plan* plan = nullptr;
  GPUGA_CUDA(cudaSetDevice(h->e->device));
  int s = plan_get(h->e, P, &plan);
  if (s != GPUGA_OK) return s;
  const LaunchSet* ls = plan->ls.get();
  *kernels = 1 + (int)ls->launches.size() + (ls->folds ? 0 : 1);  // decode + items (+ fitness fold)
  return GPUGA_OK;
}

int gpuga_plan_tiles(gpuga_engine* h, int P, int* tiles, int cap, double* tune_ms) {
  CHECK_ARG(h && P > 0, "gpuga_plan_tiles: invalid argument");
  Plan* plan = nullptr;
  GPUGA_CUDA(cudaSetDevice(h->e->device));
  const int s = plan_get(h->e, P, &plan);
  if (s != GPUGA_OK) return s;
  for (int c = 0; tiles && c < cap && c < h->e->d.Nc; ++c) tiles[c] = c < (int)plan->tiles.size() ? plan->tiles[c] : 0;
  if (tune_ms) *tune_ms = plan->tune_ms;
  return GPUGA_OK;
}

int gpuga_kernel_timing(gpuga_engine* h, int P, int enable) {
  CHECK_ARG(h && P > 0, "gpuga_kernel_timing: invalid argument");
  Plan* plan = nullptr;
  GPUGA_CUDA(cudaSetDevice(h->e->device));
  int s = plan_get(h->e, P, &plan);
  if (s != GPUGA_OK) return s;
  LaunchSet* ls = plan->ls.get();
  s = launchset_collect_timing(ls);
  if (s != GPUGA_OK) return s;
  ls->timing = enable != 0;
  std::fill(ls->t_ms.begin(), ls->t_ms.end(), 0.0);
  ls->t_count = 0;
  return GPUGA_OK;
}

int gpuga_find_force64(gpuga_engine* h, const double* params, double* F, double* W, double* pe) {
  CHECK_ARG(h && params, "gpuga_find_force64: null argument");
  GPUGA_CUDA(cudaSetDevice(h->e->device));
  return plain_find_force64(h->e, params, F, W, pe);
}

int gpuga_find_force32(gpuga_engine* h, const float* params, float* F, float* W, float* pe) {
  CHECK_ARG(h && params, "gpuga_find_force32: null argument");
  GPUGA_CUDA(cudaSetDevice(h->e->device));
  return plain_find_force32(h->e, params, F, W, pe);
}

int gpuga_decode(const gpuga_engine* h, const float* x01, float* params) {
  CHECK_ARG(h && x01 && params, "gpuga_decode: null argument");
  decode_params(h->e->spec, x01, params);
  return GPUGA_OK;
}

// fitness.cu:335-390
int gpuga_predict(gpuga_engine* h, const char* dir, const float* elite01) {
  CHECK_ARG(h && dir && elite01, "gpuga_predict: null argument");
  Engine* e = h->e;
  const TrainingSet& t = e->ts;
  const int N = t.N, Nc = t.Nc;
  std::vector<float> p32(e->spec.num_vars);
  decode_params(e->spec, elite01, p32.data());
  std::vector<double> p64(p32.begin(), p32.end());
  std::vector<double> F(3 * (size_t)N), W(6 * (size_t)N), pe(N);
  GPUGA_CUDA(cudaSetDevice(e->device));
  int s = plain_find_force64(e, p64.data(), F.data(), W.data(), pe.data());
  if (s != GPUGA_OK) return s;
  std::string base(dir);
  FILE* f = fopen((base + "/force.out").c_str(), "w");
  if (!f) {
    set_error("Failed to open %s/force.out.", dir);
    return GPUGA_ERR_IO;
  }
  for (int n = 0; n < t.N_force; ++n)
    fprintf(f, "%g %g %g %g %g %g\n", (float)F[n], (float)F[n + N], (float)F[n + 2 * (size_t)N], t.force_ref[n],
            t.force_ref[n + N], t.force_ref[n + 2 * (size_t)N]);
  fclose(f);
  auto sums = [&](FILE* out, const double* data, const float* ref) {
    for (int c = t.Nc_force; c < Nc; ++c) {
      double sum = 0.0;
      for (int m = 0; m < t.Na[c]; ++m) sum += data[t.Na_sum[c] + m];
      fprintf(out, "%g %g\n", (float)sum, ref[c]);
    }
  };
  f = fopen((base + "/energy.out").c_str(), "w");
  if (!f) {
    set_error("Failed to open %s/energy.out.", dir);
    return GPUGA_ERR_IO;
  }
  sums(f, pe.data(), t.pe_ref.data());
  fclose(f);
  f = fopen((base + "/virial.out").c_str(), "w");
  if (!f) {
    set_error("Failed to open %s/virial.out.", dir);
    return GPUGA_ERR_IO;
  }
  for (int k = 0; k < 6; ++k) sums(f, W.data() + (size_t)N * k, t.virial_ref.data() + (size_t)Nc * k);
  fclose(f);
  return GPUGA_OK;
}

// --------------------------------------------------------------------- GA
static int make_ga(Engine* e, const GAParams& gp, unsigned seed, gpuga_ga** out) {
  gpuga_ga* g = new gpuga_ga;
  g->e = e;
  int s = g->g.init(e->spec.num_vars, e->spec.pmin.data(), e->spec.pmax.data(), gp, seed);
  if (s != GPUGA_OK) {
    delete g;
    return s;
  }
  g->g.eval = [g](int P, const float* pop, float* fit) {
    g->fit64.resize(P);
    int st = engine_fitness(g->e, g->e->opt.path, P, pop, g->fit64.data(), nullptr);
    if (st != GPUGA_OK) return st;
    for (int p = 0; p < P; ++p) fit[p] = (float)g->fit64[p];  // the reference ranks FP32 fitness values
    return GPUGA_OK;
  };
  *out = g;
  return GPUGA_OK;
}

int gpuga_ga_create(gpuga_engine* h, const char* dir, unsigned seed, gpuga_ga** out) {
  CHECK_ARG(h && dir && out, "gpuga_ga_create: null argument");
  GAParams gp;
  int s = read_ga_in(dir, &gp);
  if (s != GPUGA_OK) return s;
  return make_ga(h->e, gp, seed, out);
}

int gpuga_ga_create_params(gpuga_engine* h, int population_size, int parent_number, float mutation_rate,
                           int maximum_generation, unsigned seed, gpuga_ga** out) {
  CHECK_ARG(h && out, "gpuga_ga_create_params: null argument");
  GAParams gp;
  gp.population_size = population_size;
  gp.parent_number = parent_number;
  gp.mutation_rate = mutation_rate;
  gp.maximum_generation = maximum_generation;
  CHECK_ARG(maximum_generation >= 1, "maximum_generation should be positive");
  return make_ga(h->e, gp, seed, out);
}

int gpuga_ga_create_host(int num_vars, const float* pmin, const float* pmax, int population_size,
                         int parent_number, float mutation_rate, int maximum_generation, unsigned seed,
                         gpuga_fitness_cb cb, void* user, gpuga_ga** out) {
  CHECK_ARG(pmin && pmax && cb && out, "gpuga_ga_create_host: null argument");
  CHECK_ARG(maximum_generation >= 1, "maximum_generation should be positive");
  GAParams gp;
  gp.population_size = population_size;
  gp.parent_number = parent_number;
  gp.mutation_rate = mutation_rate;
  gp.maximum_generation = maximum_generation;
  gpuga_ga* g = new gpuga_ga;
  int s = g->g.init(num_vars, pmin, pmax, gp, seed);
  if (s != GPUGA_OK) {
    delete g;
    return s;
  }
  g->cb = cb;
  g->user = user;
  g->g.eval = [g](int P, const float* pop, float* fit) {
    g->cb(P, pop, fit, g->user);
    return GPUGA_OK;
  };
  *out = g;
  return GPUGA_OK;
}

int gpuga_ga_step(gpuga_ga* g, char* line_out, int line_len) {
  CHECK_ARG(g, "gpuga_ga_step: null GA");
  std::string line;
  int s = g->g.step(&line);
  if (s != GPUGA_OK) return s;
  if (line_out && line_len > 0) snprintf(line_out, line_len, "%s", line.c_str());
  return GPUGA_OK;
}

// ga.cu:150-158: screen echo of every tenth generation, numbered after the step
static void echo_line(const gpuga_ga* g, const std::string& line) {
  if (!g->e || !g->e->opt.verbose) return;
  const size_t sp = line.find(' ');
  const int gen = atoi(line.c_str()) + 1;
  if (gen % 10 == 0) printf("%d%s", gen, line.substr(sp).c_str());
}

int gpuga_ga_run(gpuga_ga* g, const char* dir) {
  CHECK_ARG(g && dir, "gpuga_ga_run: null argument");
  std::string path = std::string(dir) + "/ga.out";
  FILE* f = fopen(path.c_str(), "w");
  if (!f) {
    set_error("Failed to open %s.", path.c_str());
    return GPUGA_ERR_IO;
  }
  if (g->e && g->device_loop && g->e->opt.path == GPUGA_PATH_BATCHED) {
    int s = device_ga_advance(g->e, &g->g, &g->dga, g->g.gp.maximum_generation - g->g.generation, g->window,
                              [&](const std::string& lines) {
                                fputs(lines.c_str(), f);
                                fflush(f);
                                size_t a = 0;
                                while (a < lines.size()) {
                                  size_t b = lines.find('\n', a);
                                  echo_line(g, lines.substr(a, b - a + 1));
                                  a = b + 1;
                                }
                              });
    fclose(f);
    if (s != GPUGA_OK) return s;
  } else {
    std::string line;
    while (g->g.generation < g->g.gp.maximum_generation) {
      int s = g->g.step(&line);
      if (s != GPUGA_OK) {
        fclose(f);
        return s;
      }
      fputs(line.c_str(), f);
      fflush(f);
      echo_line(g, line);
    }
    fclose(f);
  }
  if (!g->e) return GPUGA_OK;
  gpuga_engine h{g->e};
  return gpuga_predict(&h, dir, g->g.population.data());
}

int gpuga_ga_set_device_loop(gpuga_ga* g, int enable, int window) {
  CHECK_ARG(g, "gpuga_ga_set_device_loop: null GA");
  CHECK_ARG(window >= 0, "gpuga_ga_set_device_loop: window must be >= 0");
  g->device_loop = enable ? 1 : 0;
  if (window > 0) g->window = window;
  return GPUGA_OK;
}

int gpuga_ga_advance(gpuga_ga* g, int generations, char* lines_out, long long lines_len) {
  CHECK_ARG(g, "gpuga_ga_advance: null GA");
  CHECK_ARG(g->e, "gpuga_ga_advance: the device loop needs an engine GA (not a host-callback GA)");
  CHECK_ARG(generations >= 0, "gpuga_ga_advance: generations must be >= 0");
  std::string all;
  int s = device_ga_advance(g->e, &g->g, &g->dga, generations, g->window,
                            [&](const std::string& lines) { all += lines; });
  if (s != GPUGA_OK) return s;
  if (lines_out && lines_len > 0) snprintf(lines_out, (size_t)lines_len, "%s", all.c_str());
  return GPUGA_OK;
}

int gpuga_ga_rank_device(int device, int P, const double* fitness, int* order, float* sorted) {
  CHECK_ARG(fitness && order, "gpuga_ga_rank_device: null argument");
  return device_rank(device, P, fitness, order, sorted);
}

int gpuga_ga_state(const gpuga_ga* g, int* generation, float* population_out, float* fitness_out) {
  CHECK_ARG(g, "gpuga_ga_state: null GA");
  if (generation) *generation = g->g.generation;
  if (population_out) memcpy(population_out, g->g.population.data(), sizeof(float) * g->g.population.size());
  if (fitness_out) memcpy(fitness_out, g->g.fitness.data(), sizeof(float) * g->g.fitness.size());
  return GPUGA_OK;
}

int gpuga_ga_destroy(gpuga_ga* g) {
  delete g;
  return GPUGA_OK;
}

}  // extern "C"
