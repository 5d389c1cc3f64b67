/*
 * gpuga.h -- C ABI of the B200 GPUGA fitness engine (libgpuga_b200.so).
 *
 * Plain C types only: pointers, sizes, status codes.  Every call returns an
 * int status (GPUGA_OK == 0, negative on failure); gpuga_last_error() gives
 * the message of the last failure on the calling thread.  Host buffers are
 * caller-owned; device buffers are engine-owned unless a function says it
 * takes device pointers.
 *
 * Each entry point names the reference interface it replaces
 * (GPUGA, src/<file>:<line>).
 */
#ifndef GPUGA_B200_H
#define GPUGA_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status */
#define GPUGA_OK 0
#define GPUGA_ERR_IO (-1)          /* file cannot be opened (error.cu:27-48 my_fopen) */
#define GPUGA_ERR_PARSE (-2)       /* malformed or invalid input (fitness.cu:59-314, ga.cu:214-316) */
#define GPUGA_ERR_UNSUPPORTED (-3) /* potential_type / size outside what the engine supports */
#define GPUGA_ERR_OOM (-4)         /* device or host allocation failed */
#define GPUGA_ERR_CUDA (-5)        /* a CUDA call failed (error.cuh:35-51 CHECK) */
#define GPUGA_ERR_TIMEOUT (-6)     /* a bounded device wait gave up */
#define GPUGA_ERR_NAN (-7)         /* non-finite fitness where the caller asked for a check */
#define GPUGA_ERR_ARG (-8)         /* invalid argument */
#define GPUGA_ERR_BUDGET (-9)      /* serving: job larger than the HBM budget */
#define GPUGA_ERR_CANCELLED (-10)  /* serving: job was cancelled */
#define GPUGA_ERR_NOT_READY (-11)  /* serving: job still running */

/* Potential types (potential.in, fitness.cu:220-258): 0 RI (cation +q, anion -q/2, ri.cu:40-43),
 * 1 minimal Tersoff, 2 two-element minimal Tersoff, 3 NN2B, and 4 RI with anion charge -q
 * (charge-neutral 1:1 lattices; no counterpart in the reference, which hard-codes -q/2). */

/* Evaluation paths. */
#define GPUGA_PATH_BATCHED 0 /* all individuals x all configs per generation, FP32 math + FP64 sums */
#define GPUGA_PATH_PLAIN64 1 /* one individual per launch, FP64 throughout */
#define GPUGA_PATH_PLAIN32 2 /* one individual per launch, FP32 throughout (reference-like) */

typedef struct gpuga_engine gpuga_engine;
typedef struct gpuga_ga gpuga_ga;
typedef struct gpuga_server gpuga_server;
typedef struct gpuga_potential gpuga_potential;

typedef struct gpuga_options {
  int device;          /* CUDA device ordinal */
  int path;            /* GPUGA_PATH_* used by gpuga_fitness */
  int use_graph;       /* capture each generation in a CUDA graph (batched path) */
  int nn2b_consistent; /* 1: taper the NN2B force consistently (fixes nn2b.cu:147-148) */
  float nn2b_r1;       /* NN2B taper start, reference default 7 (nn2b.cuh:36) */
  float nn2b_r2;       /* NN2B taper end, reference default 8 (nn2b.cuh:37) */
  int verbose;         /* print the reference's start-up banners */
  int neighbor_cells;  /* neighbor build: 0 cell lists for configurations of >= 2048 atoms (default),
                          1 cell lists wherever the box holds >= 3 cells of width rc per direction,
                          2 the O(Na^2) scan of neighbor.cu:30-66 everywhere; the lists are identical */
  int ri_self_energy;  /* RI (potential types 0 and 4): 1 subtracts the damped-Coulomb self energy
                          -K_C sum_i q_i^2 [alpha/sqrt(pi) + erfc(alpha rc)/rc + alpha/sqrt(pi) exp(-alpha^2 rc^2)]
                          from every atom's energy, in FP64; 0 (default) keeps ri.cu, which has none */
  int tiles;           /* Tersoff force-item tiles: 0 (default) autotuned per configuration size when a
                          population plan is built, 1 the fixed rule (the largest individuals-per-item
                          count whose scratch fits shared memory), 2 half of it, 3 a quarter, 4 32
                          individuals with the scratch in global memory, 5 the fixed rule without staged
                          geometry.  Every choice gives bit-identical results. */
  int fitness_fold;    /* where each individual's fitness is folded from its configurations' results:
                          0 (default) or 2 in a launch of its own after the item launches; 1 in the work
                          item that finishes the individual's last configuration (an atomic count per
                          individual, so that a generation is the decode launch plus the item launch;
                          the count's round trip at the end of every item measured slower than the extra
                          launch).  All choices give the same bits. */
} gpuga_options;

/* Fills *opt with the reference's semantics (batched path, graphs on, NN2B taper 7..8 A, force quirk kept). */
void gpuga_default_options(gpuga_options* opt);

const char* gpuga_last_error(void);
const char* gpuga_version(void);

/* --------------------------------------------------------------- engine set-up */
/* Replaces Fitness::Fitness(char*) (fitness.cu:30-38): reads <dir>/potential.in and
 * <dir>/train.in, builds the neighbor list on the GPU (bit-exact with neighbor.cu:30-66)
 * and uploads the training set. */
int gpuga_engine_create(const char* dir, const gpuga_options* opt, gpuga_engine** out);

/* Same, from in-memory arrays laid out as the reference stores them after parsing
 * (fitness.cu:59-161): r is SoA float[3N]; box9 is float[9*Nc] as written in train.in
 * (row k of the file matrix = 3 consecutive floats, transposed into h like fitness.cu:115-123);
 * pe_ref float[Nc]; virial_ref float[6*Nc] ([c + Nc*k]); force_ref float[3N] SoA.
 * pmin/pmax float[num_vars]; weights = {force, energy, stress}. */
int gpuga_engine_create_from_arrays(int potential_type, int num_neurons, float cutoff, const float* weights,
                                    const float* pmin, const float* pmax, int Nc, int Nc_force, const int* Na,
                                    const int* type, const float* r, const float* box9, const float* pe_ref,
                                    const float* virial_ref, const float* force_ref, const gpuga_options* opt,
                                    gpuga_engine** out);

int gpuga_engine_destroy(gpuga_engine* e);

/* Parses <dir>/potential.in, train.in and (if present) ga.in with the reference's rules
 * (fitness.cu:59-314, ga.cu:214-316) without touching the GPU.  sizes (may be NULL):
 * potential_type, num_vars, num_neurons, Nc, Nc_force, N, N_force, max_Na,
 * population_size, parent_number, maximum_generation. */
int gpuga_parse_inputs(const char* dir, int* sizes11);

/* sizes: potential_type, num_vars, num_neurons, Nc, Nc_force, N, N_force, max_Na, num_bonds, max_neighbors */
int gpuga_engine_info(const gpuga_engine* e, int* sizes10);
/* Parameter bounds (fitness.cuh:37-38) */
int gpuga_engine_bounds(const gpuga_engine* e, float* pmin, float* pmax);
/* FP64 normalisers of the relative RMSEs (fitness.cu:86-160): {force, energy, virial} */
int gpuga_engine_norms(const gpuga_engine* e, double* norms3);

/* Neighbor list as the reference stores it (neighbor.cu:61): NN int[N], NL int[max_Na*N], NL[k*N+i]. */
int gpuga_engine_neighbors(const gpuga_engine* e, int* NN, int* NL);
/* Same list in CSR form: NN int[N], nbr int[num_bonds] (ascending global indices per atom). */
int gpuga_engine_neighbors_csr(const gpuga_engine* e, int* NN, int* nbr);

/* ------------------------------------------------------------- fitness (hot path) */
/* Replaces Fitness::compute(int, float*, float*) (fitness.cu:316-333).
 * pop01: host float[P*num_vars] in [0,1]; fitness_out: host double[P].
 * Synchronous on return.  Uses opt.path. */
int gpuga_fitness(gpuga_engine* e, int P, const float* pop01, double* fitness_out);

/* Same with an explicit path and the three relative RMSEs per individual
 * (components_out double[3P] as {energy, virial, force}; may be NULL). */
int gpuga_fitness_ex(gpuga_engine* e, int path, int P, const float* pop01, double* fitness_out,
                     double* components_out);

/* Batched path on device-resident buffers (no host copies): d_pop01 device float[P*num_vars],
 * d_fitness device double[P].  Enqueued on `stream` (a cudaStream_t, NULL = legacy default);
 * returns without synchronising. */
int gpuga_fitness_device(gpuga_engine* e, int P, const float* d_pop01, double* d_fitness, void* stream);

/* Per-(individual, config) results of the last batched evaluation:
 * energy double[P*Nc], virial double[P*Nc*6] ([p][c][k], k = xx,yy,zz,xy,yz,zx; E/V configs only),
 * force_sq double[P*Nc] (sum |F-F_ref|^2 of the config's atoms; force configs only).  Any may be NULL. */
int gpuga_last_config_results(gpuga_engine* e, int P, double* energy, double* virial, double* force_sq);

/* Per-atom forces of the force configurations from the batched path for P individuals:
 * forces_out host float[P*3*N_force] ([p][xyz][i]).  Evaluates the population. */
int gpuga_batched_forces(gpuga_engine* e, int P, const float* pop01, float* forces_out);

/* Launch plan of the batched path for population size P (built on first use).
 * *n_launches = batched launches per generation (one per kernel class: force and energy/virial items
 * share a launch, and the items fold each individual's fitness; the decode launch comes on top);
 * per_launch (may be NULL) receives up to `cap` rows of 8 doubles:
 * {kind (0 Tersoff, 1 RI, 2 NN2B), register class, items (0 energy/virial, 1 force, 2 both), CTAs,
 *  (individual, atom) units, algorithmic FP32 flops, transcendental calls, mean device ms per
 *  generation while timing is on}. */
int gpuga_plan_info(gpuga_engine* e, int P, int* n_launches, double* per_launch, int cap);
/* Kernel launches per generation of the batched path for population size P: the decode, the item
 * launches and, when the items do not fold the fitness (gpuga_options.fitness_fold), the fold. */
int gpuga_plan_kernels(gpuga_engine* e, int P, int* kernels);
/* The force-item tile of every configuration (tiles[Nc], gpuga_options.tiles codes 1-5; 0 for
 * energy/virial and non-Tersoff configurations) of the plan for population size P, and the host time
 * the autotuner spent on it. */
int gpuga_plan_tiles(gpuga_engine* e, int P, int* tiles, int cap, double* tune_ms);
/* Records CUDA events around every batched launch of population size P (eager launches only:
 * gpuga_fitness_device, or gpuga_fitness with use_graph = 0).  While timing is on, the launches
 * of a generation run one after another on the caller's stream, so each duration is that
 * launch's own; enabling or disabling resets the accumulated times. */
int gpuga_kernel_timing(gpuga_engine* e, int P, int enable);
/* Measured FP32 CUDA-core FMA throughput of `device` (TFLOP/s), for roofline fractions. */
int gpuga_calibrate_fp32(int device, double* tflops);

/* Replaces Potential::update_potential + Potential::find_force (potential.cuh:22-41) for one
 * decoded parameter vector (potential.in order).  FP64 path: F double[3N], W double[6N], pe double[N]
 * (SoA, virial order xx,yy,zz,xy,yz,zx). */
int gpuga_find_force64(gpuga_engine* e, const double* params, double* F, double* W, double* pe);
/* FP32 path with the reference's float outputs. */
int gpuga_find_force32(gpuga_engine* e, const float* params, float* F, float* W, float* pe);

/* Replaces Fitness::predict(char*, float*) (fitness.cu:335-390): decodes elite01 (float[num_vars])
 * in FP32, evaluates it on the FP64 path and writes <dir>/force.out, energy.out, virial.out in
 * the reference's "%g" format. */
int gpuga_predict(gpuga_engine* e, const char* dir, const float* elite01);

/* Decode x in [0,1] to parameters exactly like fitness.cu:320-324 (FP32, no contraction). */
int gpuga_decode(const gpuga_engine* e, const float* x01, float* params);

/* -------------------------------------------------------------------- GA (ga.cu) */
/* Replaces GA::GA + GA::compute (ga.cu:27-92) one generation at a time.
 * Reads <dir>/ga.in (ga.cu:214-316).  seed: std::mt19937 seed (12345678 = the reference's -DDEBUG). */
int gpuga_ga_create(gpuga_engine* e, const char* dir, unsigned seed, gpuga_ga** out);
/* Same with explicit ga.in values. */
int gpuga_ga_create_params(gpuga_engine* e, int population_size, int parent_number, float mutation_rate,
                           int maximum_generation, unsigned seed, gpuga_ga** out);
/* Host-only GA (no engine) whose fitness comes from a caller callback: fitness_cb(P, pop01, fitness_out, user). */
typedef void (*gpuga_fitness_cb)(int P, const float* pop01, float* fitness_out, void* user);
int gpuga_ga_create_host(int num_vars, const float* pmin, const float* pmax, int population_size,
                         int parent_number, float mutation_rate, int maximum_generation, unsigned seed,
                         gpuga_fitness_cb cb, void* user, gpuga_ga** out);
/* One generation: evaluate, sort, output line, crossover, mutation (ga.cu:82-88).
 * line_out (may be NULL) receives the ga.out line for this generation. */
int gpuga_ga_step(gpuga_ga* g, char* line_out, int line_len);
/* Runs all remaining generations writing <dir>/ga.out, then predict() (ga.cu:73-92).  Engine GAs on
 * the batched path run the device-resident loop (gpuga_ga_advance) unless it was switched off. */
int gpuga_ga_run(gpuga_ga* g, const char* dir);
/* Device-resident GA loop (replaces the host round trip of every GA::compute generation, ga.cu:78-92):
 * selection (the stable insertion sort of ga.cu:105-137, NaN included), crossover and mutation run on
 * the GPU behind the batched fitness launches, from random choices the host draws from the same
 * std::mt19937 stream in the reference's order, `window` generations per batch (one CUDA graph per
 * generation, replayed).  The result -- ga.out lines, population, fitness, random stream -- is the same
 * as `generations` calls of gpuga_ga_step.  Engine GAs on the batched path only; populations up to
 * 49152.  lines_out (may be NULL) receives the concatenated ga.out lines, truncated to lines_len. */
int gpuga_ga_advance(gpuga_ga* g, int generations, char* lines_out, long long lines_len);
/* enable: whether gpuga_ga_run uses the device loop (default 1); window > 0 sets generations per batch
 * (default 32), 0 keeps it. */
int gpuga_ga_set_device_loop(gpuga_ga* g, int enable, int window);
/* The device loop's selection order on its own: fitness double[P] is rounded to FP32 and ordered as the
 * reference's stable insertion sort orders it (ga.cu:105-119; a NaN keeps its place and no value moves
 * past it).  order[r] = index of the r-th individual; sorted (may be NULL) float[P]. */
int gpuga_ga_rank_device(int device, int P, const double* fitness, int* order, float* sorted);
/* population_out float[P*num_vars] (sorted after the last step), fitness_out float[P] */
int gpuga_ga_state(const gpuga_ga* g, int* generation, float* population_out, float* fitness_out);
int gpuga_ga_destroy(gpuga_ga* g);

/* ----------------------------------------------------- reference Potential drop-in */
/* A stand-alone potential that evaluates on caller-provided DEVICE arrays in the reference's
 * layouts, for a maintainer who keeps the reference's Fitness/Neighbor and swaps the force kernel.
 * Replaces Minimal_Tersoff/RI/NN2B (minimal_tersoff.cu, ri.cu, nn2b.cu). */
int gpuga_potential_create(int potential_type, int num_neurons, gpuga_potential** out);
/* Potential::initialize(N, max_Na) (potential.cuh:25) */
int gpuga_potential_initialize(gpuga_potential* p, int N, int max_Na);
/* Potential::update_potential(const std::vector<float>&) (potential.cuh:26) */
int gpuga_potential_update(gpuga_potential* p, const float* params, int num_params);
/* Potential::find_force (potential.cuh:28-40); every pointer is a device pointer in the reference
 * layout (NL[k*N+i], r SoA, h 18 floats per config, f SoA 3N, virial 6N, pe N). */
int gpuga_potential_find_force(gpuga_potential* p, int Nc, int N, const int* Na, const int* Na_sum, int max_Na,
                               const int* type, const float* h, const int* NN, const int* NL, const float* r,
                               float* f, float* virial, float* pe, void* stream);
int gpuga_potential_destroy(gpuga_potential* p);
/* No counterpart in the reference.  Same computation as gpuga_potential_create + _update +
 * _find_force in one call that allocates nothing, for callers that cannot call cudaMalloc when
 * they need forces (a code that gives its whole device-memory budget to its own allocator, a
 * plug-in host that forbids device allocation after initialisation).  The caller passes all
 * inputs and outputs: `params` is a HOST array of num_params floats (decoded parameters in
 * potential.in order, read during the call; NN2B weights are copied from it), every other
 * pointer is a device pointer in the reference layouts.  The scratch is a fixed 64 MiB array per
 * device inside the library, so N * max_Na * 56 bytes (+ the NN2B weights) must fit in it,
 * otherwise GPUGA_ERR_ARG.  The first call on a device looks up that array's address and should
 * come before any stream capture; the address is kept for the life of the process, so do not
 * call this entry point on a device after cudaDeviceReset.  All calls on a device share the
 * array: calls whose GPU work overlaps race on it, so serialise them. */
int gpuga_potential_find_force_noalloc(int potential_type, int num_neurons, const float* params, int num_params,
                                       int Nc, int N, const int* Na, const int* Na_sum, int max_Na, const int* type,
                                       const float* h, const int* NN, const int* NL, const float* r, float* f,
                                       float* virial, float* pe, void* stream);
/* Neighbor::compute (neighbor.cu:68-83) on device arrays: NN int[N], NL int[max_Na*N]. */
int gpuga_neighbor_compute(int Nc, int N, int max_Na, const int* Na, const int* Na_sum, const float* r,
                           const float* h, float cutoff, int* NN, int* NL, void* stream);

/* ------------------------------------------------------------------ serving */
/* A device-resident server that runs many fitting jobs concurrently, admitting jobs while the
 * sum of their device footprints stays within hbm_budget_bytes and batching the generations of
 * all running jobs into shared launches: fitness and GA (selection, crossover, mutation) of every
 * resident job run on the GPU, up to 8 generations per scheduling window, from random choices the
 * host draws from each job's own std::mt19937 stream.  Jobs join and leave at window boundaries.
 * No reference counterpart (the reference fits one potential per process, main.cu:25-55). */
int gpuga_server_create(int device, double hbm_budget_bytes, int max_jobs, gpuga_server** out);
/* Submits a fitting job for <dir> (potential.in, train.in, ga.in).  generations <= 0 uses ga.in.
 * Returns the job id in *job_id. */
int gpuga_server_submit(gpuga_server* s, const char* dir, unsigned seed, int generations, int* job_id);
/* Submits a job from an existing engine's training set (shared, not copied). */
int gpuga_server_submit_engine(gpuga_server* s, gpuga_engine* e, int population_size, int parent_number,
                               float mutation_rate, int generations, unsigned seed, int* job_id);
/* Status of a job: GPUGA_OK when finished, GPUGA_ERR_NOT_READY while queued/running, or its error.
 * progress_out (may be NULL): {generations done, generations total, state(0 queued,1 running,2 done,3 failed,4 cancelled)} */
int gpuga_server_poll(gpuga_server* s, int job_id, int* progress_out);
/* Best fitness history and final elite of a finished job: best_out float[generations], elite01_out float[num_vars] */
int gpuga_server_result(gpuga_server* s, int job_id, float* best_out, float* elite01_out);
int gpuga_server_cancel(gpuga_server* s, int job_id);
/* on != 0: no new scheduling window starts (the one in flight finishes); jobs keep being admitted
 * and set up, and start together once the hold is released (on = 0). */
int gpuga_server_hold(gpuga_server* s, int on);
/* Runs the scheduler until every submitted job is finished (or timeout_s elapses, -> GPUGA_ERR_TIMEOUT). */
int gpuga_server_drain(gpuga_server* s, double timeout_s);
/* Fills stats[0 .. n-1] (n <= 13) with: {generation batches run, jobs finished, p50 and p99 of the
 *         device time of a generation of all resident jobs (ms), aggregate evals/s over the busy wall
 *         time, device bytes in use, peak jobs resident, total evals, p50 and p99 of the wall-clock time
 *         per generation as each job saw it (ms; every stall of a running job included), busy wall
 *         time (s), p50 and p99 of the time from a job's submission to the harvest of its first
 *         window of generations (ms)} */
int gpuga_server_stats(gpuga_server* s, double* stats, int n);
int gpuga_server_destroy(gpuga_server* s);

#ifdef __cplusplus
}
#endif
#endif /* GPUGA_B200_H */
