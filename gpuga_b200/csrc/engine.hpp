// Engine: one training set resident in HBM plus the buffers of the batched
// fitness evaluation.  Layout (all device arrays):
//
//   configs  Na[Nc], Na_sum[Nc], h[18 Nc] (FP32 box + inverse)
//   atoms    type[N], r[3N] (SoA, FP32 as parsed), NN[N], off[N+1] (CSR into bonds),
//            half_off[N] (first bond whose neighbor index is > i)
//   bonds    nbr[B], rev[B] (reverse bond), rev_sm[B] (the reverse bond's slot * Na + atom,
//            local to the configuration), ptype[B] (pair set / RI pair type),
//            g32[B] float4 (unit vector, d; not kept for RI), g64[B] double4 (x,y,z,d),
//            d64[B] (Tersoff: the FP64 bond length again, for the FP64 pair terms)
//            RI: rg32 / rdl / rseg, each atom's pairs of the pair types whose Buckingham or
//            Morse term can be nonzero, grouped by pair type; ri_atom_lin / ri_cfg_lin, the
//            FP64 geometric sums of the terms that are linear in the parameters
//   targets  force_ref[3N], E_ref[Nc], W_ref[6Nc] (FP64 copies of the FP32 inputs)
//
// Bond vectors use the periodic image chosen by the reference's FP32 rule and
// are then evaluated in FP64 from the FP32 positions.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <functional>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "common.hpp"

namespace gpuga {

constexpr int kBlock = 256;           // threads per CTA of the batched kernels
constexpr int kWarps = kBlock / 32;
constexpr int kResK = 8;              // per (individual, config): E, W[6], sum|dF|^2
constexpr int kMaxConsts = 32;        // per-individual FP32 constants of the batched kernels
constexpr int kRiAtomLin = 27;        // RI linear force sums per force atom: 3 pair types x 3 x xyz
constexpr int kRiCfgLin = 66;         // RI linear energy/virial sums per configuration: 3 x (4 + 3 x 6)

// Register-array size of the batched Tersoff kernels for a configuration whose atoms have at most
// z neighbors (0: beyond the supported 16).
inline int tersoff_zclass(int z) { return z <= 4 ? 4 : (z <= 8 ? 8 : (z <= 16 ? 16 : 0)); }

struct DevSet {
  int Nc = 0, Nc_force = 0, N = 0, N_force = 0, B = 0, max_Na = 0, max_Z = 0;
  int potential_type = -1, num_types = 1, num_neurons = 0, num_vars = 0;
  int* Na = nullptr;
  int* Na_sum = nullptr;
  int* type = nullptr;
  float* r = nullptr;
  float* h = nullptr;
  int* NN = nullptr;
  int* off = nullptr;
  int* half_off = nullptr;
  int* nbr = nullptr;
  int* rev = nullptr;
  int* pslot = nullptr;  // NN2B: each bond's pair-derivative slot in a force item's scratch
  int* hb = nullptr;     // NN2B: per force configuration the bonds its force items evaluate
  int* hb_off = nullptr; //   (each unordered pair once where the list is symmetric), [Nc + 1]
  int* rev_sm = nullptr;
  uint8_t* ptype = nullptr;
  float4* g32 = nullptr;
  double4* g64 = nullptr;
  double* d64 = nullptr;   // Tersoff: FP64 bond lengths (the FP64 pair terms)
  float* tdl = nullptr;    // Tersoff: d - (float)d (the FP32 pair terms' correction)
  // Tersoff: a slot-major copy of the bond geometry, per configuration c at sm_off[c] with
  // tersoff_zclass(max Z of c) slots: bond j of local atom il at sm_off[c] + j * Na + il (the
  // layout of the force kernels' staged geometry and f_ij scratch; empty slots zero)
  int* sm_off = nullptr;
  float4* g_sm = nullptr;
  float* dl_sm = nullptr;
  uint8_t* pt_sm = nullptr;
  int* rev_sm_sm = nullptr;
  // RI batched lists: per atom the pairs its work items evaluate pair by pair (the full list
  // for force configurations, the half list for energy/virial ones; only pair types whose
  // Buckingham or Morse term can be nonzero, ri_active) grouped by pair type, in list order
  // within a type: rseg[i] = (start, start of type 1, start of type 2, end) into rg32 / rdl
  float4* rg32 = nullptr;  // (unit vector, d)
  float* rdl = nullptr;    // d - (float)d
  int4* rseg = nullptr;
  int ri_active = 0;       // bit t: pair type t is evaluated pair by pair
  // RI: the damped, shifted Coulomb and the dispersion terms are linear in the per-individual
  // constants (qq_t, qq_t v_rc, qq_t dv_rc, C_t), so their geometric sums over all pairs are
  // formed once in FP64: per force atom [kRiAtomLin], per energy/virial configuration
  // [kRiCfgLin] (layouts at ri_linear_atoms, geometry.cu)
  double* ri_atom_lin = nullptr;
  double* ri_cfg_lin = nullptr;
  float* force_ref = nullptr;
  double* E_ref = nullptr;
  double* W_ref = nullptr;
  double norm_force = 0, norm_energy = 0, norm_virial = 0;
  float w_force = 0, w_energy = 0, w_stress = 0;
  // RI: per configuration sum_i (q_i / q)^2 = cations + ratio^2 anions (the self-energy weight)
  double* ri_qsum = nullptr;
};

// One CTA of a batched launch: configuration `config` of job `job` for
// individuals [p0, p0 + G).
struct WorkItem {
  int config;
  int p0;
  int G;     // individuals per item (power of two <= 32); lanes = G individuals x (32/G) atoms
  int job;   // row of the launch set's job table
  int gofs;  // force items too large for shared memory: offset of the item's f_ij scratch in the
             // job's global scratch, in units of 64 floats
};

// Read-only training-set view the batched kernels use.
struct DevView {
  int Nc, N, N_force;
  const int* Na;
  const int* Na_sum;
  const int* NN;
  const int* off;
  const int* half_off;
  const int* pslot;
  const int* hb;
  const int* hb_off;
  const int* rev_sm;
  const uint8_t* ptype;
  const float4* g32;
  const double* d64;
  const float* tdl;
  const int* sm_off;
  const float4* g_sm;
  const float* dl_sm;
  const uint8_t* pt_sm;
  const int* rev_sm_sm;
  const float4* rg32;
  const float* rdl;
  const int4* rseg;
  const double* ri_atom_lin;
  const double* ri_cfg_lin;
  const float* force_ref;
  const double* ri_qsum;
};

struct NNTaper {
  float r1, r2, pf;
  int consistent;
};

// One row of a launch set's job table: a training set, a population and the
// buffers of its evaluation.  Several jobs share the same launches.
struct JobView {
  DevView v;
  int potential_type, num_types, num_neurons, num_vars, P, Pstride, Nc_force, ri_self;
  NNTaper tp;
  const float* pop;      // [P][num_vars] in [0,1]
  const float* pmin;
  const float* pmax;
  float* consts;         // [K][Pstride]
  double* consts64;      // RI: [K64][Pstride] FP64 constants of the linear terms
  float* weights;        // NN2B [num_vars][Pstride]
  double* res;           // [P][Nc][kResK]
  float* fdump;          // optional [P][3][N_force]
  float* gscratch;       // f_ij scratch of the force items that do not fit shared memory
  const double* E_ref;
  const double* W_ref;
  double nF, nE, nW;
  float wF, wE, wW;
  double* fitness;       // [P]
  double* comps;         // [P][3]
  int* fit_count;        // [P] configurations of this generation finished per individual; the work
                         // item that finishes an individual's last one folds its fitness (reset to
                         // 0 there).  Null: a partial launch set (no fold).
};

struct Launch {
  int kind = 0;        // 0 Tersoff, 1 RI, 2 NN2B
  int zclass = 4;      // Tersoff register-array size
  int nmax = 0;        // NN2B register-array size; Tersoff: number of atom types
  int force = 0;       // the launch's items: 0 energy/virial, 1 force (gather pass), 2 both
  bool lo = false;     // Tersoff: carry the FP64 remainders of the derived constants
  size_t smem = 0;
  int count = 0;
  size_t first = 0;    // offset of the launch's items in the set's item array
  double units = 0;    // (individual, atom) pairs per launch
  double flops = 0;    // algorithmic FP32 flops per launch (FMA = 2)
  double sfu = 0;      // transcendental calls per launch
};

// Launches of one generation over one or more jobs (a job table on the device).
struct LaunchSet {
  std::vector<Launch> launches;
  std::vector<JobView> jobs;   // host copy of the table
  JobView* d_jobs = nullptr;
  JobView* h_jobs = nullptr;   // pinned staging for table updates
  WorkItem* d_items = nullptr;
  int2* d_indmap = nullptr;    // global individual -> (job, p)
  int total_individuals = 0;
  bool folds = true;           // the items fold every individual's fitness (no fitness_jobs launch)
  cudaStream_t side = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
  bool timing = false;               // event pair around every launch (eager launches)
  std::vector<cudaEvent_t> tev;      // 2 per launch
  std::vector<double> t_ms;          // accumulated device time per launch
  int t_count = 0;
  bool t_pending = false;
  ~LaunchSet();
};

// Tile of a Tersoff force configuration's work items: individuals per item G and where the
// f_ij scratch and geometry live (batched.cu, job_items).  Every tile gives the same results bit
// for bit (same per-atom arithmetic, canonical force-error sum); the autotuner picks per
// configuration size.
enum TileMode {
  kTileDefault = 1,   // the largest G whose scratch fits shared memory, geometry staged when it fits
  kTileHalf = 2,      // half that G (staged when it fits)
  kTileQuarter = 3,   // a quarter of it
  kTileGlobal = 4,    // 32 individuals, scratch in global memory
  kTileUnstaged = 5,  // the default G, geometry read from the slot-major global copy
};
const char* tile_mode_name(int m);

struct ItemCache;  // batched.cu: a plan's work items, computed once

// Per (engine, population size) buffers plus the engine's own launch set.
struct Plan {
  int P = 0;
  int Pstride = 0;
  float* d_consts = nullptr;   // [K][Pstride] per-individual constants
  double* d_consts64 = nullptr; // RI: [K64][Pstride] FP64 constants of the linear terms
  float* d_weights = nullptr;  // NN2B weights [num_vars][Pstride]
  double* d_res = nullptr;     // [P][Nc][kResK]
  double* d_fitness = nullptr; // [P]
  double* d_comps = nullptr;   // [P][3]
  int* d_fitcnt = nullptr;     // [P] per-generation completion counts (JobView::fit_count)
  float* d_pop = nullptr;      // [P][d] staging
  float* h_pop = nullptr;      // pinned
  double* h_fit = nullptr;     // pinned [4P]: fitness + 3 components
  float* d_fdump = nullptr;    // optional per-atom forces of force configs [P][3][N_force]
  float* d_gscratch = nullptr; // f_ij scratch of force items too large for shared memory
  size_t gscratch_floats = 0;
  bool dump = false;           // pass d_fdump to the kernels (eager launches only)
  cudaGraphExec_t graph = nullptr;
  std::unique_ptr<LaunchSet> ls;
  std::vector<int8_t> tiles;   // per configuration: the force-item TileMode (empty: default rule)
  std::shared_ptr<ItemCache> items;  // the work items of this plan (launchset_build)
  double tune_ms = 0;          // host time the autotuner took
  ~Plan();
};

struct Engine {
  gpuga_options opt{};
  PotentialSpec spec;
  TrainingSet ts;
  DevSet d;
  int device = 0;
  cudaStream_t stream = nullptr;
  float* d_pmin = nullptr;
  float* d_pmax = nullptr;
  std::vector<int> h_NN, h_off, h_nbr, h_zmax;  // host copies of the neighbor list
  std::vector<char> h_pair_sym;                 // NN2B: per configuration, bond list symmetric
  std::map<int, std::unique_ptr<Plan>> plans;    // keyed by population size
  size_t device_bytes = 0;
  std::vector<void*> allocations;
  std::map<void*, size_t> allocation_bytes;
  // plain-path scratch
  double* s64 = nullptr;  // per-bond scratch (S, A, f_ij x/y/z) FP64
  float* s32 = nullptr;
  double* p64_F = nullptr;
  double* p64_W = nullptr;
  double* p64_pe = nullptr;
  float* p32_F = nullptr;
  float* p32_W = nullptr;
  float* p32_pe = nullptr;
  double* p_out = nullptr;  // per-individual fitness + components of the plain path [4P]
  int p_out_cap = 0;
  void* p_w = nullptr;      // plain-path NN2B weights of the evaluated parameter vectors
  size_t p_w_bytes = 0;
  ~Engine();
  int dalloc(void** p, size_t bytes);
  void dfree(void* p);  // frees an allocation made by dalloc before the engine's end
  template <class T>
  int alloc(T** p, size_t n) {
    return dalloc(reinterpret_cast<void**>(p), n * sizeof(T));
  }
};

// geometry.cu
int build_geometry(Engine* e);
// FP32 neighbor rule of neighbor.cu:30-66 on reference-layout device arrays.
int neighbor_reference_layout(int Nc, int N, int max_Na, const int* Na, const int* Na_sum, const float* r,
                              const float* h, float cutoff, int* NN, int* NL, cudaStream_t st);

int ref_layout_geometry(int Nc, int N, const int* Na, const int* Na_sum, const float* h, const float* r,
                        const int* NN, const int* NL, double4* g64, int* rev, cudaStream_t st);

// The reference's Potential interface on caller-owned device arrays in the
// reference layouts (potential.cuh:22-41); scratch is supplied by the caller.
struct RefPotentialScratch {
  double4* g64;  // [max_Na * N]
  int* rev;      // [max_Na * N]
  float* f5;     // [5 * max_Na * N]: per-bond S, A, f_ij x/y/z
  float* w;      // NN2B weights [num_vars]
};
size_t ref_potential_scratch_bytes(int potential_type, int num_neurons, int N, int max_Na);
int ref_potential_find_force(int potential_type, int num_neurons, const float* params, const PotentialSpec& nn_opts,
                             int Nc, int N, const int* Na, const int* Na_sum, int max_Na, const int* type,
                             const float* h, const int* NN, const int* NL, const float* r, float* f, float* virial,
                             float* pe, const RefPotentialScratch& s, cudaStream_t st);

// batched.cu
int plan_build(Engine* e, int P, Plan** out);
int consts_per_individual(const DevSet& d);
int consts64_per_individual(const DevSet& d);
JobView make_job_view(const Engine* e, const Plan* plan);
// Builds the shared launches of the given jobs (one engine + plan each); `targets`, when given,
// names each job's population and fitness buffers (default: the plan's own).
int launchset_build(const std::vector<std::pair<Engine*, Plan*>>& jobs, LaunchSet* ls,
                    const std::vector<std::pair<const float*, double*>>* targets = nullptr,
                    const std::vector<char>* only = nullptr);
// Enqueues one generation of every job of the set on `st` (force launches on a side stream).
int launchset_enqueue(LaunchSet* ls, cudaStream_t st);
int launchset_collect_timing(LaunchSet* ls);
// Points job row `job` at new population / fitness / force-dump buffers (enqueued on `st`).
int launchset_retarget(LaunchSet* ls, int job, const float* d_pop, double* d_fitness, float* fdump,
                       cudaStream_t st);
int plan_get(Engine* e, int P, Plan** out);

// plain.cu
int plain_fitness(Engine* e, bool fp64, int P, const float* pop01, double* fitness, double* comps);
int plain_find_force64(Engine* e, const double* params, double* F, double* W, double* pe);
int plain_find_force32(Engine* e, const float* params, float* F, float* W, float* pe);

// ga_device.cu: device-resident GA loop (selection, crossover, mutation on the GPU
// from host-drawn plans) for one GA or a batch of jobs sharing the launches.
struct GA;
struct DeviceGA;
struct GABatch;
// One GA: `generations` generations in windows; `sink` receives the ga.out lines of each window.
int device_ga_advance(Engine* e, GA* ga, DeviceGA** state, int generations, int window,
                      const std::function<void(const std::string&)>& sink);
void device_ga_free(DeviceGA* s);
// The GA's stable ascending order of FP32-rounded fitness values on the device: order[r] = i.
int device_rank(int device, int P, const double* fitness, int* order, float* sorted);
// Batches: per-job state (two plan stages of `window` generations), then one batch of jobs whose
// fitness comes from `ls` (job k of the launch set = job k of the batch).
int device_ga_setup(const GA& ga, int window, DeviceGA** out);
float* device_ga_population(DeviceGA* s);
double* device_ga_fitness64(DeviceGA* s);
const float* device_ga_history(const DeviceGA* s, int b);  // [n][1 + d] after ga_batch_wait
void device_ga_draw(GA& ga, DeviceGA* s, int b, int g0, int n);
int device_ga_upload(DeviceGA* s, int b, int n, cudaStream_t st);
int device_ga_sync_host(GA* ga, DeviceGA* s, int generations, cudaStream_t st);
int ga_batch_build(const std::vector<DeviceGA*>& jobs, LaunchSet* ls, GABatch** out);
void ga_batch_free(GABatch* b);
int ga_batch_window(GABatch* B, int b, int n, bool use_graph, bool timed, cudaStream_t st);
int ga_batch_wait(GABatch* B, int b);
// device time of each generation of the last timed window on plan buffer b
int ga_batch_generation_ms(GABatch* B, int b, int n, std::vector<double>* ms);

// engine.cu
int engine_create(const PotentialSpec& spec, TrainingSet&& ts, const gpuga_options& opt, Engine** out);
int engine_fitness(Engine* e, int path, int P, const float* pop01, double* fitness, double* comps);

}  // namespace gpuga
