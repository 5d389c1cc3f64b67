// Batched fitness evaluation: every individual x every configuration of the
// training set per generation.
//
// Decomposition.  A work item is (configuration c, group of G individuals).
// Inside a CTA each warp lane is one individual (G = 32) or, for force
// configurations whose per-bond force scratch would not fit in shared memory
// for 32 individuals, G individuals x 32/G atoms.  With G = 32 a warp walks
// one atom at a time for 32 parameter vectors: every geometry load is a
// warp-uniform broadcast and the neighbor loops never diverge.  Per-lane
// energy / virial / force-error sums are FP64 (registers, or shared memory for
// the Tersoff energy/virial CTAs); a fixed-order shared-memory reduction
// produces the (individual, configuration) results, and a second kernel folds
// them into the weighted relative-RMSE fitness in a fixed order, so a result
// never depends on what else shares the launch.
//
// Precision.  Pair, bond-order and three-body arithmetic is FP32 on CUDA cores
// (accurate libdevice exp/erfc/tanh, no fast-math) except where FP32 rounding
// would dominate: the bond-order power takes a double-float exponent
// (powf_dd.cuh) and the RI exponentials double-float arguments.  Tersoff site
// energies and virials are summed per atom in FP32 and across atoms in FP64,
// pair-potential sums per atom in compensated FP32 and then FP64; the loss and
// normalisers are FP64.
//
// Geometry (unit vectors, distances, reverse-bond positions, RI Coulomb terms
// and type-grouped RI pair copies) is parameter-independent and precomputed
// once (geometry.cu); three-body cosines are dot products of the FP32 unit
// vectors, formed in registers.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <tuple>
#include <type_traits>

#include <cuda_pipeline.h>

#include "engine.hpp"
#include "exp_d.cuh"
#include "powf_dd.cuh"

namespace gpuga {

// ----------------------------------------------------------------- per-individual constants
// Tersoff (minimal_tersoff.cu:39-75): per pair set s: lr = sqrt(2S)*A, la = sqrt(2/S)*A,
// cr = D0/(S-1), ca = S*D0/(S-1), r0; then n, beta, h, R1, R2, pi/(R2-R1), -1/(2n); then the
// FP64 remainders of lr, la, cr, ca and -1/(2n).  The FP32 rounding of these derived constants
// is the same for every bond of an individual, so it does not average out: cr, ca and lr, la
// enter fr' - b fa', which cancels near equilibrium, and -1/(2n) every bond order.  Without
// the remainders the fitness of a parameter set with S != 2 was off by up to 1e-5 relative.
enum { TC_LR = 0, TC_LA = 2, TC_CR = 4, TC_CA = 6, TC_R0 = 8, TC_EN = 10, TC_BETA, TC_H, TC_R1, TC_R2, TC_PF,
       TC_MHON, TC_LRL, TC_LAL = TC_LRL + 2, TC_CRL = TC_LAL + 2, TC_CAL = TC_CRL + 2, TC_MHONL = TC_CAL + 2,
       TC_COUNT };
static_assert(TC_COUNT <= kMaxConsts, "per-individual Tersoff constants");
// RI (ri.cu:36-110), pair-by-pair part in FP32: Buckingham A[3], b[3] = 1/rho and its FP64
// remainder (the exponent d/rho reaches ~20, where the FP32 rounding of b alone would move
// e^{-d/rho} by ~1e-6), the cation-anion Morse constants lr, la (with remainders), cr, ca (with
// remainders) and r0.  The linear part (damped shifted Coulomb and dispersion) takes FP64
// constants: qq[3] (K_C included), C[3], v_rc, dv_rc, rc and the self-energy coefficient.
enum { RC_A = 0, RC_B = 3, RC_BLO = 6, RC_LR = 9, RC_LA, RC_LRLO, RC_LALO, RC_CR, RC_CA, RC_CRLO, RC_CALO, RC_R0,
       RC_COUNT };
static_assert(RC_COUNT <= kMaxConsts, "per-individual RI constants");
enum { R64_QQ = 0, R64_C = 3, R64_VRC = 6, R64_DVRC, R64_RC, R64_SELF, R64_COUNT };

int consts_per_individual(const DevSet& d) {
  if (d.potential_type == 1 || d.potential_type == 2) return TC_COUNT;
  if (is_ri_type(d.potential_type)) return RC_COUNT;
  return 1;
}
int consts64_per_individual(const DevSet& d) { return is_ri_type(d.potential_type) ? R64_COUNT : 0; }

__device__ __forceinline__ float decode1(float mn, float mx, float x) {
  return __fadd_rn(mn, __fmul_rn(__fsub_rn(mx, mn), x));  // fitness.cu:320-324, no contraction
}

// One thread per individual of every job of the set: FP32 decode exactly like
// the reference, derived constants in FP64 rounded once to FP32.
__global__ void decode_jobs(const JobView* __restrict__ jobs, const int2* __restrict__ indmap, int total) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= total) return;
  const int2 jp = indmap[t];
  const JobView& J = jobs[jp.x];
  const int p = jp.y, nv = J.num_vars, Pstride = J.Pstride, potential_type = J.potential_type;
  const int num_types = J.num_types;
  const float* __restrict__ pmin = J.pmin;
  const float* __restrict__ pmax = J.pmax;
  float* __restrict__ consts = J.consts;
  float* __restrict__ weights = J.weights;
  const float* x = J.pop + (size_t)p * nv;
  auto par = [&](int m) { return (double)decode1(pmin[m], pmax[m], x[m]); };
  auto put = [&](int k, double v) { consts[(size_t)k * Pstride + p] = (float)v; };
  auto put_lo = [&](int k, double v) { consts[(size_t)k * Pstride + p] = (float)(v - (double)(float)v); };
  if (potential_type == 1 || potential_type == 2) {
    const int off = num_types == 2 ? 4 : 0;
    for (int s = 0; s < 2; ++s) {
      const int q = (num_types == 2 && s == 1) ? 4 : 0;
      const double D0 = par(q + 0), A = par(q + 1), R0 = par(q + 2), S = par(q + 3);
      put(TC_LR + s, sqrt(2.0 * S) * A);
      put(TC_LA + s, sqrt(2.0 / S) * A);
      put(TC_CR + s, D0 / (S - 1.0));
      put(TC_CA + s, S * D0 / (S - 1.0));
      put(TC_R0 + s, R0);
      put_lo(TC_LRL + s, sqrt(2.0 * S) * A);
      put_lo(TC_LAL + s, sqrt(2.0 / S) * A);
      put_lo(TC_CRL + s, D0 / (S - 1.0));
      put_lo(TC_CAL + s, S * D0 / (S - 1.0));
    }
    const double en = par(4 + off), R1 = par(7 + off), R2 = par(8 + off);
    put(TC_EN, en);
    put(TC_BETA, par(5 + off));
    put(TC_H, par(6 + off));
    put(TC_R1, R1);
    put(TC_R2, R2);
    put(TC_PF, M_PI / (R2 - R1));
    put(TC_MHON, -0.5 / en);
    put_lo(TC_MHONL, -0.5 / en);
  } else if (is_ri_type(potential_type)) {
    double* __restrict__ c64 = J.consts64;
    auto put64 = [&](int k, double v) { c64[(size_t)k * Pstride + p] = v; };
    const double q0 = par(0), ratio = ri_charge_ratio(potential_type);
    const double kc = 14.399645;  // ri.cu:29
    put64(R64_QQ + 0, q0 * q0 * kc);
    put64(R64_QQ + 1, ratio * q0 * q0 * kc);
    put64(R64_QQ + 2, ratio * ratio * q0 * q0 * kc);
    for (int t = 0; t < 3; ++t) {
      put(RC_A + t, par(1 + 3 * t));
      put(RC_B + t, 1.0 / par(2 + 3 * t));
      put_lo(RC_BLO + t, 1.0 / par(2 + 3 * t));
      put64(R64_C + t, par(3 + 3 * t));
    }
    const double rc = par(10), alpha = 0.2, pif = 0.225675833419103;
    put64(R64_VRC, erfc(alpha * rc) / rc);
    put64(R64_DVRC, -erfc(alpha * rc) / (rc * rc) - pif * exp(-alpha * alpha * rc * rc) / rc);
    put64(R64_RC, rc);
    const double d0 = par(11), al = par(12), r0 = par(13), s = par(14);
    put(RC_LR, sqrt(2.0 * s) * al);
    put(RC_LA, sqrt(2.0 / s) * al);
    put_lo(RC_LRLO, sqrt(2.0 * s) * al);
    put_lo(RC_LALO, sqrt(2.0 / s) * al);
    put(RC_CR, d0 / (s - 1.0));
    put(RC_CA, s * d0 / (s - 1.0));
    put_lo(RC_CRLO, d0 / (s - 1.0));
    put_lo(RC_CALO, s * d0 / (s - 1.0));
    put(RC_R0, r0);
    // damped-Coulomb self energy per unit (q_i / q)^2 (develop/hfo2/find_E.m:10-13)
    put64(R64_SELF, J.ri_self ? q0 * q0 * kc *
                                    (alpha / sqrt(M_PI) + erfc(alpha * rc) / rc +
                                     0.5 * pif * exp(-alpha * alpha * rc * rc))
                              : 0.0);
  } else {
    for (int m = 0; m < nv; ++m) weights[(size_t)m * Pstride + p] = decode1(pmin[m], pmax[m], x[m]);
  }
}

struct Consts {
  const float* base;
  int stride;
  int p;
  __device__ __forceinline__ float operator[](int k) const { return __ldg(base + (size_t)k * stride + p); }
};

// --------------------------------------------------------------------------- Tersoff
// The lane's Tersoff constants.  The pair terms fr = cr e^{-lr t}, fa = ca e^{-la t} come in two
// forms (tersoff_atom, PM): FP64 with FP64 constants (the FP32 value plus its FP64 remainder), or
// FP32 with the remainders applied as first-order corrections.  The remainders are exactly zero
// when S = 2, where the constants are FP32 parameters times powers of two.
// Pair-term forms of the Tersoff items (tersoff_atom).
enum PairMode { kPair32 = 0, kPair64 = 1 };

struct TersoffC {
  double cr64[2], ca64[2], lr64[2], la64[2], r064[2];
  float cr[2], ca[2], lr[2], la[2], r0[2], crl[2], cal[2], lrl[2], lal[2];
  float en, beta, h, r1, r2, pf, mhon, mhonl;
};

// LO: the derived constants carry FP64 remainders (S not fixed at 2); PM: pair-term form (PairMode).
template <bool LO, int PM>
__device__ __forceinline__ void load_tersoff(const Consts& k, TersoffC& C) {
  auto wide = [&](int hi, int lo) { return LO ? (double)k[hi] + (double)k[lo] : (double)k[hi]; };
#pragma unroll
  for (int s = 0; s < 2; ++s) {
    if (PM == kPair64) {
      C.ca64[s] = wide(TC_CA + s, TC_CAL + s);
      C.la64[s] = wide(TC_LA + s, TC_LAL + s);
      C.r064[s] = (double)k[TC_R0 + s];
      if (LO) {  // S = 2: cr = ca / 2 and lr = 2 la, not needed
        C.cr64[s] = wide(TC_CR + s, TC_CRL + s);
        C.lr64[s] = wide(TC_LR + s, TC_LRL + s);
      }
    } else {
      C.ca[s] = k[TC_CA + s];
      C.la[s] = k[TC_LA + s];
      C.r0[s] = k[TC_R0 + s];
      C.cr[s] = k[TC_CR + s];
      C.lr[s] = k[TC_LR + s];
      if (LO) {
        C.crl[s] = k[TC_CRL + s];
        C.cal[s] = k[TC_CAL + s];
        C.lrl[s] = k[TC_LRL + s];
        C.lal[s] = k[TC_LAL + s];
      }
    }
  }
  C.en = k[TC_EN];
  C.beta = k[TC_BETA];
  C.h = k[TC_H];
  C.r1 = k[TC_R1];
  C.r2 = k[TC_R2];
  C.pf = k[TC_PF];
  C.mhon = k[TC_MHON];
  C.mhonl = k[TC_MHONL];
}

// The SFU's base-2 logarithm and exponential (PTX lg2.approx / ex2.approx, subnormals flushed).
// The force items' bond-order powers and pair exponentials use them directly: their arguments and
// results are normal numbers (zeta >= 1e-16 where the result is kept, 1 + zeta^n >= 1, exponents
// of a few units), where the library functions' extra range handling does nothing.
__device__ __forceinline__ float lg2_sfu(float x) {
  float y;
  asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float ex2_sfu(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
constexpr float kLog2e = 1.4426950408889634f;

// cutoff function of minimal_tersoff.cu:77-90
__device__ __forceinline__ void cutoff_fn(float r1, float r2, float pf, float d, float& fc, float& fcp) {
  if (d < r1) {
    fc = 1.0f;
    fcp = 0.0f;
  } else if (d < r2) {
    float s, c;
    sincosf(pf * (d - r1), &s, &c);
    fc = 0.5f * c + 0.5f;
    fcp = -0.5f * pf * s;
  } else {
    fc = 0.0f;
    fcp = 0.0f;
  }
}

// WorkItem::G packs the individuals per item (bits 0-7), whether the item's
// geometry is staged in shared memory (bit 8), the byte size of the force
// scratch that precedes the staged geometry, in 16-byte units (bits 9-23),
// whether the force scratch lives in global memory instead (bit 24), log2 of
// the G of the configuration's default-rule tile (bits 25-27), whose summation
// order every tile of a force item reproduces, whether the item is a force
// item (bit 28; energy/virial items otherwise) and, for an NN2B force item, whether its
// configuration's bond list is symmetric, so that each unordered pair is evaluated once (bit 29).
__host__ __device__ __forceinline__ int item_G(const WorkItem& it) { return it.G & 0xff; }
__host__ __device__ __forceinline__ bool item_staged(const WorkItem& it) { return (it.G >> 8) & 1; }
__host__ __device__ __forceinline__ size_t item_fbytes(const WorkItem& it) { return (size_t)((it.G >> 9) & 0x7fff) * 16; }
__host__ __device__ __forceinline__ bool item_global(const WorkItem& it) { return (it.G >> 24) & 1; }
__host__ __device__ __forceinline__ int item_Grule(const WorkItem& it) { return 1 << ((it.G >> 25) & 7); }
__host__ __device__ __forceinline__ bool item_force(const WorkItem& it) { return (it.G >> 28) & 1; }
__host__ __device__ __forceinline__ bool item_pairs_once(const WorkItem& it) { return (it.G >> 29) & 1; }
__host__ __device__ __forceinline__ int pack_G(int G, bool staged, size_t fbytes, bool global, int Grule, bool force,
                                               bool once = false) {
  int lg = 0;
  while ((1 << lg) < (Grule ? Grule : G)) ++lg;
  return G | (staged ? 1 << 8 : 0) | (int)(((fbytes + 15) / 16) << 9) | (global ? 1 << 24 : 0) | (lg << 25) |
         (force ? 1 << 28 : 0) | (once ? 1 << 29 : 0);
}

// Fixed-order fold of per-lane partial sums held in shared memory as
// red[k * blockDim.x + thread] into res[p][c][k], one warp per k: lane l first adds
// the partials of lane l of every warp (warp order), then a butterfly over the lanes
// of the same individual (l mod G) adds across atom slots.  Both partners of a
// butterfly step form the same sum, so the result is deterministic, and every chain is
// short (a sequential fold over 32/G atom slots per warp stalled the CTA).
// GT: G as a compile-time constant (0: read from the item).
template <int GT>
__device__ __forceinline__ void fold_item(const WorkItem& it, int P, int Nc, const double* red,
                                          double* __restrict__ res) {
  __syncthreads();
  const int G = GT ? GT : item_G(it), nw = blockDim.x >> 5;
  const int lane = threadIdx.x & 31;
  for (int k = threadIdx.x >> 5; k < kResK; k += nw) {
    double s = 0.0;
    for (int w = 0; w < nw; ++w) s += red[(size_t)k * blockDim.x + w * 32 + lane];
    for (int o = G; o < 32; o <<= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    const int p = it.p0 + lane;
    if (lane < G && p < P) res[((size_t)p * Nc + it.config) * kResK + k] = s;
  }
}

// Same for partial sums held in registers (they are first written out).
template <int GT>
__device__ __forceinline__ void reduce_item(const WorkItem& it, int P, int Nc, double (&acc)[kResK],
                                            unsigned char* smem, double* __restrict__ res) {
  __syncthreads();
  double* red = reinterpret_cast<double*>(smem);
#pragma unroll
  for (int k = 0; k < kResK; ++k) red[(size_t)k * blockDim.x + threadIdx.x] = acc[k];
  fold_item<GT>(it, P, Nc, red, res);
}

// Geometry of one configuration as a CTA sees it.  Unstaged: the global CSR
// arrays offset to the configuration's first atom / bond (bond j of local atom
// il at boff[il] - bond0 + j).  Staged: a slot-major copy in shared memory
// (bond j of atom il at j * Na + il, `stride` = Na), so that the lanes of a warp,
// which hold consecutive atoms, read consecutive entries without bank conflicts.
// ST: 1 staged, 0 CSR, -1 decided at run time by `stride`.
template <int ST>
struct GeoT {
  const float4* g;     // (unit vector, d)
  const double* d64;   // d in FP64
  const float* dlo;    // d - (float)d
  const uint8_t* pt;   // pair set
  const int* rev;      // slot * Na + atom of the reverse bond (force scratch position)
  const int* nn;       // [Na]
  const int* boff;     // [Na] bond offset (global numbering; subtract bond0), unstaged only
  int bond0;
  int stride;          // Na when staged (slot-major), 0 for the CSR arrays
  __device__ __forceinline__ int base(int il) const {
    if constexpr (ST == 1) return il;
    else if constexpr (ST == 0) return boff[il] - bond0;
    else return stride ? il : boff[il] - bond0;
  }
  __device__ __forceinline__ int step() const {
    if constexpr (ST == 1) return stride;
    else if constexpr (ST == 0) return 1;
    else return stride ? stride : 1;
  }
};
using Geo = GeoT<-1>;

// Copies configuration c's geometry into shared memory, slot-major with ZC
// slots, with all threads of the CTA (independent loads, then one barrier).
// D64: the FP64 bond lengths (FP64 pair terms), else their FP32 remainders.
template <int ZC, bool D64>
__device__ __forceinline__ Geo stage_geometry(const DevView& S, int c, int atom0, int Na, bool force,
                                              unsigned char* base) {
  const int n = ZC * Na;
  float4* sg = reinterpret_cast<float4*>(base);
  double* sd = reinterpret_cast<double*>(sg + n);
  float* sl = reinterpret_cast<float*>(sd + (D64 ? n : 0));
  int* snn = reinterpret_cast<int*>(sl + (D64 ? 0 : n));
  int* srev = snn + Na;
  uint8_t* spt = reinterpret_cast<uint8_t*>(srev + (force ? n : 0));
  if (!D64 && S.g_sm) {
    // a straight copy of the slot-major global layout
    const int o = S.sm_off[c];
    for (int t = threadIdx.x; t < n; t += blockDim.x) {
      sg[t] = __ldg(&S.g_sm[o + t]);
      sl[t] = __ldg(&S.dl_sm[o + t]);
      spt[t] = S.pt_sm[o + t];
      if (force) srev[t] = S.rev_sm_sm[o + t];
    }
  } else {
    for (int t = threadIdx.x; t < n; t += blockDim.x) {
      const int j = t / Na, il = t - j * Na, i = atom0 + il;
      if (j < S.NN[i]) {
        const int b = S.off[i] + j;
        sg[t] = __ldg(&S.g32[b]);
        if (D64) sd[t] = __ldg(&S.d64[b]);
        else sl[t] = __ldg(&S.tdl[b]);
        spt[t] = S.ptype[b];
        if (force) srev[t] = S.rev_sm[b];
      }
    }
  }
  for (int k = threadIdx.x; k < Na; k += blockDim.x) snn[k] = S.NN[atom0 + k];
  __syncthreads();
  return Geo{sg, sd, sl, spt, srev, snn, nullptr, 0, Na};
}

// One atom of the minimal Tersoff potential (minimal_tersoff.cu:122-405) for
// the lane's parameter vector.  Returns the site energy (FP64); writes the partial
// forces f_ij (FORCE) or adds -r_ij (x) f_ij into v[6] (energy/virial items).
//
// With unit vectors u and the bond scalars
//   S_k = b'_k fa_k, T_k = S_k fc_k, A'_j = fc'_j (fr_j - b_j fa_j) + fc_j (fr'_j - b_j fa'_j)
// the reference's f_ij (minimal_tersoff.cu:250-307) is
//   f_ij = 1/2 [ (A'_j - fc'_j sum_k T_k g_jk - m_j sum_k q_jk cos_jk) u_j + m_j sum_k q_jk u_k ]
// with q_jk = beta (cos_jk - h) (S_j fc_k + T_k) and m_j = -2 fc_j / d_j.
//
// Precision.  Near equilibrium fr - b fa and fr' - b fa' are small differences of large
// terms, and the virial sums the radial forces of thousands of bonds, so the pair terms are
// evaluated in FP64 (FP64 bond length and constants, FP64 exponentials exp_d.cuh; when S = 2,
// lr = 2 la and one exponential serves both terms): the site energy and A'_j are rounded once, after the
// cancellation.  Measured on the 500-configuration Si set, this took the relative fitness error
// of individuals near the fitted optimum from 8.5e-7 to 2.4e-7; the bond order and the
// three-body terms stay FP32 (b to ~1 ulp, powf_dd.cuh).
//
// FULL: every one of the ZC bond slots is present (Z == ZC, e.g. all atoms of a diamond
// lattice), so that the per-slot guards fold away at compile time.
//
// INNER: every bond of the atom lies inside r1 (fc = 1, fc' = 0; most atoms of a set near
// equilibrium), so that the cutoff branches and the fc' terms drop out.  The expressions that
// involve fc or fc' are written with explicit roundings, so that for such an atom both forms give
// the same bits: the force-item tiles, which group atoms into warps differently, stay identical.
template <int ZC, int NT, bool FORCE, bool FULL, bool LO, int PM, bool INNER, class GEO>
__device__ __forceinline__ double tersoff_bonds(const GEO& geo, const TersoffC& C, int il, int Na, float* fsm, int G,
                                                int g, float (&v)[6], int Z, int b0, int bs, const float (&ux)[ZC],
                                                const float (&uy)[ZC], const float (&uz)[ZC], const float (&dd)[ZC],
                                                const double (&d64)[PM == kPair64 ? ZC : 1], const int (&st)[ZC]) {
  // pass A: cutoff of every bond
  float fc[ZC], fcp[ZC];
#pragma unroll
  for (int j = 0; j < ZC; ++j) {
    if constexpr (INNER) {
      fc[j] = 1.0f;
      fcp[j] = 0.0f;
    } else {
      fc[j] = fcp[j] = 0.f;
      if (j < Z) cutoff_fn(C.r1, C.r2, C.pf, dd[j], fc[j], fcp[j]);
    }
  }
  // pass B: bond order, site energy and the per-bond force scalars
  // cos(theta_jik) = u_j . u_k from the FP32 unit vectors (as accurate as a stored FP32 cosine);
  // the expression is symmetric bit for bit, so with up to 4 bonds the 6 distinct cosines are
  // formed once and kept in registers for both passes
  constexpr bool kSym = ZC == 4;
  float cs[kSym ? ZC : 1][kSym ? ZC : 1];
  if constexpr (kSym) {
#pragma unroll
    for (int j = 0; j < ZC; ++j)
#pragma unroll
      for (int k = j + 1; k < ZC; ++k)
        cs[j][k] = cs[k][j] = fmaf(uz[j], uz[k], fmaf(uy[j], uy[k], ux[j] * ux[k]));
  }
  auto cosine = [&](int j, int k) {
    if constexpr (kSym) return cs[j][k];
    else return fmaf(uz[j], uz[k], fmaf(uy[j], uy[k], ux[j] * ux[k]));
  };
  float Ap[ZC], Sb[ZC], Tb[ZC];
  double pe = 0.0;    // FP64 pair terms
  float pe32 = 0.f;   // FP32 pair terms
#pragma unroll
  for (int j = 0; j < ZC; ++j) {
    Ap[j] = Sb[j] = Tb[j] = 0.f;
    if (j < Z) {
      float zeta = 0.f;
#pragma unroll
      for (int k = 0; k < ZC; ++k) {
        if (k < Z && k != j) {
          const float x = cosine(j, k) - C.h;
          zeta = fmaf(fc[k] * C.beta, x * x, zeta);
        }
      }
      // b = 1, b' = 0 below zeta = 1e-16 (minimal_tersoff.cu:178-185), selected after the
      // evaluation rather than branched around it (the threshold is almost never met).
      // Force items: FP32 through the SFU's log2 / exp2 (on the 500-configuration Si set the
      // fitness error against FP64 stays at 1.1e-7 for random individuals and 3.1e-7 near the
      // optimum, for 7 % less time per generation than the library log2f / exp2f / expf);
      // energy/virial items: powf_dd (double-float log2 and exponent)
      float zn, opz, b;
      if constexpr (PM == kPair32) {
        zn = ex2_sfu(C.en * lg2_sfu(zeta));
        opz = 1.0f + zn;
        const float lg = lg2_sfu(opz);
        b = ex2_sfu(fmaf(C.mhon, lg, C.mhonl * lg));
      } else {
        zn = powf_dd(zeta, C.en);
        opz = 1.0f + zn;
        b = powf_dd(opz, C.mhon, C.mhonl);
      }
      float bp = __fdividef(-0.5f * b * zn, opz * zeta);
      if (zeta < 1.0e-16f) {
        b = 1.f;
        bp = 0.f;
      }
      // pair terms fr = cr e^{-lr t}, fa = ca e^{-la t}, t = d - r0.  With S = 2 (!LO) lr = 2 la
      // and cr = ca / 2, so fr = fa e^{-la t} / 2 from the one exponential.
      const int s = NT == 2 ? st[j] : 0;
      float fa32;
      if constexpr (PM == kPair64) {
        // exponentials to 7e-12 (exp_d.cuh), far below the FP32 rounding of A'_j
        const double t = d64[j] - (s ? C.r064[1] : C.r064[0]);
        const double la = s ? C.la64[1] : C.la64[0];
        const double ea = exp_d_clamped<9>(-la * t);
        const double fa = (s ? C.ca64[1] : C.ca64[0]) * ea;
        const double bd = b;
        double e, dA;  // fr - b fa and fr' - b fa'
        if constexpr (LO) {
          const double lr = s ? C.lr64[1] : C.lr64[0];
          const double fr = (s ? C.cr64[1] : C.cr64[0]) * exp_d_clamped<9>(-lr * t);
          e = fma(-bd, fa, fr);
          dA = fma(bd * la, fa, -lr * fr);
        } else {
          // S = 2: fr = fa e / 2 and fr' - b fa' = la (b fa - 2 fr) = -la (e + fr)
          const double fr = 0.5 * fa * ea;
          e = fma(-bd, fa, fr);
          dA = -la * (e + fr);
        }
        if (INNER || (fc[j] == 1.0f && fcp[j] == 0.0f)) {  // inside r1: no conversions of fc, fc'
          pe = fma(0.5, e, pe);
          Ap[j] = (float)dA;
        } else {
          pe = fma(0.5 * (double)fc[j], e, pe);
          Ap[j] = (float)fma((double)fcp[j], e, (double)fc[j] * dA);
        }
        fa32 = (float)fa;
      } else {
        // FP32 (force items; exponentials through the SFU, ex2_sfu): the FP64 remainder of d as a
        // first-order correction e^{-l (t + d_lo)} = e^{-l t} (1 - l d_lo); with S = 2 (lr = 2 la) one exponential,
        // e^{-lr t} = (e^{-la t})^2 (the same fitness error as two exponentials on the
        // 500-configuration Si set, 1.4 % less time); for S != 2 two, and the remainders of the
        // constants c e^{-l t} = c_h E + (c_l - c_h l_l t) E, l f = l_h f + l_l f
        const float t = dd[j] - (s ? C.r0[1] : C.r0[0]), dlo = geo.dlo[b0 + j * bs];
        const float lr = s ? C.lr[1] : C.lr[0], la = s ? C.la[1] : C.la[0];
        const float cr = s ? C.cr[1] : C.cr[0], ca = s ? C.ca[1] : C.ca[0];
        float er, ea;
        if constexpr (!LO) {
          ea = ex2_sfu(-la * t * kLog2e);
          ea = fmaf(-la * dlo, ea, ea);
          er = ea * ea;
        } else {
          er = ex2_sfu(-lr * t * kLog2e);
          ea = ex2_sfu(-la * t * kLog2e);
          er = fmaf(-lr * dlo, er, er);
          ea = fmaf(-la * dlo, ea, ea);
        }
        float fr = cr * er, fa = ca * ea;
        float frp = -lr * fr, fap = -la * fa;
        if constexpr (LO) {
          fr = fmaf(fmaf(-cr * (s ? C.lrl[1] : C.lrl[0]), t, s ? C.crl[1] : C.crl[0]), er, fr);
          fa = fmaf(fmaf(-ca * (s ? C.lal[1] : C.lal[0]), t, s ? C.cal[1] : C.cal[0]), ea, fa);
          frp = fmaf(-(s ? C.lrl[1] : C.lrl[0]), fr, -lr * fr);
          fap = fmaf(-(s ? C.lal[1] : C.lal[0]), fa, -la * fa);
        }
        const float e = fr - b * fa;
        pe32 = fmaf(0.5f * fc[j], e, pe32);
        const float dA = __fmaf_rn(-b, fap, frp);  // fr' - b fa'
        if constexpr (INNER) Ap[j] = dA;
        else Ap[j] = __fmaf_rn(fcp[j], e, __fmul_rn(fc[j], dA));
        fa32 = fa;
      }
      Sb[j] = bp * fa32;
      Tb[j] = Sb[j] * fc[j];
    }
  }
  // pass C: three-body force terms
#pragma unroll
  for (int j = 0; j < ZC; ++j) {
    if (j < Z) {
      float sumG = 0.f, accC = 0.f, Vx = 0.f, Vy = 0.f, Vz = 0.f;
      const float Sj = Sb[j];
#pragma unroll
      for (int k = 0; k < ZC; ++k) {
        if (k < Z && k != j) {
          const float cjk = cosine(j, k);
          const float bx = C.beta * (cjk - C.h);
          // S_j fc_k + T_k: with fc_k = 1 an explicit add (a folded fmaf(S_j, 1, T_k) could be
          // contracted with the products S_j, T_k, unlike the general form)
          const float q = bx * (INNER ? __fadd_rn(Sj, Tb[k]) : __fmaf_rn(Sj, fc[k], Tb[k]));
          if constexpr (!INNER) sumG = fmaf(Tb[k], bx * (cjk - C.h), sumG);
          accC = fmaf(q, cjk, accC);
          Vx = fmaf(q, ux[k], Vx);
          Vy = fmaf(q, uy[k], Vy);
          Vz = fmaf(q, uz[k], Vz);
        }
      }
      const float m = __fdividef(-2.0f * fc[j], dd[j]);
      const float cu = 0.5f * __fmaf_rn(-m, accC, INNER ? Ap[j] : __fmaf_rn(-fcp[j], sumG, Ap[j]));
      if (FORCE) {
        const float cv = 0.5f * m;
        const float fx = fmaf(cu, ux[j], cv * Vx);
        const float fy = fmaf(cu, uy[j], cv * Vy);
        const float fz = fmaf(cu, uz[j], cv * Vz);
        // slot-major scratch [slot][atom][xyz][G]: the lanes of a warp (consecutive atoms,
        // same slot) write consecutive words
        const int bl = j * Na + il;
        fsm[(bl * 3 + 0) * G + g] = fx;
        fsm[(bl * 3 + 1) * G + g] = fy;
        fsm[(bl * 3 + 2) * G + g] = fz;
      } else {
        // -r_ij (x) f_ij = u_j (x) t_j with t_j = a u_j + fc_j V_j, a = -d_j cu_j (r_j = d_j u_j,
        // f_ij = cu u_j + (m_j / 2) V_j and -d_j m_j / 2 = fc_j), components xx yy zz xy yz zx
        const float a = -dd[j] * cu;
        const float tx = INNER ? __fmaf_rn(a, ux[j], Vx) : __fmaf_rn(a, ux[j], __fmul_rn(fc[j], Vx));
        const float ty = INNER ? __fmaf_rn(a, uy[j], Vy) : __fmaf_rn(a, uy[j], __fmul_rn(fc[j], Vy));
        const float tz = INNER ? __fmaf_rn(a, uz[j], Vz) : __fmaf_rn(a, uz[j], __fmul_rn(fc[j], Vz));
        v[0] = fmaf(ux[j], tx, v[0]);
        v[1] = fmaf(uy[j], ty, v[1]);
        v[2] = fmaf(uz[j], tz, v[2]);
        v[3] = fmaf(ux[j], ty, v[3]);
        v[4] = fmaf(uy[j], tz, v[4]);
        v[5] = fmaf(uz[j], tx, v[5]);
      }
    }
  }
  return pe + (double)pe32;
}

template <int ZC, int NT, bool FORCE, bool FULL, bool LO, int PM, class GEO>
__device__ __forceinline__ double tersoff_atom(const GEO& geo, const TersoffC& C, int il, int Na, float* fsm, int G,
                                               int g, float (&v)[6]) {
  const int Z = FULL ? ZC : geo.nn[il];
  const int b0 = geo.base(il), bs = geo.step();  // bond j at b0 + j * bs
  float ux[ZC], uy[ZC], uz[ZC], dd[ZC];
  double d64[PM == kPair64 ? ZC : 1];  // FP64 lengths, loaded with the rest of the geometry
  int st[ZC];
#pragma unroll
  for (int j = 0; j < ZC; ++j) {
    st[j] = 0;
    if (j < Z) {
      const float4 q = geo.g[b0 + j * bs];
      ux[j] = q.x;
      uy[j] = q.y;
      uz[j] = q.z;
      dd[j] = q.w;
      if constexpr (PM == kPair64) d64[j] = geo.d64[b0 + j * bs];
      if (NT == 2) st[j] = geo.pt[b0 + j * bs];
    } else {
      ux[j] = uy[j] = uz[j] = 0.f;
      dd[j] = 1.0f;
      if constexpr (PM == kPair64) d64[j] = 1.0;
    }
  }
  if constexpr (FULL) {
    bool inside = true;
#pragma unroll
    for (int j = 0; j < ZC; ++j) inside = inside && dd[j] < C.r1;
    // the lanes that reach this point take one form together
    if (__all_sync(__activemask(), inside))
      return tersoff_bonds<ZC, NT, FORCE, FULL, LO, PM, true>(geo, C, il, Na, fsm, G, g, v, Z, b0, bs, ux, uy, uz, dd,
                                                               d64, st);
  }
  return tersoff_bonds<ZC, NT, FORCE, FULL, LO, PM, false>(geo, C, il, Na, fsm, G, g, v, Z, b0, bs, ux, uy, uz, dd,
                                                            d64, st);
}

// Energy/virial items (FORCE = false) keep their FP64 per-lane sums in shared
// memory (red[k][thread]) to save registers; a staged item's geometry follows
// that region.  Force items put the f_ij scratch first, the staged geometry
// after it, and reuse the start of shared memory for the final fold.
// GT: the item's individuals per item G as a compile-time constant (0: read from the item), so
// that the force scratch addressing and the atom-slot split fold into shifts and constants;
// ST: staged (1) or in-place CSR (0) geometry, or decided per item (-1).
// Bytes of the force items' shared-memory table of per-individual constants (G entries).
__host__ __device__ constexpr size_t tersoff_table_bytes(int G) { return ((size_t)G * sizeof(TersoffC) + 15) & ~(size_t)15; }
// A force item whose G differs from its configuration's default-rule G keeps the
// per-(individual, atom) squared force errors in a table, row g = the item's atoms: shared-memory
// items in the f_ij scratch once every f_ij has been read, an item with its scratch in global
// memory after it.
__host__ __device__ constexpr int ferr_row(int Na) { return Na; }
// Atoms per thread in a shared-memory force item's gather pass, at most: their squared errors
// wait in registers until the scratch is free.  The host's G rule keeps Na * G <= 256 * this.
__host__ __device__ constexpr int ferr_steps(int zc) { return zc == 4 ? 6 : (zc == 8 ? 4 : 2); }

// Pair-term form of the two kinds of Tersoff items (tersoff_atom, PairMode).  Energy/virial items
// take the FP64 pair terms: the configuration virial sums the radial forces of all bonds, whose
// cancellation near equilibrium amplifies FP32 rounding.  Force items stay FP32: their force error
// was the same with FP64 pair terms (500-configuration Si set, individuals near the optimum: 2.2e-7
// vs 2.3e-7 of the force RMSE) at 40 % more time.
constexpr int kPairModeEV = kPair64;
constexpr int kPairModeForce = kPair32;

template <int ZC, int NT, bool FORCE, int BLK, int GT, int ST, bool LO>
__device__ __forceinline__ void tersoff_item(const JobView* __restrict__ jobs, const WorkItem& it,
                                             unsigned char* smem) {
  constexpr int NW = BLK / 32;
  constexpr int PM = FORCE ? kPairModeForce : kPairModeEV;
  const JobView& J = jobs[it.job];
  const DevView S = J.v;
  const int P = J.P;
  double* __restrict__ res = J.res;
  float* __restrict__ fdump = J.fdump;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int G = GT ? GT : item_G(it), A = 32 / G;
  const int g = lane & (G - 1), aslot = lane / G;
  const int p = it.p0 + g;
  const Consts kc{J.consts, J.Pstride, p < P ? p : it.p0};
  TersoffC Creg;
  load_tersoff<LO, PM>(kc, Creg);
  const int c = it.config, atom0 = S.Na_sum[c], Na = S.Na[c];
  const int bond0 = S.off[atom0];
  // Force items keep the G individuals' constants in a shared-memory table at the start of the
  // dynamic shared memory, read where used: the force kernel runs at its register bound, and
  // constants held in registers across the atom loop were spilled to local memory.
  const size_t tab = FORCE ? tersoff_table_bytes(G) : 0;
  TersoffC* ctab = reinterpret_cast<TersoffC*>(smem);
  if (FORCE && warp == 0 && aslot == 0) ctab[g] = Creg;
  // force scratch: shared memory, or for configurations too large for it the item's own
  // region of global memory (visible to the whole CTA after __syncthreads as well)
  const bool glob = FORCE && item_global(it);
  float* fsm = glob ? J.gscratch + (size_t)it.gofs * 64 : reinterpret_cast<float*>(smem + tab);
  double* red = reinterpret_cast<double*>(smem);
  const size_t front = FORCE ? tab + item_fbytes(it) : (size_t)BLK * kResK * sizeof(double);
  if (FORCE) __syncthreads();  // the constants table
  const TersoffC& C = FORCE ? ctab[g] : Creg;
  if (!FORCE) {
#pragma unroll
    for (int k = 0; k < 7; ++k) red[k * BLK + threadIdx.x] = 0.0;
  }
  GeoT<ST> geo;
  if ((ST == 1 || ST == -1) && item_staged(it)) {
    const Geo s0 = stage_geometry<ZC, PM == kPair64>(S, c, atom0, Na, FORCE, smem + front);
    geo = GeoT<ST>{s0.g, s0.d64, s0.dlo, s0.pt, s0.rev, s0.nn, s0.boff, s0.bond0, s0.stride};
  } else if (FORCE && ST != 0) {
    // force items read the slot-major global copy: the lanes of a warp hold consecutive atoms and
    // read consecutive words, as from the staged copy
    const int o = S.sm_off[c];
    geo = GeoT<ST>{S.g_sm + o, nullptr, S.dl_sm + o, S.pt_sm + o, S.rev_sm_sm + o, S.NN + atom0, nullptr, 0, Na};
  } else {
    geo = GeoT<ST>{S.g32 + bond0, S.d64 + bond0, S.tdl + bond0, S.ptype + bond0, S.rev_sm + bond0, S.NN + atom0,
                   S.off + atom0, bond0, 0};
  }
  for (int base = warp * A; base < Na; base += NW * A) {
    const int il = base + aslot;
    // warp-uniform choice of the guard-free form (no divergence between the two)
    const bool full = __all_sync(0xffffffffu, il >= Na || geo.nn[il] == ZC);
    if (il < Na) {
      float v[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
      const double pe = full ? tersoff_atom<ZC, NT, FORCE, true, LO, PM>(geo, C, il, Na, fsm, G, g, v)
                            : tersoff_atom<ZC, NT, FORCE, false, LO, PM>(geo, C, il, Na, fsm, G, g, v);
      if (!FORCE) {
        red[threadIdx.x] += pe;
#pragma unroll
        for (int k = 0; k < 6; ++k) red[(k + 1) * BLK + threadIdx.x] += (double)v[k];
      }
    }
  }
  if (!FORCE) {
    red[7 * BLK + threadIdx.x] = 0.0;
    fold_item<GT>(it, P, S.Nc, red, res);
    return;
  }
  __syncthreads();
  const int N = S.N, Nf = S.N_force;
  const int Gr = item_Grule(it);
  // gather pass: F_i = sum_j (f_ij - f_ji) of (individual g, atom il) and its squared error
  auto atom_error = [&](int il) -> double {
    const int i = atom0 + il;
    const int b0 = geo.base(il), bs = geo.step(), Z = geo.nn[il];
    float Fx = 0.f, Fy = 0.f, Fz = 0.f;
    int rls[ZC];
#pragma unroll
    for (int j = 0; j < ZC; ++j) rls[j] = j < Z ? geo.rev[b0 + j * bs] : 0;
#pragma unroll
    for (int j = 0; j < ZC; ++j) {
      if (j < Z) {
        const int bl = j * Na + il, rl = rls[j];
        Fx += fsm[(bl * 3 + 0) * G + g] - fsm[(rl * 3 + 0) * G + g];
        Fy += fsm[(bl * 3 + 1) * G + g] - fsm[(rl * 3 + 1) * G + g];
        Fz += fsm[(bl * 3 + 2) * G + g] - fsm[(rl * 3 + 2) * G + g];
      }
    }
    const double dx = (double)Fx - (double)S.force_ref[i];
    const double dy = (double)Fy - (double)S.force_ref[i + N];
    const double dz = (double)Fz - (double)S.force_ref[i + 2 * (size_t)N];
    if (fdump && p < P) {
      fdump[((size_t)p * 3 + 0) * Nf + i] = Fx;
      fdump[((size_t)p * 3 + 1) * Nf + i] = Fy;
      fdump[((size_t)p * 3 + 2) * Nf + i] = Fz;
    }
    return dx * dx + dy * dy + dz * dz;
  };
  // Each individual's squared force errors are summed in the order of the configuration's
  // default-rule tile (Gr individuals per item, Ar = 32 / Gr atoms per warp step, 8 warps): per
  // thread the atoms w Ar + a + 8 Ar k in k order, then the 8 warps' sums in warp order
  // (fold_item), then a butterfly over the Ar atom slots (a pairwise tree in slot order: each
  // step adds two partners' values, and a + b == b + a).  An item of that tile sums in that
  // order as it goes; any other tile (another G, or 32 individuals with global scratch) keeps the
  // errors in a table and one warp per Gr individuals replays the order.  Every tile therefore
  // gives the same bits, and the default tile pays nothing for it.
  if (G == Gr) {
    double ferr = 0.0;
    for (int base = warp * A; base < Na; base += NW * A) {
      const int il = base + aslot;
      if (il < Na) ferr += atom_error(il);
    }
    __syncthreads();  // the fold overwrites the f_ij scratch
#pragma unroll
    for (int k = 0; k < 7; ++k) red[k * BLK + threadIdx.x] = 0.0;
    red[7 * BLK + threadIdx.x] = ferr;
    fold_item<GT>(it, P, S.Nc, red, res);
    return;
  }
  auto replay = [&](const double* ftab) {
    const int Ar = 32 / Gr, gr = lane & (Gr - 1), a = lane / Gr;
    for (int gb = warp * Gr; gb < G; gb += NW * Gr) {  // warp-uniform: every lane takes the shuffles
      const int gg = gb + gr;
      double s = 0.0;
      if (gg < G) {
        for (int w = 0; w < NW; ++w) {
          double t = 0.0;
          for (int il = w * Ar + a; il < Na; il += NW * Ar) t += ftab[(size_t)gg * Na + il];
          s += t;
        }
      }
      for (int o = Gr; o < 32; o <<= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
      const int pp = it.p0 + gg;
      if (a == 0 && gg < G && pp < P) {
        double* r = res + ((size_t)pp * S.Nc + c) * kResK;
#pragma unroll
        for (int k = 0; k < 7; ++k) r[k] = 0.0;
        r[7] = s;
      }
    }
  };
  if (glob) {
    double* ftab = reinterpret_cast<double*>(fsm + (size_t)ZC * Na * 3 * 32);
    for (int base = warp * A; base < Na; base += NW * A) {
      const int il = base + aslot;
      if (il < Na) ftab[(size_t)g * Na + il] = atom_error(il);
    }
    __syncthreads();
    replay(ftab);
  } else {
    // the errors wait in registers (at most ferr_steps per thread, by the host's G rule) until
    // every f_ij has been read, then take the scratch's place
    constexpr int KS = ferr_steps(ZC);
    if (Na > KS * NW * A) {  // outside the host's G rule: a NaN fitness rather than a wrong one
      for (int gg = threadIdx.x; gg < G; gg += BLK)
        if (it.p0 + gg < P) res[((size_t)(it.p0 + gg) * S.Nc + c) * kResK + 7] = __longlong_as_double(0x7ff8000000000000LL);
      return;
    }
    double ev[KS];
#pragma unroll
    for (int k = 0; k < KS; ++k) {
      const int il = (warp + k * NW) * A + aslot;
      ev[k] = il < Na ? atom_error(il) : 0.0;
    }
    __syncthreads();
    double* ftab = reinterpret_cast<double*>(smem + tab);
#pragma unroll
    for (int k = 0; k < KS; ++k) {
      const int il = (warp + k * NW) * A + aslot;
      if (il < Na) ftab[g * Na + il] = ev[k];
    }
    __syncthreads();
    replay(ftab);
  }
}

// fitness.cu:329-331, 437-555 in FP64 for individual p, by one warp: lane c sums configurations
// c, c + 32, ... in order, then a butterfly; the same order whichever warp or launch folds, and
// the same operations: every product and sum is an explicit intrinsic, so that the compiler's
// choice of contracting a * b + c into an FMA cannot differ between the kernels this is inlined in.
// Reads go through L2 (ld.cg): other CTAs of the same launch wrote the results.
__device__ __forceinline__ void fold_fitness(const JobView& J, int p, int lane) {
  const int Nc = J.v.Nc, Nc_force = J.Nc_force;
  const double* __restrict__ res = J.res;
  const double* __restrict__ E_ref = J.E_ref;
  const double* __restrict__ W_ref = J.W_ref;
  double eE = 0, eW = 0, eF = 0;
  for (int c = lane; c < Nc; c += 32) {
    const double* r = res + ((size_t)p * Nc + c) * kResK;
    if (c >= Nc_force) {
      const double de = __ldcg(r) - E_ref[c];
      eE = __fma_rn(de, de, eE);
#pragma unroll
      for (int k = 0; k < 6; ++k) {
        const double dw = __ldcg(r + 1 + k) - W_ref[c + (size_t)Nc * k];
        eW = __fma_rn(dw, dw, eW);
      }
    } else {
      eF += __ldcg(r + 7);
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    eE += __shfl_xor_sync(0xffffffffu, eE, o);
    eW += __shfl_xor_sync(0xffffffffu, eW, o);
    eF += __shfl_xor_sync(0xffffffffu, eF, o);
  }
  if (lane == 0) {
    const double rE = sqrt(eE / J.nE), rW = sqrt(eW / J.nW), rF = sqrt(eF / J.nF);
    J.fitness[p] = __dadd_rn(__dadd_rn(__dmul_rn((double)J.wE, rE), __dmul_rn((double)J.wW, rW)),
                             __dmul_rn((double)J.wF, rF));
    if (J.comps) {
      J.comps[3 * (size_t)p + 0] = rE;
      J.comps[3 * (size_t)p + 1] = rW;
      J.comps[3 * (size_t)p + 2] = rF;
    }
  }
}

// End of every work item: its results for individuals p0 .. p0 + G - 1 are written.  Each of those
// individuals' completion count goes up by one with a release-acquire atomic (the CTA barrier
// orders every thread's writes before it, and release is cumulative); the item that brings an individual to Nc
// configurations folds its fitness and resets the count for the next generation.  Nothing waits.
// Release-acquire increment at device scope: releases the CTA's writes ordered before it (by the
// preceding CTA barrier) and acquires the writes released by earlier increments.
__device__ __forceinline__ int atomic_add_acq_rel(int* a, int v) {
  int old;
  asm volatile("atom.acq_rel.gpu.global.add.s32 %0, [%1], %2;" : "=r"(old) : "l"(a), "r"(v) : "memory");
  return old;
}

__device__ __forceinline__ void finish_item(const JobView* __restrict__ jobs, const WorkItem& it, int G) {
  const JobView& J = jobs[it.job];
  if (!J.fit_count) return;
  __shared__ int s_last[32];
  __syncthreads();
  if (threadIdx.x < 32) {
    const int p = it.p0 + threadIdx.x;
    int last = 0;
    if (threadIdx.x < G && p < J.P) last = atomic_add_acq_rel(&J.fit_count[p], 1) == J.v.Nc - 1;
    s_last[threadIdx.x] = last;
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  for (int g = threadIdx.x >> 5; g < G; g += blockDim.x >> 5) {
    if (!s_last[g]) continue;  // warp-uniform
    __threadfence();
    fold_fitness(J, it.p0 + g, lane);
    if (lane == 0) J.fit_count[it.p0 + g] = 0;
  }
}

// Energy/virial Tersoff items read their geometry through L1: staging it in shared memory
// would cap the CTAs per SM without making the per-atom loads cheaper (measured).
constexpr bool kStageEV = false;

// LO: the job's derived constants need their FP64 remainders (tersoff_consts_exact).  One launch
// holds both kinds of items (item_force), 256 threads each: three CTAs per SM for ZC = 4 bound
// both bodies to 80 registers (the energy/virial body measured as fast there as in 128-thread
// CTAs at 96 registers, five per SM).
template <int ZC, int NT, bool LO>
__global__ void __launch_bounds__(kBlock, ZC == 4 ? 3 : 1) tersoff_batched(const JobView* __restrict__ jobs,
                                                                          const WorkItem* __restrict__ items) {
  extern __shared__ __align__(16) unsigned char smem[];
  const WorkItem it = items[blockIdx.x];
  if (!item_force(it)) {
    // energy/virial items: always 32 individuals (the run-time geometry form: the CSR-only
    // specialisation spilled at this kernel's register bound and ran 5 % slower)
    tersoff_item<ZC, NT, false, kBlock, 32, -1, LO>(jobs, it, smem);
  } else if constexpr (ZC == 4) {
#define GPUGA_TI(GG)                                    \
  case GG:                                              \
    tersoff_item<ZC, NT, true, kBlock, GG, 1, LO>(jobs, it, smem); \
    break;
    switch (item_G(it)) {
      GPUGA_TI(32)
      GPUGA_TI(16)
      GPUGA_TI(8)
      GPUGA_TI(4)
      GPUGA_TI(2)
      default: GPUGA_TI(1)
    }
#undef GPUGA_TI
  } else {
    tersoff_item<ZC, NT, true, kBlock, 0, -1, LO>(jobs, it, smem);
  }
  finish_item(jobs, it, item_G(it));
}

// --------------------------------------------------------------------------- RI / NN2B
// RI pair by pair (ri.cu:77-110): only the terms that are not linear in the per-individual
// constants, the Buckingham repulsion A e^{-d/rho} and, for cation-anion pairs, the Morse pair
// cr e^{-lr (d - r0)} - ca e^{-la (d - r0)}.  The damped shifted Coulomb and the dispersion
// -C/d^6 enter through their FP64 geometric sums (ri_linear_atoms, geometry.cu), so the large
// alternating Coulomb terms never pass through FP32 arithmetic.
//
// The exponents d/rho and lr (d - r0), la (d - r0) reach ~20, so their FP32 rounding alone
// would move exp() by ~1e-6 relative; they are formed as hi + lo (exact FMA residuals, the FP64
// remainders of d, 1/rho, lr and la) and exp(-(hi + lo)) = exp(-hi) (1 - lo).
struct RIC {  // the lane's RI constants, loaded once per work item
  float a[3], b[3], blo[3], lr, la, lrlo, lalo, cr, ca, crlo, calo, r0;
};

__device__ __forceinline__ void load_ri(const Consts& k, RIC& R) {
#pragma unroll
  for (int t = 0; t < 3; ++t) {
    R.a[t] = k[RC_A + t];
    R.b[t] = k[RC_B + t];
    R.blo[t] = k[RC_BLO + t];
  }
  R.lr = k[RC_LR];
  R.la = k[RC_LA];
  R.lrlo = k[RC_LRLO];
  R.lalo = k[RC_LALO];
  R.cr = k[RC_CR];
  R.ca = k[RC_CA];
  R.crlo = k[RC_CRLO];
  R.calo = k[RC_CALO];
  R.r0 = k[RC_R0];
}

// exp(-x y) for x = xh + xl, y = yh + yl (double-float), to ~1 ulp of exp
__device__ __forceinline__ float exp_neg_dd(float xh, float xl, float yh, float yl) {
  const float p = xh * yh;
  const float lo = fmaf(xh, yh, -p) + fmaf(xh, yl, xl * yh);
  const float e = expf(-p);
  return fmaf(-lo, e, e);
}

// Pair type T (0 cation-cation, 1 cation-anion with Morse, 2 anion-anion) at compile time:
// the lane's constants of that type stay in registers and the Morse terms exist only for T = 1.
// Returns the pair energy in p2 and dU/dd in fd.  MORSE32 (force items): the Morse exponentials
// in plain FP32 -- their arguments lr (d - r0) are small near equilibrium, so the FP32 rounding of
// the argument costs little, unlike the Buckingham argument d / rho (~7), whose double-float form
// stays: on the 300-configuration set the fitness error was the same (random 8.0e-8, near the
// optimum 7.7e-7) and the generation 10 % shorter; an FP32 Buckingham exponent as well gave 2e-6
// near the optimum.
template <int T, bool MORSE32 = false>
__device__ __forceinline__ void ri_pair(const RIC& R, float d, float dlo, float& p2, float& fd) {
  const float ex = R.a[T] * exp_neg_dd(d, dlo, R.b[T], R.blo[T]);
  p2 = ex;
  fd = -fmaf(ex, R.b[T], ex * R.blo[T]);
  if constexpr (T == 1 && MORSE32) {
    const float dr = d - R.r0;
    const float er = expf(-dr * R.lr), ea = expf(-dr * R.la);
    const float fr = R.cr * er, fa = R.ca * ea;
    p2 += fr - fa;
    fd += R.la * fa - R.lr * fr;
  } else if constexpr (T == 1) {
    // d - r0 as hi + lo (TwoSum), then the two Morse exponentials
    const float drh = d - R.r0;
    const float bb = drh - d;
    const float drl = ((d - (drh - bb)) + (-R.r0 - bb)) + dlo;
    const float er = exp_neg_dd(drh, drl, R.lr, R.lrlo), ea = exp_neg_dd(drh, drl, R.la, R.lalo);
    const float fr = fmaf(R.crlo, er, R.cr * er), fa = fmaf(R.calo, ea, R.ca * ea);
    p2 += fr - fa;
    fd += fmaf(R.la, fa, R.lalo * fa) - fmaf(R.lr, fr, R.lrlo * fr);
  }
}

// FP64 linear part of one (individual, energy/virial configuration): energy and virial from the
// configuration's geometric sums g[kRiCfgLin] (per pair type t: sum ec, count, sum d, sum 1/d^6,
// then sum d gc uu, sum d uu, sum uu / d^6) and the lane's FP64 constants.
__device__ __forceinline__ void ri_linear_config(const double* __restrict__ g, const double* __restrict__ c64,
                                                 int stride, double (&acc)[kResK]) {
  const double vrc = c64[R64_VRC * (size_t)stride], dvrc = c64[R64_DVRC * (size_t)stride],
               rc = c64[R64_RC * (size_t)stride];
#pragma unroll
  for (int t = 0; t < 3; ++t) {
    const double qq = c64[(R64_QQ + t) * (size_t)stride], C = c64[(R64_C + t) * (size_t)stride];
    const double* gt = g + 22 * t;
    // U_lin = qq ec + qq (dv_rc rc - v_rc) - qq dv_rc d - C / d^6
    acc[0] += qq * gt[0] + qq * (dvrc * rc - vrc) * gt[1] - qq * dvrc * gt[2] - C * gt[3];
    // W = -sum d dU/dd uu with dU/dd = -qq (gc + dv_rc) + 6 C / d^7
#pragma unroll
    for (int k = 0; k < 6; ++k) acc[1 + k] += qq * gt[4 + k] + qq * dvrc * gt[10 + k] - 6.0 * C * gt[16 + k];
  }
}

// FP64 linear part of the force on one atom: F_i = sum_t [-qq_t (sum gc u + dv_rc sum u) + 6 C_t sum u / d^7].
__device__ __forceinline__ void ri_linear_force(const double* __restrict__ g, const double* __restrict__ c64,
                                                int stride, double (&F)[3]) {
  const double dvrc = c64[R64_DVRC * (size_t)stride];
  F[0] = F[1] = F[2] = 0.0;
#pragma unroll
  for (int t = 0; t < 3; ++t) {
    const double qq = c64[(R64_QQ + t) * (size_t)stride], C = c64[(R64_C + t) * (size_t)stride];
#pragma unroll
    for (int a = 0; a < 3; ++a) F[a] += -qq * (g[9 * t + a] + dvrc * g[9 * t + 3 + a]) + 6.0 * C * g[9 * t + 6 + a];
  }
}

// bonds per chunk of the RI pair pipeline (one bond per lane); two stages per warp
constexpr int kPairChunk = 32;
constexpr size_t kPairStageOne = (size_t)kPairChunk * (sizeof(float4) + sizeof(float));  // geometry | d lo
constexpr size_t kPairStageBytes = (size_t)kWarps * 2 * kPairStageOne;

// Compensated FP32 sum (Kahan): the running error c is subtracted from each
// new term; value() is the sum in FP64.  Error about 2 eps sum|x| for any
// order of terms, against (n - 1) eps sum|x| for a plain FP32 sum.
struct KSum {
  float s = 0.f, c = 0.f;
  __device__ __forceinline__ void add(float x) {
    const float y = x - c;
    const float t = s + y;
    c = (t - s) - y;
    s = t;
  }
  __device__ __forceinline__ double value() const { return (double)s - (double)c; }
};

// NN2B value and derivative (nn2b.cu:49-78) for the lane's weights, held in
// shared memory as float4 groups so that each 16-byte load feeds eight FMAs:
//   W1[a][m/4][lane] (hidden-to-hidden, row a), V[v][a/4][lane] for v = w0, b0, b1, w2,
//   b2[lane]; NMAX pads n to a multiple of 4 with zero weights.
template <int NMAX>
struct NNSmem {
  static constexpr int Q = NMAX / 4;
  static constexpr size_t floats = (size_t)32 * (NMAX * NMAX + 4 * NMAX + 1);
  // float offset of parameter m (nn2b.cu:33-46 order) of lane l
  __device__ static size_t offset(int m, int n, int l) {
    auto vec = [&](int v, int a) { return ((size_t)((v * Q + a / 4) * 32 + l)) * 4 + a % 4; };
    const size_t w1_floats = (size_t)NMAX * Q * 32 * 4;
    if (m < n) return w1_floats + vec(0, m);
    if (m < 2 * n) return w1_floats + vec(1, m - n);
    if (m < 2 * n + n * n) {
      const int idx = m - 2 * n, a = idx / n, mm = idx % n;
      return ((size_t)((a * Q + mm / 4) * 32 + l)) * 4 + mm % 4;
    }
    if (m < n * (n + 3)) return w1_floats + vec(2, m - n * (n + 2));
    if (m < n * (n + 4)) return w1_floats + vec(3, m - n * (n + 3));
    return w1_floats + (size_t)4 * Q * 32 * 4 + l;
  }
};

// How nn_pairs forms the pair energy p2 = sum_a w2_a tanh(x2_a - b1_a) - b2.  Near a fitted
// optimum the sum and b2 cancel: most pairs lie near the cutoff, where the network's output
// must be small, while its terms are of the size of w2.  The FP32 rounding of those terms and
// partial sums (eps |w2|, coherent over the pairs of a shell) then set the fitness error of
// the best individuals (1e-5 relative at fitness 0.04 on the 10-neuron set).  Each product of
// two floats is exact in FP64, so an FP64 sum of the terms leaves only the FP32 errors of
// x2t itself, which do not cancel.  The force needs p2 only inside the taper shell (fcp != 0):
// `with_p2` (warp-uniform) skips it elsewhere.

// NP pairs of the same lane at once: every weight loaded from shared memory
// feeds the NP pairs (the hidden-to-hidden loads, not the FMAs, bound a
// single pair).  Each pair's arithmetic is the same sequence as for NP = 1.
// NR: the network width as a compile-time constant (0: n at run time, with the padding columns
// of the last float4 group evaluated on their zero weights); with it the row loop unrolls and the
// padding columns drop out.
template <int NMAX, int NP, int NR>
__device__ __forceinline__ void nn_pairs(const float* __restrict__ wsm, int lane, int n, const float (&d)[NP],
                                         bool with_p2, float (&p2)[NP], float (&f2)[NP]) {
  if (NR) n = NR;
  constexpr int Q = NMAX / 4;
  constexpr int NC = NR ? NR : NMAX;  // columns evaluated
  const float4* W1 = reinterpret_cast<const float4*>(wsm);
  const float4* V = W1 + NMAX * Q * 32;
  const float b2 = wsm[(size_t)(NMAX * Q * 32 + 4 * Q * 32) * 4 + lane];
  float x1[NP][NMAX], y1[NP][NMAX];
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const float4 w0 = V[(0 * Q + q) * 32 + lane];
    const float4 b0 = V[(1 * Q + q) * 32 + lane];
    const float w0c[4] = {w0.x, w0.y, w0.z, w0.w}, b0c[4] = {b0.x, b0.y, b0.z, b0.w};
#pragma unroll
    for (int u = 0; u < NP; ++u)
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        if (4 * q + c < NC) {
          x1[u][4 * q + c] = tanhf(w0c[c] * d[u] - b0c[c]);
          y1[u][4 * q + c] = (1.0f - x1[u][4 * q + c] * x1[u][4 * q + c]) * w0c[c];
        } else {
          x1[u][4 * q + c] = y1[u][4 * q + c] = 0.f;
        }
      }
  }
  double p2d[NP];
#pragma unroll
  for (int u = 0; u < NP; ++u) {
    p2[u] = f2[u] = 0.f;
    p2d[u] = 0.0;
  }
  const int qa_end = (n + 3) >> 2;
#pragma unroll (NR ? NMAX / 4 : 1)
  for (int qa = 0; qa < qa_end; ++qa) {
    const float4 b1 = V[(2 * Q + qa) * 32 + lane];
    const float4 w2 = V[(3 * Q + qa) * 32 + lane];
    const float b1c[4] = {b1.x, b1.y, b1.z, b1.w}, w2c[4] = {w2.x, w2.y, w2.z, w2.w};
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const int a = 4 * qa + c;
      if (a < n) {
        float x2[NP], y2[NP];
#pragma unroll
        for (int u = 0; u < NP; ++u) x2[u] = y2[u] = 0.f;
#pragma unroll
        for (int q = 0; q < Q; ++q) {
          const float4 w = W1[(a * Q + q) * 32 + lane];
          const float wc[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
          for (int u = 0; u < NP; ++u)
#pragma unroll
            for (int m = 0; m < 4; ++m)
              if (4 * q + m < NC) {
                x2[u] = fmaf(wc[m], x1[u][4 * q + m], x2[u]);
                y2[u] = fmaf(wc[m], y1[u][4 * q + m], y2[u]);
              }
        }
#pragma unroll
        for (int u = 0; u < NP; ++u) {
          const float x2t = tanhf(x2[u] - b1c[c]);
          const float y2t = y2[u] * (1.0f - x2t * x2t);
          if (with_p2) p2d[u] = fma((double)w2c[c], (double)x2t, p2d[u]);
          f2[u] = fmaf(w2c[c], y2t, f2[u]);
        }
      }
    }
  }
#pragma unroll
  for (int u = 0; u < NP; ++u) p2[u] = with_p2 ? (float)(p2d[u] - (double)b2) : 0.f;
}

template <int KIND, int NMAX, bool FORCE>
__device__ __forceinline__ void pair_item(const JobView* __restrict__ jobs, const WorkItem& it, unsigned char* smem) {
  const JobView& J = jobs[it.job];
  const DevView S = J.v;
  const int P = J.P, Pstride = J.Pstride, nn = J.num_neurons, nv = J.num_vars;
  const NNTaper tp = J.tp;
  const float* __restrict__ weights = J.weights;
  double* __restrict__ res = J.res;
  float* __restrict__ fdump = J.fdump;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int p = it.p0 + lane;
  const int pl = p < P ? p : it.p0;
  const Consts kc{J.consts, Pstride, pl};
  RIC R;
  if (KIND == 1) load_ri(kc, R);
  float* wsm = reinterpret_cast<float*>(smem + (size_t)kWarps * 32 * kResK * sizeof(double));
  if (KIND == 2) {
    for (size_t t = threadIdx.x; t < NNSmem<NMAX>::floats; t += blockDim.x) wsm[t] = 0.f;  // zero padding
    __syncthreads();
    for (int t = threadIdx.x; t < nv * 32; t += blockDim.x) {
      const int m = t >> 5, l = t & 31;
      const int pp = it.p0 + l < P ? it.p0 + l : it.p0;
      wsm[NNSmem<NMAX>::offset(m, nn, l)] = weights[(size_t)m * Pstride + pp];
    }
    __syncthreads();
  }
  const int c = it.config, atom0 = S.Na_sum[c], Na = S.Na[c];
  const int N = S.N;
  double acc[kResK];
#pragma unroll
  for (int k = 0; k < kResK; ++k) acc[k] = 0.0;
  // RI energy/virial items cover all atoms of their configuration, so warp 0 adds the linear
  // part (Coulomb, dispersion) and the self energy -K_C q^2 S sum_i (q_i / q)^2 once per
  // individual, in FP64
  const double* __restrict__ c64 = KIND == 1 ? J.consts64 + pl : nullptr;
  if (KIND == 1 && !FORCE && warp == 0) {
    if (J.ri_self) acc[0] = -c64[R64_SELF * (size_t)Pstride] * S.ri_qsum[c];
    ri_linear_config(S.ri_cfg_lin + (size_t)c * kRiCfgLin, c64, Pstride, acc);
  }
  // per-atom sums over the atom's pairs in FP32, added to the FP64 accumulators once per atom
  // (a per-pair FP64 add would cost two FP32->FP64 conversions per term, which run at a
  // fraction of the FP32 rate).  The energy is compensated (Kahan).  For the rigid ion the force
  // and virial components are compensated as well: once the Coulomb and dispersion terms moved to
  // the FP64 linear part, the FP32 summation of the large nearest-neighbour Buckingham terms set
  // the error of individuals near the fitted optimum (300-configuration set: max 1.5e-6 with FMA
  // sums, 7.6e-7 compensated, for 16 % of the pair time).  NN2B keeps FMA sums (its error is set
  // by the per-pair terms: compensation left it unchanged).
  constexpr int NK = FORCE ? 3 : 7;
  auto consume = [&](KSum* ks, const float4& q, float p2, float fd) {
    if (KIND == 1 && FORCE) {
      ks[0].add(fd * q.x);
      ks[1].add(fd * q.y);
      ks[2].add(fd * q.z);
    } else if (KIND == 1) {
      ks[0].add(p2);
      const float s = -q.w * fd;
      const float sx = s * q.x, sy = s * q.y, sz = s * q.z;
      ks[1].add(sx * q.x);
      ks[2].add(sy * q.y);
      ks[3].add(sz * q.z);
      ks[4].add(sx * q.y);
      ks[5].add(sy * q.z);
      ks[6].add(sz * q.x);
    } else if (FORCE) {
      ks[0].s = fmaf(fd, q.x, ks[0].s);
      ks[1].s = fmaf(fd, q.y, ks[1].s);
      ks[2].s = fmaf(fd, q.z, ks[2].s);
    } else {
      // unordered pair: full U and -r (x) r f2 with f2 = fd / d, i.e. -d fd u (x) u
      ks[0].add(p2);
      const float s = -q.w * fd;
      const float sx = s * q.x, sy = s * q.y, sz = s * q.z;
      ks[1].s = fmaf(sx, q.x, ks[1].s);
      ks[2].s = fmaf(sy, q.y, ks[2].s);
      ks[3].s = fmaf(sz, q.z, ks[3].s);
      ks[4].s = fmaf(sx, q.y, ks[4].s);
      ks[5].s = fmaf(sy, q.z, ks[5].s);
      ks[6].s = fmaf(sz, q.x, ks[6].s);
    }
  };
  auto finish_atom = [&](int il, KSum* ks) {
    if (FORCE) {
      const int i = atom0 + il;
      double F[3] = {0.0, 0.0, 0.0};
      if (KIND == 1) ri_linear_force(S.ri_atom_lin + (size_t)i * kRiAtomLin, c64, Pstride, F);
#pragma unroll
      for (int a = 0; a < 3; ++a) F[a] += ks[a].value();
      const double dx = F[0] - (double)S.force_ref[i];
      const double dy = F[1] - (double)S.force_ref[i + N];
      const double dz = F[2] - (double)S.force_ref[i + 2 * (size_t)N];
      acc[7] += dx * dx + dy * dy + dz * dz;
      if (fdump && p < P) {
        const int Nf = S.N_force;
        fdump[((size_t)p * 3 + 0) * Nf + i] = (float)F[0];
        fdump[((size_t)p * 3 + 1) * Nf + i] = (float)F[1];
        fdump[((size_t)p * 3 + 2) * Nf + i] = (float)F[2];
      }
    } else {
#pragma unroll
      for (int k = 0; k < 7; ++k) acc[k] += ks[k].value();
    }
#pragma unroll
    for (int k = 0; k < NK; ++k) ks[k] = KSum{};
  };
  KSum ks[NK];
  if constexpr (KIND == 1) {
    // The warp's pairs (atoms warp, warp + 8, ... and each atom's bonds) stream through a
    // two-stage shared-memory buffer of kPairChunk bonds: while the warp evaluates one chunk,
    // asynchronous copies (cp.async, 16 B per lane) bring the next one, so the L2 latency of the
    // per-bond geometry is hidden behind the pair arithmetic.  Every atom yields at least one
    // chunk (possibly empty: force items still owe the atom's force error).
    // [stage][geometry float4 | d lo float][kPairChunk]
    unsigned char* buf = smem + (size_t)kWarps * 32 * kResK * sizeof(double) + (size_t)warp * 2 * kPairStageOne;
    auto stage_g = [&](int st) { return reinterpret_cast<float4*>(buf + st * kPairStageOne); };
    auto stage_dl = [&](int st) {
      return reinterpret_cast<float*>(buf + st * kPairStageOne + kPairChunk * sizeof(float4));
    };
    // the atom's pairs come grouped by pair type (rseg), so a chunk splits into at most three
    // runs of one type each, evaluated with that type's constants hoisted
    int4 f_seg = make_int4(0, 0, 0, 0);
    int f_il = warp, f_b = 0;
    if (f_il < Na) {
      f_seg = S.rseg[atom0 + f_il];
      f_b = f_seg.x;
    }
    int q_il[2], q_b[2], q_n[2], q_s1[2], q_s2[2];
    bool q_last[2], q_has[2];
    auto fetch = [&](int st) {
      q_has[st] = f_il < Na;
      if (!q_has[st]) return;
      q_il[st] = f_il;
      q_b[st] = f_b;
      q_n[st] = min(kPairChunk, f_seg.w - f_b);
      q_s1[st] = f_seg.y;
      q_s2[st] = f_seg.z;
      f_b += q_n[st];
      q_last[st] = f_b >= f_seg.w;
      if (q_last[st]) {
        f_il += kWarps;
        if (f_il < Na) {
          f_seg = S.rseg[atom0 + f_il];
          f_b = f_seg.x;
        }
      }
      if (lane < q_n[st]) {
        const int bnd = q_b[st] + lane;
        __pipeline_memcpy_async(stage_g(st) + lane, S.rg32 + bnd, sizeof(float4));
        __pipeline_memcpy_async(stage_dl(st) + lane, S.rdl + bnd, sizeof(float));
      }
    };
    fetch(0);
    __pipeline_commit();
    fetch(1);
    __pipeline_commit();
    for (int st = 0; q_has[st]; st ^= 1) {
      __pipeline_wait_prior(1);  // the older of the two groups in flight (stage st) has landed
      __syncwarp();
      const float4* g = stage_g(st);
      const float* w = stage_dl(st);
      const int n = q_n[st], b0 = q_b[st];
      const int k1 = min(max(q_s1[st] - b0, 0), n), k2 = min(max(q_s2[st] - b0, 0), n);
      auto run = [&](auto type, int kb, int ke) {
        constexpr int T = decltype(type)::value;
#pragma unroll 4  // four pairs' shared-memory loads in flight (2 measured 1 % slower)
        for (int k = kb; k < ke; ++k) {
          const float4 q = g[k];
          float p2, fd;
          ri_pair<T, FORCE>(R, q.w, w[k], p2, fd);
          consume(ks, q, p2, fd);
        }
      };
      run(std::integral_constant<int, 0>{}, 0, k1);
      run(std::integral_constant<int, 1>{}, k1, k2);
      run(std::integral_constant<int, 2>{}, k2, n);
      if (q_last[st]) finish_atom(q_il[st], ks);
      __syncwarp();  // every lane is done with stage st before it is refilled
      fetch(st);
      __pipeline_commit();
    }
  } else {
    // pairs through the MLP: each pair's tapered energy and radial derivative go to
    // use(bond, geometry, p2, fd); two pairs per weight load up to 16 neurons (registers allow
    // it), one above
    constexpr int NP = NMAX <= 16 ? 2 : 1;
    // bond_of(k) for k in [kbeg, kend) in steps of `step`: the bonds to evaluate
    auto eval_list = [&](int kbeg, int kend, int step, auto&& bond_of, auto&& use) {
      for (int b = kbeg; b < kend; b += step) {
        float4 q[NP];
        float d[NP], p2[NP], f2raw[NP];
        int bd[NP];
#pragma unroll
        for (int u = 0; u < NP; ++u) {
          bd[u] = bond_of(min(b + u, kend - 1));
          q[u] = __ldg(&S.g32[bd[u]]);
          d[u] = q[u].w;
        }
        // force items: p2 enters only through the taper derivative (warp-uniform test: the
        // 32 lanes share the pairs)
        bool need_p2 = !FORCE;
#pragma unroll
        for (int u = 0; u < NP; ++u) need_p2 |= d[u] >= tp.r1;
        // the class's full width, the reference's largest width (10), or any other at run time
        if (nn == NMAX)
          nn_pairs<NMAX, NP, NMAX>(wsm, lane, nn, d, need_p2, p2, f2raw);
        else if (NMAX == 12 && nn == 10)
          nn_pairs<NMAX, NP, NMAX == 12 ? 10 : 0>(wsm, lane, nn, d, need_p2, p2, f2raw);
        else
          nn_pairs<NMAX, NP, 0>(wsm, lane, nn, d, need_p2, p2, f2raw);
#pragma unroll
        for (int u = 0; u < NP; ++u) {
          if (b + u < kend) {
            float fc, fcp, fd;
            cutoff_fn(tp.r1, tp.r2, tp.pf, d[u], fc, fcp);
            float pu = p2[u];
            if (tp.consistent) {
              fd = f2raw[u] * fc + pu * fcp;
              pu *= fc;
            } else {  // nn2b.cu:147-148: p2 is tapered before it enters the force
              pu *= fc;
              fd = f2raw[u] * fc + pu * fcp;
            }
            use(bd[u], q[u], pu, fd);
          }
        }
      }
    };
    if constexpr (FORCE) {
      // Force items evaluate the pairs into the item's scratch [bond][individual] in global
      // memory, then gather F_i = sum_j fd u_ij over i's full list in list order.  When the
      // configuration's bond list is symmetric (every bond's reverse is the same pair with the
      // negated vector, hence the same FP32 length; item_pairs_once), each unordered pair is
      // evaluated once, from its lower atom, and the gather reads the reverse bond's slot for
      // j < i (DevView::pslot): the same terms in the same order as evaluating every directed pair, with half the
      // network evaluations.  Otherwise every directed pair is evaluated into its own slot.
      // Pass 1 takes the configuration's list of bonds to evaluate (DevView::hb) in consecutive
      // groups of NP per warp: balanced across warps, and one partial group per configuration
      // instead of one per atom.
      float* __restrict__ scr = J.gscratch + (size_t)it.gofs * 64;
      const int bond0 = S.off[atom0];
      const bool once = item_pairs_once(it);
      const int* __restrict__ hb = S.hb + S.hb_off[c];
      const int nh = S.hb_off[c + 1] - S.hb_off[c];
      for (int k0 = warp * NP; k0 < nh; k0 += kWarps * NP)
        eval_list(k0, min(k0 + NP, nh), NP, [&](int k) { return __ldg(&hb[k]); },
                  [&](int b, const float4&, float, float fd) { scr[(size_t)(b - bond0) * 32 + lane] = fd; });
      __syncthreads();  // every pair's fd is in the scratch (plain loads below: written by this launch)
      for (int il = warp; il < Na; il += kWarps) {
        const int i = atom0 + il;
        const int be = S.off[i + 1];
#pragma unroll 4
        for (int b = S.off[i]; b < be; ++b) {
          const int cb = once ? __ldg(&S.pslot[b]) : b - bond0;
          consume(ks, __ldg(&S.g32[b]), 0.f, scr[(size_t)cb * 32 + lane]);
        }
        finish_atom(il, ks);
      }
    } else {
      // energy/virial items need the configuration's totals only: consecutive groups of the
      // unordered-pair list per warp, the compensated energy and FMA virial sums flushed to FP64
      // every 16 groups (FP32 chains as short as an atom's half list)
      const int* __restrict__ hb = S.hb + S.hb_off[c];
      const int nh = S.hb_off[c + 1] - S.hb_off[c];
      int groups = 0;
      for (int k0 = warp * NP; k0 < nh; k0 += kWarps * NP) {
        eval_list(k0, min(k0 + NP, nh), NP, [&](int k) { return __ldg(&hb[k]); },
                  [&](int, const float4& q, float pu, float fd) { consume(ks, q, pu, fd); });
        if (++groups == 16) {
          groups = 0;
          finish_atom(0, ks);
        }
      }
      finish_atom(0, ks);
    }
  }
  reduce_item<32>(it, P, S.Nc, acc, smem, res);  // pair items hold 32 individuals
}

// RI: three CTAs per SM (at most 85 registers); NN2B: two (128 registers, two pairs per weight
// load) -- each measured faster than the unbounded register allocation, and than NN2B at three
// CTAs per SM (with either one or two pairs per weight load).  NN2B's two kinds of items share a
// launch; the rigid ion's go in two launches of single-kind instantiations (job_items).
// ONLY: 0 both kinds of items (item_force), 1 force items only, 2 energy/virial items only (one
// body, so its own register allocation).
template <int KIND, int NMAX, int ONLY>
__global__ void __launch_bounds__(kBlock, KIND == 1 ? 3 : 2) pair_batched(const JobView* __restrict__ jobs,
                                                                         const WorkItem* __restrict__ items) {
  extern __shared__ __align__(16) unsigned char smem[];
  const WorkItem it = items[blockIdx.x];
  if (ONLY == 1 || (ONLY == 0 && item_force(it)))
    pair_item<KIND, NMAX, true>(jobs, it, smem);
  else
    pair_item<KIND, NMAX, false>(jobs, it, smem);
  finish_item(jobs, it, 32);
}

// --------------------------------------------------------------------------- fitness
// The fitness of every individual in a launch of its own: for launch sets that compute only part
// of the configurations' results (full sets fold in their work items, finish_item).
__global__ void fitness_jobs(const JobView* __restrict__ jobs, const int2* __restrict__ indmap, int total) {
  const int t = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
  if (t >= total) return;
  const int2 jp = indmap[t];
  fold_fitness(jobs[jp.x], jp.y, threadIdx.x & 31);
}

// --------------------------------------------------------------------------- planning
namespace {
constexpr size_t kRedBytes = (size_t)kWarps * 32 * kResK * sizeof(double);
// Force items with up to 4 bonds per atom: three 256-thread CTAs per SM (at most 85 registers
// per thread, 74 KB of shared memory each) beat two CTAs with twice the individuals per item
// (measured).  Larger register classes would spill under that bound and keep two CTAs per SM.
size_t force_smem_target(int zc) { return zc == 4 ? 72 * 1024 : 96 * 1024; }
size_t stage_target(int zc) { return zc == 4 ? 74 * 1024 : 110 * 1024; }  // force scratch + staged geometry
constexpr size_t kSmemMax = 220 * 1024;

int zclass_of(int z) { return tersoff_zclass(z); }
}  // namespace

const char* tile_mode_name(int m) {
  switch (m) {
    case kTileDefault: return "default";
    case kTileHalf: return "half-G";
    case kTileQuarter: return "quarter-G";
    case kTileGlobal: return "global-32";
    case kTileUnstaged: return "unstaged";
    default: return "?";
  }
}

namespace {
// register classes of the NN2B MLP width (12 covers the reference's largest width, 10)
int nmax_of(int n) { return n <= 8 ? 8 : (n <= 12 ? 12 : (n <= 16 ? 16 : (n <= 32 ? 32 : 0))); }
}  // namespace

DevView make_view(const DevSet& d) {
  DevView v;
  v.Nc = d.Nc;
  v.N = d.N;
  v.N_force = d.N_force;
  v.Na = d.Na;
  v.Na_sum = d.Na_sum;
  v.NN = d.NN;
  v.off = d.off;
  v.half_off = d.half_off;
  v.pslot = d.pslot;
  v.hb = d.hb;
  v.hb_off = d.hb_off;
  v.rev_sm = d.rev_sm;
  v.ptype = d.ptype;
  v.g32 = d.g32;
  v.d64 = d.d64;
  v.tdl = d.tdl;
  v.sm_off = d.sm_off;
  v.g_sm = d.g_sm;
  v.dl_sm = d.dl_sm;
  v.pt_sm = d.pt_sm;
  v.rev_sm_sm = d.rev_sm_sm;
  v.rg32 = d.rg32;
  v.rdl = d.rdl;
  v.rseg = d.rseg;
  v.ri_atom_lin = d.ri_atom_lin;
  v.ri_cfg_lin = d.ri_cfg_lin;
  v.force_ref = d.force_ref;
  v.ri_qsum = d.ri_qsum;
  return v;
}

JobView make_job_view(const Engine* e, const Plan* plan) {
  const DevSet& d = e->d;
  JobView j{};
  j.v = make_view(d);
  j.potential_type = d.potential_type;
  j.num_types = d.num_types;
  j.num_neurons = d.num_neurons;
  j.num_vars = d.num_vars;
  j.P = plan->P;
  j.Pstride = plan->Pstride;
  j.Nc_force = d.Nc_force;
  j.ri_self = e->spec.ri_self;
  j.tp = NNTaper{e->spec.nn_r1, e->spec.nn_r2, (float)(M_PI / ((double)e->spec.nn_r2 - e->spec.nn_r1)),
                 e->spec.nn_consistent};
  j.pop = plan->d_pop;
  j.pmin = e->d_pmin;
  j.pmax = e->d_pmax;
  j.consts = plan->d_consts;
  j.consts64 = plan->d_consts64;
  j.weights = plan->d_weights;
  j.res = plan->d_res;
  j.fdump = plan->dump ? plan->d_fdump : nullptr;
  j.gscratch = plan->d_gscratch;
  j.E_ref = d.E_ref;
  j.W_ref = d.W_ref;
  j.nF = d.norm_force;
  j.nE = d.norm_energy;
  j.nW = d.norm_virial;
  j.wF = d.w_force;
  j.wE = d.w_energy;
  j.wW = d.w_stress;
  j.fitness = plan->d_fitness;
  j.comps = plan->d_comps;
  j.fit_count = plan->d_fitcnt;
  return j;
}

LaunchSet::~LaunchSet() {
  if (d_jobs) cudaFree(d_jobs);
  if (h_jobs) cudaFreeHost(h_jobs);
  if (d_items) cudaFree(d_items);
  if (d_indmap) cudaFree(d_indmap);
  if (side) cudaStreamDestroy(side);
  if (fork) cudaEventDestroy(fork);
  if (join) cudaEventDestroy(join);
  for (auto ev : tev)
    if (ev) cudaEventDestroy(ev);
}

Plan::~Plan() {
  if (graph) cudaGraphExecDestroy(graph);
  if (h_pop) cudaFreeHost(h_pop);
  if (h_fit) cudaFreeHost(h_fit);
}

struct ItemSpec {
  WorkItem w;
  double cost, units, flops, sfu;
};
struct LaunchKey {
  int kind, zclass, nmax, force, lo;
  bool operator<(const LaunchKey& o) const {
    return std::tie(kind, zclass, nmax, force, lo) < std::tie(o.kind, o.zclass, o.nmax, o.force, o.lo);
  }
};
// A plan's work items grouped by launch (job index 0), with their shared-memory and global-scratch needs.
struct ItemCache {
  std::map<LaunchKey, std::vector<ItemSpec>> groups;
  std::map<LaunchKey, size_t> smem_need;
  size_t need = 0;
};

namespace {

// True when every derived Tersoff constant of every individual is exact in FP32: S fixed at 2 by
// its bounds, so that lr = 2A, la = A, cr = D0, ca = 2 D0 are FP32 parameters times powers of two.
// (S = 2 is the only such value: sqrt(2S) sqrt(2/S) = 2 leaves S = 2^(2a-1) for powers of two, and
// S - 1 a power of two only for a = 1.)  Otherwise the kernels carry the constants' FP64
// remainders (the LO instantiation).
static bool tersoff_consts_exact(const PotentialSpec& sp, int num_types) {
  for (int s = 0; s < num_types; ++s) {
    const int m = 4 * s + 3;
    if ((int)sp.pmin.size() <= m || sp.pmin[m] != 2.0f || sp.pmax[m] != 2.0f) return false;
  }
  return true;
}

// Work items of one job, grouped by kernel.
//   Algorithmic work per (individual, atom), counted on the batched formulation
//   (FMA = 2 flops; exp/pow/erfc/tanh/sin-cos calls counted as SFU work):
//     Tersoff: 60 flops + 4 transcendentals per bond, 21 flops per ordered triplet
//     RI:      per pair of an active type 20 flops + 1 exp, cation-anion pairs 20 more + 2 exp
//              (Morse); the linear terms are FP64 sums formed once per training set
//     NN2B:    4n^2 + 13n + 10 flops + 2n tanh per pair
// modes: per configuration the force-item tile (TileMode; empty: the default rule for all);
// only: when given, the configurations whose items are built (the autotuner's trial launches).
int job_items(const Engine* e, int P, int job, std::map<LaunchKey, std::vector<ItemSpec>>& groups,
              std::map<LaunchKey, size_t>& smem_need, size_t* gscratch_floats, const std::vector<int8_t>* modes,
              const std::vector<char>* only) {
  *gscratch_floats = 0;
  const DevSet& d = e->d;
  const TrainingSet& ts = e->ts;
  const bool tersoff = d.potential_type == 1 || d.potential_type == 2;
  const int kind = tersoff ? 0 : (is_ri_type(d.potential_type) ? 1 : 2);
  // NN2B: register-array size of the MLP; Tersoff: number of atom types (kernel template)
  const int nmax = kind == 2 ? nmax_of(d.num_neurons) : (kind == 0 ? d.num_types : 0);
  const bool lo = kind == 0 && !tersoff_consts_exact(e->spec, d.num_types);
  if (kind == 2 && nmax == 0) {
    set_error("batched NN2B supports up to 32 neurons per layer (got %d).", d.num_neurons);
    return GPUGA_ERR_UNSUPPORTED;
  }
  std::vector<double> atom_flops(ts.N), atom_sfu(ts.N), atom_flops_half(ts.N), atom_sfu_half(ts.N);
  for (int i = 0; i < ts.N; ++i) {
    const double Z = e->h_NN[i];
    if (kind == 0) {
      atom_flops[i] = 60.0 * Z + 21.0 * Z * (Z - 1.0);
      atom_sfu[i] = 4.0 * Z;
    } else if (kind == 1) {
      // evaluated pairs only (ri_active), by pair type
      double f = 0, sf = 0, fh = 0, sfh = 0;
      for (int b = e->h_off[i]; b < e->h_off[i + 1]; ++b) {
        const int t = ts.type[i] + ts.type[e->h_nbr[b]];
        if (!((d.ri_active >> t) & 1)) continue;
        const double pf = t == 1 ? 40.0 : 20.0, ps = t == 1 ? 3.0 : 1.0;
        f += pf;
        sf += ps;
        if (e->h_nbr[b] > i) {
          fh += pf;
          sfh += ps;
        }
      }
      atom_flops[i] = f;
      atom_sfu[i] = sf;
      atom_flops_half[i] = fh;
      atom_sfu_half[i] = sfh;
    } else {
      const double nn = d.num_neurons;
      const double fpp = 4.0 * nn * nn + 13.0 * nn + 10.0;
      const double spp = 2.0 * nn;
      int half = 0;
      for (int b = e->h_off[i]; b < e->h_off[i + 1]; ++b) half += e->h_nbr[b] > i;
      atom_flops[i] = fpp * Z;
      atom_sfu[i] = spp * Z;
      atom_flops_half[i] = fpp * half;
      atom_sfu_half[i] = spp * half;
    }
  }
  // NN2B force configurations whose bond list is symmetric (engine set-up, geometry.cu): their
  // force items evaluate each unordered pair once (pair_item)
  const std::vector<char>& pair_sym = e->h_pair_sym;
  for (int c = 0; c < ts.Nc; ++c) {
    if (only && !(*only)[c]) continue;
    const bool force = c < ts.Nc_force;
    const int Na = ts.Na[c];
    const int mode = (modes && !modes->empty() && (*modes)[c] > 0) ? (*modes)[c] : kTileDefault;
    int zc = 0, G = 32, Grule = 32;
    size_t smem = kRedBytes;
    bool staged = false, global = false, once = false;
    size_t fbytes = 0, item_floats = 0;
    if (kind == 0) {
      zc = zclass_of(e->h_zmax[c]);
      if (zc == 0) {
        set_error("configuration %d has an atom with %d neighbors; the batched Tersoff path supports 16.", c,
                  e->h_zmax[c]);
        return GPUGA_ERR_UNSUPPORTED;
      }
      // slot-major staged geometry: zc slots per atom of (float4, the FP64 length (FP64 pair terms)
      // or its FP32 remainder, pair set[, reverse position]) + counts
      const bool d64 = (force ? kPairModeForce : kPairModeEV) == kPair64;
      const size_t stage =
          ((size_t)zc * Na * (16 + (d64 ? 8 : 4) + 1 + (force ? 4 : 0)) + (size_t)Na * 4 + 15) & ~(size_t)15;
      // per individual: the f_ij scratch (slot-major, padded to max Z), which afterwards holds the
      // squared-error rows (ferr_row)
      const size_t per_ind = std::max((size_t)e->h_zmax[c] * Na * 3 * sizeof(float),
                                      (size_t)ferr_row(Na) * sizeof(double));
      // force items: the constants table (tersoff_table_bytes), the f_ij scratch, the staged geometry
      auto scratch = [&](int g) { return tersoff_table_bytes(g) + ((per_ind * g + 15) & ~(size_t)15); };
      // the gather pass holds at most ferr_steps(zc) atoms per thread (8 warps of 32 / g atoms)
      auto fits = [&](int g) {
        return scratch(g) <= force_smem_target(zc) && (size_t)Na * g <= (size_t)ferr_steps(zc) * kBlock;
      };
      // default rule: the largest G whose scratch fits, and the geometry staged too when it fits
      // beside the scratch of >= 4 individuals; 32 individuals with global scratch when not even
      // one individual's scratch fits.  Its G fixes the summation order of every tile.
      const bool rule_global = !fits(1);
      if (force && !rule_global) {
        while (Grule > 1 && !fits(Grule)) Grule >>= 1;
        int Gs = Grule;
        while (Gs > 4 && scratch(Gs) + stage > stage_target(zc)) Gs >>= 1;
        if (scratch(Gs) + stage <= stage_target(zc)) Grule = Gs;
      }
      if (force && (rule_global || mode == kTileGlobal)) {
        // 32 individuals per item (lane = individual, one atom per warp step, coalesced scratch
        // rows) with the scratch (ZC slots) and the squared-error table in global memory
        global = true;
        item_floats = ((size_t)zc * Na * 3 * 32 + (size_t)2 * ferr_row(Na) * 32 + 63) & ~(size_t)63;
        smem = std::max(smem, kRedBytes + tersoff_table_bytes(32));
      } else if (force) {
        G = Grule;
        if (mode == kTileHalf) G = std::max(1, G / 2);
        if (mode == kTileQuarter) G = std::max(1, G / 4);
        staged = mode != kTileUnstaged && scratch(G) + stage <= stage_target(zc);
        fbytes = (per_ind * G + 15) & ~(size_t)15;
        smem = std::max(smem, scratch(G) + (staged ? stage : 0));
      } else {
        // energy/virial items (always G = 32, which tersoff_batched compiles in): per-lane FP64
        // sums of the 256-thread CTA, then (optionally; kStageEV) the geometry
        smem = (size_t)kBlock * kResK * sizeof(double);
        if (kStageEV && stage <= stage_target(zc)) {
          staged = true;
          smem += stage;
        }
      }
    } else if (kind == 2) {
      smem += (size_t)32 * (nmax * nmax + 4 * nmax + 1) * sizeof(float);  // NNSmem<nmax>::floats
      if (force) {
        // the pairs' fd in a [bond][individual] global scratch, each unordered pair once when the
        // bond list is symmetric
        global = true;
        once = pair_sym[c] != 0;
        const long long Bc = (long long)e->h_off[ts.Na_sum[c] + Na] - e->h_off[ts.Na_sum[c]];
        item_floats = ((size_t)Bc * 32 + 63) & ~(size_t)63;
      }
    } else {
      smem += kPairStageBytes;  // RI: the warps' two-stage pair buffers
    }
    // force and energy/virial items share a launch, except the rigid ion's: its two bodies under
    // one register allocation spilled more and ran 3 % slower than two single-kind kernels on two
    // streams (300-configuration set: 5.92 vs 5.74 ms per generation)
    const LaunchKey key{kind, zc, nmax, kind == 1 && force ? 1 : 0, lo ? 1 : 0};
    smem_need[key] = std::max(smem_need[key], smem);
    double cf = 0, cs = 0;
    const bool half = kind != 0 && (!force || once);  // unordered pairs evaluated once
    for (int k = 0; k < Na; ++k) {
      const int i = ts.Na_sum[c] + k;
      cf += half ? atom_flops_half[i] : atom_flops[i];
      cs += half ? atom_sfu_half[i] : atom_sfu[i];
    }
    for (int p0 = 0; p0 < P; p0 += G) {
      const int cnt = std::min(G, P - p0);
      int gofs = 0;
      if (global) {
        if (*gscratch_floats / 64 > (size_t)INT32_MAX) {
          set_error("global force scratch exceeds the addressable size.");
          return GPUGA_ERR_UNSUPPORTED;
        }
        gofs = (int)(*gscratch_floats / 64);
        *gscratch_floats += item_floats;
      }
      groups[key].push_back(
          {WorkItem{c, p0, pack_G(G, staged, fbytes, global, Grule, force, once), job, gofs}, cf * cnt, (double)Na * cnt, cf * cnt, cs * cnt});
    }
  }
  return GPUGA_OK;
}

template <class K>
int set_smem(K kernel) {
  GPUGA_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemMax));
  return GPUGA_OK;
}

// configure_only: raise the dynamic shared-memory limit of the launch's kernel
// (done when a launch set is built, never inside a stream capture).
int launch_one(const LaunchSet* ls, const Launch& L, cudaStream_t st, bool configure_only) {
  const dim3 grid(L.count), block(kBlock);
  const WorkItem* items = ls->d_items + L.first;
#define GPUGA_TERSOFF1(ZC, NT)                                                          \
  do {                                                                                  \
    if (configure_only) {                                                               \
      if (L.lo) GPUGA_TRY(set_smem(tersoff_batched<ZC, NT, true>));                     \
      else GPUGA_TRY(set_smem(tersoff_batched<ZC, NT, false>));                         \
      break;                                                                            \
    }                                                                                   \
    if (L.lo)                                                                           \
      tersoff_batched<ZC, NT, true><<<grid, block, L.smem, st>>>(ls->d_jobs, items);     \
    else                                                                                \
      tersoff_batched<ZC, NT, false><<<grid, block, L.smem, st>>>(ls->d_jobs, items);    \
  } while (0)
#define GPUGA_TERSOFF(ZC)                                                             \
  do {                                                                                \
    if (L.nmax == 2) GPUGA_TERSOFF1(ZC, 2); else GPUGA_TERSOFF1(ZC, 1);               \
  } while (0)
#define GPUGA_PAIR1(KD, NM, ON)                                                       \
  do {                                                                                \
    if (configure_only) {                                                             \
      GPUGA_TRY(set_smem(pair_batched<KD, NM, ON>));                                  \
      break;                                                                          \
    }                                                                                 \
    pair_batched<KD, NM, ON><<<grid, block, L.smem, st>>>(ls->d_jobs, items);         \
  } while (0)
#define GPUGA_PAIR(KD, NM) GPUGA_PAIR1(KD, NM, 0)
  if (L.kind == 0) {
    if (L.zclass == 4) GPUGA_TERSOFF(4);
    else if (L.zclass == 8) GPUGA_TERSOFF(8);
    else GPUGA_TERSOFF(16);
  } else if (L.kind == 1) {  // the rigid ion's two kinds in launches of their own (job_items)
    if (L.force == 1) GPUGA_PAIR1(1, 8, 1); else GPUGA_PAIR1(1, 8, 2);
  } else if (L.nmax == 8) {
    GPUGA_PAIR(2, 8);
  } else if (L.nmax == 12) {
    GPUGA_PAIR(2, 12);
  } else if (L.nmax == 16) {
    GPUGA_PAIR(2, 16);
  } else {
    GPUGA_PAIR(2, 32);
  }
#undef GPUGA_TERSOFF
#undef GPUGA_TERSOFF1
#undef GPUGA_PAIR
#undef GPUGA_PAIR1
  GPUGA_CUDA(cudaGetLastError());
  return GPUGA_OK;
}

}  // namespace

int launchset_build(const std::vector<std::pair<Engine*, Plan*>>& jobs, LaunchSet* ls,
                    const std::vector<std::pair<const float*, double*>>* targets, const std::vector<char>* only) {
  std::map<LaunchKey, std::vector<ItemSpec>> groups;
  std::map<LaunchKey, size_t> smem_need;
  std::vector<int2> indmap;
  ls->jobs.clear();
  for (size_t j = 0; j < jobs.size(); ++j) {
    Engine* e = jobs[j].first;
    Plan* plan = jobs[j].second;
    size_t need = 0;
    // a plan's items depend only on its training set, population size and tiles: computed once
    // (a pass over every atom and bond) and reused by every launch set the job joins
    if (only || !plan->items) {
      std::shared_ptr<ItemCache> cache(new ItemCache);
      GPUGA_TRY(job_items(e, plan->P, 0, cache->groups, cache->smem_need, &cache->need, &plan->tiles, only));
      if (!only) plan->items = cache;
      for (auto& kv : cache->groups)
        for (ItemSpec t : kv.second) {
          t.w.job = (int)j;
          groups[kv.first].push_back(t);
        }
      for (auto& kv : cache->smem_need) smem_need[kv.first] = std::max(smem_need[kv.first], kv.second);
      need = cache->need;
    } else {
      const ItemCache& cache = *plan->items;
      for (auto& kv : cache.groups) {
        std::vector<ItemSpec>& dst = groups[kv.first];
        for (ItemSpec t : kv.second) {
          t.w.job = (int)j;
          dst.push_back(t);
        }
      }
      for (auto& kv : cache.smem_need) smem_need[kv.first] = std::max(smem_need[kv.first], kv.second);
      need = cache.need;
    }
    if (need > plan->gscratch_floats) {
      GPUGA_TRY(e->alloc(&plan->d_gscratch, need));
      plan->gscratch_floats = need;
    }
    ls->jobs.push_back(make_job_view(e, plan));
    if (targets) {  // the job's population / fitness live elsewhere (a device GA's buffers)
      ls->jobs.back().pop = (*targets)[j].first;
      ls->jobs.back().fitness = (*targets)[j].second;
    }
    for (int p = 0; p < jobs[j].second->P; ++p) indmap.push_back(make_int2((int)j, p));
  }
  std::vector<WorkItem> all;
  ls->launches.clear();
  for (auto& kv : groups) {
    auto& v = kv.second;
    std::stable_sort(v.begin(), v.end(), [](const ItemSpec& a, const ItemSpec& b) { return a.cost > b.cost; });
    Launch L;
    L.kind = kv.first.kind;
    L.zclass = kv.first.zclass;
    L.nmax = kv.first.nmax;
    L.lo = kv.first.lo != 0;
    int nforce = 0;
    for (auto& t : v) nforce += item_force(t.w) ? 1 : 0;
    L.force = nforce == 0 ? 0 : (nforce == (int)v.size() ? 1 : 2);
    L.smem = smem_need[kv.first];
    L.count = (int)v.size();
    L.first = all.size();
    for (auto& t : v) {
      all.push_back(t.w);
      L.units += t.units;
      L.flops += t.flops;
      L.sfu += t.sfu;
    }
    ls->launches.push_back(L);
  }
  // longest launches first so that the side stream starts the big ones early
  std::stable_sort(ls->launches.begin(), ls->launches.end(),
                   [](const Launch& a, const Launch& b) { return a.flops > b.flops; });
  ls->total_individuals = (int)indmap.size();
  // where the fitness is folded (gpuga_options.fitness_fold; a partial set never folds in its items).
  // The fold launch is the default: the count's round trip at the end of every item holds the
  // item's CTA slot, which measured slower than the extra launch at every size (B200: 62 170 items
  // 4.79 vs 4.63 ms per generation, 290 items 0.069 vs 0.062 ms).
  const int fold_opt = jobs.empty() ? 0 : jobs[0].first->opt.fitness_fold;
  ls->folds = !only && fold_opt == 1;
  if (!ls->folds)
    for (JobView& jv : ls->jobs) jv.fit_count = nullptr;
  GPUGA_CUDA(cudaMalloc(&ls->d_items, sizeof(WorkItem) * std::max<size_t>(all.size(), 1)));
  GPUGA_CUDA(cudaMemcpy(ls->d_items, all.data(), sizeof(WorkItem) * all.size(), cudaMemcpyHostToDevice));
  GPUGA_CUDA(cudaMalloc(&ls->d_indmap, sizeof(int2) * std::max<size_t>(indmap.size(), 1)));
  GPUGA_CUDA(cudaMemcpy(ls->d_indmap, indmap.data(), sizeof(int2) * indmap.size(), cudaMemcpyHostToDevice));
  GPUGA_CUDA(cudaMalloc(&ls->d_jobs, sizeof(JobView) * std::max<size_t>(ls->jobs.size(), 1)));
  GPUGA_CUDA(cudaMallocHost(&ls->h_jobs, sizeof(JobView) * std::max<size_t>(ls->jobs.size(), 1)));
  GPUGA_CUDA(cudaMemcpy(ls->d_jobs, ls->jobs.data(), sizeof(JobView) * ls->jobs.size(), cudaMemcpyHostToDevice));
  GPUGA_CUDA(cudaStreamCreateWithFlags(&ls->side, cudaStreamNonBlocking));
  GPUGA_CUDA(cudaEventCreateWithFlags(&ls->fork, cudaEventDisableTiming));
  GPUGA_CUDA(cudaEventCreateWithFlags(&ls->join, cudaEventDisableTiming));
  ls->tev.assign(2 * ls->launches.size(), nullptr);
  for (auto& ev : ls->tev) GPUGA_CUDA(cudaEventCreate(&ev));
  ls->t_ms.assign(ls->launches.size(), 0.0);
  for (const Launch& L : ls->launches) GPUGA_TRY(launch_one(ls, L, nullptr, true));
  return GPUGA_OK;
}

int launchset_retarget(LaunchSet* ls, int job, const float* d_pop, double* d_fitness, float* fdump,
                       cudaStream_t st) {
  JobView& j = ls->jobs[job];
  if (j.pop == d_pop && j.fitness == d_fitness && j.fdump == fdump) return GPUGA_OK;
  j.pop = d_pop;
  j.fitness = d_fitness;
  j.fdump = fdump;
  // staged through pinned memory; the previous copy has completed once the stream reached it
  GPUGA_CUDA(cudaStreamSynchronize(st));
  ls->h_jobs[job] = j;
  GPUGA_CUDA(cudaMemcpyAsync(ls->d_jobs + job, ls->h_jobs + job, sizeof(JobView), cudaMemcpyHostToDevice, st));
  return GPUGA_OK;
}

// Folds the event pairs of the previous timed generation into the per-launch totals.
int launchset_collect_timing(LaunchSet* ls) {
  if (!ls->t_pending) return GPUGA_OK;
  for (size_t k = 0; k < ls->launches.size(); ++k) {
    GPUGA_CUDA(cudaEventSynchronize(ls->tev[2 * k + 1]));
    float ms = 0.f;
    GPUGA_CUDA(cudaEventElapsedTime(&ms, ls->tev[2 * k], ls->tev[2 * k + 1]));
    ls->t_ms[k] += ms;
  }
  ls->t_count += 1;
  ls->t_pending = false;
  return GPUGA_OK;
}

// One generation of every job of the set: decode, the batched launches
// (energy/virial launches on `st`, force launches on the side stream), then
// the fitness fold.  While per-launch timing is on, every launch runs on `st`
// one after another, so that each event pair brackets that launch alone.
int launchset_enqueue(LaunchSet* ls, cudaStream_t st) {
  const int total = ls->total_individuals;
  decode_jobs<<<(total + 127) / 128, 128, 0, st>>>(ls->d_jobs, ls->d_indmap, total);
  GPUGA_CUDA(cudaGetLastError());
  // several launches (job mixes with several kernel classes): every second one on the side stream
  const bool any_side = ls->launches.size() > 1 && !ls->timing;
  if (any_side) {
    GPUGA_CUDA(cudaEventRecord(ls->fork, st));
    GPUGA_CUDA(cudaStreamWaitEvent(ls->side, ls->fork, 0));
  }
  GPUGA_TRY(launchset_collect_timing(ls));
  for (size_t k = 0; k < ls->launches.size(); ++k) {
    const Launch& L = ls->launches[k];
    cudaStream_t s = (k & 1) && any_side ? ls->side : st;
    if (ls->timing) GPUGA_CUDA(cudaEventRecord(ls->tev[2 * k], s));
    GPUGA_TRY(launch_one(ls, L, s, false));
    if (ls->timing) GPUGA_CUDA(cudaEventRecord(ls->tev[2 * k + 1], s));
  }
  ls->t_pending = ls->timing;
  if (any_side) {
    GPUGA_CUDA(cudaEventRecord(ls->join, ls->side));
    GPUGA_CUDA(cudaStreamWaitEvent(st, ls->join, 0));
  }
  if (!ls->folds) {  // a partial set: the fitness of every individual in one more launch
    fitness_jobs<<<(total + 3) / 4, 128, 0, st>>>(ls->d_jobs, ls->d_indmap, total);
    GPUGA_CUDA(cudaGetLastError());
  }
  return GPUGA_OK;
}

namespace {

__global__ void fill_value(float* __restrict__ p, size_t n, float v) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = v;
}

// Device time (ms) of the force launches of the configurations in `only`, with the plan's current
// tiles: the best of three launches after one warm-up, on `st`.
int time_force_items(Engine* e, Plan* plan, const std::vector<char>& only, cudaStream_t st, double* ms) {
  LaunchSet ls;
  GPUGA_TRY(launchset_build({{e, plan}}, &ls, nullptr, &only));
  const int total = ls.total_individuals;
  decode_jobs<<<(total + 127) / 128, 128, 0, st>>>(ls.d_jobs, ls.d_indmap, total);
  GPUGA_CUDA(cudaGetLastError());
  cudaEvent_t a = nullptr, b = nullptr;
  GPUGA_CUDA(cudaEventCreate(&a));
  GPUGA_CUDA(cudaEventCreate(&b));
  double best = 1e30;
  int s = GPUGA_OK;
  for (int r = 0; r < 4 && s == GPUGA_OK; ++r) {
    cudaEventRecord(a, st);
    for (const Launch& L : ls.launches)
      if (s == GPUGA_OK) s = launch_one(&ls, L, st, false);
    cudaEventRecord(b, st);
    const cudaError_t ce = cudaEventSynchronize(b);
    if (ce != cudaSuccess) s = cuda_status(ce, "cudaEventSynchronize", __FILE__, __LINE__);
    float t = 0.f;
    if (s == GPUGA_OK) cudaEventElapsedTime(&t, a, b);
    if (r > 0) best = std::min(best, (double)t);
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  *ms = best;
  return s;
}

// The autotuner: per size of force configuration (their atom count), time the force items of those
// configurations under every tile (TileMode) on the first plan of a population size, and keep the
// fastest; a tile replaces the default rule only when it is at least 3 % faster (timing noise).
// Tiles never change a result bit, so the choice is free to follow the clock.
int tune_tiles(Engine* e, Plan* plan) {
  const TrainingSet& ts = e->ts;
  const auto t0 = std::chrono::steady_clock::now();
  cudaStream_t st = e->stream;
  const size_t npop = (size_t)plan->P * e->d.num_vars;
  fill_value<<<(unsigned)((npop + 255) / 256), 256, 0, st>>>(plan->d_pop, npop, 0.5f);  // mid-range individuals
  GPUGA_CUDA(cudaGetLastError());
  std::map<int, std::vector<int>> classes;
  for (int c = 0; c < ts.Nc_force; ++c) classes[ts.Na[c]].push_back(c);
  plan->tiles.assign(ts.Nc, 0);
  for (int c = 0; c < ts.Nc_force; ++c) plan->tiles[c] = kTileDefault;
  for (const auto& kv : classes) {
    std::vector<char> only(ts.Nc, 0);
    for (int c : kv.second) only[c] = 1;
    int best_mode = kTileDefault;
    double best_ms = 0.0, default_ms = 0.0;
    for (int mode : {kTileDefault, kTileHalf, kTileQuarter, kTileGlobal, kTileUnstaged}) {
      for (int c : kv.second) plan->tiles[c] = (int8_t)mode;
      double ms = 0.0;
      GPUGA_TRY(time_force_items(e, plan, only, st, &ms));
      if (mode == kTileDefault) {
        default_ms = best_ms = ms;
      } else if (ms < best_ms && ms < 0.97 * default_ms) {
        best_ms = ms;
        best_mode = mode;
      }
    }
    for (int c : kv.second) plan->tiles[c] = (int8_t)best_mode;
  }
  plan->tune_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  return GPUGA_OK;
}

}  // namespace

int plan_build(Engine* e, int P, Plan** out) {
  const DevSet& d = e->d;
  std::unique_ptr<Plan> plan(new Plan);
  plan->P = P;
  plan->Pstride = (P + 31) & ~31;
  const int K = consts_per_individual(d);
  GPUGA_TRY(e->alloc(&plan->d_consts, (size_t)K * plan->Pstride));
  if (const int K64 = consts64_per_individual(d)) GPUGA_TRY(e->alloc(&plan->d_consts64, (size_t)K64 * plan->Pstride));
  if (d.potential_type == 3) GPUGA_TRY(e->alloc(&plan->d_weights, (size_t)d.num_vars * plan->Pstride));
  GPUGA_TRY(e->alloc(&plan->d_res, (size_t)P * d.Nc * kResK));
  GPUGA_TRY(e->alloc(&plan->d_fitness, (size_t)P));
  GPUGA_TRY(e->alloc(&plan->d_comps, (size_t)3 * P));
  GPUGA_TRY(e->alloc(&plan->d_fitcnt, (size_t)P));
  GPUGA_CUDA(cudaMemset(plan->d_fitcnt, 0, sizeof(int) * (size_t)P));
  GPUGA_TRY(e->alloc(&plan->d_pop, (size_t)P * d.num_vars));
  GPUGA_CUDA(cudaMallocHost(&plan->h_pop, sizeof(float) * (size_t)P * d.num_vars));
  GPUGA_CUDA(cudaMallocHost(&plan->h_fit, sizeof(double) * 4 * (size_t)P));
  const bool tersoff = d.potential_type == 1 || d.potential_type == 2;
  const int tiles = e->opt.tiles;
  if (tersoff && tiles == 0 && e->ts.Nc_force > 0) {
    GPUGA_TRY(tune_tiles(e, plan.get()));
    // the trial launches may have grown the global scratch beyond what the chosen tiles need
    if (plan->d_gscratch) {
      GPUGA_CUDA(cudaStreamSynchronize(e->stream));
      e->dfree(plan->d_gscratch);
      plan->d_gscratch = nullptr;
      plan->gscratch_floats = 0;
    }
  } else if (tersoff && tiles >= kTileDefault && tiles <= kTileUnstaged) {
    plan->tiles.assign(e->ts.Nc, 0);
    for (int c = 0; c < e->ts.Nc_force; ++c) plan->tiles[c] = (int8_t)tiles;
  } else if (tiles < 0 || tiles > kTileUnstaged) {
    set_error("gpuga_options.tiles must be 0..5 (got %d).", tiles);
    return GPUGA_ERR_ARG;
  }
  if (e->opt.fitness_fold < 0 || e->opt.fitness_fold > 2) {
    set_error("gpuga_options.fitness_fold must be 0..2 (got %d).", e->opt.fitness_fold);
    return GPUGA_ERR_ARG;
  }
  plan->ls.reset(new LaunchSet);
  GPUGA_TRY(launchset_build({{e, plan.get()}}, plan->ls.get()));
  *out = plan.release();
  return GPUGA_OK;
}

}  // namespace gpuga
