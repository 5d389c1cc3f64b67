// Plain path: one parameter vector per launch sequence, one thread per atom,
// every arithmetic step in the template type T.  T = double is the FP64
// reference on the device (gpuga_find_force64, gpuga_predict) and the
// denominator of the batched engine's speed-up ("plain FP64, one individual per
// launch"); T = float serves the reference's FP32 Potential entry points.
//
// The formulation is the batched engine's (batched.cu): unit bond vectors,
// the bond-order derivative folded into per-bond scalars and each partial
// force f_ij assembled from a radial and a perpendicular part.  The per-bond
// scalars live in global scratch instead of registers, so an atom may have any
// number of neighbors.  Output layouts are the reference's (potential.cuh:28-40):
// F[3][N], W[6][N] (xx, yy, zz, xy, yz, zx) and pe[N] per atom.
#include <cmath>

#include "engine.hpp"

namespace gpuga {

// -------------------------------------------------------------------- math by argument type
__device__ __forceinline__ float m_exp(float x) { return expf(x); }
__device__ __forceinline__ double m_exp(double x) { return exp(x); }
__device__ __forceinline__ float m_log(float x) { return logf(x); }
__device__ __forceinline__ double m_log(double x) { return log(x); }
__device__ __forceinline__ float m_log1p(float x) { return log1pf(x); }
__device__ __forceinline__ double m_log1p(double x) { return log1p(x); }
__device__ __forceinline__ float m_erfc(float x) { return erfcf(x); }
__device__ __forceinline__ double m_erfc(double x) { return erfc(x); }
__device__ __forceinline__ float m_tanh(float x) { return tanhf(x); }
__device__ __forceinline__ double m_tanh(double x) { return tanh(x); }
__device__ __forceinline__ void m_sincos(float x, float* s, float* c) { sincosf(x, s, c); }
__device__ __forceinline__ void m_sincos(double x, double* s, double* c) { sincos(x, s, c); }

// Cosine taper between r1 and r2 (minimal_tersoff.cu:77-90; nn2b.cu:80-92 with its own r1, r2):
// 1 below r1, 0 from r2 on, (1 + cos(pf (d - r1))) / 2 between; dfc = d fc / d d.
template <class T>
__device__ __forceinline__ void taper(T r1, T r2, T pf, T d, T& fc, T& dfc) {
  fc = T(0);
  dfc = T(0);
  if (d < r1) {
    fc = T(1);
  } else if (d < r2) {
    T s, c;
    m_sincos(pf * (d - r1), &s, &c);
    fc = T(0.5) * (T(1) + c);
    dfc = T(-0.5) * pf * s;
  }
}

// ------------------------------------------------------------------------ parameter sets
// Minimal Tersoff (minimal_tersoff.cu:39-75) as the engine derives it: per pair set s (0 for
// equal types, 1 otherwise) fr = cr e^{-lr (d - r0)}, fa = ca e^{-la (d - r0)} with
// lr = sqrt(2S) A, la = sqrt(2/S) A, cr = D0/(S-1), ca = S D0/(S-1); then the bond order
// b = (1 + zeta^n)^mhon, mhon = -1/(2n), zeta = sum fc beta (cos - h)^2.
template <class T>
struct TersoffSet {
  T cr[2], ca[2], lr[2], la[2], r0[2];
  T n, beta, h, r1, r2, pf, mhon;
};

template <class T>
TersoffSet<T> tersoff_set(const double* p, int num_types) {
  TersoffSet<T> t;
  const int off = num_types == 2 ? 4 : 0;
  for (int s = 0; s < 2; ++s) {
    const double* q = p + ((num_types == 2 && s == 1) ? 4 : 0);  // D0, A, r0, S of the set
    const double D0 = q[0], A = q[1], R0 = q[2], S = q[3];
    t.cr[s] = (T)(D0 / (S - 1.0));
    t.ca[s] = (T)(S * D0 / (S - 1.0));
    t.lr[s] = (T)(sqrt(2.0 * S) * A);
    t.la[s] = (T)(sqrt(2.0 / S) * A);
    t.r0[s] = (T)R0;
  }
  const double n = p[4 + off], r1 = p[7 + off], r2 = p[8 + off];
  t.n = (T)n;
  t.beta = (T)p[5 + off];
  t.h = (T)p[6 + off];
  t.r1 = (T)r1;
  t.r2 = (T)r2;
  t.pf = (T)(M_PI / (r2 - r1));
  t.mhon = (T)(-0.5 / n);
  return t;
}

// Rigid ion (ri.cu:21-110): per pair type t = type_i + type_j Buckingham A, 1/rho, C and the
// charge product qq (K_C included), the shifted damped Coulomb term with cutoff rc, and the
// cation-anion Morse pair with the Tersoff-style constants above; self = K_C S(rc) of the optional
// self energy (0 when off).
template <class T>
struct RigidIon {
  T A[3], inv_rho[3], C[3], qq[3];
  T rc, v_rc, dv_rc, cr, ca, lr, la, r0, self;
};

constexpr double kCoulomb = 14.399645;      // ri.cu:29
constexpr double kAlpha = 0.2;              // ri.cu:26
constexpr double kTwoOverSqrtPi = 1.1283791670955126;

// Damped-Coulomb self energy per K_C q_i^2 (develop/hfo2/find_E.m:10-13).
inline double ri_self_factor(double rc) {
  return kAlpha / sqrt(M_PI) + erfc(kAlpha * rc) / rc + 0.5 * (kTwoOverSqrtPi * kAlpha) * exp(-kAlpha * kAlpha * rc * rc);
}

template <class T>
RigidIon<T> rigid_ion_set(const double* p, int potential_type, bool with_self) {
  RigidIon<T> r;
  const double q2 = p[0] * p[0] * kCoulomb, ratio = ri_charge_ratio(potential_type);
  r.qq[0] = (T)q2;
  r.qq[1] = (T)(ratio * q2);
  r.qq[2] = (T)(ratio * ratio * q2);
  for (int t = 0; t < 3; ++t) {
    r.A[t] = (T)p[1 + 3 * t];
    r.inv_rho[t] = (T)(1.0 / p[2 + 3 * t]);
    r.C[t] = (T)p[3 + 3 * t];
  }
  const double rc = p[10], D0 = p[11], al = p[12], S = p[14];
  const double erfc_rc = erfc(kAlpha * rc);
  r.rc = (T)rc;
  r.v_rc = (T)(erfc_rc / rc);
  r.dv_rc = (T)(-erfc_rc / (rc * rc) - kTwoOverSqrtPi * kAlpha * exp(-kAlpha * kAlpha * rc * rc) / rc);
  r.cr = (T)(D0 / (S - 1.0));
  r.ca = (T)(S * D0 / (S - 1.0));
  r.lr = (T)(sqrt(2.0 * S) * al);
  r.la = (T)(sqrt(2.0 / S) * al);
  r.r0 = (T)p[13];
  r.self = with_self ? (T)ri_self_factor(rc) : T(0);
  return r;
}

// NN 2-body taper (nn2b.cuh:36-38 by default) and the force order of nn2b.cu:147-148.
struct MlpTaper {
  double r1, r2, pf;
  int consistent;
};

// --------------------------------------------------------------------------- list layouts
// The engine's CSR lists, or the reference's NL[k*N + i] (neighbor.cu:61) for the
// drop-in Potential entry points.  A bond's slot indexes the per-bond arrays
// (geometry, reverse slot, scratch).
struct CsrLayout {
  const int* off;
  const int* nbr;
  __device__ __forceinline__ int count(int i) const { return off[i + 1] - off[i]; }
  __device__ __forceinline__ int slot(int i, int k) const { return off[i] + k; }
  __device__ __forceinline__ int nb(int i, int k) const { return nbr[off[i] + k]; }
};
struct RefLayout {
  int N;
  const int* NN;
  const int* NL;
  __device__ __forceinline__ int count(int i) const { return NN[i]; }
  __device__ __forceinline__ int slot(int i, int k) const { return k * N + i; }
  __device__ __forceinline__ int nb(int i, int k) const { return NL[(size_t)k * N + i]; }
};

// Bond geometry (x, y, z, d) in FP64 as unit vector and length in T.
template <class T>
struct Bond {
  T ux, uy, uz, d;
  __device__ __forceinline__ explicit Bond(const double4& q) {
    const double inv = 1.0 / q.w;
    ux = (T)(q.x * inv);
    uy = (T)(q.y * inv);
    uz = (T)(q.z * inv);
    d = (T)q.w;
  }
  __device__ __forceinline__ T dot(const Bond& o) const { return ux * o.ux + uy * o.uy + uz * o.uz; }
};

// ------------------------------------------------------------------------------- Tersoff
// Per atom i, two passes over its bonds.
//   1. bond order of every bond j: zeta_j = sum_{k != j} fc_k beta (cos_jk - h)^2,
//      b_j = (1 + zeta_j^n)^mhon, db_j = d b / d zeta; the site energy
//      pe_i = 1/2 sum_j fc_j (fr_j - b_j fa_j); per bond the scalars S_j = db_j fa_j and
//      A_j = dfc_j (fr_j - b_j fa_j) + fc_j (fr'_j - b_j fa'_j) go to scratch.
//   2. f_ij = dE_i / dr_ij = 1/2 [(A_j - dfc_j sum_k T_k g_jk - m_j sum_k q_jk cos_jk) u_j
//                                 + m_j sum_k q_jk u_k]
//      with T_k = S_k fc_k, g = beta (cos - h)^2, q_jk = beta (cos_jk - h)(S_j fc_k + T_k),
//      m_j = -2 fc_j / d_j (the derivative of cos_jk along r_ij is (u_k - cos_jk u_j) / d_j).
template <class T, class Lay>
__global__ void plain_tersoff_bonds(int N, int num_types, const int* __restrict__ type, Lay L,
                                    const double4* __restrict__ g, TersoffSet<T> P, T* __restrict__ sS,
                                    T* __restrict__ sA, T* __restrict__ fx, T* __restrict__ fy, T* __restrict__ fz,
                                    T* __restrict__ pe) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const int Z = L.count(i), ti = type[i];
  T site = T(0);
  for (int j = 0; j < Z; ++j) {
    const int sj = L.slot(i, j);
    const Bond<T> bj(g[sj]);
    T zeta = T(0);
    for (int k = 0; k < Z; ++k) {
      if (k == j) continue;
      const Bond<T> bk(g[L.slot(i, k)]);
      T fck, dfck;
      taper(P.r1, P.r2, P.pf, bk.d, fck, dfck);
      const T x = bj.dot(bk) - P.h;
      zeta += fck * P.beta * x * x;
    }
    T b = T(1), db = T(0);
    if (!(zeta < T(1.0e-16))) {  // minimal_tersoff.cu:178-185: b = 1, b' = 0 below 1e-16
      const T zn = m_exp(P.n * m_log(zeta));
      b = m_exp(P.mhon * m_log1p(zn));
      db = T(-0.5) * b * zn / ((T(1) + zn) * zeta);
    }
    const int s = (num_types == 2 && ti != type[L.nb(i, j)]) ? 1 : 0;
    const T t = bj.d - P.r0[s];
    const T fr = P.cr[s] * m_exp(-P.lr[s] * t), fa = P.ca[s] * m_exp(-P.la[s] * t);
    T fcj, dfcj;
    taper(P.r1, P.r2, P.pf, bj.d, fcj, dfcj);
    const T e = fr - b * fa;
    site += T(0.5) * fcj * e;
    sS[sj] = db * fa;
    sA[sj] = dfcj * e + fcj * (-P.lr[s] * fr + b * P.la[s] * fa);
  }
  pe[i] = site;
  for (int j = 0; j < Z; ++j) {
    const int sj = L.slot(i, j);
    const Bond<T> bj(g[sj]);
    T fcj, dfcj;
    taper(P.r1, P.r2, P.pf, bj.d, fcj, dfcj);
    const T Sj = sS[sj];
    T sum_tg = T(0), sum_qc = T(0), vx = T(0), vy = T(0), vz = T(0);
    for (int k = 0; k < Z; ++k) {
      if (k == j) continue;
      const int sk = L.slot(i, k);
      const Bond<T> bk(g[sk]);
      T fck, dfck;
      taper(P.r1, P.r2, P.pf, bk.d, fck, dfck);
      const T Tk = sS[sk] * fck;
      const T c = bj.dot(bk);
      const T bx = P.beta * (c - P.h);
      const T q = bx * (Sj * fck + Tk);
      sum_tg += Tk * bx * (c - P.h);
      sum_qc += q * c;
      vx += q * bk.ux;
      vy += q * bk.uy;
      vz += q * bk.uz;
    }
    const T m = T(-2) * fcj / bj.d;
    const T radial = T(0.5) * (sA[sj] - dfcj * sum_tg - m * sum_qc), perp = T(0.5) * m;
    fx[sj] = radial * bj.ux + perp * vx;
    fy[sj] = radial * bj.uy + perp * vy;
    fz[sj] = radial * bj.uz + perp * vz;
  }
}

// F_i = sum_j (f_ij - f_ji); the per-atom virial of the reference's output layout
// (minimal_tersoff.cu:377-404): W_i,ab = -1/2 sum_j r_ij,a (f_ij - f_ji)_b in the order
// xx, yy, zz, xy, yz, zx (not symmetrised).
template <class T, class Lay>
__global__ void plain_tersoff_gather(int N, Lay L, const int* __restrict__ rev, const double4* __restrict__ g,
                                     const T* __restrict__ fx, const T* __restrict__ fy, const T* __restrict__ fz,
                                     T* __restrict__ F, T* __restrict__ W) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  T f[3] = {T(0), T(0), T(0)}, w[6] = {T(0), T(0), T(0), T(0), T(0), T(0)};
  const int Z = L.count(i);
  for (int j = 0; j < Z; ++j) {
    const int sj = L.slot(i, j), sr = rev[sj];
    const double4 q = g[sj];
    const T r[3] = {(T)q.x, (T)q.y, (T)q.z};
    const T df[3] = {fx[sj] - fx[sr], fy[sj] - fy[sr], fz[sj] - fz[sr]};
    for (int a = 0; a < 3; ++a) {
      f[a] += df[a];
      w[a] -= T(0.5) * r[a] * df[a];          // xx, yy, zz
      w[3 + a] -= T(0.5) * r[a] * df[(a + 1) % 3];  // xy, yz, zx
    }
  }
  for (int a = 0; a < 3; ++a) F[i + (size_t)a * N] = f[a];
  for (int k = 0; k < 6; ++k) W[i + (size_t)k * N] = w[k];
}

// --------------------------------------------------------------------------- pair models
// Rigid-ion pair energy U(d) and dU/dd for pair type t (0 cation-cation, 1 cation-anion with
// Morse, 2 anion-anion): A e^{-d/rho} - C/d^6 + qq (erfc(alpha d)/d - v_rc - dv_rc (d - rc)).
template <class T>
__device__ __forceinline__ void rigid_ion_pair(const RigidIon<T>& R, int t, T d, T& U, T& dU) {
  const T id = T(1) / d, id6 = id * id * id * id * id * id;
  const T buck = R.A[t] * m_exp(-d * R.inv_rho[t]);
  const T coul = m_erfc(T(kAlpha) * d) * id;
  U = buck - R.C[t] * id6 + R.qq[t] * (coul - R.v_rc - R.dv_rc * (d - R.rc));
  dU = -R.inv_rho[t] * buck + T(6) * R.C[t] * id6 * id -
       R.qq[t] * (coul * id + T(kTwoOverSqrtPi * kAlpha) * m_exp(T(-kAlpha * kAlpha) * d * d) * id + R.dv_rc);
  if (t == 1) {
    const T x = d - R.r0;
    const T rep = R.cr * m_exp(-R.lr * x), att = R.ca * m_exp(-R.la * x);
    U += rep - att;
    dU += R.la * att - R.lr * rep;
  }
}

// 1 -> n -> n -> 1 tanh network of the distance (nn2b.cu:49-78 parameter order: w0[n], b0[n],
// W1[n][n] row-major, b1[n], w2[n], b2) and its derivative, forward mode.
template <class T>
__device__ __forceinline__ void mlp_pair(const T* __restrict__ w, int n, T d, T& U, T& dU) {
  T h1[32], dh1[32];
  for (int m = 0; m < n; ++m) {
    h1[m] = m_tanh(w[m] * d - w[n + m]);
    dh1[m] = (T(1) - h1[m] * h1[m]) * w[m];
  }
  const T* W1 = w + 2 * n;
  const T* b1 = W1 + n * n;
  const T* w2 = b1 + n;
  U = T(0);
  dU = T(0);
  for (int a = 0; a < n; ++a) {
    T z = T(0), dz = T(0);
    for (int m = 0; m < n; ++m) {
      z += W1[a * n + m] * h1[m];
      dz += W1[a * n + m] * dh1[m];
    }
    const T h2 = m_tanh(z - b1[a]);
    U += w2[a] * h2;
    dU += w2[a] * (T(1) - h2 * h2) * dz;
  }
  U -= w2[n];
}

// Owner-computes pair loop: every atom walks its full list.  pe_i = 1/2 sum_j U_ij,
// F_i = sum_j dU_ij u_ij, W_i = -1/2 sum_j d_ij dU_ij u_ij (x) u_ij (reference order).
// KIND 0 rigid ion, 1 NN 2-body.
template <class T, int KIND, class Lay>
__global__ void plain_pair(int N, const int* __restrict__ type, Lay L, const double4* __restrict__ g, RigidIon<T> R,
                           const T* __restrict__ w, int n, MlpTaper tp, T* __restrict__ F, T* __restrict__ W,
                           T* __restrict__ pe) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  T e = T(0), f[3] = {T(0), T(0), T(0)}, v[6] = {T(0), T(0), T(0), T(0), T(0), T(0)};
  const int Z = L.count(i);
  for (int j = 0; j < Z; ++j) {
    const Bond<T> bj(g[L.slot(i, j)]);
    T U, dU;
    if (KIND == 0) {
      rigid_ion_pair(R, type[i] + type[L.nb(i, j)], bj.d, U, dU);
    } else {
      T Uraw, dUraw, fc, dfc;
      mlp_pair(w, n, bj.d, Uraw, dUraw);
      taper((T)tp.r1, (T)tp.r2, (T)tp.pf, bj.d, fc, dfc);
      U = Uraw * fc;
      // nn2b.cu:147-148 tapers the energy before it enters the force term
      dU = dUraw * fc + (tp.consistent ? Uraw : U) * dfc;
    }
    const T u[3] = {bj.ux, bj.uy, bj.uz};
    const T s = T(-0.5) * bj.d * dU;
    for (int a = 0; a < 3; ++a) {
      f[a] += dU * u[a];
      v[a] += s * u[a] * u[a];
      v[3 + a] += s * u[a] * u[(a + 1) % 3];
    }
    e += T(0.5) * U;
  }
  if (KIND == 0) e -= R.qq[type[i] == 0 ? 0 : 2] * R.self;  // self energy K_C q_i^2 S(rc)
  for (int a = 0; a < 3; ++a) F[i + (size_t)a * N] = f[a];
  for (int k = 0; k < 6; ++k) W[i + (size_t)k * N] = v[k];
  pe[i] = e;
}

// ----------------------------------------------------------------- per-individual fitness
// One CTA per configuration: FP64 sums of site energies / virials and of the
// squared force error, then one thread folds them into the fitness
// (fitness.cu:392-555 with FP64 accumulation).
template <class T>
__global__ void p_config_errors(int N, int Nc, int Nc_force, const int* __restrict__ Na,
                                const int* __restrict__ Na_sum, const T* __restrict__ F, const T* __restrict__ W,
                                const T* __restrict__ pe, const float* __restrict__ force_ref,
                                const double* __restrict__ E_ref, const double* __restrict__ W_ref,
                                double* __restrict__ cfg) {
  __shared__ double red[8][256];
  const int c = blockIdx.x;
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int i = Na_sum[c] + threadIdx.x; i < Na_sum[c] + Na[c]; i += blockDim.x) {
    if (c >= Nc_force) {
      acc[0] += (double)pe[i];
      for (int k = 0; k < 6; ++k) acc[1 + k] += (double)W[i + (size_t)N * k];
    } else {
      const double dx = (double)F[i] - force_ref[i];
      const double dy = (double)F[i + N] - force_ref[i + N];
      const double dz = (double)F[i + 2 * (size_t)N] - force_ref[i + 2 * (size_t)N];
      acc[7] += dx * dx + dy * dy + dz * dz;
    }
  }
  for (int k = 0; k < 8; ++k) red[k][threadIdx.x] = acc[k];
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s)
      for (int k = 0; k < 8; ++k) red[k][threadIdx.x] += red[k][threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    double eE = 0, eW = 0;
    if (c >= Nc_force) {
      const double de = red[0][0] - E_ref[c];
      eE = de * de;
      for (int k = 0; k < 6; ++k) {
        const double dw = red[1 + k][0] - W_ref[c + (size_t)Nc * k];
        eW += dw * dw;
      }
    }
    cfg[3 * c + 0] = eE;
    cfg[3 * c + 1] = eW;
    cfg[3 * c + 2] = red[7][0];
  }
}

__global__ void p_fitness(int Nc, const double* __restrict__ cfg, double nF, double nE, double nW, float wF,
                          float wE, float wW, double* __restrict__ out) {
  if (threadIdx.x != 0) return;
  double eE = 0, eW = 0, eF = 0;
  for (int c = 0; c < Nc; ++c) {
    eE += cfg[3 * c];
    eW += cfg[3 * c + 1];
    eF += cfg[3 * c + 2];
  }
  const double rE = sqrt(eE / nE), rW = sqrt(eW / nW), rF = sqrt(eF / nF);
  out[0] = (double)wE * rE + (double)wW * rW + (double)wF * rF;
  out[1] = rE;
  out[2] = rW;
  out[3] = rF;
}

namespace {

// Device buffers of one evaluation: per-bond scratch (S, A, f_ij x/y/z), per-atom outputs.
template <class T>
struct Scratch {
  T *S, *A, *fx, *fy, *fz, *F, *W, *pe;
};

template <class T>
Scratch<T> carve(T* bonds, size_t B, T* F, T* W, T* pe) {
  return Scratch<T>{bonds, bonds + B, bonds + 2 * B, bonds + 3 * B, bonds + 4 * B, F, W, pe};
}

template <class T>
int ensure_scratch(Engine* e, Scratch<T>* s);

template <>
int ensure_scratch<double>(Engine* e, Scratch<double>* s) {
  const size_t B = std::max(e->d.B, 1), N = e->d.N;
  if (!e->s64) {
    GPUGA_TRY(e->alloc(&e->s64, 5 * B));
    GPUGA_TRY(e->alloc(&e->p64_F, 3 * N));
    GPUGA_TRY(e->alloc(&e->p64_W, 6 * N));
    GPUGA_TRY(e->alloc(&e->p64_pe, N));
  }
  *s = carve(e->s64, B, e->p64_F, e->p64_W, e->p64_pe);
  return GPUGA_OK;
}

template <>
int ensure_scratch<float>(Engine* e, Scratch<float>* s) {
  const size_t B = std::max(e->d.B, 1), N = e->d.N;
  if (!e->s32) {
    GPUGA_TRY(e->alloc(&e->s32, 5 * B));
    GPUGA_TRY(e->alloc(&e->p32_F, 3 * N));
    GPUGA_TRY(e->alloc(&e->p32_W, 6 * N));
    GPUGA_TRY(e->alloc(&e->p32_pe, N));
  }
  *s = carve(e->s32, B, e->p32_F, e->p32_W, e->p32_pe);
  return GPUGA_OK;
}

MlpTaper mlp_taper(const PotentialSpec& sp) {
  return MlpTaper{sp.nn_r1, sp.nn_r2, M_PI / ((double)sp.nn_r2 - sp.nn_r1), sp.nn_consistent};
}

// Enqueues the force launches of one parameter vector p (decoded, FP64) on `st`.  NN2B reads its
// weights from the device array w (already in T).
template <class T, class Lay>
int enqueue_force(int potential_type, int num_neurons, const double* p, const PotentialSpec& sp, int N,
                  const int* type, Lay L, const int* rev, const double4* g, const T* w, const Scratch<T>& s,
                  cudaStream_t st) {
  const int grid = (N + 127) / 128;
  if (potential_type == 1 || potential_type == 2) {
    const int num_types = potential_type == 2 ? 2 : 1;
    const TersoffSet<T> P = tersoff_set<T>(p, num_types);
    plain_tersoff_bonds<T><<<grid, 128, 0, st>>>(N, num_types, type, L, g, P, s.S, s.A, s.fx, s.fy, s.fz, s.pe);
    plain_tersoff_gather<T><<<grid, 128, 0, st>>>(N, L, rev, g, s.fx, s.fy, s.fz, s.F, s.W);
  } else if (is_ri_type(potential_type)) {
    const RigidIon<T> R = rigid_ion_set<T>(p, potential_type, sp.ri_self != 0);
    plain_pair<T, 0><<<grid, 128, 0, st>>>(N, type, L, g, R, nullptr, 0, MlpTaper{}, s.F, s.W, s.pe);
  } else if (potential_type == 3) {
    if (num_neurons < 1 || num_neurons > 32) {
      set_error("the plain NN2B path supports 1 to 32 neurons per layer (got %d).", num_neurons);
      return GPUGA_ERR_UNSUPPORTED;
    }
    plain_pair<T, 1><<<grid, 128, 0, st>>>(N, type, L, g, RigidIon<T>{}, w, num_neurons, mlp_taper(sp), s.F, s.W,
                                           s.pe);
  } else {
    set_error("unsupported potential type %d.", potential_type);
    return GPUGA_ERR_UNSUPPORTED;
  }
  GPUGA_CUDA(cudaGetLastError());
  return GPUGA_OK;
}

// Device copy of P parameter vectors in T for NN2B (the kernels read weights from HBM).
template <class T>
int upload_weights(Engine* e, const std::vector<double>& host, T** out) {
  const size_t need = host.size() * sizeof(T);
  if (e->p_w_bytes < need) {
    if (e->p_w) cudaFree(e->p_w);
    e->p_w = nullptr;
    e->p_w_bytes = 0;
    GPUGA_CUDA(cudaMalloc(&e->p_w, need));
    e->p_w_bytes = need;
  }
  std::vector<T> conv(host.begin(), host.end());
  GPUGA_CUDA(cudaMemcpy(e->p_w, conv.data(), need, cudaMemcpyHostToDevice));
  *out = static_cast<T*>(e->p_w);
  return GPUGA_OK;
}

template <class T>
int plain_fitness_t(Engine* e, int P, const float* pop01, double* fitness, double* comps) {
  Scratch<T> s;
  GPUGA_TRY(ensure_scratch<T>(e, &s));
  const DevSet& d = e->d;
  const int nv = d.num_vars;
  cudaStream_t st = e->stream;
  if (e->p_out_cap < P) {
    if (e->p_out) cudaFree(e->p_out);
    e->p_out = nullptr;
    GPUGA_CUDA(cudaMalloc(&e->p_out, sizeof(double) * (4 * (size_t)P + 3 * (size_t)d.Nc)));
    e->p_out_cap = P;
  }
  double* cfg = e->p_out + 4 * (size_t)P;
  // FP32 decode as the reference does (fitness.cu:320-324), then the individual's parameters in T
  std::vector<double> params((size_t)P * nv);
  std::vector<float> p32(nv);
  for (int p = 0; p < P; ++p) {
    decode_params(e->spec, pop01 + (size_t)p * nv, p32.data());
    for (int m = 0; m < nv; ++m) params[(size_t)p * nv + m] = p32[m];
  }
  T* w = nullptr;
  if (d.potential_type == 3) GPUGA_TRY(upload_weights<T>(e, params, &w));
  const CsrLayout L{d.off, d.nbr};
  for (int p = 0; p < P; ++p) {
    GPUGA_TRY(enqueue_force<T>(d.potential_type, d.num_neurons, params.data() + (size_t)p * nv, e->spec, d.N, d.type,
                               L, d.rev, d.g64, w ? w + (size_t)p * nv : nullptr, s, st));
    p_config_errors<T><<<d.Nc, 256, 0, st>>>(d.N, d.Nc, d.Nc_force, d.Na, d.Na_sum, s.F, s.W, s.pe, d.force_ref,
                                             d.E_ref, d.W_ref, cfg);
    p_fitness<<<1, 32, 0, st>>>(d.Nc, cfg, d.norm_force, d.norm_energy, d.norm_virial, d.w_force, d.w_energy,
                                d.w_stress, e->p_out + 4 * (size_t)p);
    GPUGA_CUDA(cudaGetLastError());
  }
  std::vector<double> out(4 * (size_t)P);
  GPUGA_CUDA(cudaMemcpyAsync(out.data(), e->p_out, sizeof(double) * 4 * P, cudaMemcpyDeviceToHost, st));
  GPUGA_CUDA(cudaStreamSynchronize(st));
  for (int p = 0; p < P; ++p) {
    fitness[p] = out[4 * (size_t)p];
    if (comps)
      for (int k = 0; k < 3; ++k) comps[3 * (size_t)p + k] = out[4 * (size_t)p + 1 + k];
  }
  return GPUGA_OK;
}

// One parameter vector on the engine's training set; outputs copied to the host.
template <class T>
int plain_find_force_t(Engine* e, const std::vector<double>& params, T* F, T* W, T* pe) {
  Scratch<T> s;
  GPUGA_TRY(ensure_scratch<T>(e, &s));
  const DevSet& d = e->d;
  cudaStream_t st = e->stream;
  T* w = nullptr;
  if (d.potential_type == 3) GPUGA_TRY(upload_weights<T>(e, params, &w));
  GPUGA_TRY(enqueue_force<T>(d.potential_type, d.num_neurons, params.data(), e->spec, d.N, d.type,
                             CsrLayout{d.off, d.nbr}, d.rev, d.g64, w, s, st));
  const size_t N = d.N;
  if (F) GPUGA_CUDA(cudaMemcpyAsync(F, s.F, sizeof(T) * 3 * N, cudaMemcpyDeviceToHost, st));
  if (W) GPUGA_CUDA(cudaMemcpyAsync(W, s.W, sizeof(T) * 6 * N, cudaMemcpyDeviceToHost, st));
  if (pe) GPUGA_CUDA(cudaMemcpyAsync(pe, s.pe, sizeof(T) * N, cudaMemcpyDeviceToHost, st));
  GPUGA_CUDA(cudaStreamSynchronize(st));
  return GPUGA_OK;
}

}  // namespace

int plain_fitness(Engine* e, bool fp64, int P, const float* pop01, double* fitness, double* comps) {
  return fp64 ? plain_fitness_t<double>(e, P, pop01, fitness, comps)
              : plain_fitness_t<float>(e, P, pop01, fitness, comps);
}

// FP64 parameters stay exact: the constants are derived from them directly.
int plain_find_force64(Engine* e, const double* params, double* F, double* W, double* pe) {
  return plain_find_force_t<double>(e, std::vector<double>(params, params + e->d.num_vars), F, W, pe);
}

int plain_find_force32(Engine* e, const float* params, float* F, float* W, float* pe) {
  return plain_find_force_t<float>(e, std::vector<double>(params, params + e->d.num_vars), F, W, pe);
}

// --------------------------------------------------------------- reference-layout Potential
size_t ref_potential_scratch_bytes(int potential_type, int num_neurons, int N, int max_Na) {
  const size_t slots = (size_t)N * (size_t)max_Na;
  const int nv = std::max(num_vars_for(potential_type, num_neurons), 1);
  auto up = [](size_t b) { return (b + 255) & ~(size_t)255; };
  return up(slots * sizeof(double4)) + up(slots * sizeof(int)) + up(5 * slots * sizeof(float)) +
         up((size_t)nv * sizeof(float));
}

// Potential::find_force (potential.cuh:28-40) in FP32 on the reference's
// layouts: bond geometry from the FP32 image rule, then the Tersoff passes or
// the pair loop, all enqueued on `st`; nothing is allocated here.  `params` is a
// host array (decoded parameters in potential.in order); NN2B weights are copied
// from it into the scratch.
int ref_potential_find_force(int potential_type, int num_neurons, const float* params, const PotentialSpec& nn_opts,
                             int Nc, int N, const int* Na, const int* Na_sum, int max_Na, const int* type,
                             const float* h, const int* NN, const int* NL, const float* r, float* f, float* virial,
                             float* pe, const RefPotentialScratch& s, cudaStream_t st) {
  const int nv = num_vars_for(potential_type, num_neurons);
  if (nv < 0) {
    set_error("unsupported potential type %d.", potential_type);
    return GPUGA_ERR_UNSUPPORTED;
  }
  GPUGA_TRY(ref_layout_geometry(Nc, N, Na, Na_sum, h, r, NN, NL, s.g64, s.rev, st));
  const size_t slots = (size_t)N * (size_t)max_Na;
  Scratch<float> sc{s.f5, s.f5 + slots, s.f5 + 2 * slots, s.f5 + 3 * slots, s.f5 + 4 * slots, f, virial, pe};
  if (potential_type == 3 && num_neurons >= 1 && num_neurons <= 32)
    GPUGA_CUDA(cudaMemcpyAsync(s.w, params, sizeof(float) * nv, cudaMemcpyHostToDevice, st));
  const std::vector<double> p(params, params + nv);
  return enqueue_force<float>(potential_type, num_neurons, p.data(), nn_opts, N, type, RefLayout{N, NN, NL}, s.rev,
                              s.g64, s.w, sc, st);
}

}  // namespace gpuga
