// Plain path: one individual per launch sequence, one thread per atom, the
// reference's three-step Tersoff structure (minimal_tersoff.cu:122-405) and
// owner-computes pair loops (ri.cu:112-189, nn2b.cu:94-173), templated on the
// arithmetic type.  FP64 is the denominator of the batched engine's speed-up
// and the device-side FP64 reference; FP32 gives the reference's float outputs.
#include <cmath>

#include "engine.hpp"

namespace gpuga {

template <class T>
struct PT {  // minimal Tersoff constants
  T D0[2], A[2], R0[2], S[2], EN, BETA, H, R1, R2, PF, MHON;
};
template <class T>
struct PR {  // RI constants (ri.cu:21-25); self: K_C S(rc) of the optional self energy (0 when off)
  T a[3], b[3], c[3], qq[3], v_rc, dv_rc, cutoff, d0, alpha, r0, s, self;
};

// Damped-Coulomb self energy per K_C q_i^2 (develop/hfo2/find_E.m:10-13).
inline double ri_self_factor(double rc) {
  const double alpha = 0.2, pif = 0.225675833419103;
  return alpha / sqrt(M_PI) + erfc(alpha * rc) / rc + 0.5 * pif * exp(-alpha * alpha * rc * rc);
}
struct PN {
  int n;
  double r1, r2, pf;
  int consistent;
};

template <class T>
__device__ __forceinline__ T texp(T x) {
  return exp(x);
}
template <>
__device__ __forceinline__ float texp<float>(float x) {
  return expf(x);
}

template <class T>
__device__ __forceinline__ void fcut(T r1, T r2, T pf, T d, T& fc, T& fcp) {
  if (d < r1) {
    fc = 1;
    fcp = 0;
  } else if (d < r2) {
    fc = T(0.5) * cos(pf * (d - r1)) + T(0.5);
    fcp = -sin(pf * (d - r1)) * pf * T(0.5);
  } else {
    fc = 0;
    fcp = 0;
  }
}

// Neighbor-list layouts: the engine's CSR lists, or the reference's
// NL[k*N + i] (neighbor.cu:61) for the drop-in Potential entry points.  A bond
// slot indexes the per-bond arrays (geometry, reverse slot, scratch).
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

template <class T>
__device__ __forceinline__ void bond(const double4* g, int b, T& x, T& y, T& z, T& d) {
  const double4 q = g[b];
  x = (T)q.x;
  y = (T)q.y;
  z = (T)q.z;
  d = (T)q.w;
}

// step 1 (minimal_tersoff.cu:122-188): bond orders
template <class T, class Lay>
__global__ void p_tersoff1(int N, Lay L, const double4* __restrict__ g, PT<T> P, T* __restrict__ b,
                           T* __restrict__ bp) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const int Z = L.count(i);
  for (int k1 = 0; k1 < Z; ++k1) {
    const int i1 = L.slot(i, k1);
    const int n2 = L.nb(i, k1);
    T x12, y12, z12, d12;
    bond(g, i1, x12, y12, z12, d12);
    T zeta = 0;
    for (int k2 = 0; k2 < Z; ++k2) {
      const int i2 = L.slot(i, k2);
      if (L.nb(i, k2) == n2) continue;
      T x13, y13, z13, d13;
      bond(g, i2, x13, y13, z13, d13);
      const T cs = (x12 * x13 + y12 * y13 + z12 * z13) / (d12 * d13);
      T fc13, fcp13;
      fcut(P.R1, P.R2, P.PF, d13, fc13, fcp13);
      const T x = cs - P.H;
      zeta += fc13 * P.BETA * x * x;
    }
    const T bzn = pow(zeta, P.EN);
    const T bij = pow(T(1) + bzn, P.MHON);
    if (zeta < T(1.0e-16)) {
      b[i1] = 1;
      bp[i1] = 0;
    } else {
      b[i1] = bij;
      bp[i1] = -bij * bzn * T(0.5) / ((T(1) + bzn) * zeta);
    }
  }
}

// step 2 (minimal_tersoff.cu:191-316): partial forces and site energies
template <class T, class Lay>
__global__ void p_tersoff2(int N, int num_types, const int* __restrict__ type, Lay L,
                           const double4* __restrict__ g, PT<T> P, const T* __restrict__ b,
                           const T* __restrict__ bp, T* __restrict__ pe, T* __restrict__ fxs,
                           T* __restrict__ fys, T* __restrict__ fzs) {
  const int n1 = blockIdx.x * blockDim.x + threadIdx.x;
  if (n1 >= N) return;
  const int type1 = type[n1];
  const int Z = L.count(n1);
  T pot = 0;
  for (int k1 = 0; k1 < Z; ++k1) {
    const int i1 = L.slot(n1, k1);
    const int n2 = L.nb(n1, k1);
    const int s12 = (num_types == 2 && type1 != type[n2]) ? 1 : 0;
    T x12, y12, z12, d12;
    bond(g, i1, x12, y12, z12, d12);
    const T d12inv = T(1) / d12;
    T fc12, fcp12;
    fcut(P.R1, P.R2, P.PF, d12, fc12, fcp12);
    const T lr = sqrt(T(2) * P.S[s12]) * P.A[s12], la = sqrt(T(2) / P.S[s12]) * P.A[s12];
    const T fr12 = P.D0[s12] / (P.S[s12] - T(1)) * texp(-lr * (d12 - P.R0[s12]));
    const T frp12 = -lr * fr12;
    const T fa12 = P.S[s12] * P.D0[s12] / (P.S[s12] - T(1)) * texp(-la * (d12 - P.R0[s12]));
    const T fap12 = -la * fa12;
    const T b12 = b[i1];
    const T factor3 = (fcp12 * (fr12 - b12 * fa12) + fc12 * (frp12 - b12 * fap12)) * d12inv;
    T f12x = x12 * factor3 * T(0.5), f12y = y12 * factor3 * T(0.5), f12z = z12 * factor3 * T(0.5);
    pot += fc12 * (fr12 - b12 * fa12) * T(0.5);
    const T bp12 = bp[i1];
    for (int k2 = 0; k2 < Z; ++k2) {
      const int i2 = L.slot(n1, k2);
      const int n3 = L.nb(n1, k2);
      if (n3 == n2) continue;
      const int s13 = (num_types == 2 && type1 != type[n3]) ? 1 : 0;
      T x13, y13, z13, d13;
      bond(g, i2, x13, y13, z13, d13);
      T fc13, fcp13;
      fcut(P.R1, P.R2, P.PF, d13, fc13, fcp13);
      const T la13 = sqrt(T(2) / P.S[s13]) * P.A[s13];
      const T fa13 = P.S[s13] * P.D0[s13] / (P.S[s13] - T(1)) * texp(-la13 * (d13 - P.R0[s13]));
      const T bp13 = bp[i2];
      const T one_over_d12d13 = T(1) / (d12 * d13);
      const T cos123 = (x12 * x13 + y12 * y13 + z12 * z13) * one_over_d12d13;
      const T cos123_over_d12d12 = cos123 * d12inv * d12inv;
      const T xx = cos123 - P.H;
      const T g123 = P.BETA * xx * xx, gp123 = P.BETA * T(2) * xx;
      const T dc = -fc12 * bp12 * fa12 * fc13 * gp123 - fc12 * bp13 * fa13 * fc13 * gp123;
      const T dr = -fcp12 * bp13 * fa13 * g123 * fc13 * d12inv;
      T cos_d = x13 * one_over_d12d13 - x12 * cos123_over_d12d12;
      f12x += (x12 * dr + dc * cos_d) * T(0.5);
      cos_d = y13 * one_over_d12d13 - y12 * cos123_over_d12d12;
      f12y += (y12 * dr + dc * cos_d) * T(0.5);
      cos_d = z13 * one_over_d12d13 - z12 * cos123_over_d12d12;
      f12z += (z12 * dr + dc * cos_d) * T(0.5);
    }
    fxs[i1] = f12x;
    fys[i1] = f12y;
    fzs[i1] = f12z;
  }
  pe[n1] = pot;
}

// step 3 (minimal_tersoff.cu:318-405): force gather and per-atom virial
template <class T, class Lay>
__global__ void p_tersoff3(int N, Lay L, const int* __restrict__ rev, const double4* __restrict__ g,
                           const T* __restrict__ fxs, const T* __restrict__ fys, const T* __restrict__ fzs,
                           T* __restrict__ F, T* __restrict__ W) {
  const int n1 = blockIdx.x * blockDim.x + threadIdx.x;
  if (n1 >= N) return;
  T sfx = 0, sfy = 0, sfz = 0, vxx = 0, vyy = 0, vzz = 0, vxy = 0, vyz = 0, vzx = 0;
  const int Z = L.count(n1);
  for (int k1 = 0; k1 < Z; ++k1) {
    const int i1 = L.slot(n1, k1);
    T x12, y12, z12, d12;
    bond(g, i1, x12, y12, z12, d12);
    const int r = rev[i1];
    const T dx = fxs[i1] - fxs[r], dy = fys[i1] - fys[r], dz = fzs[i1] - fzs[r];
    sfx += dx;
    sfy += dy;
    sfz += dz;
    vxx -= x12 * dx * T(0.5);
    vyy -= y12 * dy * T(0.5);
    vzz -= z12 * dz * T(0.5);
    vxy -= x12 * dy * T(0.5);
    vyz -= y12 * dz * T(0.5);
    vzx -= z12 * dx * T(0.5);
  }
  F[n1] = sfx;
  F[n1 + N] = sfy;
  F[n1 + 2 * (size_t)N] = sfz;
  W[n1] = vxx;
  W[n1 + N] = vyy;
  W[n1 + 2 * (size_t)N] = vzz;
  W[n1 + 3 * (size_t)N] = vxy;
  W[n1 + 4 * (size_t)N] = vyz;
  W[n1 + 5 * (size_t)N] = vzx;
}

template <class T>
__device__ __forceinline__ void ri_p2f2(const PR<T>& q, int t, T d, T& p2, T& f2) {
  const T alpha = T(0.2), alpha_sq = T(0.04), pif = T(0.225675833419103);
  const T dsq = d * d, dinv = T(1) / d, dinv3 = dinv * dinv * dinv, dinv6 = dinv3 * dinv3, dinv7 = dinv6 * dinv;
  const T ex = texp(-d * q.b[t]);
  const T erfc_r = erfc(alpha * d) * dinv;
  p2 = q.a[t] * ex - q.c[t] * dinv6;
  f2 = T(6) * q.c[t] * dinv7 - q.a[t] * ex * q.b[t];
  p2 += q.qq[t] * (erfc_r - q.v_rc - q.dv_rc * (d - q.cutoff));
  f2 -= q.qq[t] * (erfc_r * dinv + pif * dinv * texp(-alpha_sq * dsq) + q.dv_rc);
  if (t == 1) {
    const T fr = q.d0 / (q.s - T(1)) * texp(-sqrt(T(2) * q.s) * q.alpha * (d - q.r0));
    const T frp = -sqrt(T(2) * q.s) * q.alpha * fr;
    const T fa = q.s * q.d0 / (q.s - T(1)) * texp(-sqrt(T(2) / q.s) * q.alpha * (d - q.r0));
    const T fap = -sqrt(T(2) / q.s) * q.alpha * fa;
    p2 += fr - fa;
    f2 += frp - fap;
  }
  f2 *= dinv;
}

template <class T>
__device__ void nn_p2f2(const T* __restrict__ w, int n, T d, T& p2, T& f2) {
  T x1[32], y1[32];
  for (int a = 0; a < n; ++a) {
    x1[a] = tanh(w[a] * d - w[a + n]);
    y1[a] = (T(1) - x1[a] * x1[a]) * w[a];
  }
  p2 = 0;
  f2 = 0;
  for (int a = 0; a < n; ++a) {
    T x2 = 0, y2 = 0;
    for (int m = 0; m < n; ++m) {
      x2 += w[2 * n + a * n + m] * x1[m];
      y2 += w[2 * n + a * n + m] * y1[m];
    }
    x2 = tanh(x2 - w[n * (n + 2) + a]);
    y2 *= T(1) - x2 * x2;
    p2 += w[n * (n + 3) + a] * x2;
    f2 += w[n * (n + 3) + a] * y2;
  }
  p2 = p2 - w[n * (n + 4)];
}

// ri.cu:112-189 / nn2b.cu:94-173
template <class T, class Lay>
__global__ void p_pair(int N, int kind, const int* __restrict__ type, Lay L, const double4* __restrict__ g, PR<T> q,
                       const T* __restrict__ w, PN nn, T* __restrict__ F, T* __restrict__ W, T* __restrict__ pe) {
  const int n1 = blockIdx.x * blockDim.x + threadIdx.x;
  if (n1 >= N) return;
  T e = 0, fx = 0, fy = 0, fz = 0, vxx = 0, vyy = 0, vzz = 0, vxy = 0, vyz = 0, vzx = 0;
  const int Z = L.count(n1);
  for (int k1 = 0; k1 < Z; ++k1) {
    const int i1 = L.slot(n1, k1);
    T x12, y12, z12, d12;
    bond(g, i1, x12, y12, z12, d12);
    T p2, f2;
    if (kind == 0) {
      ri_p2f2(q, type[n1] + type[L.nb(n1, k1)], d12, p2, f2);
    } else {
      nn_p2f2(w, nn.n, d12, p2, f2);
      T fc, fcp;
      fcut((T)nn.r1, (T)nn.r2, (T)nn.pf, d12, fc, fcp);
      if (nn.consistent) {
        f2 = (f2 * fc + p2 * fcp) / d12;
        p2 *= fc;
      } else {
        p2 *= fc;
        f2 = (f2 * fc + p2 * fcp) / d12;
      }
    }
    fx += x12 * f2;
    fy += y12 * f2;
    fz += z12 * f2;
    vxx -= x12 * x12 * f2 * T(0.5);
    vyy -= y12 * y12 * f2 * T(0.5);
    vzz -= z12 * z12 * f2 * T(0.5);
    vxy -= x12 * y12 * f2 * T(0.5);
    vyz -= y12 * z12 * f2 * T(0.5);
    vzx -= z12 * x12 * f2 * T(0.5);
    e += p2 * T(0.5);
  }
  F[n1] = fx;
  F[n1 + N] = fy;
  F[n1 + 2 * (size_t)N] = fz;
  W[n1] = vxx;
  W[n1 + N] = vyy;
  W[n1 + 2 * (size_t)N] = vzz;
  W[n1 + 3 * (size_t)N] = vxy;
  W[n1 + 4 * (size_t)N] = vyz;
  W[n1 + 5 * (size_t)N] = vzx;
  if (kind == 0) e -= q.qq[type[n1] == 0 ? 0 : 2] * q.self;
  pe[n1] = e;
}

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

template <class T>
PT<T> tersoff_consts(const float* p, int num_types) {
  PT<T> t;
  t.D0[0] = p[0]; t.A[0] = p[1]; t.R0[0] = p[2]; t.S[0] = p[3];
  int off = 0;
  if (num_types == 2) {
    off = 4;
    t.D0[1] = p[4]; t.A[1] = p[5]; t.R0[1] = p[6]; t.S[1] = p[7];
  } else {
    t.D0[1] = t.D0[0]; t.A[1] = t.A[0]; t.R0[1] = t.R0[0]; t.S[1] = t.S[0];
  }
  t.EN = p[4 + off];
  t.BETA = p[5 + off];
  t.H = p[6 + off];
  t.R1 = p[7 + off];
  t.R2 = p[8 + off];
  t.PF = (T)(M_PI / ((double)t.R2 - (double)t.R1));
  t.MHON = (T)(-0.5 / (double)t.EN);
  return t;
}

template <class T>
PR<T> ri_consts(const float* p, int potential_type, bool with_self) {
  PR<T> r;
  const double q0 = p[0], kc = 14.399645, alpha = 0.2, pif = 0.225675833419103;
  const double ratio = ri_charge_ratio(potential_type);
  r.qq[0] = (T)(q0 * q0 * kc);
  r.qq[1] = (T)(ratio * q0 * q0 * kc);
  r.qq[2] = (T)(ratio * ratio * q0 * q0 * kc);
  for (int t = 0; t < 3; ++t) {
    r.a[t] = p[1 + 3 * t];
    r.b[t] = (T)(1.0 / (double)p[2 + 3 * t]);
    r.c[t] = p[3 + 3 * t];
  }
  const double rc = p[10];
  r.cutoff = (T)rc;
  r.d0 = p[11];
  r.alpha = p[12];
  r.r0 = p[13];
  r.s = p[14];
  r.v_rc = (T)(erfc(alpha * rc) / rc);
  r.dv_rc = (T)(-erfc(alpha * rc) / (rc * rc) - pif * exp(-alpha * alpha * rc * rc) / rc);
  r.self = with_self ? (T)ri_self_factor(rc) : T(0);
  return r;
}

template <class T>
struct Scratch {
  T *b, *bp, *fx, *fy, *fz, *F, *W, *pe, *w;
};

template <class T>
int ensure_scratch(Engine* e, Scratch<T>* s);

template <>
int ensure_scratch<double>(Engine* e, Scratch<double>* s) {
  const size_t B = std::max(e->d.B, 1), N = e->d.N;
  if (!e->s64) {
    GPUGA_TRY(e->alloc(&e->s64, 5 * B + (size_t)std::max(e->d.num_vars, 1)));
    GPUGA_TRY(e->alloc(&e->p64_F, 3 * N));
    GPUGA_TRY(e->alloc(&e->p64_W, 6 * N));
    GPUGA_TRY(e->alloc(&e->p64_pe, N));
  }
  *s = {e->s64, e->s64 + B, e->s64 + 2 * B, e->s64 + 3 * B, e->s64 + 4 * B, e->p64_F, e->p64_W, e->p64_pe,
        e->s64 + 5 * B};
  return GPUGA_OK;
}

template <>
int ensure_scratch<float>(Engine* e, Scratch<float>* s) {
  const size_t B = std::max(e->d.B, 1), N = e->d.N;
  if (!e->s32) {
    GPUGA_TRY(e->alloc(&e->s32, 5 * B + (size_t)std::max(e->d.num_vars, 1)));
    GPUGA_TRY(e->alloc(&e->p32_F, 3 * N));
    GPUGA_TRY(e->alloc(&e->p32_W, 6 * N));
    GPUGA_TRY(e->alloc(&e->p32_pe, N));
  }
  *s = {e->s32, e->s32 + B, e->s32 + 2 * B, e->s32 + 3 * B, e->s32 + 4 * B, e->p32_F, e->p32_W, e->p32_pe,
        e->s32 + 5 * B};
  return GPUGA_OK;
}

// Enqueues the force launches of one individual (decoded FP32 parameters).
template <class T>
int enqueue_force(Engine* e, const float* params, const Scratch<T>& s, cudaStream_t st) {
  const DevSet& d = e->d;
  const int N = d.N, grid = (N + 127) / 128;
  if (d.potential_type == 1 || d.potential_type == 2) {
    const PT<T> P = tersoff_consts<T>(params, d.num_types);
    const CsrLayout L{d.off, d.nbr};
    p_tersoff1<T><<<grid, 128, 0, st>>>(N, L, d.g64, P, s.b, s.bp);
    p_tersoff2<T><<<grid, 128, 0, st>>>(N, d.num_types, d.type, L, d.g64, P, s.b, s.bp, s.pe, s.fx, s.fy, s.fz);
    p_tersoff3<T><<<grid, 128, 0, st>>>(N, L, d.rev, d.g64, s.fx, s.fy, s.fz, s.F, s.W);
  } else {
    PR<T> q{};
    PN nn{d.num_neurons, e->spec.nn_r1, e->spec.nn_r2, M_PI / ((double)e->spec.nn_r2 - e->spec.nn_r1),
          e->spec.nn_consistent};
    if (is_ri_type(d.potential_type)) {
      q = ri_consts<T>(params, d.potential_type, e->spec.ri_self != 0);
    } else {
      if (d.num_neurons > 32) {
        set_error("the plain NN2B path supports up to 32 neurons per layer.");
        return GPUGA_ERR_UNSUPPORTED;
      }
      std::vector<T> w(d.num_vars);
      for (int m = 0; m < d.num_vars; ++m) w[m] = params[m];
      GPUGA_CUDA(cudaMemcpyAsync(s.w, w.data(), sizeof(T) * d.num_vars, cudaMemcpyHostToDevice, st));
      GPUGA_CUDA(cudaStreamSynchronize(st));  // w is a stack buffer
    }
    p_pair<T><<<grid, 128, 0, st>>>(N, is_ri_type(d.potential_type) ? 0 : 1, d.type, CsrLayout{d.off, d.nbr}, d.g64, q,
                                    s.w, nn, s.F, s.W, s.pe);
  }
  GPUGA_CUDA(cudaGetLastError());
  return GPUGA_OK;
}

template <class T>
int plain_fitness_t(Engine* e, int P, const float* pop01, double* fitness, double* comps) {
  Scratch<T> s;
  GPUGA_TRY(ensure_scratch<T>(e, &s));
  const DevSet& d = e->d;
  cudaStream_t st = e->stream;
  if (e->p_out_cap < P) {
    if (e->p_out) cudaFree(e->p_out);
    e->p_out = nullptr;
    GPUGA_CUDA(cudaMalloc(&e->p_out, sizeof(double) * (4 * (size_t)P + 3 * (size_t)d.Nc)));
    e->p_out_cap = P;
  }
  double* cfg = e->p_out + 4 * (size_t)P;
  std::vector<float> params(d.num_vars);
  for (int p = 0; p < P; ++p) {
    decode_params(e->spec, pop01 + (size_t)p * d.num_vars, params.data());
    GPUGA_TRY(enqueue_force<T>(e, params.data(), s, st));
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

}  // namespace

int plain_fitness(Engine* e, bool fp64, int P, const float* pop01, double* fitness, double* comps) {
  return fp64 ? plain_fitness_t<double>(e, P, pop01, fitness, comps)
              : plain_fitness_t<float>(e, P, pop01, fitness, comps);
}

int plain_find_force64(Engine* e, const double* params, double* F, double* W, double* pe) {
  Scratch<double> s;
  GPUGA_TRY(ensure_scratch<double>(e, &s));
  // The FP64 path takes FP64 parameters: keep them exact by going through the
  // double constants directly.
  const DevSet& d = e->d;
  cudaStream_t st = e->stream;
  const int N = d.N, grid = (N + 127) / 128;
  if (d.potential_type == 1 || d.potential_type == 2) {
    PT<double> P;
    P.D0[0] = params[0]; P.A[0] = params[1]; P.R0[0] = params[2]; P.S[0] = params[3];
    int off = 0;
    if (d.num_types == 2) {
      off = 4;
      P.D0[1] = params[4]; P.A[1] = params[5]; P.R0[1] = params[6]; P.S[1] = params[7];
    } else {
      P.D0[1] = P.D0[0]; P.A[1] = P.A[0]; P.R0[1] = P.R0[0]; P.S[1] = P.S[0];
    }
    P.EN = params[4 + off];
    P.BETA = params[5 + off];
    P.H = params[6 + off];
    P.R1 = params[7 + off];
    P.R2 = params[8 + off];
    P.PF = M_PI / (P.R2 - P.R1);
    P.MHON = -0.5 / P.EN;
    const CsrLayout L{d.off, d.nbr};
    p_tersoff1<double><<<grid, 128, 0, st>>>(N, L, d.g64, P, s.b, s.bp);
    p_tersoff2<double><<<grid, 128, 0, st>>>(N, d.num_types, d.type, L, d.g64, P, s.b, s.bp, s.pe, s.fx, s.fy,
                                             s.fz);
    p_tersoff3<double><<<grid, 128, 0, st>>>(N, L, d.rev, d.g64, s.fx, s.fy, s.fz, s.F, s.W);
  } else {
    PR<double> q{};
    PN nn{d.num_neurons, e->spec.nn_r1, e->spec.nn_r2, M_PI / ((double)e->spec.nn_r2 - e->spec.nn_r1),
          e->spec.nn_consistent};
    if (is_ri_type(d.potential_type)) {
      const double q0 = params[0], kc = 14.399645, alpha = 0.2, pif = 0.225675833419103;
      const double ratio = ri_charge_ratio(d.potential_type);
      q.qq[0] = q0 * q0 * kc;
      q.qq[1] = ratio * q0 * q0 * kc;
      q.qq[2] = ratio * ratio * q0 * q0 * kc;
      for (int t = 0; t < 3; ++t) {
        q.a[t] = params[1 + 3 * t];
        q.b[t] = 1.0 / params[2 + 3 * t];
        q.c[t] = params[3 + 3 * t];
      }
      q.cutoff = params[10];
      q.d0 = params[11];
      q.alpha = params[12];
      q.r0 = params[13];
      q.s = params[14];
      q.v_rc = erfc(alpha * q.cutoff) / q.cutoff;
      q.dv_rc = -erfc(alpha * q.cutoff) / (q.cutoff * q.cutoff) -
                pif * exp(-alpha * alpha * q.cutoff * q.cutoff) / q.cutoff;
      q.self = e->spec.ri_self ? ri_self_factor(q.cutoff) : 0.0;
    } else {
      if (d.num_neurons > 32) {
        set_error("the plain NN2B path supports up to 32 neurons per layer.");
        return GPUGA_ERR_UNSUPPORTED;
      }
      GPUGA_CUDA(cudaMemcpyAsync(s.w, params, sizeof(double) * d.num_vars, cudaMemcpyHostToDevice, st));
    }
    p_pair<double><<<grid, 128, 0, st>>>(N, is_ri_type(d.potential_type) ? 0 : 1, d.type, CsrLayout{d.off, d.nbr}, d.g64,
                                         q, s.w, nn, s.F, s.W, s.pe);
  }
  GPUGA_CUDA(cudaGetLastError());
  if (F) GPUGA_CUDA(cudaMemcpyAsync(F, s.F, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost, st));
  if (W) GPUGA_CUDA(cudaMemcpyAsync(W, s.W, sizeof(double) * 6 * N, cudaMemcpyDeviceToHost, st));
  if (pe) GPUGA_CUDA(cudaMemcpyAsync(pe, s.pe, sizeof(double) * N, cudaMemcpyDeviceToHost, st));
  GPUGA_CUDA(cudaStreamSynchronize(st));
  return GPUGA_OK;
}

int plain_find_force32(Engine* e, const float* params, float* F, float* W, float* pe) {
  Scratch<float> s;
  GPUGA_TRY(ensure_scratch<float>(e, &s));
  cudaStream_t st = e->stream;
  const int N = e->d.N;
  GPUGA_TRY(enqueue_force<float>(e, params, s, st));
  if (F) GPUGA_CUDA(cudaMemcpyAsync(F, s.F, sizeof(float) * 3 * N, cudaMemcpyDeviceToHost, st));
  if (W) GPUGA_CUDA(cudaMemcpyAsync(W, s.W, sizeof(float) * 6 * N, cudaMemcpyDeviceToHost, st));
  if (pe) GPUGA_CUDA(cudaMemcpyAsync(pe, s.pe, sizeof(float) * N, cudaMemcpyDeviceToHost, st));
  GPUGA_CUDA(cudaStreamSynchronize(st));
  return GPUGA_OK;
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
// layouts: bond geometry from the FP32 image rule, then the three Tersoff steps
// or the pair loop, all enqueued on `st`; nothing is allocated here.
int ref_potential_find_force(int potential_type, int num_neurons, const float* params, const PotentialSpec& nn_opts,
                             int Nc, int N, const int* Na, const int* Na_sum, int max_Na, const int* type,
                             const float* h, const int* NN, const int* NL, const float* r, float* f, float* virial,
                             float* pe, const RefPotentialScratch& s, cudaStream_t st) {
  (void)max_Na;
  GPUGA_TRY(ref_layout_geometry(Nc, N, Na, Na_sum, h, r, NN, NL, s.g64, s.rev, st));
  const size_t slots = (size_t)N * (size_t)max_Na;
  float* b = s.f5;
  float* bp = s.f5 + slots;
  float* fx = s.f5 + 2 * slots;
  float* fy = s.f5 + 3 * slots;
  float* fz = s.f5 + 4 * slots;
  const RefLayout L{N, NN, NL};
  const int grid = (N + 127) / 128;
  if (potential_type == 1 || potential_type == 2) {
    const int num_types = potential_type == 2 ? 2 : 1;
    const PT<float> P = tersoff_consts<float>(params, num_types);
    p_tersoff1<float><<<grid, 128, 0, st>>>(N, L, s.g64, P, b, bp);
    p_tersoff2<float><<<grid, 128, 0, st>>>(N, num_types, type, L, s.g64, P, b, bp, pe, fx, fy, fz);
    p_tersoff3<float><<<grid, 128, 0, st>>>(N, L, s.rev, s.g64, fx, fy, fz, f, virial);
  } else if (is_ri_type(potential_type) || potential_type == 3) {
    PR<float> q{};
    PN nn{num_neurons, nn_opts.nn_r1, nn_opts.nn_r2, M_PI / ((double)nn_opts.nn_r2 - nn_opts.nn_r1),
          nn_opts.nn_consistent};
    if (is_ri_type(potential_type)) {
      q = ri_consts<float>(params, potential_type, nn_opts.ri_self != 0);
    } else {
      if (num_neurons > 32) {
        set_error("the NN2B Potential entry points support up to 32 neurons per layer.");
        return GPUGA_ERR_UNSUPPORTED;
      }
      GPUGA_CUDA(cudaMemcpyAsync(s.w, params, sizeof(float) * num_vars_for(3, num_neurons), cudaMemcpyHostToDevice,
                                 st));
    }
    p_pair<float><<<grid, 128, 0, st>>>(N, is_ri_type(potential_type) ? 0 : 1, type, L, s.g64, q, s.w, nn, f, virial, pe);
  } else {
    set_error("unsupported potential type %d.", potential_type);
    return GPUGA_ERR_UNSUPPORTED;
  }
  GPUGA_CUDA(cudaGetLastError());
  return GPUGA_OK;
}

}  // namespace gpuga
