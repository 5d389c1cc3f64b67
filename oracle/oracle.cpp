// GPUGA fitness-path ORACLE — test infrastructure only.
//
// This file is a plain CPU restatement of the reference algorithm (GPUGA,
// src/*.cu) used as the checker for the CUDA engine in gpuga_b200/.  Only the
// test suite, the smoke check and the CPU-baseline leg of bench.py load it.
// Nothing in the product links it.
//
//   * Parsers of potential.in / train.in follow src/fitness.cu:220-314 and
//     src/fitness.cu:59-182 (fscanf order, validation, FP32 storage).
//   * The box inverse follows src/fitness.cu:40-57 in FP32.
//   * The neighbor list follows src/neighbor.cu:30-66 + src/mic.cuh:20-32 in
//     FP32 with an explicit, selectable FMA contraction pattern, so that the
//     list can be pinned bit-for-bit against the reference build.
//   * Forces/energies/virials are FP64 restatements of
//     src/minimal_tersoff.cu:39-405, src/ri.cu:36-189, src/nn2b.cu:33-173.
//   * The fitness follows src/fitness.cu:316-331 and 392-555 in FP64.
//   * The GA follows src/ga.cu:27-212 with libstdc++'s std::mt19937 and the
//     same distribution objects (the reference's own RNG dependency).
//
// Build: see oracle/Makefile (g++ -O2 -fopenmp -ffp-contract=off).
#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

struct OSet {
  // potential.in
  int potential_type = -1;  // 0 RI, 1/2 Tersoff, 3 NN2B, 4 RI with anion charge -q (extension)
  int ri_self = 0;          // RI: subtract the damped-Coulomb self energy (opt-in extension)
  int num_neurons = 0;
  int num_vars = 0;
  float cutoff = 0.f;
  float w_force = 0.f, w_energy = 0.f, w_stress = 0.f;
  std::vector<float> pmin, pmax;
  // train.in
  int Nc = 0, Nc_force = 0, N = 0, N_force = 0, max_Na = 0;
  std::vector<int> Na, Na_sum, type;
  std::vector<float> r;  // SoA [x(N) y(N) z(N)], fitness.cu:130-148
  std::vector<float> h;  // 18 per config, fitness.cu:115-125
  std::vector<float> pe_ref, virial_ref, force_ref;  // virial_ref[c + Nc*k]
  double fss = 0, pss = 0, vss = 0;  // FP64 normalisers (fitness.cu:86-160)
  // neighbor list (CSR in ascending n2 order) + per-bond image and FP64 geometry
  std::vector<int> NN, off, nl;  // nl: global atom index
  std::vector<double> bx, by, bz, bd;
  // NN2B options (reference defaults: taper 7..8 A, force quirk reproduced)
  double nn_r1 = 7.0, nn_r2 = 8.0;
  int nn_consistent = 0;
  int fma_mode = 0;
  std::string err;
};

bool fail(OSet* s, const char* msg) {
  s->err = msg;
  return false;
}

// ---------------------------------------------------------------- parsers
bool read_potential(OSet* s, const char* dir) {
  std::string path = std::string(dir) + "/potential.in";
  FILE* f = fopen(path.c_str(), "r");
  if (!f) return fail(s, "cannot open potential.in");
  char name[256];
  if (fscanf(f, "%255s%d", name, &s->potential_type) != 2) { fclose(f); return fail(s, "potential.in: type"); }
  switch (s->potential_type) {
    case 0:
    case 4: s->num_vars = 15; break;
    case 1: s->num_vars = 9; break;
    case 2: s->num_vars = 13; break;
    case 3:
      if (fscanf(f, "%255s%d", name, &s->num_neurons) != 2) { fclose(f); return fail(s, "potential.in: neurons"); }
      s->num_vars = s->num_neurons * (s->num_neurons + 4) + 1;
      break;
    default: fclose(f); return fail(s, "unsupported potential type");
  }
  s->pmin.assign(s->num_vars, 0.f);
  s->pmax.assign(s->num_vars, 0.f);
  if (fscanf(f, "%255s%f", name, &s->cutoff) != 2) { fclose(f); return fail(s, "potential.in: cutoff"); }
  if (fscanf(f, "%255s%f", name, &s->w_force) != 2 || s->w_force < 0) { fclose(f); return fail(s, "potential.in: weight_force"); }
  if (fscanf(f, "%255s%f", name, &s->w_energy) != 2 || s->w_energy < 0) { fclose(f); return fail(s, "potential.in: weight_energy"); }
  if (fscanf(f, "%255s%f", name, &s->w_stress) != 2 || s->w_stress < 0) { fclose(f); return fail(s, "potential.in: weight_stress"); }
  for (int n = 0; n < s->num_vars; ++n) {
    if (s->potential_type != 3) {
      if (fscanf(f, "%255s%f%f", name, &s->pmin[n], &s->pmax[n]) != 3) { fclose(f); return fail(s, "potential.in: bounds"); }
    } else {
      s->pmin[n] = -3.0f;
      s->pmax[n] = 3.0f;
    }
  }
  fclose(f);
  return true;
}

// fitness.cu:40-57, FP32 without contraction (x86-64 host code).
void get_inverse(float* h) {
  h[9] = h[4] * h[8] - h[5] * h[7];
  h[10] = h[2] * h[7] - h[1] * h[8];
  h[11] = h[1] * h[5] - h[2] * h[4];
  h[12] = h[5] * h[6] - h[3] * h[8];
  h[13] = h[0] * h[8] - h[2] * h[6];
  h[14] = h[2] * h[3] - h[0] * h[5];
  h[15] = h[3] * h[7] - h[4] * h[6];
  h[16] = h[1] * h[6] - h[0] * h[7];
  h[17] = h[0] * h[4] - h[1] * h[3];
  float volume = h[0] * (h[4] * h[8] - h[5] * h[7]) + h[1] * (h[5] * h[6] - h[3] * h[8]) +
                 h[2] * (h[3] * h[7] - h[4] * h[6]);
  for (int n = 9; n < 18; n++) h[n] /= volume;
}

bool read_train(OSet* s, const char* dir) {
  std::string path = std::string(dir) + "/train.in";
  FILE* f = fopen(path.c_str(), "r");
  if (!f) return fail(s, "cannot open train.in");
  if (fscanf(f, "%d%d", &s->Nc, &s->Nc_force) != 2) { fclose(f); return fail(s, "train.in: Nc"); }
  if (s->Nc < 2) { fclose(f); return fail(s, "Nc < 2"); }
  if (s->Nc_force < 1 || s->Nc_force > s->Nc - 1) { fclose(f); return fail(s, "bad Nc_force"); }
  const int Nc = s->Nc;
  s->Na.assign(Nc, 0);
  s->Na_sum.assign(Nc, 0);
  s->N = 0;
  s->max_Na = 0;
  for (int c = 0; c < Nc; ++c) {
    if (fscanf(f, "%d", &s->Na[c]) != 1) { fclose(f); return fail(s, "train.in: Na"); }
    if (s->Na[c] < 2) { fclose(f); return fail(s, "Na < 2"); }
    s->N += s->Na[c];
    s->max_Na = std::max(s->max_Na, s->Na[c]);
  }
  for (int c = 1; c < Nc; ++c) s->Na_sum[c] = s->Na_sum[c - 1] + s->Na[c - 1];
  s->N_force = 0;
  for (int c = 0; c < s->Nc_force; ++c) s->N_force += s->Na[c];
  const int N = s->N;
  s->type.assign(N, 0);
  s->r.assign(3 * (size_t)N, 0.f);
  s->h.assign(18 * (size_t)Nc, 0.f);
  s->pe_ref.assign(Nc, 0.f);
  s->virial_ref.assign(6 * (size_t)Nc, 0.f);
  s->force_ref.assign(3 * (size_t)N, 0.f);
  float emin = 0.0f;
  for (int c = 0; c < Nc; ++c) {
    if (c >= s->Nc_force) {
      float* v = s->virial_ref.data();
      if (fscanf(f, "%f%f%f%f%f%f%f", &s->pe_ref[c], &v[c], &v[c + Nc], &v[c + 2 * Nc], &v[c + 3 * Nc],
                 &v[c + 4 * Nc], &v[c + 5 * Nc]) != 7) {
        fclose(f);
        return fail(s, "train.in: energy/virial");
      }
      if (s->pe_ref[c] < emin) emin = s->pe_ref[c];
    }
    float t[9];
    for (int k = 0; k < 9; ++k)
      if (fscanf(f, "%f", &t[k]) != 1) { fclose(f); return fail(s, "train.in: box"); }
    float* h = s->h.data() + 18 * (size_t)c;
    h[0] = t[0]; h[3] = t[1]; h[6] = t[2];
    h[1] = t[3]; h[4] = t[4]; h[7] = t[5];
    h[2] = t[6]; h[5] = t[7]; h[8] = t[8];
    get_inverse(h);
    for (int k = 0; k < s->Na[c]; ++k) {
      int i = s->Na_sum[c] + k;
      if (c < s->Nc_force) {
        if (fscanf(f, "%d%f%f%f%f%f%f", &s->type[i], &s->r[i], &s->r[i + N], &s->r[i + 2 * N], &s->force_ref[i],
                   &s->force_ref[i + N], &s->force_ref[i + 2 * N]) != 7) {
          fclose(f);
          return fail(s, "train.in: force atom");
        }
        double fx = s->force_ref[i], fy = s->force_ref[i + N], fz = s->force_ref[i + 2 * N];
        s->fss += fx * fx + fy * fy + fz * fz;
      } else {
        if (fscanf(f, "%d%f%f%f", &s->type[i], &s->r[i], &s->r[i + N], &s->r[i + 2 * N]) != 4) {
          fclose(f);
          return fail(s, "train.in: atom");
        }
      }
    }
  }
  fclose(f);
  for (int c = s->Nc_force; c < Nc; ++c) {
    double e = (double)s->pe_ref[c] - (double)emin;
    s->pss += e * e;
    for (int k = 0; k < 6; ++k) {
      double v = s->virial_ref[c + Nc * k];
      s->vss += v * v;
    }
  }
  return true;
}

// ---------------------------------------------------------------- neighbor list
// Three-term dot product a0*b0 + a1*b1 + a2*b2 in FP32 with a fixed contraction.
//   mode 0: fma(a2,b2, fma(a0,b0, a1*b1))   (multiply-add fused onto the left product)
//   mode 1: fma(a2,b2, fma(a1,b1, a0*b0))   (left-to-right accumulation)
//   mode 2: ((a0*b0 + a1*b1) + a2*b2)        (no contraction)
inline float dot3(int mode, float a0, float b0, float a1, float b1, float a2, float b2) {
  switch (mode) {
    case 0: return std::fmaf(a2, b2, std::fmaf(a0, b0, a1 * b1));
    case 1: return std::fmaf(a2, b2, std::fmaf(a1, b1, a0 * b0));
    default: {
      float t = a0 * b0;
      float u = a1 * b1;
      float v = a2 * b2;
      return (t + u) + v;
    }
  }
}

// mic.cuh:20-32 in FP32; returns the image shift so FP64 geometry can use it.
inline void mic32(int mode, const float* h, float& x, float& y, float& z, float& ix, float& iy, float& iz) {
  float sx = dot3(mode, h[9], x, h[10], y, h[11], z);
  float sy = dot3(mode, h[12], x, h[13], y, h[14], z);
  float sz = dot3(mode, h[15], x, h[16], y, h[17], z);
  ix = std::nearbyint(sx);
  iy = std::nearbyint(sy);
  iz = std::nearbyint(sz);
  sx -= ix;
  sy -= iy;
  sz -= iz;
  x = dot3(mode, h[0], sx, h[1], sy, h[2], sz);
  y = dot3(mode, h[3], sx, h[4], sy, h[5], sz);
  z = dot3(mode, h[6], sx, h[7], sy, h[8], sz);
}

// neighbor.cu:30-66 (+ neighbor.cu:72-74 for rc^2 in FP32), then FP64 bond
// geometry for the image the FP32 rule picked.
void build_neighbors(OSet* s) {
  const int N = s->N;
  const float rc2 = s->cutoff * s->cutoff;
  std::vector<std::vector<int>> lists(N);
  std::vector<std::vector<float>> imgs(N);
#pragma omp parallel for schedule(dynamic, 16)
  for (int c = 0; c < s->Nc; ++c) {
    const float* h = s->h.data() + 18 * (size_t)c;
    const int n_begin = s->Na_sum[c], n_end = n_begin + s->Na[c];
    for (int n1 = n_begin; n1 < n_end; ++n1) {
      float x1 = s->r[n1], y1 = s->r[n1 + N], z1 = s->r[n1 + 2 * N];
      for (int n2 = n_begin; n2 < n_end; ++n2) {
        if (n2 == n1) continue;
        float x12 = s->r[n2] - x1, y12 = s->r[n2 + N] - y1, z12 = s->r[n2 + 2 * N] - z1;
        float ix, iy, iz;
        mic32(s->fma_mode, h, x12, y12, z12, ix, iy, iz);
        float d2 = dot3(s->fma_mode, x12, x12, y12, y12, z12, z12);
        if (d2 < rc2) {
          lists[n1].push_back(n2);
          imgs[n1].push_back(ix);
          imgs[n1].push_back(iy);
          imgs[n1].push_back(iz);
        }
      }
    }
  }
  s->NN.assign(N, 0);
  s->off.assign(N + 1, 0);
  for (int i = 0; i < N; ++i) {
    s->NN[i] = (int)lists[i].size();
    s->off[i + 1] = s->off[i] + s->NN[i];
  }
  const int B = s->off[N];
  s->nl.assign(B, 0);
  s->bx.assign(B, 0);
  s->by.assign(B, 0);
  s->bz.assign(B, 0);
  s->bd.assign(B, 0);
  for (int c = 0; c < s->Nc; ++c) {
    const float* h = s->h.data() + 18 * (size_t)c;
    for (int i = s->Na_sum[c]; i < s->Na_sum[c] + s->Na[c]; ++i) {
      for (int k = 0; k < s->NN[i]; ++k) {
        int b = s->off[i] + k, j = lists[i][k];
        double ix = imgs[i][3 * k], iy = imgs[i][3 * k + 1], iz = imgs[i][3 * k + 2];
        double dx = (double)s->r[j] - (double)s->r[i];
        double dy = (double)s->r[j + N] - (double)s->r[i + N];
        double dz = (double)s->r[j + 2 * N] - (double)s->r[i + 2 * N];
        // r = (x_j - x_i) - H * image, H columns are the cell vectors
        dx -= (double)h[0] * ix + (double)h[1] * iy + (double)h[2] * iz;
        dy -= (double)h[3] * ix + (double)h[4] * iy + (double)h[5] * iz;
        dz -= (double)h[6] * ix + (double)h[7] * iy + (double)h[8] * iz;
        s->nl[b] = j;
        s->bx[b] = dx;
        s->by[b] = dy;
        s->bz[b] = dz;
        s->bd[b] = std::sqrt(dx * dx + dy * dy + dz * dz);
      }
    }
  }
}

// ---------------------------------------------------------------- potentials (FP64)
struct TersoffP {
  double D0[2], A[2], R0[2], S[2], EN, BETA, H, R1, R2, PF, MHON;
};

// minimal_tersoff.cu:39-60 (set 1 only exists for the two-element form; the
// one-element form uses set 0 for every pair, see the parity notes).
TersoffP tersoff_params(const double* p, int num_types) {
  TersoffP t;
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
  t.PF = M_PI / (t.R2 - t.R1);
  t.MHON = -0.5 / t.EN;
  return t;
}

inline void fc_fcp(double r1, double r2, double pf, double d, double& fc, double& fcp) {
  if (d < r1) { fc = 1.0; fcp = 0.0; }
  else if (d < r2) { fc = 0.5 * std::cos(pf * (d - r1)) + 0.5; fcp = -std::sin(pf * (d - r1)) * pf * 0.5; }
  else { fc = 0.0; fcp = 0.0; }
}

void tersoff_force(const OSet* s, const double* p, double* F, double* W, double* pe) {
  const int num_types = s->potential_type == 2 ? 2 : 1;
  const TersoffP t = tersoff_params(p, num_types);
  const int N = s->N;
  const int B = s->off[N];
  std::vector<double> b(B), bp(B), fx(B), fy(B), fz(B);
  // step 1: bond orders, minimal_tersoff.cu:122-188
#pragma omp parallel for schedule(static)
  for (int n1 = 0; n1 < N; ++n1) {
    for (int i1 = s->off[n1]; i1 < s->off[n1 + 1]; ++i1) {
      double d12 = s->bd[i1];
      double zeta = 0.0;
      for (int i2 = s->off[n1]; i2 < s->off[n1 + 1]; ++i2) {
        if (s->nl[i2] == s->nl[i1]) continue;
        double d13 = s->bd[i2];
        double cos123 = (s->bx[i1] * s->bx[i2] + s->by[i1] * s->by[i2] + s->bz[i1] * s->bz[i2]) / (d12 * d13);
        double fc13, fcp13;
        fc_fcp(t.R1, t.R2, t.PF, d13, fc13, fcp13);
        double x = cos123 - t.H;
        zeta += fc13 * t.BETA * x * x;
      }
      double bzn = std::pow(zeta, t.EN);
      double bij = std::pow(1.0 + bzn, t.MHON);
      if (zeta < 1.0e-16) { b[i1] = 1.0; bp[i1] = 0.0; }
      else { b[i1] = bij; bp[i1] = -bij * bzn * 0.5 / ((1.0 + bzn) * zeta); }
    }
  }
  // step 2: partial forces and site energies, minimal_tersoff.cu:191-316
#pragma omp parallel for schedule(static)
  for (int n1 = 0; n1 < N; ++n1) {
    const int type1 = s->type[n1];
    double pot = 0.0;
    for (int i1 = s->off[n1]; i1 < s->off[n1 + 1]; ++i1) {
      const int n2 = s->nl[i1];
      const int set12 = (num_types == 2 && type1 != s->type[n2]) ? 1 : 0;
      const double x12 = s->bx[i1], y12 = s->by[i1], z12 = s->bz[i1], d12 = s->bd[i1];
      const double d12inv = 1.0 / d12;
      double fc12, fcp12;
      fc_fcp(t.R1, t.R2, t.PF, d12, fc12, fcp12);
      const double D0 = t.D0[set12], A = t.A[set12], R0 = t.R0[set12], S = t.S[set12];
      const double fr12 = D0 / (S - 1.0) * std::exp(-std::sqrt(2.0 * S) * A * (d12 - R0));
      const double frp12 = -std::sqrt(2.0 * S) * A * fr12;
      const double fa12 = S * D0 / (S - 1.0) * std::exp(-std::sqrt(2.0 / S) * A * (d12 - R0));
      const double fap12 = -std::sqrt(2.0 / S) * A * fa12;
      const double b12 = b[i1];
      const double factor3 = (fcp12 * (fr12 - b12 * fa12) + fc12 * (frp12 - b12 * fap12)) * d12inv;
      double f12x = x12 * factor3 * 0.5, f12y = y12 * factor3 * 0.5, f12z = z12 * factor3 * 0.5;
      pot += fc12 * (fr12 - b12 * fa12) * 0.5;
      const double bp12 = bp[i1];
      for (int i2 = s->off[n1]; i2 < s->off[n1 + 1]; ++i2) {
        const int n3 = s->nl[i2];
        if (n3 == n2) continue;
        const int set13 = (num_types == 2 && type1 != s->type[n3]) ? 1 : 0;
        const double x13 = s->bx[i2], y13 = s->by[i2], z13 = s->bz[i2], d13 = s->bd[i2];
        double fc13, fcp13;
        fc_fcp(t.R1, t.R2, t.PF, d13, fc13, fcp13);
        const double D0b = t.D0[set13], Ab = t.A[set13], R0b = t.R0[set13], Sb = t.S[set13];
        const double fa13 = Sb * D0b / (Sb - 1.0) * std::exp(-std::sqrt(2.0 / Sb) * Ab * (d13 - R0b));
        const double bp13 = bp[i2];
        const double one_over_d12d13 = 1.0 / (d12 * d13);
        const double cos123 = (x12 * x13 + y12 * y13 + z12 * z13) * one_over_d12d13;
        const double cos123_over_d12d12 = cos123 * d12inv * d12inv;
        const double xx = cos123 - t.H;
        const double g123 = t.BETA * xx * xx, gp123 = t.BETA * 2.0 * xx;
        const double dc = -fc12 * bp12 * fa12 * fc13 * gp123 - fc12 * bp13 * fa13 * fc13 * gp123;
        const double dr = -fcp12 * bp13 * fa13 * g123 * fc13 * d12inv;
        double cos_d = x13 * one_over_d12d13 - x12 * cos123_over_d12d12;
        f12x += (x12 * dr + dc * cos_d) * 0.5;
        cos_d = y13 * one_over_d12d13 - y12 * cos123_over_d12d12;
        f12y += (y12 * dr + dc * cos_d) * 0.5;
        cos_d = z13 * one_over_d12d13 - z12 * cos123_over_d12d12;
        f12z += (z12 * dr + dc * cos_d) * 0.5;
      }
      fx[i1] = f12x;
      fy[i1] = f12y;
      fz[i1] = f12z;
    }
    pe[n1] = pot;
  }
  // step 3: gather F_i = sum_j (f_ij - f_ji) and the per-atom virial, minimal_tersoff.cu:318-405
#pragma omp parallel for schedule(static)
  for (int n1 = 0; n1 < N; ++n1) {
    double sfx = 0, sfy = 0, sfz = 0, vxx = 0, vyy = 0, vzz = 0, vxy = 0, vyz = 0, vzx = 0;
    for (int i1 = s->off[n1]; i1 < s->off[n1 + 1]; ++i1) {
      const int n2 = s->nl[i1];
      const double x12 = s->bx[i1], y12 = s->by[i1], z12 = s->bz[i1];
      int rev = s->off[n2];  // reference falls back to slot 0 when not found (minimal_tersoff.cu:368)
      for (int k = s->off[n2]; k < s->off[n2 + 1]; ++k)
        if (s->nl[k] == n1) { rev = k; break; }
      const double dx = fx[i1] - fx[rev], dy = fy[i1] - fy[rev], dz = fz[i1] - fz[rev];
      sfx += dx; sfy += dy; sfz += dz;
      vxx -= x12 * dx * 0.5;
      vyy -= y12 * dy * 0.5;
      vzz -= z12 * dz * 0.5;
      vxy -= x12 * dy * 0.5;
      vyz -= y12 * dz * 0.5;
      vzx -= z12 * dx * 0.5;
    }
    F[n1] = sfx; F[n1 + N] = sfy; F[n1 + 2 * N] = sfz;
    W[n1] = vxx; W[n1 + N] = vyy; W[n1 + 2 * N] = vzz;
    W[n1 + 3 * N] = vxy; W[n1 + 4 * N] = vyz; W[n1 + 5 * N] = vzx;
  }
}

// ri.cu:26-29 constants, ri.cu:36-74 parameter set-up
struct RIP {
  double a[3], b[3], c[3], qq[3], v_rc, dv_rc, cutoff, d0, alpha, r0, s, self;
};
const double RI_ALPHA = 0.2, RI_ALPHA_SQ = 0.04, RI_PIF = 0.225675833419103, RI_KC = 14.399645;

// Charges: cation +q, anion -q/2 (ri.cu:40-43) for potential_type 0; anion -q for the neutral
// variant 4.  self: the damped-Coulomb self-energy factor of develop/hfo2/find_E.m:10-13 (the
// teacher there multiplies it by 0): E_self = -K_C sum_i q_i^2 self.
RIP ri_params(const double* p, int potential_type, bool with_self) {
  RIP r;
  const double q0 = p[0];
  const double ratio = potential_type == 4 ? -1.0 : -0.5;
  r.qq[0] = q0 * q0 * RI_KC;
  r.qq[1] = ratio * q0 * q0 * RI_KC;
  r.qq[2] = ratio * ratio * q0 * q0 * RI_KC;
  for (int t = 0; t < 3; ++t) {
    r.a[t] = p[1 + 3 * t];
    r.b[t] = 1.0 / p[2 + 3 * t];
    r.c[t] = p[3 + 3 * t];
  }
  r.cutoff = p[10];
  r.d0 = p[11]; r.alpha = p[12]; r.r0 = p[13]; r.s = p[14];
  r.v_rc = std::erfc(RI_ALPHA * r.cutoff) / r.cutoff;
  r.dv_rc = -std::erfc(RI_ALPHA * r.cutoff) / (r.cutoff * r.cutoff);
  r.dv_rc -= RI_PIF * std::exp(-RI_ALPHA_SQ * r.cutoff * r.cutoff) / r.cutoff;
  const double rc = r.cutoff, erfc_rc = std::erfc(RI_ALPHA * rc);
  r.self = with_self ? RI_ALPHA / std::sqrt(M_PI) + 0.5 * erfc_rc / rc +
                           0.5 * (erfc_rc / rc + RI_PIF * std::exp(-RI_ALPHA_SQ * rc * rc))
                     : 0.0;
  return r;
}

// ri.cu:77-110
inline void ri_p2_f2(const RIP& q, int t, double d, double& p2, double& f2) {
  const double dsq = d * d, dinv = 1.0 / d, dinv3 = dinv * dinv * dinv, dinv6 = dinv3 * dinv3, dinv7 = dinv6 * dinv;
  const double ex = std::exp(-d * q.b[t]);
  const double erfc_r = std::erfc(RI_ALPHA * d) * dinv;
  p2 = q.a[t] * ex - q.c[t] * dinv6;
  f2 = 6.0 * q.c[t] * dinv7 - q.a[t] * ex * q.b[t];
  p2 += q.qq[t] * (erfc_r - q.v_rc - q.dv_rc * (d - q.cutoff));
  f2 -= q.qq[t] * (erfc_r * dinv + RI_PIF * dinv * std::exp(-RI_ALPHA_SQ * dsq) + q.dv_rc);
  if (t == 1) {
    const double fr = q.d0 / (q.s - 1.0) * std::exp(-std::sqrt(2.0 * q.s) * q.alpha * (d - q.r0));
    const double frp = -std::sqrt(2.0 * q.s) * q.alpha * fr;
    const double fa = q.s * q.d0 / (q.s - 1.0) * std::exp(-std::sqrt(2.0 / q.s) * q.alpha * (d - q.r0));
    const double fap = -std::sqrt(2.0 / q.s) * q.alpha * fa;
    p2 += fr - fa;
    f2 += frp - fap;
  }
  f2 *= dinv;
}

// nn2b.cu:33-46 unpacking is index arithmetic on p; nn2b.cu:49-92 values
inline void nn_p2_f2(const double* p, int n, double d, double& p2, double& f2) {
  std::vector<double> x1(n), y1(n);
  for (int a = 0; a < n; ++a) {
    x1[a] = std::tanh(p[a] * d - p[a + n]);
    y1[a] = (1.0 - x1[a] * x1[a]) * p[a];
  }
  p2 = 0.0;
  f2 = 0.0;
  for (int a = 0; a < n; ++a) {
    double x2 = 0.0, y2 = 0.0;
    for (int m = 0; m < n; ++m) {
      const double w = p[2 * n + a * n + m];
      x2 += w * x1[m];
      y2 += w * y1[m];
    }
    x2 = std::tanh(x2 - p[n * (n + 2) + a]);
    y2 *= 1.0 - x2 * x2;
    p2 += p[n * (n + 3) + a] * x2;
    f2 += p[n * (n + 3) + a] * y2;
  }
  p2 = p2 - p[n * (n + 4)];
}

// ri.cu:112-189 and nn2b.cu:94-173: owner-computes pair loop over the full list
void pair_force(const OSet* s, const double* p, double* F, double* W, double* pe) {
  const int N = s->N;
  const bool is_ri = s->potential_type == 0 || s->potential_type == 4;
  RIP q;
  if (is_ri) q = ri_params(p, s->potential_type, s->ri_self != 0);
  const int n = s->num_neurons;
  const double pf = M_PI / (s->nn_r2 - s->nn_r1);
#pragma omp parallel for schedule(static)
  for (int n1 = 0; n1 < N; ++n1) {
    double e = 0, fx = 0, fy = 0, fz = 0, vxx = 0, vyy = 0, vzz = 0, vxy = 0, vyz = 0, vzx = 0;
    for (int i1 = s->off[n1]; i1 < s->off[n1 + 1]; ++i1) {
      const int n2 = s->nl[i1];
      const double x12 = s->bx[i1], y12 = s->by[i1], z12 = s->bz[i1], d12 = s->bd[i1];
      double p2, f2;
      if (is_ri) {
        ri_p2_f2(q, s->type[n1] + s->type[n2], d12, p2, f2);
      } else {
        nn_p2_f2(p, n, d12, p2, f2);
        double fc, fcp;
        fc_fcp(s->nn_r1, s->nn_r2, pf, d12, fc, fcp);
        if (s->nn_consistent) {
          f2 = (f2 * fc + p2 * fcp) / d12;
          p2 *= fc;
        } else {  // nn2b.cu:147-148 order: p2 is tapered before it enters f2
          p2 *= fc;
          f2 = (f2 * fc + p2 * fcp) / d12;
        }
      }
      fx += x12 * f2; fy += y12 * f2; fz += z12 * f2;
      vxx -= x12 * x12 * f2 * 0.5;
      vyy -= y12 * y12 * f2 * 0.5;
      vzz -= z12 * z12 * f2 * 0.5;
      vxy -= x12 * y12 * f2 * 0.5;
      vyz -= y12 * z12 * f2 * 0.5;
      vzx -= z12 * x12 * f2 * 0.5;
      e += p2 * 0.5;
    }
    F[n1] = fx; F[n1 + N] = fy; F[n1 + 2 * N] = fz;
    W[n1] = vxx; W[n1 + N] = vyy; W[n1 + 2 * N] = vzz;
    W[n1 + 3 * N] = vxy; W[n1 + 4 * N] = vyz; W[n1 + 5 * N] = vzx;
    if (is_ri) e -= (s->type[n1] == 0 ? q.qq[0] : q.qq[2]) * q.self;
    pe[n1] = e;
  }
}

void find_force(const OSet* s, const double* p, double* F, double* W, double* pe) {
  if (s->potential_type == 1 || s->potential_type == 2) tersoff_force(s, p, F, W, pe);
  else pair_force(s, p, F, W, pe);
}

// fitness.cu:316-325: parameters[m] = min + (max - min) * x in FP32 (no contraction)
void decode(const OSet* s, const float* x, double* p) {
  for (int m = 0; m < s->num_vars; ++m) {
    volatile float a = s->pmin[m];
    volatile float b = s->pmax[m] - a;
    volatile float bx = b * x[m];
    float v = a + bx;
    p[m] = v;
  }
}

// fitness.cu:329-331, 392-555 in FP64.  comps (optional) = {rrmse_E, rrmse_W, rrmse_F}.
double fitness_one(const OSet* s, const double* F, const double* W, const double* pe, double* comps) {
  const int N = s->N, Nc = s->Nc;
  double errE = 0, errW = 0, errF = 0;
  for (int c = s->Nc_force; c < Nc; ++c) {
    double e = 0;
    double w[6] = {0, 0, 0, 0, 0, 0};
    for (int i = s->Na_sum[c]; i < s->Na_sum[c] + s->Na[c]; ++i) {
      e += pe[i];
      for (int k = 0; k < 6; ++k) w[k] += W[i + (size_t)N * k];
    }
    double de = e - (double)s->pe_ref[c];
    errE += de * de;
    for (int k = 0; k < 6; ++k) {
      double dw = w[k] - (double)s->virial_ref[c + Nc * k];
      errW += dw * dw;
    }
  }
  for (int i = 0; i < s->N_force; ++i) {
    double dx = F[i] - s->force_ref[i], dy = F[i + N] - s->force_ref[i + N], dz = F[i + 2 * N] - s->force_ref[i + 2 * N];
    errF += dx * dx + dy * dy + dz * dz;
  }
  const double rE = std::sqrt(errE / s->pss), rW = std::sqrt(errW / s->vss), rF = std::sqrt(errF / s->fss);
  if (comps) { comps[0] = rE; comps[1] = rW; comps[2] = rF; }
  return (double)s->w_energy * rE + (double)s->w_stress * rW + (double)s->w_force * rF;
}

}  // namespace

// ====================================================================== C ABI
extern "C" {

void* oracle_load(const char* dir, int fma_mode, char* errbuf, int errlen) {
  OSet* s = new OSet;
  s->fma_mode = fma_mode;
  if (!read_potential(s, dir) || !read_train(s, dir)) {
    if (errbuf && errlen > 0) snprintf(errbuf, errlen, "%s", s->err.c_str());
    delete s;
    return nullptr;
  }
  build_neighbors(s);
  return s;
}

void oracle_free(void* h) { delete (OSet*)h; }

// info: potential_type, num_vars, num_neurons, Nc, Nc_force, N, N_force, max_Na, num_bonds
void oracle_info(void* h, int* info) {
  OSet* s = (OSet*)h;
  info[0] = s->potential_type; info[1] = s->num_vars; info[2] = s->num_neurons;
  info[3] = s->Nc; info[4] = s->Nc_force; info[5] = s->N; info[6] = s->N_force;
  info[7] = s->max_Na; info[8] = s->off[s->N];
}

// fw: cutoff, w_force, w_energy, w_stress; norms: force, energy, virial (FP64)
void oracle_scalars(void* h, float* fw, double* norms) {
  OSet* s = (OSet*)h;
  fw[0] = s->cutoff; fw[1] = s->w_force; fw[2] = s->w_energy; fw[3] = s->w_stress;
  norms[0] = s->fss; norms[1] = s->pss; norms[2] = s->vss;
}

void oracle_bounds(void* h, float* mn, float* mx) {
  OSet* s = (OSet*)h;
  for (int m = 0; m < s->num_vars; ++m) { mn[m] = s->pmin[m]; mx[m] = s->pmax[m]; }
}

// Parsed arrays: Na, Na_sum, type (N), r (3N), h (18 Nc), pe_ref (Nc), virial_ref (6 Nc), force_ref (3N)
void oracle_arrays(void* hh, int* Na, int* Na_sum, int* type, float* r, float* h, float* pe_ref, float* virial_ref,
                   float* force_ref) {
  OSet* s = (OSet*)hh;
  if (Na) std::copy(s->Na.begin(), s->Na.end(), Na);
  if (Na_sum) std::copy(s->Na_sum.begin(), s->Na_sum.end(), Na_sum);
  if (type) std::copy(s->type.begin(), s->type.end(), type);
  if (r) std::copy(s->r.begin(), s->r.end(), r);
  if (h) std::copy(s->h.begin(), s->h.end(), h);
  if (pe_ref) std::copy(s->pe_ref.begin(), s->pe_ref.end(), pe_ref);
  if (virial_ref) std::copy(s->virial_ref.begin(), s->virial_ref.end(), virial_ref);
  if (force_ref) std::copy(s->force_ref.begin(), s->force_ref.end(), force_ref);
}

// Neighbor list in CSR form: NN[N], nl[num_bonds] (global atom indices, ascending)
void oracle_neighbors(void* h, int* NN, int* nl) {
  OSet* s = (OSet*)h;
  std::copy(s->NN.begin(), s->NN.end(), NN);
  std::copy(s->nl.begin(), s->nl.end(), nl);
}

void oracle_set_ri_self(void* h, int on) { static_cast<OSet*>(h)->ri_self = on; }

void oracle_set_nn2b(void* h, double r1, double r2, int consistent) {
  OSet* s = (OSet*)h;
  s->nn_r1 = r1; s->nn_r2 = r2; s->nn_consistent = consistent;
}

void oracle_decode(void* h, const float* x01, double* params) { decode((OSet*)h, x01, params); }

void oracle_find_force(void* h, const double* params, double* F, double* W, double* pe) {
  find_force((OSet*)h, params, F, W, pe);
}

// Per-config totals from per-atom arrays: E[Nc], Wc[6*Nc] ([c + Nc*k])
void oracle_config_sums(void* h, const double* W, const double* pe, double* E, double* Wc) {
  OSet* s = (OSet*)h;
  for (int c = 0; c < s->Nc; ++c) {
    double e = 0, w[6] = {0, 0, 0, 0, 0, 0};
    for (int i = s->Na_sum[c]; i < s->Na_sum[c] + s->Na[c]; ++i) {
      e += pe[i];
      for (int k = 0; k < 6; ++k) w[k] += W[i + (size_t)s->N * k];
    }
    E[c] = e;
    for (int k = 0; k < 6; ++k) Wc[c + (size_t)s->Nc * k] = w[k];
  }
}

// Batched fitness in FP64: pop01 is [P][num_vars] in [0,1]; comps (optional) [P][3]
void oracle_fitness(void* h, int P, const float* pop01, double* fitness, double* comps) {
  OSet* s = (OSet*)h;
  std::vector<double> F(3 * (size_t)s->N), W(6 * (size_t)s->N), pe(s->N), p(s->num_vars);
  for (int n = 0; n < P; ++n) {
    decode(s, pop01 + (size_t)n * s->num_vars, p.data());
    find_force(s, p.data(), F.data(), W.data(), pe.data());
    fitness[n] = fitness_one(s, F.data(), W.data(), pe.data(), comps ? comps + 3 * (size_t)n : nullptr);
  }
}

// Fitness of already-computed per-atom arrays.
double oracle_fitness_arrays(void* h, const double* F, const double* W, const double* pe, double* comps) {
  return fitness_one((OSet*)h, F, W, pe, comps);
}

int oracle_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

// FP32 MIC of mic.cuh:20-32 plus the squared distance of neighbor.cu:59 for n
// inputs: h[18n], in[3n] -> out[4n] = (x, y, z, d^2), with contraction `mode`.
void oracle_mic_batch(int mode, int n, const float* h, const float* in, float* out) {
  for (int k = 0; k < n; ++k) {
    float x = in[3 * k], y = in[3 * k + 1], z = in[3 * k + 2], ix, iy, iz;
    mic32(mode, h + 18 * (size_t)k, x, y, z, ix, iy, iz);
    out[4 * k] = x;
    out[4 * k + 1] = y;
    out[4 * k + 2] = z;
    out[4 * k + 3] = dot3(mode, x, x, y, y, z, z);
  }
}

// ---------------------------------------------------------------- GA (ga.cu:27-212)
// Runs `generations` generations of the reference GA with a fixed seed and a
// fitness supplied by the caller through a callback; writes ga.out-style lines
// into `out` (caller-owned, out_len bytes).  fitness_cb(P, pop, fitness, user).
typedef void (*oracle_fitness_cb)(int, const float*, float*, void*);

int oracle_ga_run(int num_vars, const float* pmin, const float* pmax, int population_size, int parent_number,
                  float mutation_rate, int maximum_generation, int generations_to_run, unsigned seed,
                  oracle_fitness_cb cb, void* user, char* out, int out_len, float* final_population) {
  const int P = population_size, d = num_vars;
  const int child_number = P - parent_number;
  std::vector<float> fitness(P), cum(parent_number), pop((size_t)P * d), popc((size_t)P * d);
  std::vector<int> index(P);
  float numerator = 0.0;
  float denominator = (1.0 + parent_number) * parent_number / 2.0;
  for (int n = 0; n < parent_number; ++n) {
    numerator += parent_number - n;
    cum[n] = numerator / denominator;
  }
  std::mt19937 rng(seed);
  {
    std::uniform_real_distribution<float> r1(0, 1);
    for (int n = 0; n < P * d; ++n) pop[n] = r1(rng);
  }
  auto get_a_parent = [&]() {
    int parent = 0;
    std::uniform_real_distribution<float> r1(0, 1);
    float ref = r1(rng);
    for (int n = 0; n < parent_number; ++n)
      if (cum[n] > ref) { parent = n; break; }
    return parent;
  };
  std::string text;
  char buf[64];
  for (int g = 0; g < generations_to_run; ++g) {
    cb(P, pop.data(), fitness.data(), user);
    // ga.cu:105-137 stable insertion sort + permutation
    for (int n = 0; n < P; ++n) index[n] = n;
    for (int i = 1; i < P; i++) {
      float key = fitness[i];
      int j = i - 1;
      while (j >= 0 && fitness[j] > key) {
        fitness[j + 1] = fitness[j];
        index[j + 1] = index[j];
        --j;
      }
      fitness[j + 1] = key;
      index[j + 1] = i;
    }
    popc = pop;
    for (int n = 0; n < P; ++n)
      for (int m = 0; m < d; ++m) pop[(size_t)n * d + m] = popc[(size_t)index[n] * d + m];
    // ga.cu:138-147 output line
    snprintf(buf, sizeof buf, "%d %g ", g, fitness[0]);
    text += buf;
    for (int m = 0; m < d; ++m) {
      volatile float a = pmin[m];
      volatile float b = pmax[m] - a;
      volatile float bx = b * pop[m];
      float v = a + bx;
      snprintf(buf, sizeof buf, "%g ", v);
      text += buf;
    }
    text += "\n";
    // ga.cu:161-186 crossover
    for (int m = 0; m < child_number; m += 2) {
      int p1 = get_a_parent();
      int p2 = get_a_parent();
      while (p2 == p1) p2 = get_a_parent();
      std::uniform_int_distribution<int> r1(1, d - 1);
      int cp = r1(rng);
      int c1 = parent_number + m, c2 = c1 + 1;
      for (int n = 0; n < cp; ++n) {
        pop[(size_t)c1 * d + n] = pop[(size_t)p1 * d + n];
        pop[(size_t)c2 * d + n] = pop[(size_t)p2 * d + n];
      }
      for (int n = cp; n < d; ++n) {
        pop[(size_t)c1 * d + n] = pop[(size_t)p2 * d + n];
        pop[(size_t)c2 * d + n] = pop[(size_t)p1 * d + n];
      }
    }
    // ga.cu:188-198 mutation; the index is drawn before the value (C++14 order)
    float rate_n = mutation_rate * (1.0 - float(g) / maximum_generation);
    int mm = P * d;
    int num_mut = (int)std::round(mm * rate_n);
    for (int n = 0; n < num_mut; ++n) {
      std::uniform_int_distribution<int> r1(d, mm - 1);
      std::uniform_real_distribution<float> r2(0, 1);
      int idx = r1(rng);
      float val = r2(rng);
      pop[idx] = val;
    }
  }
  if (final_population) std::copy(pop.begin(), pop.end(), final_population);
  if ((int)text.size() + 1 > out_len) return -(int)text.size() - 1;
  memcpy(out, text.c_str(), text.size() + 1);
  return (int)text.size();
}

}  // extern "C"
