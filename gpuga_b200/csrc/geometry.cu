// Neighbor list and parameter-independent geometry.
//
// The list is built with the reference's FP32 rule (neighbor.cu:30-66,
// mic.cuh:20-32): same-config atoms, ascending n2, strict d^2 < rc^2 in FP32,
// nearest image by round-half-even of the fractional coordinates.  Every FP32
// operation is an explicit round-to-nearest intrinsic so the compiler cannot
// fuse differently from the pinned pattern (kMicMode).
//
// From the list the engine derives, once per training set, everything that
// does not depend on the potential parameters: FP64 bond vectors for the
// image the FP32 rule picked, unit vectors and distances in FP32, reverse-bond
// indices (and their positions in the batched force scratch) and the
// fixed-damping Coulomb terms of the RI potential.
#include <algorithm>
#include <cmath>
#include <numeric>
#include <vector>

#include "engine.hpp"

namespace gpuga {

// Contraction pattern of the three-term dot products in the FP32 MIC and the
// squared distance; pinned against the reference build.
//   0: fma(a2,b2, fma(a0,b0, a1*b1))   1: fma(a2,b2, fma(a1,b1, a0*b0))   2: no fusion
#ifndef GPUGA_MIC_MODE
#define GPUGA_MIC_MODE 0
#endif
constexpr int kMicMode = GPUGA_MIC_MODE;

template <int MODE>
__device__ __forceinline__ float dot3(float a0, float b0, float a1, float b1, float a2, float b2) {
  if (MODE == 0) return __fmaf_rn(a2, b2, __fmaf_rn(a0, b0, __fmul_rn(a1, b1)));
  if (MODE == 1) return __fmaf_rn(a2, b2, __fmaf_rn(a1, b1, __fmul_rn(a0, b0)));
  return __fadd_rn(__fadd_rn(__fmul_rn(a0, b0), __fmul_rn(a1, b1)), __fmul_rn(a2, b2));
}

// mic.cuh:20-32; also returns the image shift that was removed.
template <int MODE>
__device__ __forceinline__ void mic32(const float* h, float& x, float& y, float& z, float& ix, float& iy,
                                      float& iz) {
  float sx = dot3<MODE>(h[9], x, h[10], y, h[11], z);
  float sy = dot3<MODE>(h[12], x, h[13], y, h[14], z);
  float sz = dot3<MODE>(h[15], x, h[16], y, h[17], z);
  ix = rintf(sx);
  iy = rintf(sy);
  iz = rintf(sz);
  sx = __fsub_rn(sx, ix);
  sy = __fsub_rn(sy, iy);
  sz = __fsub_rn(sz, iz);
  x = dot3<MODE>(h[0], sx, h[1], sy, h[2], sz);
  y = dot3<MODE>(h[3], sx, h[4], sy, h[5], sz);
  z = dot3<MODE>(h[6], sx, h[7], sy, h[8], sz);
}

// The reference's pair test (neighbor.cu:51-60): FP32 difference, nearest
// image, strict d^2 < rc^2.  Returns the image shift removed.
template <int MODE>
__device__ __forceinline__ bool pair_within(const float* hh, float rc2, const float* __restrict__ r, int N,
                                            float x1, float y1, float z1, int n2, float& ix, float& iy, float& iz) {
  float x12 = __fsub_rn(r[n2], x1);
  float y12 = __fsub_rn(r[n2 + N], y1);
  float z12 = __fsub_rn(r[n2 + 2 * (size_t)N], z1);
  mic32<MODE>(hh, x12, y12, z12, ix, iy, iz);
  return dot3<MODE>(x12, x12, y12, y12, z12, z12) < rc2;
}

// One CTA per configuration, atoms strided over the threads.  Pass 0 counts,
// pass 1 writes the CSR list and the image shifts.  Configurations listed in
// `skip` (cell-list configurations) are left to neighbor_cells.
template <int MODE, bool FILL>
__global__ void neighbor_scan(int N, const int* __restrict__ Na, const int* __restrict__ Na_sum,
                              float rc2, const float* __restrict__ box, const float* __restrict__ r,
                              int* __restrict__ NN, const int* __restrict__ off, int* __restrict__ nbr,
                              float* __restrict__ img, const uint8_t* __restrict__ skip) {
  const int c = blockIdx.x;
  if (skip && skip[c]) return;
  const int n_begin = Na_sum[c], n_end = n_begin + Na[c];
  const float* h = box + 18 * (size_t)c;
  float hh[18];
#pragma unroll
  for (int k = 0; k < 18; ++k) hh[k] = h[k];
  for (int n1 = n_begin + threadIdx.x; n1 < n_end; n1 += blockDim.x) {
    const float x1 = r[n1], y1 = r[n1 + N], z1 = r[n1 + 2 * (size_t)N];
    int count = 0;
    int base = FILL ? off[n1] : 0;
    for (int n2 = n_begin; n2 < n_end; ++n2) {
      if (n2 == n1) continue;
      float ix, iy, iz;
      if (pair_within<MODE>(hh, rc2, r, N, x1, y1, z1, n2, ix, iy, iz)) {
        if (FILL) {
          nbr[base + count] = n2;
          img[3 * (size_t)(base + count) + 0] = ix;
          img[3 * (size_t)(base + count) + 1] = iy;
          img[3 * (size_t)(base + count) + 2] = iz;
        }
        ++count;
      }
    }
    if (!FILL) NN[n1] = count;
  }
}

// Cell-list build for large configurations: one thread per atom visits the 27
// cells around its own (cell widths >= rc, >= 3 cells per direction, so every
// pair within rc is visited exactly once), applies the same FP32 pair test and,
// in the fill pass, sorts its neighbors ascending -- the list is then the
// reference's, bit for bit, in O(N) instead of O(Na^2) per configuration.
//   atoms[k]: atoms handled here; acell[k] = (cell x, y, z, grid row) of atoms[k];
//   grid[g] = (nx, ny, nz, first cell); cell_atoms[cell_start[cell] .. cell_start[cell + 1]).
template <int MODE, bool FILL>
__global__ void neighbor_cells(int N, int n_atoms, const int* __restrict__ atoms, const int4* __restrict__ acell,
                               const int4* __restrict__ grid, const int* __restrict__ grid_cfg,
                               const int* __restrict__ cell_start, const int* __restrict__ cell_atoms, float rc2,
                               const float* __restrict__ box, const float* __restrict__ r, int* __restrict__ NN,
                               const int* __restrict__ off, int* __restrict__ nbr, float* __restrict__ img) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n_atoms) return;
  const int n1 = atoms[k];
  const int4 ac = acell[k];
  const int4 gd = grid[ac.w];
  const float* h = box + 18 * (size_t)grid_cfg[ac.w];
  float hh[18];
#pragma unroll
  for (int q = 0; q < 18; ++q) hh[q] = h[q];
  const float x1 = r[n1], y1 = r[n1 + N], z1 = r[n1 + 2 * (size_t)N];
  int count = 0;
  const int base = FILL ? off[n1] : 0;
  for (int dz = -1; dz <= 1; ++dz)
    for (int dy = -1; dy <= 1; ++dy)
      for (int dx = -1; dx <= 1; ++dx) {
        const int cx = (ac.x + dx + gd.x) % gd.x, cy = (ac.y + dy + gd.y) % gd.y, cz = (ac.z + dz + gd.z) % gd.z;
        const int cell = gd.w + (cz * gd.y + cy) * gd.x + cx;
        for (int q = cell_start[cell]; q < cell_start[cell + 1]; ++q) {
          const int n2 = cell_atoms[q];
          if (n2 == n1) continue;
          float ix, iy, iz;
          if (pair_within<MODE>(hh, rc2, r, N, x1, y1, z1, n2, ix, iy, iz)) {
            if (FILL) {
              nbr[base + count] = n2;
              img[3 * (size_t)(base + count) + 0] = ix;
              img[3 * (size_t)(base + count) + 1] = iy;
              img[3 * (size_t)(base + count) + 2] = iz;
            }
            ++count;
          }
        }
      }
  if constexpr (!FILL) {
    NN[n1] = count;
  } else {
    // ascending neighbor index, as the reference's n2 loop produces them (insertion sort)
    for (int a = base + 1; a < base + count; ++a) {
      const int key = nbr[a];
      const float kx = img[3 * (size_t)a], ky = img[3 * (size_t)a + 1], kz = img[3 * (size_t)a + 2];
      int b = a - 1;
      while (b >= base && nbr[b] > key) {
        nbr[b + 1] = nbr[b];
        img[3 * (size_t)(b + 1) + 0] = img[3 * (size_t)b + 0];
        img[3 * (size_t)(b + 1) + 1] = img[3 * (size_t)b + 1];
        img[3 * (size_t)(b + 1) + 2] = img[3 * (size_t)b + 2];
        --b;
      }
      nbr[b + 1] = key;
      img[3 * (size_t)(b + 1) + 0] = kx;
      img[3 * (size_t)(b + 1) + 1] = ky;
      img[3 * (size_t)(b + 1) + 2] = kz;
    }
  }
}

// Reference layout NL[k*N + n1] (neighbor.cu:61) for the drop-in entry point.
template <int MODE>
__global__ void neighbor_reference(int N, const int* __restrict__ Na, const int* __restrict__ Na_sum, float rc2,
                                   const float* __restrict__ box, const float* __restrict__ r, int* __restrict__ NN,
                                   int* __restrict__ NL) {
  const int c = blockIdx.x;
  const int n_begin = Na_sum[c], n_end = n_begin + Na[c];
  const float* h = box + 18 * (size_t)c;
  float hh[18];
#pragma unroll
  for (int k = 0; k < 18; ++k) hh[k] = h[k];
  for (int n1 = n_begin + threadIdx.x; n1 < n_end; n1 += blockDim.x) {
    const float x1 = r[n1], y1 = r[n1 + N], z1 = r[n1 + 2 * (size_t)N];
    int count = 0;
    for (int n2 = n_begin; n2 < n_end; ++n2) {
      if (n2 == n1) continue;
      float ix, iy, iz;
      if (pair_within<MODE>(hh, rc2, r, N, x1, y1, z1, n2, ix, iy, iz)) NL[(size_t)count++ * N + n1] = n2;
    }
    NN[n1] = count;
  }
}

constexpr int kCellMinAtoms = 2048;  // automatic cell lists from this configuration size on

constexpr double kRiAlpha = 0.2;                  // ri.cu:26
constexpr double kRiPiFactor = 0.225675833419103;  // ri.cu:28, 2*alpha/sqrt(pi)

// Per atom: FP64 bond vectors for the FP32-chosen image, FP32 unit vectors,
// reverse bonds, half-list start and pair types; where asked for (dl, d64 not null)
// also the FP64 remainder d - (float)d of each bond length and the FP64 length itself.
__global__ void bond_geometry(int N, const int* __restrict__ atom_cfg, const float* __restrict__ box,
                              const float* __restrict__ r, const int* __restrict__ type, const int* __restrict__ off,
                              const int* __restrict__ nbr, const float* __restrict__ img, int potential_type,
                              int num_types, double4* __restrict__ g64, float4* __restrict__ g32,
                              float* __restrict__ dl, double* __restrict__ d64, int* __restrict__ rev,
                              int* __restrict__ half_off,
                              uint8_t* __restrict__ ptype) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const float* h = box + 18 * (size_t)atom_cfg[i];
  const double xi = r[i], yi = r[i + N], zi = r[i + 2 * (size_t)N];
  int hstart = off[i + 1];
  for (int b = off[i]; b < off[i + 1]; ++b) {
    const int j = nbr[b];
    const double ix = img[3 * (size_t)b], iy = img[3 * (size_t)b + 1], iz = img[3 * (size_t)b + 2];
    double dx = (double)r[j] - xi, dy = (double)r[j + N] - yi, dz = (double)r[j + 2 * (size_t)N] - zi;
    dx -= (double)h[0] * ix + (double)h[1] * iy + (double)h[2] * iz;
    dy -= (double)h[3] * ix + (double)h[4] * iy + (double)h[5] * iz;
    dz -= (double)h[6] * ix + (double)h[7] * iy + (double)h[8] * iz;
    const double d = sqrt(dx * dx + dy * dy + dz * dz);
    g64[b] = make_double4(dx, dy, dz, d);
    g32[b] = make_float4((float)(dx / d), (float)(dy / d), (float)(dz / d), (float)d);
    if (dl) dl[b] = (float)(d - (double)(float)d);
    if (d64) d64[b] = d;
  int rb = off[j];  // minimal_tersoff.cu:368: slot 0 when the reverse is absent
    for (int k = off[j]; k < off[j + 1]; ++k)
      if (nbr[k] == i) {
        rb = k;
        break;
      }
    rev[b] = rb;
    if (j > i && hstart == off[i + 1]) hstart = b;
    uint8_t t = 0;
    if (potential_type == 0) t = (uint8_t)(type[i] + type[j]);
    else if (num_types == 2) t = (uint8_t)(type[i] != type[j]);
    ptype[b] = t;
  }
  half_off[i] = hstart;
}

// NN2B: the slot each bond's pair derivative is read from in a force item's scratch, local to
// the configuration's first bond: the bond itself when its neighbor has a larger index, else its
// reverse (the unordered pair is evaluated from its lower atom).
__global__ void pair_slots(int N, const int* __restrict__ atom_cfg, const int* __restrict__ Na_sum,
                           const int* __restrict__ off, const int* __restrict__ nbr, const int* __restrict__ rev,
                           int* __restrict__ pslot) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const int bond0 = off[Na_sum[atom_cfg[i]]];
  for (int b = off[i]; b < off[i + 1]; ++b) pslot[b] = (nbr[b] > i ? b : rev[b]) - bond0;
}

// Position of each bond's reverse in the batched force kernel's slot-major
// scratch of its configuration: slot * Na + atom, both local to the configuration.
__global__ void reverse_slots(int N, const int* __restrict__ atom_cfg, const int* __restrict__ Na,
                              const int* __restrict__ Na_sum, const int* __restrict__ off,
                              const int* __restrict__ nbr, const int* __restrict__ rev, int* __restrict__ rev_sm) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const int c = atom_cfg[i], atom0 = Na_sum[c], na = Na[c];
  for (int b = off[i]; b < off[i + 1]; ++b) {
    const int j = nbr[b];
    rev_sm[b] = (rev[b] - off[j]) * na + (j - atom0);
  }
}

// RI: each atom's pairs that are evaluated pair by pair (full list for force
// configurations, i < N_force; half list otherwise; pair types in the `active` mask
// only) copied grouped by pair type, list order kept within a type.
__global__ void ri_group(int N, int N_force, int active, const int* __restrict__ off, const int* __restrict__ half_off,
                         const uint8_t* __restrict__ ptype, const float4* __restrict__ g32,
                         const float* __restrict__ dl, const int* __restrict__ start, float4* __restrict__ rg32,
                         float* __restrict__ rdl, int4* __restrict__ rseg) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const int bb = i < N_force ? off[i] : half_off[i], be = off[i + 1];
  int o = start[i];
  int seg[3];
  for (int t = 0; t < 3; ++t) {
    seg[t] = o;
    if (!((active >> t) & 1)) continue;
    for (int b = bb; b < be; ++b) {
      if (ptype[b] != t) continue;
      rg32[o] = g32[b];
      rdl[o] = dl[b];
      ++o;
    }
  }
  rseg[i] = make_int4(seg[0], seg[1], seg[2], o);
}

// RI terms that are linear in the per-individual constants (ri.cu:77-110): for pair type t
//   U_lin(d) = qq_t [ec(d) - v_rc - dv_rc (d - rc)] - C_t / d^6,
//   dU_lin/dd = -qq_t [gc(d) + dv_rc] + 6 C_t / d^7,
//   ec = erfc(alpha d) / d,  gc = erfc(alpha d) / d^2 + (2 alpha / sqrt(pi)) e^{-alpha^2 d^2} / d.
// Their geometric sums, in FP64, one thread per atom:
//   force atom i (full list), out_atom[i][t*9 + 3m + a]: m = 0 sum gc u_a, 1 sum u_a, 2 sum u_a / d^7
//     (F_i = sum_j dU/dd u_ij);
//   energy/virial atom i (half list, j > i), out_ev[i][t*22 + ...]: [0..3] sum ec, count, sum d,
//     sum 1/d^6; [4 + 6m + k] with m = 0 sum d gc uu, 1 sum d uu, 2 sum uu / d^6, k = xx, yy, zz,
//     xy, yz, zx (W = -sum_pairs d dU/dd u (x) u).
__global__ void ri_linear_atoms(int N, int N_force, const int* __restrict__ off, const int* __restrict__ half_off,
                                const uint8_t* __restrict__ ptype, const double4* __restrict__ g64,
                                double* __restrict__ out_atom, double* __restrict__ out_ev) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const bool force = i < N_force;
  double acc[kRiCfgLin];
  for (int k = 0; k < kRiCfgLin; ++k) acc[k] = 0.0;
  for (int b = force ? off[i] : half_off[i]; b < off[i + 1]; ++b) {
    const double4 q = g64[b];
    const double d = q.w, id = 1.0 / d, id2 = id * id, id6 = id2 * id2 * id2;
    const double u[3] = {q.x * id, q.y * id, q.z * id};
    const double ec = erfc(kRiAlpha * d) * id;
    const double gc = ec * id + kRiPiFactor * exp(-kRiAlpha * kRiAlpha * d * d) * id;
    const int t = ptype[b];
    if (force) {
      double* a = acc + 9 * t;
      for (int c = 0; c < 3; ++c) {
        a[c] += gc * u[c];
        a[3 + c] += u[c];
        a[6 + c] += id6 * id * u[c];
      }
    } else {
      double* a = acc + 22 * t;
      a[0] += ec;
      a[1] += 1.0;
      a[2] += d;
      a[3] += id6;
      const double uu[6] = {u[0] * u[0], u[1] * u[1], u[2] * u[2], u[0] * u[1], u[1] * u[2], u[2] * u[0]};
      for (int k = 0; k < 6; ++k) {
        a[4 + k] += d * gc * uu[k];
        a[10 + k] += d * uu[k];
        a[16 + k] += id6 * uu[k];
      }
    }
  }
  if (force) {
    for (int k = 0; k < kRiAtomLin; ++k) out_atom[(size_t)i * kRiAtomLin + k] = acc[k];
  } else {
    for (int k = 0; k < kRiCfgLin; ++k) out_ev[(size_t)i * kRiCfgLin + k] = acc[k];
  }
}

// Per energy/virial configuration c >= Nc_force: the atoms' sums in atom order (thread k = sum k).
__global__ void ri_linear_configs(int Nc, int Nc_force, const int* __restrict__ Na, const int* __restrict__ Na_sum,
                                  const double* __restrict__ ev, double* __restrict__ out_cfg) {
  const int c = Nc_force + blockIdx.x, k = threadIdx.x;
  if (c >= Nc || k >= kRiCfgLin) return;
  double s = 0.0;
  for (int i = Na_sum[c]; i < Na_sum[c] + Na[c]; ++i) s += ev[(size_t)i * kRiCfgLin + k];
  out_cfg[(size_t)c * kRiCfgLin + k] = s;
}

// Bond geometry for lists in the reference layout NL[k*N + i]: the FP32 rule
// picks the image, the vector is then evaluated in FP64; rev holds the slot of
// the reverse bond (slot 0 of the neighbor when absent, minimal_tersoff.cu:368).
template <int MODE>
__global__ void ref_layout_bonds(int N, const int* __restrict__ Na, const int* __restrict__ Na_sum,
                                 const float* __restrict__ box, const float* __restrict__ r,
                                 const int* __restrict__ NN, const int* __restrict__ NL, double4* __restrict__ g64,
                                 int* __restrict__ rev) {
  const int c = blockIdx.x;
  const int n_begin = Na_sum[c], n_end = n_begin + Na[c];
  const float* h = box + 18 * (size_t)c;
  float hh[18];
#pragma unroll
  for (int k = 0; k < 18; ++k) hh[k] = h[k];
  for (int i = n_begin + threadIdx.x; i < n_end; i += blockDim.x) {
    const float x1 = r[i], y1 = r[i + N], z1 = r[i + 2 * (size_t)N];
    for (int k = 0; k < NN[i]; ++k) {
      const size_t slot = (size_t)k * N + i;
      const int j = NL[slot];
      float x12 = __fsub_rn(r[j], x1), y12 = __fsub_rn(r[j + N], y1), z12 = __fsub_rn(r[j + 2 * (size_t)N], z1);
      float ix, iy, iz;
      mic32<MODE>(hh, x12, y12, z12, ix, iy, iz);
      double dx = (double)r[j] - (double)x1, dy = (double)r[j + N] - (double)y1,
             dz = (double)r[j + 2 * (size_t)N] - (double)z1;
      dx -= (double)hh[0] * ix + (double)hh[1] * iy + (double)hh[2] * iz;
      dy -= (double)hh[3] * ix + (double)hh[4] * iy + (double)hh[5] * iz;
      dz -= (double)hh[6] * ix + (double)hh[7] * iy + (double)hh[8] * iz;
      g64[slot] = make_double4(dx, dy, dz, sqrt(dx * dx + dy * dy + dz * dz));
      int rs = j;
      for (int kk = 0; kk < NN[j]; ++kk)
        if (NL[(size_t)kk * N + j] == i) {
          rs = kk * N + j;
          break;
        }
      rev[slot] = rs;
    }
  }
}

int ref_layout_geometry(int Nc, int N, const int* Na, const int* Na_sum, const float* h, const float* r,
                        const int* NN, const int* NL, double4* g64, int* rev, cudaStream_t st) {
  ref_layout_bonds<kMicMode><<<Nc, 128, 0, st>>>(N, Na, Na_sum, h, r, NN, NL, g64, rev);
  GPUGA_CUDA(cudaGetLastError());
  return GPUGA_OK;
}

int neighbor_reference_layout(int Nc, int N, int max_Na, const int* Na, const int* Na_sum, const float* r,
                              const float* h, float cutoff, int* NN, int* NL, cudaStream_t st) {
  (void)max_Na;
  const float rc2 = cutoff * cutoff;  // neighbor.cu:73 (FP32 on the host)
  neighbor_reference<kMicMode><<<Nc, 256, 0, st>>>(N, Na, Na_sum, rc2, h, r, NN, NL);
  GPUGA_CUDA(cudaGetLastError());
  return GPUGA_OK;
}

// Cell lists of the configurations that take the O(N) path: every cell at least
// rc (with a 1e-4 margin for the FP32 test) wide along each cell vector's
// normal and at least 3 cells per direction, so that the 27 cells around an
// atom hold every atom within rc exactly once under the nearest-image rule.
struct CellLists {
  std::vector<uint8_t> skip;        // per configuration: 1 = cell path
  std::vector<int> atoms;           // atoms of cell-path configurations
  std::vector<int4> acell;          // per listed atom: cell x, y, z and grid row
  std::vector<int4> grid;           // per cell-path configuration: nx, ny, nz, first cell
  std::vector<int> grid_cfg;        // configuration of each grid row
  std::vector<int> cell_start;      // [cells + 1]
  std::vector<int> cell_atoms;      // atoms by cell, ascending within a cell
};

void build_cell_lists(const Engine* e, CellLists* cl) {
  const TrainingSet& ts = e->ts;
  const int mode = e->opt.neighbor_cells;  // 0 auto, 1 wherever the grid allows, 2 never
  const double rc = e->spec.cutoff * (1.0 + 1e-4);
  cl->skip.assign(ts.Nc, 0);
  cl->cell_start.assign(1, 0);
  if (mode == 2) return;
  for (int c = 0; c < ts.Nc; ++c) {
    const int Na = ts.Na[c];
    if (mode == 0 && Na < kCellMinAtoms) continue;
    const float* h = &ts.h[18 * (size_t)c];
    // cell vectors are the columns of h; width along a = V / |b x c|, etc.
    const double a[3] = {h[0], h[3], h[6]}, b[3] = {h[1], h[4], h[7]}, cc[3] = {h[2], h[5], h[8]};
    auto cross = [](const double* u, const double* v, double* w) {
      w[0] = u[1] * v[2] - u[2] * v[1];
      w[1] = u[2] * v[0] - u[0] * v[2];
      w[2] = u[0] * v[1] - u[1] * v[0];
    };
    double bc[3], ca[3], ab[3];
    cross(b, cc, bc);
    cross(cc, a, ca);
    cross(a, b, ab);
    const double vol = std::fabs(a[0] * bc[0] + a[1] * bc[1] + a[2] * bc[2]);
    const double wa = vol / std::sqrt(bc[0] * bc[0] + bc[1] * bc[1] + bc[2] * bc[2]);
    const double wb = vol / std::sqrt(ca[0] * ca[0] + ca[1] * ca[1] + ca[2] * ca[2]);
    const double wc = vol / std::sqrt(ab[0] * ab[0] + ab[1] * ab[1] + ab[2] * ab[2]);
    const int nx = (int)std::floor(wa / rc), ny = (int)std::floor(wb / rc), nz = (int)std::floor(wc / rc);
    if (!(vol > 0) || nx < 3 || ny < 3 || nz < 3) continue;
    if ((long long)nx * ny * nz > 4LL * Na + 64) continue;  // sparse grid: the scan is as cheap
    cl->skip[c] = 1;
    const int g = (int)cl->grid.size();
    const int first = (int)cl->cell_start.size() - 1;
    const int ncell = nx * ny * nz;
    cl->grid.push_back(make_int4(nx, ny, nz, first));
    cl->grid_cfg.push_back(c);
    // fractional coordinates with the inverse of the FP32 box, in FP64
    const double det = a[0] * bc[0] + a[1] * bc[1] + a[2] * bc[2];
    std::vector<int> cell_of(Na), count(ncell, 0);
    for (int k = 0; k < Na; ++k) {
      const int i = ts.Na_sum[c] + k;
      const double x = ts.r[i], y = ts.r[i + ts.N], z = ts.r[i + 2 * (size_t)ts.N];
      // s = h^-1 r with h^-1 rows = (b x c, c x a, a x b) / det
      double s[3] = {(bc[0] * x + bc[1] * y + bc[2] * z) / det, (ca[0] * x + ca[1] * y + ca[2] * z) / det,
                     (ab[0] * x + ab[1] * y + ab[2] * z) / det};
      const int n[3] = {nx, ny, nz};
      int ci[3];
      for (int q = 0; q < 3; ++q) {
        s[q] -= std::floor(s[q]);
        ci[q] = std::min(n[q] - 1, std::max(0, (int)(s[q] * n[q])));
      }
      cell_of[k] = (ci[2] * ny + ci[1]) * nx + ci[0];
      ++count[cell_of[k]];
      cl->atoms.push_back(i);
      cl->acell.push_back(make_int4(ci[0], ci[1], ci[2], g));
    }
    std::vector<int> start(ncell + 1, 0);
    for (int q = 0; q < ncell; ++q) start[q + 1] = start[q] + count[q];
    const int base = (int)cl->cell_atoms.size();
    cl->cell_atoms.resize(base + Na);
    std::vector<int> fill(start.begin(), start.end() - 1);
    for (int k = 0; k < Na; ++k) cl->cell_atoms[base + fill[cell_of[k]]++] = ts.Na_sum[c] + k;
    for (int q = 1; q <= ncell; ++q) cl->cell_start.push_back(base + start[q]);
  }
}

// Tersoff: bond j of local atom il of configuration c copied to sm_off[c] + j * Na + il (empty
// slots zero), one thread per atom.
__global__ void slot_major_copy(int N, const int* __restrict__ atom_cfg, const int* __restrict__ Na_sum,
                                const int* __restrict__ Na, const int* __restrict__ sm_off,
                                const int* __restrict__ zc_of, const int* __restrict__ off,
                                const float4* __restrict__ g32, const float* __restrict__ tdl,
                                const uint8_t* __restrict__ ptype, const int* __restrict__ rev_sm,
                                float4* __restrict__ g_sm, float* __restrict__ dl_sm, uint8_t* __restrict__ pt_sm,
                                int* __restrict__ rev_sm_sm) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const int c = atom_cfg[i], il = i - Na_sum[c], na = Na[c];
  const int Z = off[i + 1] - off[i];
  for (int j = 0; j < zc_of[c]; ++j) {
    const size_t o = (size_t)sm_off[c] + (size_t)j * na + il;
    if (j < Z) {
      const int b = off[i] + j;
      g_sm[o] = g32[b];
      dl_sm[o] = tdl[b];
      pt_sm[o] = ptype[b];
      rev_sm_sm[o] = rev_sm[b];
    } else {
      g_sm[o] = make_float4(0.f, 0.f, 0.f, 1.f);
      dl_sm[o] = 0.f;
      pt_sm[o] = 0;
      rev_sm_sm[o] = 0;
    }
  }
}

// The slot-major copy of the Tersoff geometry (DevSet::g_sm and friends).
static int build_slot_major(Engine* e, cudaStream_t st) {
  DevSet& d = e->d;
  const TrainingSet& ts = e->ts;
  const int Nc = ts.Nc, N = ts.N;
  std::vector<int> offs(Nc), zcs(Nc), atom_cfg(N);
  long long total = 0;
  for (int c = 0; c < Nc; ++c) {
    zcs[c] = std::max(tersoff_zclass(e->h_zmax[c]), 1);  // beyond 16 neighbors: refused at planning
    if (zcs[c] == 1) zcs[c] = 16;
    offs[c] = (int)total;
    total += (long long)zcs[c] * ts.Na[c];
    for (int k = 0; k < ts.Na[c]; ++k) atom_cfg[ts.Na_sum[c] + k] = c;
  }
  if (total > (1LL << 31) - 1) {
    set_error("slot-major geometry of %lld slots exceeds int32 indexing.", total);
    return GPUGA_ERR_UNSUPPORTED;
  }
  const size_t n = std::max<long long>(total, 1);
  GPUGA_TRY(e->alloc(&d.sm_off, std::max(Nc, 1)));
  GPUGA_TRY(e->alloc(&d.g_sm, n));
  GPUGA_TRY(e->alloc(&d.dl_sm, n));
  GPUGA_TRY(e->alloc(&d.pt_sm, n));
  GPUGA_TRY(e->alloc(&d.rev_sm_sm, n));
  int *d_zc = nullptr, *d_cfg = nullptr;
  GPUGA_CUDA(cudaMalloc(&d_zc, sizeof(int) * std::max(Nc, 1)));
  GPUGA_CUDA(cudaMalloc(&d_cfg, sizeof(int) * std::max(N, 1)));
  GPUGA_CUDA(cudaMemcpyAsync(d.sm_off, offs.data(), sizeof(int) * Nc, cudaMemcpyHostToDevice, st));
  GPUGA_CUDA(cudaMemcpyAsync(d_zc, zcs.data(), sizeof(int) * Nc, cudaMemcpyHostToDevice, st));
  GPUGA_CUDA(cudaMemcpyAsync(d_cfg, atom_cfg.data(), sizeof(int) * N, cudaMemcpyHostToDevice, st));
  slot_major_copy<<<(N + 127) / 128, 128, 0, st>>>(N, d_cfg, d.Na_sum, d.Na, d.sm_off, d_zc, d.off, d.g32, d.tdl,
                                                   d.ptype, d.rev_sm, d.g_sm, d.dl_sm, d.pt_sm, d.rev_sm_sm);
  GPUGA_CUDA(cudaGetLastError());
  GPUGA_CUDA(cudaStreamSynchronize(st));
  cudaFree(d_zc);
  cudaFree(d_cfg);
  return GPUGA_OK;
}

// Pair types whose Buckingham or Morse term can be nonzero for some individual: type t is left
// out of the pair-by-pair lists when its bounds fix A_t = 0 with rho_t > 0 (A e^{-d/rho} is then
// exactly zero) and, for the cation-anion type, the Morse D0 is fixed at 0 as well.
static int ri_active_types(const PotentialSpec& sp) {
  if (sp.pmin.size() < 15 || sp.pmax.size() < 15) return 7;
  int mask = 0;
  for (int t = 0; t < 3; ++t) {
    const int a = 1 + 3 * t, rho = 2 + 3 * t;
    const bool zero_buck = sp.pmin[a] == 0.0f && sp.pmax[a] == 0.0f && sp.pmin[rho] > 0.0f;
    const bool zero_morse = t != 1 || (sp.pmin[11] == 0.0f && sp.pmax[11] == 0.0f);
    if (!(zero_buck && zero_morse)) mask |= 1 << t;
  }
  return mask;
}

int build_geometry(Engine* e) {
  DevSet& d = e->d;
  const TrainingSet& ts = e->ts;
  const int N = ts.N, Nc = ts.Nc;
  cudaStream_t st = e->stream;
  const float rc2 = e->spec.cutoff * e->spec.cutoff;

  GPUGA_TRY(e->alloc(&d.NN, N));
  GPUGA_TRY(e->alloc(&d.off, N + 1));
  CellLists cl;
  build_cell_lists(e, &cl);
  uint8_t* d_skip = nullptr;
  int *d_catoms = nullptr, *d_gcfg = nullptr, *d_cstart = nullptr, *d_cell_atoms = nullptr;
  int4 *d_acell = nullptr, *d_grid = nullptr;
  const int n_cell_atoms = (int)cl.atoms.size();
  if (n_cell_atoms > 0) {
    GPUGA_CUDA(cudaMalloc(&d_skip, Nc));
    GPUGA_CUDA(cudaMalloc(&d_catoms, sizeof(int) * n_cell_atoms));
    GPUGA_CUDA(cudaMalloc(&d_acell, sizeof(int4) * n_cell_atoms));
    GPUGA_CUDA(cudaMalloc(&d_grid, sizeof(int4) * cl.grid.size()));
    GPUGA_CUDA(cudaMalloc(&d_gcfg, sizeof(int) * cl.grid_cfg.size()));
    GPUGA_CUDA(cudaMalloc(&d_cstart, sizeof(int) * cl.cell_start.size()));
    GPUGA_CUDA(cudaMalloc(&d_cell_atoms, sizeof(int) * cl.cell_atoms.size()));
    GPUGA_CUDA(cudaMemcpy(d_skip, cl.skip.data(), Nc, cudaMemcpyHostToDevice));
    GPUGA_CUDA(cudaMemcpy(d_catoms, cl.atoms.data(), sizeof(int) * n_cell_atoms, cudaMemcpyHostToDevice));
    GPUGA_CUDA(cudaMemcpy(d_acell, cl.acell.data(), sizeof(int4) * n_cell_atoms, cudaMemcpyHostToDevice));
    GPUGA_CUDA(cudaMemcpy(d_grid, cl.grid.data(), sizeof(int4) * cl.grid.size(), cudaMemcpyHostToDevice));
    GPUGA_CUDA(cudaMemcpy(d_gcfg, cl.grid_cfg.data(), sizeof(int) * cl.grid_cfg.size(), cudaMemcpyHostToDevice));
    GPUGA_CUDA(cudaMemcpy(d_cstart, cl.cell_start.data(), sizeof(int) * cl.cell_start.size(), cudaMemcpyHostToDevice));
    GPUGA_CUDA(cudaMemcpy(d_cell_atoms, cl.cell_atoms.data(), sizeof(int) * cl.cell_atoms.size(),
                          cudaMemcpyHostToDevice));
  }
  auto free_cells = [&]() {
    cudaFree(d_skip);
    cudaFree(d_catoms);
    cudaFree(d_acell);
    cudaFree(d_grid);
    cudaFree(d_gcfg);
    cudaFree(d_cstart);
    cudaFree(d_cell_atoms);
  };
  neighbor_scan<kMicMode, false><<<Nc, 256, 0, st>>>(N, d.Na, d.Na_sum, rc2, d.h, d.r, d.NN, nullptr, nullptr,
                                                    nullptr, d_skip);
  GPUGA_CUDA(cudaGetLastError());
  if (n_cell_atoms > 0) {
    neighbor_cells<kMicMode, false><<<(n_cell_atoms + 127) / 128, 128, 0, st>>>(
        N, n_cell_atoms, d_catoms, d_acell, d_grid, d_gcfg, d_cstart, d_cell_atoms, rc2, d.h, d.r, d.NN, nullptr,
        nullptr, nullptr);
    GPUGA_CUDA(cudaGetLastError());
  }
  e->h_NN.assign(N, 0);
  GPUGA_CUDA(cudaMemcpyAsync(e->h_NN.data(), d.NN, sizeof(int) * N, cudaMemcpyDeviceToHost, st));
  GPUGA_CUDA(cudaStreamSynchronize(st));
  e->h_off.assign(N + 1, 0);
  long long total = 0;
  int max_Z = 0;
  for (int i = 0; i < N; ++i) {
    e->h_off[i] = (int)total;
    total += e->h_NN[i];
    max_Z = std::max(max_Z, e->h_NN[i]);
  }
  if (total > (1LL << 31) - 1) {
    set_error("neighbor list has %lld bonds, more than the engine indexes with int32.", total);
    return GPUGA_ERR_UNSUPPORTED;
  }
  e->h_off[N] = (int)total;
  const int B = (int)total;
  d.B = B;
  d.max_Z = max_Z;
  GPUGA_CUDA(cudaMemcpyAsync(d.off, e->h_off.data(), sizeof(int) * (N + 1), cudaMemcpyHostToDevice, st));

  float* img = nullptr;
  GPUGA_CUDA(cudaMalloc(&img, sizeof(float) * 3 * (size_t)std::max(B, 1)));
  GPUGA_TRY(e->alloc(&d.nbr, std::max(B, 1)));
  neighbor_scan<kMicMode, true><<<Nc, 256, 0, st>>>(N, d.Na, d.Na_sum, rc2, d.h, d.r, d.NN, d.off, d.nbr, img,
                                                   d_skip);
  GPUGA_CUDA(cudaGetLastError());
  if (n_cell_atoms > 0) {
    neighbor_cells<kMicMode, true><<<(n_cell_atoms + 127) / 128, 128, 0, st>>>(
        N, n_cell_atoms, d_catoms, d_acell, d_grid, d_gcfg, d_cstart, d_cell_atoms, rc2, d.h, d.r, d.NN, d.off,
        d.nbr, img);
    GPUGA_CUDA(cudaGetLastError());
  }

  // per-atom config index for the geometry kernel
  std::vector<int> atom_cfg(N);
  for (int c = 0; c < Nc; ++c)
    for (int k = 0; k < ts.Na[c]; ++k) atom_cfg[ts.Na_sum[c] + k] = c;
  int* d_atom_cfg = nullptr;
  GPUGA_CUDA(cudaMalloc(&d_atom_cfg, sizeof(int) * N));
  GPUGA_CUDA(cudaMemcpyAsync(d_atom_cfg, atom_cfg.data(), sizeof(int) * N, cudaMemcpyHostToDevice, st));

  GPUGA_TRY(e->alloc(&d.g64, std::max(B, 1)));
  // RI evaluates its type-grouped copies (rg32 / rdl, below): there g32 and dl are scratch
  const bool ri = is_ri_type(d.potential_type);
  float* dl = nullptr;
  if (ri) {
    GPUGA_CUDA(cudaMalloc(&d.g32, sizeof(float4) * std::max(B, 1)));
    GPUGA_CUDA(cudaMalloc(&dl, sizeof(float) * std::max(B, 1)));
  } else {
    GPUGA_TRY(e->alloc(&d.g32, std::max(B, 1)));
  }
  GPUGA_TRY(e->alloc(&d.rev, std::max(B, 1)));
  GPUGA_TRY(e->alloc(&d.half_off, N));
  GPUGA_TRY(e->alloc(&d.ptype, std::max(B, 1)));
  const bool tersoff = d.potential_type == 1 || d.potential_type == 2;
  if (tersoff) {
    GPUGA_TRY(e->alloc(&d.d64, std::max(B, 1)));
    GPUGA_TRY(e->alloc(&d.tdl, std::max(B, 1)));
  }
  bond_geometry<<<(N + 127) / 128, 128, 0, st>>>(N, d_atom_cfg, d.h, d.r, d.type, d.off, d.nbr, img,
                                                 ri ? 0 : d.potential_type, d.num_types, d.g64, d.g32,
                                                 ri ? dl : d.tdl, d.d64, d.rev, d.half_off, d.ptype);
  GPUGA_CUDA(cudaGetLastError());
  GPUGA_TRY(e->alloc(&d.rev_sm, std::max(B, 1)));
  reverse_slots<<<(N + 127) / 128, 128, 0, st>>>(N, d_atom_cfg, d.Na, d.Na_sum, d.off, d.nbr, d.rev, d.rev_sm);
  GPUGA_CUDA(cudaGetLastError());
  if (d.potential_type == 3) {
    GPUGA_TRY(e->alloc(&d.pslot, std::max(B, 1)));
    pair_slots<<<(N + 127) / 128, 128, 0, st>>>(N, d_atom_cfg, d.Na_sum, d.off, d.nbr, d.rev, d.pslot);
    GPUGA_CUDA(cudaGetLastError());
  }
  if (ri) {
    d.ri_active = ri_active_types(e->spec);
    std::vector<int> half(N), start(N + 1, 0);
    std::vector<uint8_t> pt(std::max(B, 1));
    GPUGA_CUDA(cudaMemcpyAsync(half.data(), d.half_off, sizeof(int) * N, cudaMemcpyDeviceToHost, st));
    GPUGA_CUDA(cudaMemcpyAsync(pt.data(), d.ptype, (size_t)B, cudaMemcpyDeviceToHost, st));
    GPUGA_CUDA(cudaStreamSynchronize(st));
    // the host has the lists already (h_off); nbr comes back below, ptype just now
    for (int i = 0; i < N; ++i) {
      int n = 0;
      for (int b = i < ts.N_force ? e->h_off[i] : half[i]; b < e->h_off[i + 1]; ++b) n += (d.ri_active >> pt[b]) & 1;
      start[i + 1] = start[i] + n;
    }
    int* d_start = nullptr;
    GPUGA_CUDA(cudaMalloc(&d_start, sizeof(int) * (N + 1)));
    GPUGA_CUDA(cudaMemcpyAsync(d_start, start.data(), sizeof(int) * (N + 1), cudaMemcpyHostToDevice, st));
    GPUGA_TRY(e->alloc(&d.rg32, std::max(start[N], 1)));
    GPUGA_TRY(e->alloc(&d.rdl, std::max(start[N], 1)));
    GPUGA_TRY(e->alloc(&d.rseg, N));
    ri_group<<<(N + 127) / 128, 128, 0, st>>>(N, ts.N_force, d.ri_active, d.off, d.half_off, d.ptype, d.g32, dl,
                                              d_start, d.rg32, d.rdl, d.rseg);
    GPUGA_CUDA(cudaGetLastError());
    // FP64 sums of the linear terms
    double* ev = nullptr;
    GPUGA_CUDA(cudaMalloc(&ev, sizeof(double) * kRiCfgLin * (size_t)std::max(N, 1)));
    GPUGA_TRY(e->alloc(&d.ri_atom_lin, (size_t)kRiAtomLin * std::max(ts.N_force, 1)));
    GPUGA_TRY(e->alloc(&d.ri_cfg_lin, (size_t)kRiCfgLin * Nc));
    GPUGA_CUDA(cudaMemsetAsync(d.ri_cfg_lin, 0, sizeof(double) * kRiCfgLin * (size_t)Nc, st));
    ri_linear_atoms<<<(N + 127) / 128, 128, 0, st>>>(N, ts.N_force, d.off, d.half_off, d.ptype, d.g64, d.ri_atom_lin,
                                                     ev);
    GPUGA_CUDA(cudaGetLastError());
    if (Nc > ts.Nc_force) {
      ri_linear_configs<<<Nc - ts.Nc_force, 96, 0, st>>>(Nc, ts.Nc_force, d.Na, d.Na_sum, ev, d.ri_cfg_lin);
      GPUGA_CUDA(cudaGetLastError());
    }
    GPUGA_CUDA(cudaStreamSynchronize(st));
    cudaFree(ev);
    cudaFree(d_start);
    cudaFree(d.g32);
    cudaFree(dl);
    d.g32 = nullptr;
  }

  GPUGA_CUDA(cudaStreamSynchronize(st));
  cudaFree(img);
  cudaFree(d_atom_cfg);
  free_cells();

  e->h_nbr.assign(std::max(B, 1), 0);
  GPUGA_CUDA(cudaMemcpy(e->h_nbr.data(), d.nbr, sizeof(int) * (size_t)B, cudaMemcpyDeviceToHost));
  e->h_zmax.assign(Nc, 0);
  for (int c = 0; c < Nc; ++c)
    for (int k = 0; k < ts.Na[c]; ++k) e->h_zmax[c] = std::max(e->h_zmax[c], e->h_NN[ts.Na_sum[c] + k]);
  if (tersoff) GPUGA_TRY(build_slot_major(e, st));
  if (d.potential_type == 3) {
    // NN2B: the bonds each configuration's work items evaluate, as one list per configuration
    // (hb, hb_off).  Energy/virial configurations: the bonds to a higher-index neighbor (the
    // unordered pairs).  Force configurations: the same when the bond list is symmetric (every
    // bond's reverse present: the nearest-image rule gives that except at exact half-box ties),
    // else all bonds.
    e->h_pair_sym.assign(Nc, 0);
    std::vector<int> hb, hb_off(Nc + 1, 0);
    for (int c = 0; c < Nc; ++c) {
      hb_off[c] = (int)hb.size();
      const int a0 = ts.Na_sum[c], a1 = a0 + ts.Na[c];
      if (c >= ts.Nc_force) {  // energy/virial items: the unordered pairs (the half lists)
        for (int i = a0; i < a1; ++i)
          for (int b = e->h_off[i]; b < e->h_off[i + 1]; ++b)
            if (e->h_nbr[b] > i) hb.push_back(b);
        continue;
      }
      bool sym = true;
      for (int i = a0; sym && i < a1; ++i)
        for (int b = e->h_off[i]; sym && b < e->h_off[i + 1]; ++b) {
          const int j = e->h_nbr[b];
          sym = j != i && std::binary_search(e->h_nbr.begin() + e->h_off[j], e->h_nbr.begin() + e->h_off[j + 1], i);
        }
      e->h_pair_sym[c] = sym;
      for (int i = a0; i < a1; ++i)
        for (int b = e->h_off[i]; b < e->h_off[i + 1]; ++b)
          if (!sym || e->h_nbr[b] > i) hb.push_back(b);
    }
    hb_off[Nc] = (int)hb.size();
    GPUGA_TRY(e->alloc(&d.hb, std::max<size_t>(hb.size(), 1)));
    GPUGA_TRY(e->alloc(&d.hb_off, (size_t)Nc + 1));
    if (!hb.empty()) GPUGA_CUDA(cudaMemcpy(d.hb, hb.data(), sizeof(int) * hb.size(), cudaMemcpyHostToDevice));
    GPUGA_CUDA(cudaMemcpy(d.hb_off, hb_off.data(), sizeof(int) * (Nc + 1), cudaMemcpyHostToDevice));
  }
  return GPUGA_OK;
}

}  // namespace gpuga
