// Probe linked against the UNMODIFIED reference sources (GPUGA src/*.cu minus
// main.cu, gpuga.cu and ga.cu) -- test and baseline infrastructure only.
//
//   ref_probe neighbors <dir> <out.bin>   dump NN[N] and NL[max_Na*N] as built by neighbor.cu
//   ref_probe mic <count> <seed> <out.bin> outputs of mic.cuh's dev_apply_mic and of the
//                                          squared-distance expression of neighbor.cu:59 on
//                                          random inputs (FP32 contraction pattern check)
//   ref_probe time <dir> <P> <steps> <warmup> <seed>
//                                          wall time of Fitness::compute (fitness.cu:316-333)
//                                          per generation, host population to host fitness,
//                                          L2 flushed between generations
//
// Built by oracle/Makefile (target `ref`) into oracle/_ref/.
#include <cuda_runtime.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <vector>

#include "fitness.cuh"
#include "mic.cuh"
#include "neighbor.cuh"

namespace {

struct Probe : public Fitness {
  explicit Probe(char* dir) : Fitness(dir) {}
  int n_atoms() const { return N; }
  int max_atoms() const { return max_Na; }
  const Neighbor& nb() const { return neighbor; }
};

__global__ void mic_kernel(int n, const float* h, const float* in, float* out) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const float* hk = h + 18 * (size_t)k;
  float x12 = in[3 * (size_t)k], y12 = in[3 * (size_t)k + 1], z12 = in[3 * (size_t)k + 2];
  dev_apply_mic(hk, x12, y12, z12);
  float distance_square = x12 * x12 + y12 * y12 + z12 * z12;
  out[4 * (size_t)k] = x12;
  out[4 * (size_t)k + 1] = y12;
  out[4 * (size_t)k + 2] = z12;
  out[4 * (size_t)k + 3] = distance_square;
}

// fitness.cu:40-57 as compiled in the reference (host code).
void inverse(float* h) {
  h[9] = h[4] * h[8] - h[5] * h[7];
  h[10] = h[2] * h[7] - h[1] * h[8];
  h[11] = h[1] * h[5] - h[2] * h[4];
  h[12] = h[5] * h[6] - h[3] * h[8];
  h[13] = h[0] * h[8] - h[2] * h[6];
  h[14] = h[2] * h[3] - h[0] * h[5];
  h[15] = h[3] * h[7] - h[4] * h[6];
  h[16] = h[1] * h[6] - h[0] * h[7];
  h[17] = h[0] * h[4] - h[1] * h[3];
  float v = h[0] * (h[4] * h[8] - h[5] * h[7]) + h[1] * (h[5] * h[6] - h[3] * h[8]) + h[2] * (h[3] * h[7] - h[4] * h[6]);
  for (int n = 9; n < 18; n++) h[n] /= v;
}

int cmd_neighbors(char* dir, const char* out) {
  Probe f(dir);
  CHECK(cudaDeviceSynchronize());
  const int N = f.n_atoms(), M = f.max_atoms();
  FILE* fo = fopen(out, "wb");
  if (!fo) return 1;
  fwrite(&N, sizeof(int), 1, fo);
  fwrite(&M, sizeof(int), 1, fo);
  fwrite(f.nb().NN, sizeof(int), N, fo);
  std::vector<int> NL((size_t)N * M, -1);
  for (int i = 0; i < N; ++i)
    for (int k = 0; k < f.nb().NN[i]; ++k) NL[(size_t)k * N + i] = f.nb().NL[(size_t)k * N + i];
  fwrite(NL.data(), sizeof(int), NL.size(), fo);
  fclose(fo);
  return 0;
}

int cmd_mic(int n, unsigned seed, const char* out) {
  std::mt19937 rng(seed);
  std::uniform_real_distribution<float> box(4.0f, 14.0f), tilt(-1.5f, 1.5f), disp(-20.0f, 20.0f);
  std::vector<float> h(18 * (size_t)n), in(3 * (size_t)n), res(4 * (size_t)n);
  for (int k = 0; k < n; ++k) {
    float* hk = &h[18 * (size_t)k];
    for (int a = 0; a < 9; ++a) hk[a] = (a % 4 == 0) ? box(rng) : tilt(rng);
    inverse(hk);
    for (int a = 0; a < 3; ++a) in[3 * (size_t)k + a] = disp(rng);
  }
  float *dh, *din, *dout;
  CHECK(cudaMalloc(&dh, sizeof(float) * h.size()));
  CHECK(cudaMalloc(&din, sizeof(float) * in.size()));
  CHECK(cudaMalloc(&dout, sizeof(float) * res.size()));
  CHECK(cudaMemcpy(dh, h.data(), sizeof(float) * h.size(), cudaMemcpyHostToDevice));
  CHECK(cudaMemcpy(din, in.data(), sizeof(float) * in.size(), cudaMemcpyHostToDevice));
  mic_kernel<<<(n + 127) / 128, 128>>>(n, dh, din, dout);
  CHECK(cudaGetLastError());
  CHECK(cudaMemcpy(res.data(), dout, sizeof(float) * res.size(), cudaMemcpyDeviceToHost));
  FILE* fo = fopen(out, "wb");
  if (!fo) return 1;
  fwrite(&n, sizeof(int), 1, fo);
  fwrite(h.data(), sizeof(float), h.size(), fo);
  fwrite(in.data(), sizeof(float), in.size(), fo);
  fwrite(res.data(), sizeof(float), res.size(), fo);
  fclose(fo);
  cudaFree(dh);
  cudaFree(din);
  cudaFree(dout);
  return 0;
}

int cmd_time(char* dir, int P, int steps, int warmup, unsigned seed) {
  Probe f(dir);
  const int d = f.number_of_variables;
  std::vector<float> pop((size_t)P * d), fit(P);
  std::mt19937 rng(seed);
  std::uniform_real_distribution<float> u(0, 1);
  for (auto& v : pop) v = u(rng);
  void* flush = nullptr;
  const size_t flush_bytes = 256u << 20;  // larger than the 126 MB L2
  CHECK(cudaMalloc(&flush, flush_bytes));
  std::vector<double> ms;
  for (int s = 0; s < warmup + steps; ++s) {
    CHECK(cudaMemset(flush, s & 0xff, flush_bytes));
    CHECK(cudaDeviceSynchronize());
    auto t0 = std::chrono::steady_clock::now();
    f.compute(P, pop.data(), fit.data());
    CHECK(cudaDeviceSynchronize());
    auto t1 = std::chrono::steady_clock::now();
    if (s >= warmup) ms.push_back(std::chrono::duration<double, std::milli>(t1 - t0).count());
  }
  cudaFree(flush);
  printf("REF_TIME {\"P\": %d, \"N\": %d, \"steps\": %d, \"ms\": [", P, f.n_atoms(), steps);
  for (size_t k = 0; k < ms.size(); ++k) printf("%s%.6f", k ? ", " : "", ms[k]);
  printf("], \"fitness0\": %.9g}\n", fit[0]);
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc >= 4 && !strcmp(argv[1], "neighbors")) return cmd_neighbors(argv[2], argv[3]);
  if (argc >= 5 && !strcmp(argv[1], "mic")) return cmd_mic(atoi(argv[2]), (unsigned)atoi(argv[3]), argv[4]);
  if (argc >= 7 && !strcmp(argv[1], "time"))
    return cmd_time(argv[2], atoi(argv[3]), atoi(argv[4]), atoi(argv[5]), (unsigned)atoi(argv[6]));
  fprintf(stderr, "usage: ref_probe neighbors <dir> <out> | mic <n> <seed> <out> | time <dir> <P> <steps> <warmup> <seed>\n");
  return 2;
}
