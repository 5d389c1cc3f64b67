// Potential::find_force for callers that cannot allocate device memory.
//
// Some hosts of this library are not allowed to call cudaMalloc at the point
// where they need forces: a molecular-dynamics code that hands every byte of a
// fixed device-memory budget to its own pool allocator, a plug-in host whose
// interface forbids device allocation after initialisation, or a real-time
// loop that must not allocate after start-up.
// gpuga_potential_find_force_noalloc serves them: the caller still owns and
// passes every input and output array, and the per-bond scratch of the force
// kernels lives in one file-scope __device__ array of fixed size (64 MiB) that
// the CUDA runtime creates when the library's module is loaded on a device and
// keeps until the process exits.
//
// The first call on a device resolves the array's device address
// (cudaGetSymbolAddress, with that device current); make that first call
// before any stream capture.  The address is kept until the process exits: a
// cudaDeviceReset unloads the module, so the entry point must not be used on
// that device afterwards.  Every call on a device uses the same array, so
// calls whose work overlaps on the GPU (two streams, two threads) race on it;
// serialise them.  Each call zeroes the part of the array it uses before use.
// `params` is a host array (read during the call; the NN2B weights are copied
// from it into the scratch), every other array a device array.
#include <mutex>

#include "engine.hpp"

namespace gpuga {
namespace {

// Upper bound of the shared scratch: 64 MiB per device.
constexpr size_t kNoAllocScratchBytes = 64u << 20;

// The scratch itself.  Host code must not use this name as an address: the
// device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
void* g_scratch_ptr[kMaxDevices] = {};

// Once per device, with that device current: resolve the device address of the scratch.
int scratch_for_current_device(void** out) {
  int dev = 0;
  GPUGA_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) {
    set_error("device ordinal %d is beyond the %d devices this entry point tracks.", dev, kMaxDevices);
    return GPUGA_ERR_UNSUPPORTED;
  }
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    cudaError_t err = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (err != cudaSuccess) return cuda_status(err, "cudaGetSymbolAddress", __FILE__, __LINE__);
    g_scratch_ptr[dev] = p;
  }
  *out = g_scratch_ptr[dev];
  return GPUGA_OK;
}

}  // namespace
}  // namespace gpuga

using namespace gpuga;

extern "C" int gpuga_potential_find_force_noalloc(int potential_type, int num_neurons, const float* params,
                                                  int num_params, int Nc, int N, const int* Na, const int* Na_sum,
                                                  int max_Na, const int* type, const float* h, const int* NN,
                                                  const int* NL, const float* r, float* f, float* virial, float* pe,
                                                  void* stream) {
  const int nv = num_vars_for(potential_type, num_neurons);
  if (nv < 0 || (potential_type == 3 && (num_neurons < 1 || num_neurons > 32))) {
    set_error("unsupported potential type %d (neurons %d).", potential_type, num_neurons);
    return GPUGA_ERR_UNSUPPORTED;
  }
  if (!params || num_params != nv || Nc < 1 || N < 1 || max_Na < 1 || !Na || !Na_sum || !type || !h || !NN || !NL ||
      !r || !f || !virial || !pe) {
    set_error("gpuga_potential_find_force_noalloc: invalid argument (expected %d parameters)", nv);
    return GPUGA_ERR_ARG;
  }
  const size_t need = ref_potential_scratch_bytes(potential_type, num_neurons, N, max_Na);
  if (need > kNoAllocScratchBytes) {
    set_error("gpuga_potential_find_force_noalloc: N=%d x max_Na=%d needs %zu bytes of scratch, above the fixed "
              "%zu-byte limit of this entry point; use gpuga_potential_find_force",
              N, max_Na, need, kNoAllocScratchBytes);
    return GPUGA_ERR_ARG;
  }
  void* base = nullptr;
  GPUGA_TRY(scratch_for_current_device(&base));
  cudaStream_t st = (cudaStream_t)stream;
  // The array keeps the previous call's contents: start every call from zeros.
  GPUGA_CUDA(cudaMemsetAsync(base, 0, need, st));
  const size_t slots = (size_t)N * (size_t)max_Na;
  auto up = [](size_t b) { return (b + 255) & ~(size_t)255; };
  char* p = static_cast<char*>(base);
  RefPotentialScratch s;
  s.g64 = reinterpret_cast<double4*>(p);
  p += up(slots * sizeof(double4));
  s.rev = reinterpret_cast<int*>(p);
  p += up(slots * sizeof(int));
  s.f5 = reinterpret_cast<float*>(p);
  p += up(5 * slots * sizeof(float));
  s.w = reinterpret_cast<float*>(p);
  PotentialSpec opts;  // NN2B taper 7..8 A with the reference's force order (nn2b.cuh:36-38, nn2b.cu:147-148)
  return ref_potential_find_force(potential_type, num_neurons, params, opts, Nc, N, Na, Na_sum, max_Na, type, h, NN,
                                  NL, r, f, virial, pe, s, st);
}
