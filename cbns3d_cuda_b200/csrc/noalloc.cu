// noalloc.cu - cbns_calc_gradient_noalloc: the 4th-order gradient of a host
// field without any device allocation.
//
// Who needs it: callers that cannot call cudaMalloc -- hosts whose device
// memory is fully owned by their own pool allocator or held to a fixed budget
// (a cudaMalloc outside the pool can fail or push the process over its
// budget), and latency-sensitive paths that cannot afford the device-wide
// synchronisation cudaMalloc/cudaFree imply.  cbns_calc_gradient allocates its
// device copies per call; this variant keeps them in a file-scope __device__
// array instead.  Like cbns_calc_gradient it is synchronous: blocking copies
// on the legacy default stream.
//
// Limits and sharing:
//   * at most CBNS_NOALLOC_MAX_POINTS grid points (IM*JM*KM); larger requests
//     return CBNS_ERR_TOO_LARGE before touching the GPU;
//   * the array (4 x CBNS_NOALLOC_MAX_POINTS doubles, 8 MiB) exists on every
//     GPU that loads this library, for the life of the process;
//   * every call on a device uses the same array, and it keeps the previous
//     call's contents; each call writes every element it later reads (the
//     input copy and all three derivative arrays), so nothing needs clearing;
//     calls that overlap on the GPU (from several host threads at once) race
//     on the array and must be serialised by the caller;
//   * the device address of the array is looked up once per device, on that
//     device's first call (with the device current);
//   * a failure returns CBNS_ERR_CUDA and records the CUDA error text for
//     cbns_status_string, as the other entry points do.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/cbns_b200.h"
#include "setup.cuh"

namespace cbns {
void set_last_error(const char* what, cudaError_t e);  // abi.cu
}

namespace {

constexpr unsigned long long kMaxPoints = CBNS_NOALLOC_MAX_POINTS;

// f, fx, fy, fz for up to kMaxPoints nodes each
static __device__ __align__(256) double g_noalloc_scratch[4 * kMaxPoints];

constexpr int kMaxDevices = 64;
double* g_scratch_ptr[kMaxDevices] = {nullptr};
std::mutex g_scratch_mu;

// Device address of g_noalloc_scratch on the current device (set up once).
cudaError_t scratch_for_current_device(double** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_ptr[dev]) {
    double* p = nullptr;
    e = cudaGetSymbolAddress(reinterpret_cast<void**>(&p), g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_ptr[dev] = p;
  }
  *out = g_scratch_ptr[dev];
  return cudaSuccess;
}

}  // namespace

extern "C" int cbns_calc_gradient_noalloc(unsigned IM, unsigned JM, unsigned KM, const double* f, double* fx,
                                          double* fy, double* fz) {
  if (!f || !fx || !fy || !fz || IM < 2 || JM < 2 || KM < 2) return CBNS_ERR_ARG;
  const unsigned long long N = (unsigned long long)IM * JM * KM;
  if (N > kMaxPoints) return CBNS_ERR_TOO_LARGE;
  double* s = nullptr;
  cudaError_t e = scratch_for_current_device(&s);
  if (e != cudaSuccess) {
    cbns::set_last_error("cudaGetSymbolAddress(g_noalloc_scratch)", e);
    return CBNS_ERR_CUDA;
  }
  const size_t bytes = N * sizeof(double);
  e = cudaMemcpy(s, f, bytes, cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cbns::launch_gradient_dense((int)IM, (int)JM, (int)KM, s, s + kMaxPoints, s + 2 * kMaxPoints,
                                    s + 3 * kMaxPoints, 0);
  if (e == cudaSuccess) e = cudaMemcpy(fx, s + kMaxPoints, bytes, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(fy, s + 2 * kMaxPoints, bytes, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(fz, s + 3 * kMaxPoints, bytes, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) {
    cbns::set_last_error("cbns_calc_gradient_noalloc", e);
    return CBNS_ERR_CUDA;
  }
  return CBNS_OK;
}
