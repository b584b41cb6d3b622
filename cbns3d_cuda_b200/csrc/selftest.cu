// selftest.cu - the time-out path of the library's bounded waits, run on the
// GPU without a fault: one thread waits on mbarriers that nothing completes --
// the tensor-core MMA barrier with the sensor's two wait windows (tc_mlp.cuh)
// and the stage kernel's TMA transaction barrier after an arrival that
// announces bytes no copy will bring (tma.cuh) -- records what each wait
// returned and how long it took, and exits.  No copy or MMA was ever issued,
// so nothing is in flight on either barrier when the CTA exits, and the
// context stays usable; the host reads the record.
#include <cuda_runtime.h>

#include "../../include/cbns_b200.h"
#include "tc_mlp.cuh"
#include "tma.cuh"

namespace cbns {

void set_last_error(const char* what, cudaError_t e);  // abi.cu

namespace {

// out[0], out[1]: 1 when the MMA-barrier wait, the TMA-barrier wait reported a
// time-out; clk[0], clk[1]: the waits' lengths in globaltimer nanoseconds
struct WaitRecord {
  int out[2];
  unsigned long long clk[2];
};

__global__ void wait_timeout_kernel(WaitRecord* rec) {
  int* out = rec->out;
  unsigned long long* clk = rec->clk;
  __shared__ alignas(8) unsigned long long bar[2];
  if (threadIdx.x != 0) return;
  tc::mbar_init(&bar[0]);   // expects one arrival; none comes
  tma::bar_init(&bar[1]);
  tma::fence_init();
  tma::bar_expect(&bar[1], 16);  // the arrival, with 16 bytes no copy brings
  unsigned long long t0, t1, t2;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
  const bool mma_done = tc::mbar_wait(&bar[0], 0) || tc::mbar_wait(&bar[0], 0);
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t1));
  const bool tma_done = tma::bar_wait(&bar[1], 0);
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t2));
  out[0] = mma_done ? 0 : 1;
  out[1] = tma_done ? 0 : 1;
  clk[0] = t1 - t0;
  clk[1] = t2 - t1;
}

}  // namespace
}  // namespace cbns

extern "C" int cbns_selftest_waits(int* mma_timed_out, int* tma_timed_out, double* mma_seconds,
                                   double* tma_seconds) {
  if (!mma_timed_out || !tma_timed_out) return CBNS_ERR_ARG;
  cbns::WaitRecord* d_rec = nullptr;
  cudaError_t e = cudaMalloc(&d_rec, sizeof(cbns::WaitRecord));
  if (e != cudaSuccess) {
    cbns::set_last_error("cbns_selftest_waits: cudaMalloc", e);
    return CBNS_ERR_CUDA;
  }
  cbns::WaitRecord h{{-1, -1}, {0, 0}};
  e = cudaMemcpy(d_rec, &h, sizeof(h), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    cbns::wait_timeout_kernel<<<1, 32>>>(d_rec);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaMemcpy(&h, d_rec, sizeof(h), cudaMemcpyDeviceToHost);
  cudaFree(d_rec);
  if (e != cudaSuccess) {
    cbns::set_last_error("cbns_selftest_waits", e);
    return CBNS_ERR_CUDA;
  }
  *mma_timed_out = h.out[0];
  *tma_timed_out = h.out[1];
  if (mma_seconds) *mma_seconds = 1e-9 * (double)h.clk[0];
  if (tma_seconds) *tma_seconds = 1e-9 * (double)h.clk[1];
  return CBNS_OK;
}
