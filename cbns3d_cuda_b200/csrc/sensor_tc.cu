// sensor_tc.cu - the sensor network's forward pass on the tcgen05 tensor
// cores for a batch of feature vectors (BF16 operands, FP32 accumulation).
// The same tile routine (tc_mlp.cuh) runs inside the hybrid stage kernel; this
// kernel serves validation against the FP32 predictor and batch inference.
#include "sensor_kernels.cuh"
#include "tc_mlp.cuh"

namespace cbns {

namespace {

__global__ void __launch_bounds__(128) mlp_predict_tc_kernel(const float* __restrict__ P, const float* __restrict__ X,
                                                             unsigned n, float* __restrict__ out, int* fail) {
  extern __shared__ unsigned char raw[];
  tc::Smem& s = *reinterpret_cast<tc::Smem*>((reinterpret_cast<uintptr_t>(raw) + 127) & ~uintptr_t(127));
  const int t = threadIdx.x;
  if (t < 32) tc::tmem_alloc(&s.tmem, tc::TMEM_COLS);
  if (t == 0) tc::mbar_init(&s.bar);
  tc::load_weights(s, P, t, 128);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  unsigned phase = 0;
  const unsigned ntiles = (n + 127) / 128;
  for (unsigned tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const unsigned sidx = tile * 128 + t;
    float f[SN_IN];
#pragma unroll
    for (int k = 0; k < SN_IN; ++k) f[k] = sidx < n ? X[(size_t)sidx * SN_IN + k] : 0.f;
    tc::put_features(s, t, f);
    float z = 0.f;
    if (!tc::run_tile(s, t, phase, &z)) {
      if (t == 0) atomicExch(fail, 1);
      break;
    }
    if (sidx < n) out[sidx] = 1.f / (1.f + __expf(-z));
  }
  tc::fence_before_sync();
  __syncthreads();
  if (t < 32) {
    tc::fence_after_sync();
    tc::tmem_dealloc(s.tmem, tc::TMEM_COLS);
  }
}

// One 128-face tile per round: each thread forms the features of one face from
// global memory, the tile goes through the network on the tensor cores, and the
// thread writes its face's decision.
__global__ void __launch_bounds__(128) sensor_mask_kernel(const MaskArgs a) {
  if (a.check_done && a.st->done) return;
  extern __shared__ unsigned char raw[];
  tc::Smem& s = *reinterpret_cast<tc::Smem*>((reinterpret_cast<uintptr_t>(raw) + 127) & ~uintptr_t(127));
  const int t = threadIdx.x;
  if (t < 32) tc::tmem_alloc(&s.tmem, tc::TMEM_COLS);
  if (t == 0) tc::mbar_init(&s.bar);
  tc::load_weights(s, a.params, t, 128);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const Dims& d = a.d;
  const long nf = total_faces(d);
  const long ntiles = (nf + 127) / 128;
  // p >= tau  <=>  logit >= log(tau / (1 - tau))
  const float zcut = logf(a.tau / (1.f - a.tau));
  unsigned phase = 0;
  unsigned nweno = 0;
  for (long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const long e = tile * 128 + t;
    int dir, i, j, k;
    float f[SN_IN];
    if (decode_face(d, e, dir, i, j, k)) {
      const long sd = dir == 0 ? 1 : (dir == 1 ? d.PX : d.PL);
      const long oa = node_off(d, i, j, k), ob = oa + sd;
      auto ld = [&](int p, int n) -> float { return (float)__ldg(a.q + n * d.VOL + oa + (p - 2) * sd); };
      const float nx = (float)(0.5 * (__ldg(a.area[3 * dir] + oa) + __ldg(a.area[3 * dir] + ob)));
      const float ny = (float)(0.5 * (__ldg(a.area[3 * dir + 1] + oa) + __ldg(a.area[3 * dir + 1] + ob)));
      const float nz = (float)(0.5 * (__ldg(a.area[3 * dir + 2] + oa) + __ldg(a.area[3 * dir + 2] + ob)));
      const float in = rsqrtf(nx * nx + ny * ny + nz * nz);
      face_features(ld, nx * in, ny * in, nz * in, a.gamma, a.gam1, f);
    } else {
#pragma unroll
      for (int m = 0; m < SN_IN; ++m) f[m] = 0.f;
    }
    tc::put_features(s, t, f);
    float z = 0.f;
    if (!tc::run_tile(s, t, phase, &z)) {
      if (t == 0) {  // decisions incomplete: the step takes WENO5 everywhere
        atomicExch(&a.st->sensor_fail, 1);
        atomicExch(&a.st->force_weno, 1);
      }
      break;
    }
    if (e < nf) {
      // non-finite features (e.g. a non-physical state) fall back to WENO5
      const unsigned char dec = (z >= zcut || !(z == z)) ? 1 : 0;
      a.mask[e] = dec;
      nweno += dec;
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) nweno += __shfl_xor_sync(0xffffffffu, nweno, o);
  if ((t & 31) == 0 && nweno) atomicAdd(&a.st->weno_faces, (unsigned long long)nweno);
  tc::fence_before_sync();
  __syncthreads();
  if (t < 32) {
    tc::fence_after_sync();
    tc::tmem_dealloc(s.tmem, tc::TMEM_COLS);
  }
}

}  // namespace

cudaError_t launch_sensor_mask(const MaskArgs& a, cudaStream_t s) {
  const int smem = (int)sizeof(tc::Smem) + 128;
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(sensor_mask_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  const long nf = (long)(a.d.IM - 1) * (a.d.JM - 2) * (a.d.KM - 2) + (long)(a.d.IM - 2) * (a.d.JM - 1) * (a.d.KM - 2) +
                  (long)(a.d.IM - 2) * (a.d.JM - 2) * (a.d.KM - 1);
  const long ntiles = (nf + 127) / 128;
  // 8 CTAs per SM fill the 512 TMEM columns (64 each) and hide the MMA round trips
  const unsigned grid = (unsigned)(ntiles < 148L * 8 ? ntiles : 148L * 8);
  sensor_mask_kernel<<<grid, 128, smem, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_mlp_predict_tc(const float* P, const float* X, unsigned n, float* out, int* fail, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  const int smem = (int)sizeof(tc::Smem) + 128;
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(mlp_predict_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  const unsigned ntiles = (n + 127) / 128;
  const unsigned grid = ntiles < 592u ? ntiles : 592u;
  mlp_predict_tc_kernel<<<grid, 128, smem, s>>>(P, X, n, out, fail);
  return cudaGetLastError();
}

}  // namespace cbns
