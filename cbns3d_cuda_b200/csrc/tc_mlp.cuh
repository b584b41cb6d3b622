// tc_mlp.cuh - the sensor network on the 5th-generation tensor cores
// (tcgen05, sm_100a): BF16 operands in shared memory, FP32 accumulators in
// tensor memory, one elected thread issuing the MMAs, completion through an
// mbarrier with a bounded wait.
//
// One tile = 128 faces (MMA M = 128).  Layer 1: D1[128x32] = X[128x16] W1'[32x16]^T
// where column 15 of X is 1 and column 15 of W1' is b1 (bias folded into K).
// Layer 2: D2[128x32] = relu(D1)[128x32] W2[32x32]^T (two K = 16 MMAs) plus
// b2 through a third MMA, ONE[128x16] B2'[32x16]^T, where columns 0 and 1 of
// ONE are 1 and of B2' the BF16 high and low parts of b2 (b2 to ~16 bits).
// The output layer (32 -> 1, plus b3) runs on the CUDA cores from the FP32
// accumulators.
//
// Shared-memory operands use the canonical K-major layout without swizzle:
// 8-row x 16-byte core matrices, element (r, k) at
//   (r / 8) * SBO + (k / 8) * 128 + (r % 8) * 16 + (k % 8) * 2   bytes,
// LBO = 128 (next 8 K-elements), SBO = 128 * K / 8 (next 8 rows).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "sensor.cuh"

namespace cbns {
namespace tc {

// bytes of one operand tile
constexpr int X_BYTES = 128 * 16 * 2;   // layer-1 A: 128 x 16
constexpr int H_BYTES = 128 * 32 * 2;   // layer-2 A: 128 x 32
constexpr int W1_BYTES = 32 * 16 * 2;   // layer-1 B: 32 x 16
constexpr int W2_BYTES = 32 * 32 * 2;   // layer-2 B: 32 x 32
constexpr int B2_BYTES = 32 * 16 * 2;   // layer-2 bias B: 32 x 16
constexpr unsigned TMEM_COLS = 64;      // D1 at columns 0..31, D2 at 32..63
constexpr unsigned WAIT_LIMIT = 1u << 20;

// instruction descriptor: D = F32, A = B = BF16, both K-major, N = 32, M = 128
constexpr unsigned IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((32u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

// shared-memory matrix descriptor: start, LBO, SBO (bytes), version 1, no swizzle
__device__ __forceinline__ unsigned long long sdesc(unsigned addr, unsigned lbo, unsigned sbo) {
  return (unsigned long long)((addr >> 4) & 0x3FFFu) | ((unsigned long long)((lbo >> 4) & 0x3FFFu) << 16) |
         ((unsigned long long)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// byte offset of element (r, k) in a K-major no-swizzle tile with K columns
__device__ __forceinline__ int kmajor_off(int r, int k, int K) {
  return (r >> 3) * (16 * K) + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2;
}

__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// warp-collective TMEM allocation; the address lands in *slot (shared)
__device__ __forceinline__ void tmem_alloc(unsigned* slot, unsigned ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)), "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(unsigned taddr, unsigned ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void mbar_init(unsigned long long* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Wait for the given phase with an iteration limit; false on timeout.  Each
// try_wait may suspend the thread (SUSPEND_NS is the hint) before it returns
// false, so the wait costs few instructions; it is bounded by WAIT_LIMIT
// tries (4.2 s measured on a B200, whose try_wait suspends about 4 us).
constexpr unsigned SUSPEND_NS = 1000;
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned phase) {
  const unsigned a = smem_u32(bar);
  for (unsigned it = 0; it < WAIT_LIMIT; ++it) {
    unsigned done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(phase), "r"(SUSPEND_NS)
        : "memory");
    if (done) return true;
  }
  return false;
}

// one MMA: D[tmem] (+)= A * B^T, issued by the calling thread
__device__ __forceinline__ void mma_bf16(unsigned d_tmem, unsigned long long adesc, unsigned long long bdesc,
                                         bool accumulate) {
  const unsigned acc = accumulate ? 1u : 0u, z = 0u;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
      ::"r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(IDESC), "r"(acc), "r"(z), "r"(z), "r"(z), "r"(z)
      : "memory");
}

__device__ __forceinline__ void mma_commit(unsigned long long* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

// 32 consecutive FP32 columns of this thread's TMEM lane (warp w of a
// warpgroup reads lanes 32w .. 32w+31)
__device__ __forceinline__ void tmem_ld32(unsigned taddr, float v[32]) {
  unsigned r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// 16 consecutive FP32 columns of this thread's TMEM lane
__device__ __forceinline__ void tmem_ld16(unsigned taddr, float v[16]) {
  unsigned r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Shared memory of the tensor-core MLP (all operand tiles 128-byte aligned).
struct alignas(128) Smem {
  unsigned char x[X_BYTES];    // layer-1 A (features + constant 1)
  unsigned char h[H_BYTES];    // layer-2 A (relu(D1))
  unsigned char one[X_BYTES];  // bias A (columns 0, 1 = 1)
  unsigned char w1[W1_BYTES];  // layer-1 B ([W1 | b1])
  unsigned char w2[W2_BYTES];  // layer-2 B (W2)
  unsigned char b2[B2_BYTES];  // bias B (columns 0, 1 = b2 high, low)
  alignas(16) float w3[SN_H];
  float b3;
  unsigned long long bar;
  unsigned tmem;
  int failed;
};

// Stage the weights (FP32 parameter vector P) into the B operands.
__device__ __forceinline__ void load_weights(Smem& s, const float* P, int t, int nthreads) {
  for (int e = t; e < SN_H * 16; e += nthreads) {
    const int n = e >> 4, k = e & 15;
    const float v = k < SN_IN ? P[SP_W1 + n * SN_IN + k] : P[SP_B1 + n];
    *reinterpret_cast<__nv_bfloat16*>(s.w1 + kmajor_off(n, k, 16)) = __float2bfloat16_rn(v);
  }
  for (int e = t; e < SN_H * SN_H; e += nthreads) {
    const int n = e >> 5, k = e & 31;
    *reinterpret_cast<__nv_bfloat16*>(s.w2 + kmajor_off(n, k, 32)) = __float2bfloat16_rn(P[SP_W2 + e]);
  }
  for (int e = t; e < SN_H * 16; e += nthreads) {
    const int n = e >> 4, k = e & 15;
    const float b = P[SP_B2 + n];
    const __nv_bfloat16 hi = __float2bfloat16_rn(b);
    const float v = k == 0 ? b : (k == 1 ? b - __bfloat162float(hi) : 0.0f);
    *reinterpret_cast<__nv_bfloat16*>(s.b2 + kmajor_off(n, k, 16)) = __float2bfloat16_rn(v);
  }
  for (int e = t; e < 128 * 16; e += nthreads) {
    const int r = e >> 4, k = e & 15;
    *reinterpret_cast<__nv_bfloat16*>(s.one + kmajor_off(r, k, 16)) = __float2bfloat16_rn(k < 2 ? 1.0f : 0.0f);
  }
  for (int e = t; e < SN_H; e += nthreads) s.w3[e] = P[SP_W3 + e];
  if (t == 0) s.b3 = P[SP_B3];
}

// Write one feature row (15 features, then the constant 1) of the layer-1 A tile.
__device__ __forceinline__ void put_features(Smem& s, int row, const float f[SN_IN]) {
#pragma unroll
  for (int k = 0; k < 16; k += 2) {
    const float a = f[k], b = k + 1 < SN_IN ? f[k + 1] : 1.0f;
    *reinterpret_cast<__nv_bfloat162*>(s.x + kmajor_off(row, k, 16)) = __floats2bfloat162_rn(a, b);
  }
}

// Run both layers for the 128-row tile in s.x.  Called by all threads of the
// CTA; warps 0..3 hold the 128 rows (thread 32w+l <-> row 32w+l) and return
// the logit of their row in *logit.  phase: the mbarrier phase parity to wait
// for next (flips twice per call).  Returns false if a wait timed out.
__device__ __forceinline__ bool run_tile(Smem& s, int t, unsigned& phase, float* logit) {
  fence_async_smem();
  fence_before_sync();
  __syncthreads();
  const unsigned tmem = s.tmem;
  if (t == 0) {
    fence_after_sync();
    mma_bf16(tmem, sdesc(smem_u32(s.x), 128, 256), sdesc(smem_u32(s.w1), 128, 256), false);
    mma_commit(&s.bar);
  }
  // warp 0 waits on the barrier, the other warps at the CTA barrier (which
  // issues nothing); every thread then takes the same branch.  A wait that
  // runs out is given a second bounded window: an MMA whose commit has not
  // arrived may still own its accumulator columns, and the caller frees TMEM
  // once this returns false, so the MMA gets every chance to retire first; if
  // it has not after both windows, the tensor pipe is making no progress and
  // the caller's failure flag is the only recourse.
  const int warp = t >> 5;
  bool ok = warp == 0 ? (mbar_wait(&s.bar, phase) || mbar_wait(&s.bar, phase)) : true;
  phase ^= 1u;
  if (!__syncthreads_and(ok)) return false;
  fence_after_sync();
  if (warp < 4) {
    const int row = t;
#pragma unroll
    for (int half = 0; half < 2; ++half) {  // two 16-column loads keep register pressure down
      float d1[16];
      tmem_ld16(tmem + ((unsigned)(32 * warp) << 16) + 16 * half, d1);
#pragma unroll
      for (int k = 0; k < 16; k += 2) {
        *reinterpret_cast<__nv_bfloat162*>(s.h + kmajor_off(row, 16 * half + k, 32)) =
            __floats2bfloat162_rn(fmaxf(d1[k], 0.f), fmaxf(d1[k + 1], 0.f));
      }
    }
  }
  fence_async_smem();
  fence_before_sync();
  __syncthreads();
  if (t == 0) {
    fence_after_sync();
    const unsigned ha = smem_u32(s.h), wa = smem_u32(s.w2);
    mma_bf16(tmem + 32, sdesc(ha, 128, 512), sdesc(wa, 128, 512), false);
    mma_bf16(tmem + 32, sdesc(ha + 256, 128, 512), sdesc(wa + 256, 128, 512), true);
    mma_bf16(tmem + 32, sdesc(smem_u32(s.one), 128, 256), sdesc(smem_u32(s.b2), 128, 256), true);
    mma_commit(&s.bar);
  }
  ok = warp == 0 ? (mbar_wait(&s.bar, phase) || mbar_wait(&s.bar, phase)) : true;
  phase ^= 1u;
  if (!__syncthreads_and(ok)) return false;
  fence_after_sync();
  if (warp < 4) {
    float z = s.b3;
    const float4* w3 = reinterpret_cast<const float4*>(s.w3);
#pragma unroll
    for (int half = 0; half < 2; ++half) {
      float d2[16];
      tmem_ld16(tmem + ((unsigned)(32 * warp) << 16) + 32 + 16 * half, d2);
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const float4 w = w3[4 * half + k];
        z += w.x * fmaxf(d2[4 * k], 0.f) + w.y * fmaxf(d2[4 * k + 1], 0.f) + w.z * fmaxf(d2[4 * k + 2], 0.f) +
             w.w * fmaxf(d2[4 * k + 3], 0.f);
      }
    }
    *logit = z;
  }
  fence_before_sync();
  __syncthreads();  // the next tile may overwrite x, h and the accumulators
  return ok;
}

}  // namespace tc
}  // namespace cbns
