// tma.cuh - tensor-memory-accelerator (TMA) tile loads into shared memory
// with mbarrier completion, for the stage kernel's plane staging.
//
// A 4-D tiled tensor map describes one family of node arrays in the library's
// layout (cbns_common.cuh): dim 0 = x (the padded row, PX elements), dim 1 =
// the JG rows, dim 2 = the KG planes, dim 3 = the fields (VOL elements apart).
// One cp.async.bulk.tensor copies a box of that tensor -- (x, rows, 1 plane,
// fields) -- into shared memory and signals the transferred bytes on an
// mbarrier.  Rules kept by every caller: the box's x coordinate times the
// element size is a multiple of 16 bytes, every shared-memory destination is
// 128-byte aligned, and the tensor maps describe this GPU's own memory (no
// cluster multicast anywhere).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

namespace cbns {
namespace tma {

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void bar_init(unsigned long long* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void bar_inval(unsigned long long* bar) {
  asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}
// make the initialised barriers visible to the async proxy (the TMA unit)
__device__ __forceinline__ void fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
// order this thread's earlier generic-proxy shared-memory accesses (made
// visible to it by a CTA barrier) before the async-proxy writes it issues next
__device__ __forceinline__ void fence_proxy() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// the issuing thread's arrival, announcing `bytes` of transactions
__device__ __forceinline__ void bar_expect(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

// Wait for the phase of the given parity with an iteration limit; false on
// timeout.  Each try_wait may suspend the thread for up to kSuspendNs, so the
// wait is bounded by kWaitLimit tries (4.2 s measured on a B200, whose
// try_wait suspends about 4 us per try).
constexpr unsigned kWaitLimit = 1u << 20;
constexpr unsigned kSuspendNs = 1000;
__device__ __forceinline__ bool bar_wait(unsigned long long* bar, unsigned parity) {
  const unsigned a = smem_u32(bar);
  for (unsigned it = 0; it < kWaitLimit; ++it) {
    unsigned done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity), "r"(kSuspendNs)
        : "memory");
    if (done) return true;
  }
  return false;
}

// box of the 4-D tensor at (x, y, z, f) -> dst, completion on bar
__device__ __forceinline__ void load_4d(void* dst, const CUtensorMap* map, int x, int y, int z, int f,
                                        unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(z), "r"(f), "r"(smem_u32(bar))
      : "memory");
}

}  // namespace tma

// Host: encode a 4-D tiled tensor map over `fields` node arrays of element
// size `esize` (4 or 8 bytes) that start at `base`, VOL elements apart, with
// the box (bx, by, 1, bf).  Returns false if the driver rejects it.
bool encode_node_map(CUtensorMap* map, const void* base, int esize, long PX, long JG, long KG, long VOL, int fields,
                     unsigned bx, unsigned by, unsigned bf);

}  // namespace cbns
