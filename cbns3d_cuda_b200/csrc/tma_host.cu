// tma_host.cu - host-side encoding of the 4-D tiled tensor maps of tma.cuh,
// through the driver's cuTensorMapEncodeTiled (looked up once through the
// runtime, so the library needs no link against libcuda).
#include <cudaTypedefs.h>

#include <mutex>

#include "tma.cuh"

namespace cbns {

namespace {
PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
std::once_flag g_once;
}  // namespace

bool encode_node_map(CUtensorMap* map, const void* base, int esize, long PX, long JG, long KG, long VOL, int fields,
                     unsigned bx, unsigned by, unsigned bf) {
  std::call_once(g_once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    cudaGetLastError();
  });
  if (!g_encode || (esize != 4 && esize != 8)) return false;
  const cuuint64_t dims[4] = {(cuuint64_t)PX, (cuuint64_t)JG, (cuuint64_t)KG, (cuuint64_t)fields};
  const cuuint64_t strides[3] = {(cuuint64_t)(PX * esize), (cuuint64_t)(PX * JG * esize), (cuuint64_t)(VOL * esize)};
  const cuuint32_t box[4] = {bx, by, 1u, bf};
  const cuuint32_t estr[4] = {1u, 1u, 1u, 1u};
  const CUresult r = g_encode(map, esize == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4,
                              const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                              CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

}  // namespace cbns
