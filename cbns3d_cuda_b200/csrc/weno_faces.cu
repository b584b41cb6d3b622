// weno_faces.cu - the WENO5 faces of a hybrid stage, evaluated ahead of the
// stage kernel.
//
// The learned sensor sends about one face in eight to the characteristic
// WENO5 flux (the reference's rec_riemann kernels, src/rec_riemann_kernel.cu,
// called from calc_numerical_flux, src/calc_numerical_flux.cu:15-74) and the
// rest to the linear upwind-5 flux.  Evaluating both inside the stage kernel
// gives the whole stage kernel the register budget and the control flow of
// WENO5 while most of its work is linear.  So, per step, the faces whose
// decision byte is set are listed once (weno_list_kernel), and per stage this
// pass evaluates the listed faces into a face array (8 floats per face, 5
// used: one 16-byte and one 4-byte access), where the stage kernel, which
// holds only the linear flux, reads them.  While force_weno is set (the audit
// rejected the step's decisions, or the sensor timed out) the pass evaluates
// every face.
//
// Stencils are read from the stage input in FP64 and rounded to FP32 as the
// stage kernel rounds its staged copies, and the face normals are formed from
// the same FP32 area vectors, so a face gets the flux the stage kernel would
// compute for it.
#include "cbns_common.cuh"
#include "face_flux.cuh"
#include "sensor_kernels.cuh"
#include "stage.cuh"

namespace cbns {

namespace {

constexpr int LT = 256;       // list kernel: threads
constexpr int LB = 16;        // decision bytes per thread (one 16-byte load)
constexpr int LCH = LT * LB;  // faces per CTA
constexpr int WT = 256;       // evaluation kernel: threads

// A list entry: the face index and, packed, its kind (0 i-, 1 j-, 2 k-face,
// bits 30-31) and the node offset of its low node (bits 0-29; contexts of the
// hybrid precision keep VOL below 2^30).
__device__ __forceinline__ int2 list_entry(long e, int kind, long oa) {
  return make_int2((int)e, (int)(((unsigned)kind << 30) | (unsigned)oa));
}

// Walks faces in index order: the kind and low-node offset of a face, decoded
// by 32-bit divisions at the start and wherever a row or a kind ends, stepped
// along the row otherwise (faces of every kind are numbered i fastest).
struct FaceCursor {
  long e;        // face index
  int kind;      // 0 i, 1 j, 2 k
  int i, ni;     // position in the row and row length
  long oa;       // low-node offset
  long kind_end; // first face index of the next kind
};

__device__ __forceinline__ void cursor_set(const Dims& d, long nfi, long nfj, long e, FaceCursor& c) {
  c.e = e;
  if (e < nfi) {
    const unsigned ni = (unsigned)(d.IM - 1), nj = (unsigned)(d.JM - 2);
    const unsigned u = (unsigned)e, r = u / ni;
    c.kind = 0;
    c.i = (int)(u - r * ni);
    c.ni = (int)ni;
    c.oa = node_off(d, c.i, (int)(r % nj) + 1, (int)(r / nj) + 1);
    c.kind_end = nfi;
  } else if (e < nfi + nfj) {
    const unsigned ni = (unsigned)(d.IM - 2), nj = (unsigned)(d.JM - 1);
    const unsigned u = (unsigned)(e - nfi), r = u / ni;
    c.kind = 1;
    c.i = (int)(u - r * ni);
    c.ni = (int)ni;
    c.oa = node_off(d, c.i + 1, (int)(r % nj), (int)(r / nj) + 1);
    c.kind_end = nfi + nfj;
  } else {
    const unsigned ni = (unsigned)(d.IM - 2), nj = (unsigned)(d.JM - 2);
    const unsigned u = (unsigned)(e - nfi - nfj), r = u / ni;
    c.kind = 2;
    c.i = (int)(u - r * ni);
    c.ni = (int)ni;
    c.oa = node_off(d, c.i + 1, (int)(r % nj) + 1, (int)(r / nj));
    c.kind_end = 0x7fffffffffffffffL;
  }
}

// The faces of one kind: the first face index and the count (i-faces, then
// j-faces, then k-faces in the global face numbering).
__host__ __device__ __forceinline__ void kind_range(const Dims& d, int kind, long* first, long* count) {
  const long nfi = (long)(d.IM - 1) * (d.JM - 2) * (d.KM - 2);
  const long nfj = (long)(d.IM - 2) * (d.JM - 1) * (d.KM - 2);
  const long nfk = (long)(d.IM - 2) * (d.JM - 2) * (d.KM - 1);
  *first = kind == 0 ? 0 : (kind == 1 ? nfi : nfi + nfj);
  *count = kind == 0 ? nfi : (kind == 1 ? nfj : nfk);
}

// CTAs of the list kernel for one kind: chunks of LCH faces from the kind's
// first face rounded down to a 16-byte boundary of the mask.
__host__ __device__ __forceinline__ int list_ctas_kind(const Dims& d, int kind) {
  long first, count;
  kind_range(d, kind, &first, &count);
  const long a = first & ~15L;
  return (int)((first + count - a + LCH - 1) / LCH);
}

// List the faces whose decision is set, each kind in its own list (the list
// array's range from the kind's first face index on), so that the evaluation
// pass can walk the three kinds side by side, plane by plane.  One 16-byte
// load of decisions per thread; a CTA-wide scan of the counts and one global
// atomic per CTA place the CTA's faces in its kind's list, in face order
// within the CTA.  The decisions change only on the steps the network runs
// (sensor_step), so on the others the lists of the last such step stand.
__device__ __forceinline__ void list_body(const Dims& d, const unsigned char* __restrict__ mask, long nf, StepState* st,
                                          int2* __restrict__ list, int check_done, unsigned every, unsigned bx) {
  __shared__ int wsum[LT / 32];
  __shared__ int cbase;
  if ((check_done && st->done) || !sensor_step(st, every)) return;
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  int kind = 0;
  unsigned chunk = bx;
  for (; kind < 2; ++kind) {
    const unsigned ck = (unsigned)list_ctas_kind(d, kind);
    if (chunk < ck) break;
    chunk -= ck;
  }
  long first, count;
  kind_range(d, kind, &first, &count);
  const long f0 = (first & ~15L) + (long)chunk * LCH + (long)t * LB;  // 16-byte aligned
  unsigned bits = 0;
  if (f0 + LB <= nf) {
    const uint4 v = __ldg(reinterpret_cast<const uint4*>(mask + f0));
    const unsigned w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
      for (int b = 0; b < 4; ++b)
        if ((w[q] >> (8 * b)) & 0xffu) bits |= 1u << (4 * q + b);
  } else {
    for (int b = 0; b < LB && f0 + b < nf; ++b)
      if (__ldg(mask + f0 + b)) bits |= 1u << b;
  }
  // only this kind's faces
#pragma unroll
  for (int b = 0; b < LB; ++b)
    if (f0 + b < first || f0 + b >= first + count) bits &= ~(1u << b);
  const int n = __popc(bits);
  int incl = n;
#pragma unroll
  for (int s = 1; s < 32; s <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, incl, s);
    if (lane >= s) incl += y;
  }
  if (lane == 31) wsum[warp] = incl;
  __syncthreads();
  if (t == 0) {
    int tot = 0;
    for (int w = 0; w < LT / 32; ++w) {
      const int c = wsum[w];
      wsum[w] = tot;
      tot += c;
    }
    cbase = tot ? (int)atomicAdd(&st->weno_listed[kind], (unsigned)tot) : 0;
  }
  __syncthreads();
  long pos = first + cbase + wsum[warp] + incl - n;
  if (!bits) return;
  const long nfi = (long)(d.IM - 1) * (d.JM - 2) * (d.KM - 2);
  const long nfj = (long)(d.IM - 2) * (d.JM - 1) * (d.KM - 2);
  // the cursor starts at the thread's first face of this kind
  const int b0 = __ffs(bits) - 1;
  FaceCursor c;
  cursor_set(d, nfi, nfj, f0 + b0, c);
  for (int b = b0; b < LB; ++b) {
    if ((bits >> b) & 1u) list[pos++] = list_entry(c.e, c.kind, c.oa);
    if (b == LB - 1 || !(bits >> (b + 1))) break;
    // advance to face f0 + b + 1
    if (c.e + 1 == c.kind_end || c.i + 1 == c.ni) {
      cursor_set(d, nfi, nfj, c.e + 1, c);  // next kind, or next row (which may start a new plane)
    } else {
      ++c.e;
      ++c.i;
      ++c.oa;
    }
  }
}

__global__ void __launch_bounds__(LT) weno_list_kernel(const Dims d, const unsigned char* __restrict__ mask, long nf,
                                                       StepState* st, int2* __restrict__ list, int check_done,
                                                       unsigned every) {
  list_body(d, mask, nf, st, list, check_done, every, blockIdx.x);
}

// Zero the lists' lengths on the steps the lists are built anew.
__global__ void weno_list_reset(StepState* st, int check_done, unsigned every) {
  if (threadIdx.x < 3 && !(check_done && st->done) && sensor_step(st, every)) st->weno_listed[threadIdx.x] = 0;
}

// Many blocks: zero every block's count, then list every block's faces (block
// b owning CTAs cta[b] .. cta[b+1]-1).
__global__ void weno_list_reset_batched(const ListArgs* args, int nblocks) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b < nblocks && !(args[b].check_done && args[b].st->done) && sensor_step(args[b].st, args[b].every))
    for (int k = 0; k < 3; ++k) args[b].st->weno_listed[k] = 0;
}

__global__ void __launch_bounds__(LT) weno_list_batched(const ListArgs* args, const int* cta, int nblocks) {
  const int b = block_of_cta(cta, nblocks, (int)blockIdx.x);
  const ListArgs& a = args[b];
  list_body(a.d, a.mask, a.nf, a.st, a.list, a.check_done, a.every, blockIdx.x - (unsigned)__ldg(cta + b));
}

// The WENO5 flux of one face of a's stage input into a.wflux: face w of the
// list (or, with all set, face w of the block).  Each thread stages its face's
// stencil in FP32 in its own column of shared memory (my, stride WT), so the
// flux reads it there instead of keeping it in registers.
__device__ __forceinline__ void weno_face(const StageArgs& a, bool all, long w, const int2* list, float* my) {
  const Dims& d = a.d;
  const long VOL = d.VOL;
  long e, oa;
  int kind;
  if (all) {
    const long nfi = (long)(d.IM - 1) * (d.JM - 2) * (d.KM - 2);
    const long nfj = (long)(d.IM - 2) * (d.JM - 1) * (d.KM - 2);
    FaceCursor c;
    cursor_set(d, nfi, nfj, w, c);
    e = w;
    kind = c.kind;
    oa = c.oa;
  } else {
    const int2 le = __ldg(list + w);
    e = le.x;
    kind = (int)((unsigned)le.y >> 30);
    oa = (long)((unsigned)le.y & 0x3fffffffu);
  }
  long o0, s;  // first stencil node and the stride along the face normal
  float nx, ny, nz;
  if (kind == 0) {
    // i-face between node oa and the next along i
    o0 = oa - 2;
    s = 1;
    nx = 0.5f * (__ldg(a.area32[0] + oa) + __ldg(a.area32[0] + oa + 1));
    ny = 0.5f * (__ldg(a.area32[1] + oa) + __ldg(a.area32[1] + oa + 1));
    nz = 0.5f * (__ldg(a.area32[2] + oa) + __ldg(a.area32[2] + oa + 1));
  } else if (kind == 1) {
    // j-face between node oa and the next along j
    o0 = oa - 2 * d.PX;
    s = d.PX;
    nx = 0.5f * (__ldg(a.area32[3] + oa) + __ldg(a.area32[3] + oa + d.PX));
    ny = 0.5f * (__ldg(a.area32[4] + oa) + __ldg(a.area32[4] + oa + d.PX));
    nz = 0.5f * (__ldg(a.area32[5] + oa) + __ldg(a.area32[5] + oa + d.PX));
  } else {
    // k-face between node oa and the next along k
    o0 = oa - 2 * d.PL;
    s = d.PL;
    nx = 0.5f * ((float)__ldg(a.area[6] + oa) + (float)__ldg(a.area[6] + oa + d.PL));
    ny = 0.5f * ((float)__ldg(a.area[7] + oa) + (float)__ldg(a.area[7] + oa + d.PL));
    nz = 0.5f * ((float)__ldg(a.area[8] + oa) + (float)__ldg(a.area[8] + oa + d.PL));
  }
  // the stencil in FP32: all 30 loads in flight at once, each value converted once
  {
    const double* sp = a.src + o0;
#pragma unroll
    for (int q = 0; q < NEQ; ++q)
#pragma unroll
      for (int p = 0; p < 6; ++p) my[(q * 6 + p) * WT] = (float)__ldg(sp + q * VOL + p * s);
  }
  auto ld = [&](int p, int q) -> float { return my[(q * 6 + p) * WT]; };
  const FluxConsts<float> C{(float)a.gamma, (float)a.gam1, (float)a.gam1_inv};
  float f[5];
  face_flux<float>(ld, nx, ny, nz, C, f);
  float* out = a.wflux + 8 * e;
  *reinterpret_cast<float4*>(out) = make_float4(f[0], f[1], f[2], f[3]);
  out[4] = f[4];
}

// One thread per listed face, or per face while force_weno is set.  The CTAs
// are shared out among the three kinds' lists in proportion to their lengths
// (at least one for a kind with faces), and each kind's CTAs walk its list
// grid-stride, so the three kinds advance through the grid's planes side by
// side and the stencils they share stay in L2.  Built for 3 CTAs per SM (80
// registers): the faces' stencil loads are the wait, and 24 warps per SM hide
// more of it than 16 (10% faster on the bench grid); the staged stencils take
// 30 KB of shared memory per CTA.
__global__ void __launch_bounds__(WT, 3) weno_faces_kernel(const __grid_constant__ StageArgs a, int mode, long nf,
                                                           const int2* list) {
  __shared__ float stn[NEQ * 6][WT];
  const StepState* st = a.st;
  if (mode != 0 && st->done) return;
  const bool all = st->force_weno != 0;
  long first[3], len[3];
  for (int k = 0; k < 3; ++k) {
    long cnt;
    kind_range(a.d, k, &first[k], &cnt);
    len[k] = all ? cnt : (long)st->weno_listed[k];
  }
  const long tot = len[0] + len[1] + len[2];
  if (tot == 0) return;
  const int G = gridDim.x;
  int b1 = (int)((len[0] * G + tot - 1) / tot), b2 = (int)(((len[0] + len[1]) * G + tot - 1) / tot);
  b1 = min(max(b1, len[0] > 0 ? 1 : 0), G - (len[1] > 0 ? 1 : 0) - (len[2] > 0 ? 1 : 0));
  b2 = min(max(b2, b1 + (len[1] > 0 ? 1 : 0)), G - (len[2] > 0 ? 1 : 0));
  const int c = blockIdx.x;
  const int k = c < b1 ? 0 : (c < b2 ? 1 : 2);
  const int base = k == 0 ? 0 : (k == 1 ? b1 : b2);
  const int g = k == 0 ? b1 : (k == 1 ? b2 - b1 : G - b2);
  for (long w = (long)(c - base) * WT + threadIdx.x; w < len[k]; w += (long)g * WT)
    weno_face(a, all, first[k] + w, list, &stn[0][threadIdx.x]);
}

int g_weno_grid = 0;  // persistent grid of the evaluation kernel: resident CTAs of the device

}  // namespace

cudaError_t weno_prepare() {
  if (g_weno_grid) return cudaSuccess;
  int per_sm = 0, dev = 0, nsm = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, weno_faces_kernel, WT, 0);
  if (e == cudaSuccess) e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return e;
  g_weno_grid = nsm * (per_sm > 0 ? per_sm : 1);
  return cudaSuccess;
}

cudaError_t launch_weno_list(const Dims& d, const unsigned char* mask, long nfaces, StepState* st, int2* list,
                             bool check_done, unsigned every, cudaStream_t s) {
  weno_list_reset<<<1, 32, 0, s>>>(st, check_done, every);
  if (nfaces > 0)
    weno_list_kernel<<<(unsigned)weno_list_ctas(d), LT, 0, s>>>(d, mask, nfaces, st, list, check_done, every);
  return cudaGetLastError();
}

int weno_list_ctas(const Dims& d) { return list_ctas_kind(d, 0) + list_ctas_kind(d, 1) + list_ctas_kind(d, 2); }

cudaError_t launch_weno_list_batched(const ListArgs* args, const int* cta, int nblocks, int total, cudaStream_t s) {
  weno_list_reset_batched<<<(nblocks + 255) / 256, 256, 0, s>>>(args, nblocks);
  if (total > 0) weno_list_batched<<<total, LT, 0, s>>>(args, cta, nblocks);
  return cudaGetLastError();
}

cudaError_t launch_weno_faces(const StageArgs& a, int mode, long nfaces, const int2* list, cudaStream_t s) {
  cudaError_t e = weno_prepare();
  if (e != cudaSuccess || nfaces <= 0) return e;
  weno_faces_kernel<<<g_weno_grid, WT, 0, s>>>(a, mode, nfaces, list);
  return cudaGetLastError();
}

}  // namespace cbns
