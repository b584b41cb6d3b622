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

// Per-step decisions of the hybrid flux, in directional sweeps.  A work item
// is up to SW_CH tiles of 128 faces:
//   i-faces: 128 consecutive faces of SW_CH grid rows (j, k); each row's node
//            primitives (i0-2 .. i0+130) are staged in shared memory, the
//            next row's loads in flight while the current row is classified;
//   j-faces: a segment of 128 i-columns at one k, SW_CH consecutive faces
//            along j; every thread keeps its column's 6-node window of
//            primitives in registers and loads one node ahead per face;
//   k-faces: the same along k at one j.
// So each node's primitives are formed once per direction, and a tile's
// loads are coalesced along i.  A tile whose faces all have flat stencils is
// decided linear at once; any other tile goes through the network on the
// tensor cores and each thread writes the decision byte of its face.
constexpr int SW_T = 128;  // faces per tile = threads per CTA
constexpr int SW_CH = 30;  // tiles per work item (a multiple of the 6-face window rotation)

struct RowSmem {
  float pr[5][SW_T + 8];  // r, p, u, v, w of nodes i0-2 .. i0+130
  float ax[3][SW_T + 4];  // J grad(xi) of nodes i0 .. i0+128
};

// The window sweeps stream each column's nodes through a per-thread ring of
// SW_D slots filled by asynchronous copies (cp.async), SW_D faces ahead: slot
// u % SW_D holds the 5 state values of node f0+3+u and the area vector of
// node f0+1+u for face f0+u.  Two slots keep the sweep at 5 CTAs per SM (16
// KB of ring; four slots and 4 CTAs per SM measured 2% slower).
constexpr int SW_D = 2;
struct WinSmem {
  double v[SW_D][8][SW_T];
};

__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(tc::smem_u32(smem)), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_ring() {
  asm volatile("cp.async.wait_group %0;" ::"n"(SW_D - 1) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

struct SweepCtx {
  tc::Smem* s;
  unsigned phase;
  float zcut;
  unsigned char* mask;
};

// Decision of the thread's face e (when valid) from its features f; false if
// a tensor-core wait timed out.  Called by all threads of the CTA.
__device__ __forceinline__ bool classify(SweepCtx& c, int t, const float f[SN_IN], bool valid, long e) {
  unsigned char dec = 0;
  const bool flat = feature_l1(f) < SN_FLAT;  // false for NaN features
  if (!__syncthreads_and(!valid || flat)) {
    tc::put_features(*c.s, t, f);
    float z = 0.f;
    if (!tc::run_tile(*c.s, t, c.phase, &z)) return false;
    // non-finite features (e.g. a non-physical state) fall back to WENO5
    dec = (!flat && (z >= c.zcut || !(z == z))) ? 1 : 0;
  }
  if (valid) c.mask[e] = dec;
  return true;
}

// One work item (KIND 0: i-face rows; KIND 1: j- or k-face window sweeps) of
// the block a: its decisions into a.mask.  Called by all threads of the CTA;
// false if a tensor-core wait timed out (the CTA then classifies nothing more).
template <int KIND>
__device__ __forceinline__ bool mask_item(const MaskArgs& a, long item, SweepCtx& cx, RowSmem& rs, WinSmem& ws, int t) {
  const Dims& d = a.d;
  const int IM = d.IM, JM = d.JM, KM = d.KM;
  const long VOL = d.VOL;
  const long nfi = (long)(IM - 1) * (JM - 2) * (KM - 2);
  const long nfj = (long)(IM - 2) * (JM - 1) * (KM - 2);
  const int nseg0 = (IM - 1 + SW_T - 1) / SW_T, nseg = (IM - 2 + SW_T - 1) / SW_T;
  const int rows = (JM - 2) * (KM - 2);
  const long n0 = (long)nseg0 * ((rows + SW_CH - 1) / SW_CH);
  const long n1 = (long)nseg * (KM - 2) * ((JM - 1 + SW_CH - 1) / SW_CH);
  const long n2 = (long)nseg * (JM - 2) * ((KM - 1 + SW_CH - 1) / SW_CH);
  const float gamma = a.gamma, gam1 = a.gam1;
  bool ok = true;

  auto load_q = [&](const double* p, double q[5]) {
#pragma unroll
    for (int n = 0; n < 5; ++n) q[n] = __ldg(p + n * VOL);
  };
  auto prim_of = [&](const double q[5]) {
    return node_prim((float)q[0], (float)q[1], (float)q[2], (float)q[3], (float)q[4], gam1);
  };

  float f[SN_IN];
  if (KIND == 0) {  // i-faces, row by row
    const int seg = (int)(item % nseg0), rc = (int)(item / nseg0);
    const int i0 = seg * SW_T;
    const int r0 = rc * SW_CH, r1 = min(rows, (rc + 1) * SW_CH);
    // this thread's share of a row: node x = t (and x = SW_T + t for t < 5)
    // and the area vector of node x = t (and x = SW_T for t = 0); the next
    // row's share is loaded while the current row goes through the network
    double q0[5], q1[5], a0[3], a1[3];
    auto fetch = [&](int r) {
      const int j = 1 + r % (JM - 2), k = 1 + r / (JM - 2);
      const int ia = i0 - 2 + t, ib = i0 - 2 + SW_T + t;
      if (ia <= IM + 1) load_q(a.q + node_off(d, ia, j, k), q0);
      if (t < 5 && ib <= IM + 1) load_q(a.q + node_off(d, ib, j, k), q1);
      if (i0 + t <= IM + 1) {
        const long o = node_off(d, i0 + t, j, k);
#pragma unroll
        for (int m = 0; m < 3; ++m) a0[m] = __ldg(a.area[m] + o);
      }
      if (t == 0 && i0 + SW_T <= IM + 1) {
        const long o = node_off(d, i0 + SW_T, j, k);
#pragma unroll
        for (int m = 0; m < 3; ++m) a1[m] = __ldg(a.area[m] + o);
      }
    };
    auto put = [&](int x, const double q[5]) {
      const NodePrim p = prim_of(q);
      rs.pr[0][x] = p.r;
      rs.pr[1][x] = p.p;
      rs.pr[2][x] = p.u;
      rs.pr[3][x] = p.v;
      rs.pr[4][x] = p.w;
    };
    fetch(r0);
    for (int r = r0; ok && r < r1; ++r) {
      const int j = 1 + r % (JM - 2), k = 1 + r / (JM - 2);
      __syncthreads();  // the previous row's staging is no longer read
      if (i0 - 2 + t <= IM + 1) put(t, q0);
      if (t < 5 && i0 - 2 + SW_T + t <= IM + 1) put(SW_T + t, q1);
      if (i0 + t <= IM + 1) {
#pragma unroll
        for (int m = 0; m < 3; ++m) rs.ax[m][t] = (float)a0[m];
      }
      if (t == 0 && i0 + SW_T <= IM + 1) {
#pragma unroll
        for (int m = 0; m < 3; ++m) rs.ax[m][SW_T] = (float)a1[m];
      }
      if (r + 1 < r1) fetch(r + 1);
      __syncthreads();
      const int i = i0 + t;
      const bool valid = i <= IM - 2;
      if (valid) {
        const float A[3] = {rs.ax[0][t], rs.ax[1][t], rs.ax[2][t]};
        const float B[3] = {rs.ax[0][t + 1], rs.ax[1][t + 1], rs.ax[2][t + 1]};
        float nx, ny, nz;
        face_unit_normal(A, B, nx, ny, nz);
        auto P = [&](int q) {
          NodePrim p;
          p.r = rs.pr[0][t + q];
          p.p = rs.pr[1][t + q];
          p.u = rs.pr[2][t + q];
          p.v = rs.pr[3][t + q];
          p.w = rs.pr[4][t + q];
          return p;
        };
        features_of(P, nx, ny, nz, gamma, f);
      } else {
#pragma unroll
        for (int m = 0; m < SN_IN; ++m) f[m] = 0.f;
      }
      ok = classify(cx, t, f, valid, i + (long)(IM - 1) * ((j - 1) + (long)(JM - 2) * (k - 1)));
    }
  } else {  // j- or k-faces: a window sweep along the direction
    const bool dj = item < n0 + n1;
    const long it = dj ? item - n0 : item - n0 - n1;
    const int seg = (int)(it % nseg);
    const long r2 = it / nseg;
    // dj: c = k (1..KM-2), faces along j; else c = j (1..JM-2), faces along k
    const int cdim = dj ? KM - 2 : JM - 2;
    const int c = 1 + (int)(r2 % cdim), ch = (int)(r2 / cdim);
    const int nface = dj ? JM - 1 : KM - 1;
    const int f0 = ch * SW_CH, f1 = min(nface, f0 + SW_CH);
    const int i = 1 + seg * SW_T + t;
    const bool valid = i <= IM - 2;
    const long sd = dj ? d.PX : d.PL;
    const int am = dj ? 3 : 6;  // J grad(eta) or J grad(zeta)
    // offset of the sweep's position 0 for this column; face fc has global
    // index e0 + fc * es
    const long obase = dj ? node_off(d, valid ? i : 1, 0, c) : node_off(d, valid ? i : 1, c, 0);
    const long e0 = dj ? nfi + (i - 1) + (long)(IM - 2) * (JM - 1) * (c - 1) : nfi + nfj + (i - 1) + (long)(IM - 2) * (c - 1);
    const long es = dj ? (long)(IM - 2) : (long)(IM - 2) * (JM - 2);
    NodePrim W0, W1, W2, W3, W4, W5;
    float Aa[3], Ab[3];
    // step u (face f0+u) consumes node f0+3+u and the area vector of node f0+1+u
    auto issue = [&](int u) {
      if (valid && f0 + u < f1) {
        const int slot = u % SW_D;
        const long on = obase + (long)(f0 + 3 + u) * sd, oa = obase + (long)(f0 + 1 + u) * sd;
#pragma unroll
        for (int n = 0; n < 5; ++n) cp_async8(&ws.v[slot][n][t], a.q + n * VOL + on);
#pragma unroll
        for (int m = 0; m < 3; ++m) cp_async8(&ws.v[slot][5 + m][t], a.area[am + m] + oa);
      }
      cp_async_commit();  // one group per step, empty or not
    };
#pragma unroll
    for (int u = 0; u < SW_D; ++u) issue(u);
    if (valid) {
      double qq[5];
      load_q(a.q + obase + (long)(f0 - 2) * sd, qq);
      W0 = prim_of(qq);
      load_q(a.q + obase + (long)(f0 - 1) * sd, qq);
      W1 = prim_of(qq);
      load_q(a.q + obase + (long)f0 * sd, qq);
      W2 = prim_of(qq);
      load_q(a.q + obase + (long)(f0 + 1) * sd, qq);
      W3 = prim_of(qq);
      load_q(a.q + obase + (long)(f0 + 2) * sd, qq);
      W4 = prim_of(qq);
#pragma unroll
      for (int m = 0; m < 3; ++m) Aa[m] = (float)__ldg(a.area[am + m] + obase + (long)f0 * sd);
    }
    // One face: the window (w0..w4 hold positions fc-2..fc+2, wn receives
    // fc+3), the area vectors of positions fc (A0) and fc+1 (A1 receives).
    // The unrolled loop below rotates the roles instead of moving values.
    auto face = [&](int fc, NodePrim& w0, NodePrim& w1, NodePrim& w2, NodePrim& w3, NodePrim& w4, NodePrim& wn,
                    float* A0, float* A1) {
      const int u = fc - f0;
      cp_async_wait_ring();  // the copies of step u have landed
      if (valid) {
        const int slot = u % SW_D;
        double nq[5];
#pragma unroll
        for (int n = 0; n < 5; ++n) nq[n] = ws.v[slot][n][t];
        wn = prim_of(nq);
#pragma unroll
        for (int m = 0; m < 3; ++m) A1[m] = (float)ws.v[slot][5 + m][t];
      }
      issue(u + SW_D);  // refill the slot just read
      if (valid) {
        float nx, ny, nz;
        face_unit_normal(A0, A1, nx, ny, nz);
        auto P = [&](int q) { return q == 0 ? w0 : q == 1 ? w1 : q == 2 ? w2 : q == 3 ? w3 : q == 4 ? w4 : wn; };
        features_of(P, nx, ny, nz, gamma, f);
      } else {
#pragma unroll
        for (int m = 0; m < SN_IN; ++m) f[m] = 0.f;
      }
      return classify(cx, t, f, valid, e0 + fc * es);
    };
    for (int fc = f0; ok && fc < f1; fc += 6) {
      ok = face(fc, W0, W1, W2, W3, W4, W5, Aa, Ab);
      if (!ok || fc + 1 >= f1) break;
      ok = face(fc + 1, W1, W2, W3, W4, W5, W0, Ab, Aa);
      if (!ok || fc + 2 >= f1) break;
      ok = face(fc + 2, W2, W3, W4, W5, W0, W1, Aa, Ab);
      if (!ok || fc + 3 >= f1) break;
      ok = face(fc + 3, W3, W4, W5, W0, W1, W2, Ab, Aa);
      if (!ok || fc + 4 >= f1) break;
      ok = face(fc + 4, W4, W5, W0, W1, W2, W3, Aa, Ab);
      if (!ok || fc + 5 >= f1) break;
      ok = face(fc + 5, W5, W0, W1, W2, W3, W4, Ab, Aa);
    }
    cp_async_wait_all();  // the ring is reused by the next item
  }
  return ok;
}

// The items of one kind of a block: [*it0, *it1) of the numbering both kinds share.
__device__ __forceinline__ void mask_items(const Dims& d, int kind, long* it0, long* it1) {
  const int nseg0 = (d.IM - 1 + SW_T - 1) / SW_T, nseg = (d.IM - 2 + SW_T - 1) / SW_T;
  const int rows = (d.JM - 2) * (d.KM - 2);
  const long n0 = (long)nseg0 * ((rows + SW_CH - 1) / SW_CH);
  const long n1 = (long)nseg * (d.KM - 2) * ((d.JM - 1 + SW_CH - 1) / SW_CH);
  const long n2 = (long)nseg * (d.JM - 2) * ((d.KM - 1 + SW_CH - 1) / SW_CH);
  *it0 = kind == 0 ? 0 : n0;
  *it1 = kind == 0 ? n0 : n0 + n1 + n2;
}

__device__ __forceinline__ float logit_cut(float tau) { return logf(tau / (1.f - tau)); }  // p >= tau <=> logit >= cut

__device__ __forceinline__ void mask_fail(StepState* st) {  // decisions incomplete: the step takes WENO5 everywhere
  atomicExch(&st->sensor_fail, 1);
  atomicExch(&st->force_weno, 1);
}

// CTA set-up of the sweeps: TMEM columns, the mbarrier, the network's weights.
struct MaskSmem {
  tc::Smem* s;
  RowSmem* rs;
  WinSmem* ws;
};
__device__ __forceinline__ MaskSmem mask_setup(const float* params, int t) {
  extern __shared__ unsigned char raw[];
  unsigned char* base = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(raw) + 127) & ~uintptr_t(127));
  MaskSmem m{reinterpret_cast<tc::Smem*>(base), reinterpret_cast<RowSmem*>(base + sizeof(tc::Smem)),
             reinterpret_cast<WinSmem*>(base + sizeof(tc::Smem))};
  if (t < 32) tc::tmem_alloc(&m.s->tmem, tc::TMEM_COLS);
  if (t == 0) tc::mbar_init(&m.s->bar);
  tc::load_weights(*m.s, params, t, SW_T);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  return m;
}

__device__ __forceinline__ void mask_teardown(const MaskSmem& m, int t) {
  tc::fence_before_sync();
  __syncthreads();
  if (t < 32) {
    tc::fence_after_sync();
    tc::tmem_dealloc(m.s->tmem, tc::TMEM_COLS);
  }
}

// KIND 0: the i-face rows; KIND 1: the j- and k-face window sweeps (two
// launches, so that each path gets its own register allocation; both at 5
// CTAs per SM).
template <int KIND>
__global__ void __launch_bounds__(SW_T, 5) sensor_mask_kernel(const MaskArgs a) {
  if ((a.check_done && a.st->done) || !sensor_step(a.st, a.every)) return;
  const int t = threadIdx.x;
  const MaskSmem m = mask_setup(a.params, t);
  SweepCtx cx{m.s, 0u, logit_cut(a.tau), a.mask};
  long it0, it1;
  mask_items(a.d, KIND, &it0, &it1);
  bool ok = true;
  for (long item = it0 + blockIdx.x; ok && item < it1; item += gridDim.x)
    ok = mask_item<KIND>(a, item, cx, *m.rs, *m.ws, t);
  if (!ok && t == 0) mask_fail(a.st);
  mask_teardown(m, t);
}

// Many blocks in one launch: the work items of every block that takes the
// network this step (block b's items of this kind numbered ipre[b] ..
// ipre[b+1]-1), handed out round robin to a grid sized for the device.  The
// weights are loaded once per CTA, from args[0] (every block of a batch
// carries the same network).  After a tensor-core wait timed out, a CTA
// marks the block of each item it still owns as failed (WENO5 everywhere).
template <int KIND>
__global__ void __launch_bounds__(SW_T, 5) sensor_mask_batched(const MaskArgs* args, const long* ipre,
                                                                              int nblocks) {
  const int t = threadIdx.x;
  const long total = ipre[nblocks];
  if ((long)blockIdx.x >= total) return;
  const MaskSmem m = mask_setup(args[0].params, t);
  SweepCtx cx{m.s, 0u, 0.f, nullptr};
  bool ok = true;
  int b = 0;  // the block of item g: g only grows, so does b
  for (long g = blockIdx.x; g < total; g += gridDim.x) {
    while (ipre[b + 1] <= g) ++b;
    const MaskArgs& a = args[b];
    if ((a.check_done && a.st->done) || !sensor_step(a.st, a.every)) continue;
    if (ok) {
      cx.zcut = logit_cut(a.tau);
      cx.mask = a.mask;
      long it0, it1;
      mask_items(a.d, KIND, &it0, &it1);
      ok = mask_item<KIND>(a, it0 + (g - ipre[b]), cx, *m.rs, *m.ws, t);
    }
    if (!ok && t == 0) mask_fail(a.st);
  }
  mask_teardown(m, t);
}

}  // namespace

constexpr int kMaskSmem0 = (int)(sizeof(tc::Smem) + sizeof(RowSmem)) + 128;
constexpr int kMaskSmem1 = (int)(sizeof(tc::Smem) + sizeof(WinSmem)) + 128;
// at most 8 CTAs per SM hold TMEM (64 columns each of 512); the two launches
// of a sweep run back to back on the stream
constexpr long kMaskCap0 = 148L * 5, kMaskCap1 = 148L * 5;

cudaError_t mask_prepare() {
  static bool attr = false;
  if (attr) return cudaSuccess;
  cudaError_t e = cudaFuncSetAttribute(sensor_mask_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaskSmem0);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(sensor_mask_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaskSmem1);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(sensor_mask_batched<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaskSmem0);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(sensor_mask_batched<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaskSmem1);
  attr = e == cudaSuccess;
  return e;
}

void sensor_mask_items(const Dims& d, long* items0, long* items1) {
  const long rows = (long)(d.JM - 2) * (d.KM - 2);
  const long nseg0 = (d.IM - 1 + SW_T - 1) / SW_T, nseg = (d.IM - 2 + SW_T - 1) / SW_T;
  *items0 = nseg0 * ((rows + SW_CH - 1) / SW_CH);
  *items1 = nseg * (d.KM - 2) * ((d.JM - 1 + SW_CH - 1) / SW_CH) + nseg * (d.JM - 2) * ((d.KM - 1 + SW_CH - 1) / SW_CH);
}

cudaError_t launch_sensor_mask(const MaskArgs& a, cudaStream_t s) {
  cudaError_t e = mask_prepare();
  if (e != cudaSuccess) return e;
  long items0, items1;
  sensor_mask_items(a.d, &items0, &items1);
  sensor_mask_kernel<0><<<(unsigned)(items0 < kMaskCap0 ? items0 : kMaskCap0), SW_T, kMaskSmem0, s>>>(a);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  sensor_mask_kernel<1><<<(unsigned)(items1 < kMaskCap1 ? items1 : kMaskCap1), SW_T, kMaskSmem1, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_sensor_mask_batched(const MaskArgs* args, const long* ipre0, const long* ipre1, long total0,
                                       long total1, int nblocks, cudaStream_t s) {
  cudaError_t e = mask_prepare();
  if (e != cudaSuccess) return e;
  if (total0 > 0)
    sensor_mask_batched<0><<<(unsigned)(total0 < kMaskCap0 ? total0 : kMaskCap0), SW_T, kMaskSmem0, s>>>(args, ipre0,
                                                                                                       nblocks);
  e = cudaGetLastError();
  if (e != cudaSuccess || total1 <= 0) return e;
  sensor_mask_batched<1><<<(unsigned)(total1 < kMaskCap1 ? total1 : kMaskCap1), SW_T, kMaskSmem1, s>>>(args, ipre1,
                                                                                                     nblocks);
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
