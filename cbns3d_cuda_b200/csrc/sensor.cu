// sensor.cu - training side of the learned shock sensor: face sampling with
// features and WENO-weight labels from a solver state, the network's loss and
// gradient over a batch (forward and backward by hand), the Adam update, and
// an FP32 forward pass.  See sensor.cuh for the features, label and layout.
#include "face_flux.cuh"
#include "sensor.cuh"
#include "sensor_kernels.cuh"

namespace cbns {

namespace {

// ---------------------------------------------------------------- sampling
__global__ void sample_faces_kernel(const SampleArgs a) {
  const Dims& d = a.d;
  const long ni = (long)(d.IM - 1) * (d.JM - 2) * (d.KM - 2);
  const long nj = (long)(d.IM - 2) * (d.JM - 1) * (d.KM - 2);
  const long nk = (long)(d.IM - 2) * (d.JM - 2) * (d.KM - 1);
  const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (e >= ni + nj + nk || (e % a.stride) != a.offset) return;
  int dir, i, j, k;
  if (e < ni) {  // face between (i, j+1, k+1) and (i+1, j+1, k+1)
    dir = 0;
    i = (int)(e % (d.IM - 1));
    j = 1 + (int)((e / (d.IM - 1)) % (d.JM - 2));
    k = 1 + (int)(e / ((long)(d.IM - 1) * (d.JM - 2)));
  } else if (e < ni + nj) {
    const long r = e - ni;
    dir = 1;
    i = 1 + (int)(r % (d.IM - 2));
    j = (int)((r / (d.IM - 2)) % (d.JM - 1));
    k = 1 + (int)(r / ((long)(d.IM - 2) * (d.JM - 1)));
  } else {
    const long r = e - ni - nj;
    dir = 2;
    i = 1 + (int)(r % (d.IM - 2));
    j = 1 + (int)((r / (d.IM - 2)) % (d.JM - 2));
    k = (int)(r / ((long)(d.IM - 2) * (d.JM - 2)));
  }
  const long sd = dir == 0 ? 1 : (dir == 1 ? d.PX : d.PL);
  const long oa = node_off(d, i, j, k), ob = oa + sd;
  const double* q = a.q;
  const long V = d.VOL;
  auto ld = [&](int p, int n) -> float { return (float)q[n * V + oa + (p - 2) * sd]; };
  // the same FP32 arithmetic as the per-step sensor sweep, so that inference
  // sees exactly the features the network was trained on
  const float A[3] = {(float)a.area[3 * dir][oa], (float)a.area[3 * dir + 1][oa], (float)a.area[3 * dir + 2][oa]};
  const float B[3] = {(float)a.area[3 * dir][ob], (float)a.area[3 * dir + 1][ob], (float)a.area[3 * dir + 2][ob]};
  float ux, uy, uz;
  face_unit_normal(A, B, ux, uy, uz);
  float f[SN_IN];
  face_features(ld, ux, uy, uz, a.gamma, a.gam1, f);
  const float dev = face_weno_deviation(ld, 0.5f * (A[0] + B[0]), 0.5f * (A[1] + B[1]), 0.5f * (A[2] + B[2]),
                                        a.gamma, a.gam1);
  const unsigned slot = atomicAdd(a.count, 1u);
  if (slot >= a.capacity) return;
#pragma unroll
  for (int m = 0; m < SN_IN; ++m) a.feat[(long)slot * SN_IN + m] = f[m];
  a.label[slot] = dev > SN_DEV_THRESHOLD ? 1 : 0;
  if (a.dev) a.dev[slot] = dev;
  if (a.index) a.index[slot] = (unsigned)e;
}

// ---------------------------------------------------------------- loss and gradient
constexpr int TILE = 128, GT = 256, HP = SN_H + 1;

struct GradSmem {
  float x[TILE][16];
  float h1[TILE][HP], h2[TILE][HP], g2[TILE][HP], g1[TILE][HP];
  float dz[TILE];
  float W2[SN_H][SN_H];
  float w3[SN_H];
};

// Binary cross-entropy with positive-class weight, averaged over n samples:
// loss = -(1/n) sum w_i [y_i log p_i + (1 - y_i) log(1 - p_i)], p = sigmoid(z).
// Each CTA takes tiles of 128 samples: forward into shared memory, backward by
// the chain rule, per-thread partial sums of the weight gradients in registers,
// one atomic add per parameter per CTA at the end.
__global__ void __launch_bounds__(GT) mlp_grad_kernel(const float* __restrict__ P, const float* __restrict__ X,
                                                      const unsigned char* __restrict__ Y, unsigned n, float pos_w,
                                                      float inv_n, float* G, float* loss) {
  extern __shared__ __align__(16) unsigned char raw[];
  GradSmem& s = *reinterpret_cast<GradSmem*>(raw);
  const int t = threadIdx.x;
  const int c = t & 31, rb = t >> 5;  // column and first row of this thread's outputs
  for (int e = t; e < SN_H * SN_H; e += GT) s.W2[e / SN_H][e % SN_H] = P[SP_W2 + e];
  if (t < SN_H) s.w3[t] = P[SP_W3 + t];
  float w1[SN_IN], w2[SN_H];
#pragma unroll
  for (int k = 0; k < SN_IN; ++k) w1[k] = P[SP_W1 + c * SN_IN + k];
#pragma unroll
  for (int k = 0; k < SN_H; ++k) w2[k] = P[SP_W2 + c * SN_H + k];
  const float b1 = P[SP_B1 + c], b2 = P[SP_B2 + c], b3 = P[SP_B3];
  // owned gradient entries
  float gW2[4] = {0, 0, 0, 0}, gW1[2] = {0, 0}, gvec = 0.f, lsum = 0.f;
  __syncthreads();
  const unsigned ntiles = (n + TILE - 1) / TILE;
  for (unsigned tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const unsigned base = tile * TILE;
    for (int e = t; e < TILE * 16; e += GT) {
      const int r = e >> 4, k = e & 15;
      const unsigned sidx = base + r;
      s.x[r][k] = (k < SN_IN && sidx < n) ? X[(size_t)sidx * SN_IN + k] : 0.f;
    }
    __syncthreads();
    for (int r = rb; r < TILE; r += 8) {
      float h = b1;
#pragma unroll
      for (int k = 0; k < SN_IN; ++k) h += s.x[r][k] * w1[k];
      s.h1[r][c] = fmaxf(h, 0.f);
    }
    __syncthreads();
    for (int r = rb; r < TILE; r += 8) {
      float h = b2;
#pragma unroll
      for (int k = 0; k < SN_H; ++k) h += s.h1[r][k] * w2[k];
      s.h2[r][c] = fmaxf(h, 0.f);
    }
    __syncthreads();
    if (t < TILE) {
      const unsigned sidx = base + t;
      float dz = 0.f;
      if (sidx < n) {
        float z = b3;
#pragma unroll
        for (int k = 0; k < SN_H; ++k) z += s.h2[t][k] * s.w3[k];
        const float y = Y[sidx] ? 1.f : 0.f;
        const float w = Y[sidx] ? pos_w : 1.f;
        const float p = 1.f / (1.f + __expf(-z));
        // log(sigmoid(z)) and log(1 - sigmoid(z)) in a form that does not overflow
        const float lp = -log1pf(__expf(-fabsf(z))) + fminf(z, 0.f);
        const float lq = lp - z;
        lsum += -w * (y * lp + (1.f - y) * lq) * inv_n;
        dz = w * (p - y) * inv_n;
      }
      s.dz[t] = dz;
    }
    __syncthreads();
    for (int r = rb; r < TILE; r += 8) s.g2[r][c] = s.h2[r][c] > 0.f ? s.dz[r] * s.w3[c] : 0.f;
    __syncthreads();
    // dW2[cc][k] = sum_r g2[r][cc] h1[r][k]
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int e = t + GT * q, cc = e / SN_H, k = e % SN_H;
      float acc = 0.f;
      for (int r = 0; r < TILE; ++r) acc += s.g2[r][cc] * s.h1[r][k];
      gW2[q] += acc;
    }
    // per-column vectors: db1 (t<32, after g1), db2 (32..63), dw3 (64..95), db3 (96)
    if (t >= 32 && t < 64) {
      float acc = 0.f;
      for (int r = 0; r < TILE; ++r) acc += s.g2[r][t - 32];
      gvec += acc;
    } else if (t >= 64 && t < 96) {
      float acc = 0.f;
      for (int r = 0; r < TILE; ++r) acc += s.dz[r] * s.h2[r][t - 64];
      gvec += acc;
    } else if (t == 96) {
      float acc = 0.f;
      for (int r = 0; r < TILE; ++r) acc += s.dz[r];
      gvec += acc;
    }
    // g1[r][k] = (sum_c g2[r][c] W2[c][k]) * relu'(h1)
    for (int r = rb; r < TILE; r += 8) {
      float acc = 0.f;
#pragma unroll
      for (int cc = 0; cc < SN_H; ++cc) acc += s.g2[r][cc] * s.W2[cc][c];
      s.g1[r][c] = s.h1[r][c] > 0.f ? acc : 0.f;
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const int e = t + GT * q;
      if (e < SN_H * SN_IN) {
        const int cc = e / SN_IN, k = e % SN_IN;
        float acc = 0.f;
        for (int r = 0; r < TILE; ++r) acc += s.g1[r][cc] * s.x[r][k];
        gW1[q] += acc;
      }
    }
    if (t < 32) {
      float acc = 0.f;
      for (int r = 0; r < TILE; ++r) acc += s.g1[r][t];
      gvec += acc;
    }
    __syncthreads();
  }
#pragma unroll
  for (int q = 0; q < 4; ++q) atomicAdd(&G[SP_W2 + t + GT * q], gW2[q]);
#pragma unroll
  for (int q = 0; q < 2; ++q)
    if (t + GT * q < SN_H * SN_IN) atomicAdd(&G[SP_W1 + t + GT * q], gW1[q]);
  if (t < 32) atomicAdd(&G[SP_B1 + t], gvec);
  else if (t < 64) atomicAdd(&G[SP_B2 + t - 32], gvec);
  else if (t < 96) atomicAdd(&G[SP_W3 + t - 64], gvec);
  else if (t == 96) atomicAdd(&G[SP_B3], gvec);
  if (t < TILE) {
    float l = lsum;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
    if ((t & 31) == 0) atomicAdd(loss, l);
  }
}

// ---------------------------------------------------------------- widening
// Grid of one pass: x over the faces of a line along i (128 per CTA), y over
// groups of lines along the walked direction, z over (face direction, the
// third index).  Pass dim 0 and 1: the thread walks j (lines along j, groups
// of DLJ), the CTA holds k; pass dim 2: the thread walks k (groups of DLK),
// the CTA holds j.  So the widening of passes 1 and 2 runs along the thread's
// own walk as a sliding window sum (two loads per face whatever the width),
// and that of pass 0 along i from a line segment staged in shared memory with
// its halo.  No index division per face.
constexpr int DLJ = 16, DLK = 32;
__host__ __device__ __forceinline__ dim3 dilate_grid(const Dims& d, int dim) {
  const unsigned gx = (unsigned)((d.IM - 1 + 127) / 128);
  if (dim == 2) return dim3(gx, (unsigned)((d.KM - 1 + DLK - 1) / DLK), (unsigned)(3 * (d.JM - 1)));
  return dim3(gx, (unsigned)((d.JM - 1 + DLJ - 1) / DLJ), (unsigned)(3 * (d.KM - 1)));
}

// CTA (bx, by, bz) of one block's widening grid for pass a.dim
__device__ __forceinline__ void dilate_body(const DilateArgs& a, unsigned bx, unsigned by, unsigned bz) {
  if (a.check_done && a.st->done) return;
  const bool lead = bx == 0 && by == 0 && bz == 0 && threadIdx.x == 0;
  if (a.hold || !sensor_step(a.st, a.every)) {
    // decisions of an earlier step: only the statistics, that step's count
    if (a.count && lead) atomicAdd(&a.st->weno_faces, a.st->weno_last);
    return;
  }
  if (a.dim == 0 && lead) a.st->weno_last = 0;  // the last pass counts anew
  const Dims& d = a.d;
  const int IM = d.IM, JM = d.JM, KM = d.KM;
  const bool walk_k = a.dim == 2;
  const int zc = walk_k ? JM - 1 : KM - 1;
  const int dir = (int)bz / zc, fixed = (int)bz % zc;
  // extents (n0, n1, n2) and first index of this direction's faces
  const int n0 = dir == 0 ? IM - 1 : IM - 2, n1 = dir == 1 ? JM - 1 : JM - 2, n2 = dir == 2 ? KM - 1 : KM - 2;
  const long first = dir == 0 ? 0
                              : (dir == 1 ? (long)(IM - 1) * (JM - 2) * (KM - 2)
                                          : (long)(IM - 1) * (JM - 2) * (KM - 2) + (long)(IM - 2) * (JM - 1) * (KM - 2));
  if (fixed >= (walk_k ? n1 : n2)) return;  // uniform per CTA
  const int x0 = (int)bx * 128 + (int)threadIdx.x;
  const bool valid = x0 < n0;
  // the thread's walk: positions q0 .. q1-1 along j (walk_k: along k), face
  // index base + q * step
  const int nq = walk_k ? n2 : n1, dl = walk_k ? DLK : DLJ;
  const int q0 = (int)by * dl, q1 = min(nq, q0 + dl);
  const long step = walk_k ? (long)n0 * n1 : (long)n0;
  const long base = first + x0 + (walk_k ? (long)n0 * fixed : (long)n0 * n1 * fixed);
  unsigned cnt = 0;
  {
    const unsigned char* __restrict__ in = a.in;
    unsigned char* __restrict__ out = a.out;
    const int w = a.dim == dir ? a.along : a.across;
    if (a.dim == 0) {
      // along i: each line's 128 faces and a halo of w either side staged in
      // shared memory (coalesced), then each thread ORs its window there
      constexpr int WMAX = 16;
      __shared__ unsigned char row[128 + 2 * WMAX];
      const int t = threadIdx.x;
      const int xb = (int)bx * 128;  // first face of the CTA's segment
      for (int q = q0; q < q1; ++q) {
        const long e = base + q * step;  // this thread's face (x0 = xb + t)
        unsigned dec = 0;
        if (w <= WMAX) {
          __syncthreads();  // the previous line's window reads are done
          row[WMAX + t] = valid ? __ldg(in + e) : 0;
          if (t < WMAX) {
            const int xl = xb - WMAX + t, xr = xb + 128 + t;  // halo faces
            row[t] = (xl >= 0 && xl < n0) ? __ldg(in + e - WMAX) : 0;
            row[WMAX + 128 + t] = (xr < n0) ? __ldg(in + e + 128) : 0;
          }
          __syncthreads();
          if (valid)
            for (int o = -w; o <= w; ++o) dec |= row[WMAX + t + o];
        } else if (valid) {
          const int lo = max(-w, -x0), hi = min(w, n0 - 1 - x0);
          for (int o = lo; o <= hi; ++o) dec |= __ldg(in + e + o);
        }
        if (valid) {
          out[e] = (unsigned char)dec;
          cnt += dec;
        }
      }
    } else if (valid) {
      // along the walk: a sliding window sum of the 0/1 decisions
      int sum = 0;
      for (int q = max(0, q0 - w); q <= min(nq - 1, q0 + w); ++q) sum += __ldg(in + base + q * step);
      for (int q = q0; q < q1; ++q) {
        const unsigned dec = sum > 0 ? 1u : 0u;
        out[base + q * step] = (unsigned char)dec;
        cnt += dec;
        if (q - w >= 0) sum -= __ldg(in + base + (q - w) * step);
        if (q + 1 + w < nq) sum += __ldg(in + base + (q + 1 + w) * step);
      }
    }
  }
  if (a.count) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    if ((threadIdx.x & 31) == 0 && cnt) {
      atomicAdd(&a.st->weno_faces, (unsigned long long)cnt);
      atomicAdd(&a.st->weno_last, (unsigned long long)cnt);
    }
  }
}

__global__ void __launch_bounds__(128) sensor_dilate_kernel(const DilateArgs a) {
  dilate_body(a, blockIdx.x, blockIdx.y, blockIdx.z);
}

// Many blocks in one launch: block b owns CTAs cta[b] .. cta[b+1]-1, args[b]
// are its DilateArgs (all of one pass).
__global__ void __launch_bounds__(128) sensor_dilate_batched(const DilateArgs* args, const int* cta, int nblocks) {
  const int b = block_of_cta(cta, nblocks, (int)blockIdx.x);
  const DilateArgs& a = args[b];
  const dim3 g = dilate_grid(a.d, a.dim);
  const unsigned l = blockIdx.x - (unsigned)__ldg(cta + b);
  dilate_body(a, l % g.x, (l / g.x) % g.y, l / (g.x * g.y));
}

// ---------------------------------------------------------------- audit
__device__ __forceinline__ void audit_body(const AuditArgs& a, unsigned bx) {
  if (a.check_done && a.st->done) return;
  const Dims& d = a.d;
  const long nf = total_faces(d);
  // runs of 128 consecutive faces (coalesced loads): run r is audited when
  // r % stride == steps % stride
  const unsigned off = a.st->steps % a.stride;
  const long e = ((long)bx * a.stride + off) * 128 + threadIdx.x;
  float err = 0.f;
  bool audited = false;
  int dir, i, j, k;
  if (e < nf && a.mask[e] == 0 && decode_face(d, e, dir, i, j, k)) {
    const long sd = dir == 0 ? 1 : (dir == 1 ? d.PX : d.PL);
    const long oa = node_off(d, i, j, k), ob = oa + sd;
    auto ld = [&](int p, int n) -> float { return (float)__ldg(a.q + n * d.VOL + oa + (p - 2) * sd); };
    const float nx = (float)(0.5 * (__ldg(a.area[3 * dir] + oa) + __ldg(a.area[3 * dir] + ob)));
    const float ny = (float)(0.5 * (__ldg(a.area[3 * dir + 1] + oa) + __ldg(a.area[3 * dir + 1] + ob)));
    const float nz = (float)(0.5 * (__ldg(a.area[3 * dir + 2] + oa) + __ldg(a.area[3 * dir + 2] + ob)));
    const FluxConsts<float> C{a.gamma, a.gam1, a.gam1_inv};
    float fw[5], fl[5];
    face_flux<float>(ld, nx, ny, nz, C, fw);
    face_flux_linear<float>(ld, nx, ny, nz, C, fl);
    float num = 0.f, den = 0.f;
#pragma unroll
    for (int n = 0; n < 5; ++n) {
      num = fmaxf(num, fabsf(fw[n] - fl[n]));
      den = fmaxf(den, fabsf(fw[n]));
    }
    err = num / (den + 1.0e-20f);
    if (!(err == err)) err = 3.0e38f;
    audited = true;
  }
  const unsigned full = 0xffffffffu;
  const unsigned n_aud = __popc(__ballot_sync(full, audited));
  float m = err;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(full, m, o));
  if ((threadIdx.x & 31) == 0 && n_aud) {
    atomicAdd(&a.st->audit_faces, (unsigned long long)n_aud);
    atomicMax(reinterpret_cast<int*>(&a.st->audit_max), __float_as_int(m));  // m >= 0: int order = float order
    if (m > a.bound && atomicExch(&a.st->force_weno, 1) == 0) atomicAdd(&a.st->audit_fail_steps, 1u);
  }
}

__global__ void __launch_bounds__(128) sensor_audit_kernel(const AuditArgs a) { audit_body(a, blockIdx.x); }

__global__ void __launch_bounds__(128) sensor_audit_batched(const AuditArgs* args, const int* cta, int nblocks) {
  const int b = block_of_cta(cta, nblocks, (int)blockIdx.x);
  audit_body(args[b], blockIdx.x - (unsigned)__ldg(cta + b));
}

__global__ void adam_kernel(float* P, const float* G, float* M, float* V, float lr, float c1, float c2) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= SP_N) return;
  const float g = G[e];
  const float m = 0.9f * M[e] + 0.1f * g;
  const float v = 0.999f * V[e] + 0.001f * g * g;
  M[e] = m;
  V[e] = v;
  P[e] -= lr * (m * c1) / (sqrtf(v * c2) + 1.0e-8f);
}

__global__ void mlp_predict_kernel(const float* __restrict__ P, const float* __restrict__ X, unsigned n,
                                   float* __restrict__ out) {
  __shared__ float sp[SP_N];
  for (int e = threadIdx.x; e < SP_N; e += blockDim.x) sp[e] = P[e];
  __syncthreads();
  const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float x[SN_IN];
#pragma unroll
  for (int k = 0; k < SN_IN; ++k) x[k] = X[(size_t)i * SN_IN + k];
  out[i] = 1.f / (1.f + __expf(-mlp_forward(sp, x)));
}

}  // namespace

cudaError_t launch_sample_faces(const SampleArgs& a, cudaStream_t s) {
  const Dims& d = a.d;
  const long n = (long)(d.IM - 1) * (d.JM - 2) * (d.KM - 2) + (long)(d.IM - 2) * (d.JM - 1) * (d.KM - 2) +
                 (long)(d.IM - 2) * (d.JM - 2) * (d.KM - 1);
  sample_faces_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(a);
  return cudaGetLastError();
}

int sensor_audit_ctas(const AuditArgs& a) {
  const long nf = (long)(a.d.IM - 1) * (a.d.JM - 2) * (a.d.KM - 2) + (long)(a.d.IM - 2) * (a.d.JM - 1) * (a.d.KM - 2) +
                  (long)(a.d.IM - 2) * (a.d.JM - 2) * (a.d.KM - 1);
  const long runs = (nf + 127) / 128;
  return (int)((runs + a.stride - 1) / a.stride);
}

cudaError_t launch_sensor_audit(const AuditArgs& a, cudaStream_t s) {
  sensor_audit_kernel<<<(unsigned)sensor_audit_ctas(a), 128, 0, s>>>(a);
  return cudaGetLastError();
}

int sensor_dilate_ctas(const Dims& d, int dim) {
  const dim3 g = dilate_grid(d, dim);
  return (int)(g.x * g.y * g.z);
}

cudaError_t launch_sensor_dilate(const DilateArgs& a, cudaStream_t s) {
  sensor_dilate_kernel<<<dilate_grid(a.d, a.dim), 128, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_sensor_audit_batched(const AuditArgs* args, const int* cta, int nblocks, int total,
                                        cudaStream_t s) {
  if (total <= 0) return cudaSuccess;
  sensor_audit_batched<<<total, 128, 0, s>>>(args, cta, nblocks);
  return cudaGetLastError();
}

cudaError_t launch_sensor_dilate_batched(const DilateArgs* args, const int* cta, int nblocks, int total,
                                         cudaStream_t s) {
  if (total <= 0) return cudaSuccess;
  sensor_dilate_batched<<<total, 128, 0, s>>>(args, cta, nblocks);
  return cudaGetLastError();
}

cudaError_t launch_mlp_grad(const float* P, const float* X, const unsigned char* Y, unsigned n, float pos_w, float* G,
                            float* loss, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(G, 0, SP_N * sizeof(float), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(loss, 0, sizeof(float), s);
  if (e != cudaSuccess) return e;
  if (n == 0) return cudaSuccess;
  static bool attr = false;
  if (!attr) {
    e = cudaFuncSetAttribute(mlp_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(GradSmem));
    if (e != cudaSuccess) return e;
    attr = true;
  }
  const unsigned ntiles = (n + TILE - 1) / TILE;
  const unsigned grid = ntiles < 296u ? ntiles : 296u;
  mlp_grad_kernel<<<grid, GT, sizeof(GradSmem), s>>>(P, X, Y, n, pos_w, 1.0f / (float)n, G, loss);
  return cudaGetLastError();
}

cudaError_t launch_adam(float* P, const float* G, float* M, float* V, unsigned step, float lr, cudaStream_t s) {
  const float c1 = 1.0f / (1.0f - powf(0.9f, (float)step));
  const float c2 = 1.0f / (1.0f - powf(0.999f, (float)step));
  adam_kernel<<<(SP_N + 255) / 256, 256, 0, s>>>(P, G, M, V, lr, c1, c2);
  return cudaGetLastError();
}

cudaError_t launch_mlp_predict(const float* P, const float* X, unsigned n, float* out, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  mlp_predict_kernel<<<(n + 255) / 256, 256, 0, s>>>(P, X, n, out);
  return cudaGetLastError();
}

}  // namespace cbns
