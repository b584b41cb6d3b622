// sensor.cuh - the learned shock sensor: face features, WENO-weight labels and
// the MLP parameter layout shared by the training kernels (sensor.cu), the
// tensor-core inference (sensor_tc.cu) and the hybrid stage kernel.
//
// Features (15 per face).  For the face between stencil points 2 (node a) and
// 3 (node b) of the 6-point stencil a-2 .. b+2 along the face normal n:
//   f[m]      = (rho_{m+1} - rho_m) / rho_bar        m = 0..4
//   f[5 + m]  = (p_{m+1}   - p_m)   / p_bar
//   f[10 + m] = (un_{m+1}  - un_m)  / c_bar          un = velocity . unit normal
// with rho_bar, p_bar the means over a and b and c_bar = sqrt(gamma p_bar / rho_bar):
// normalised density, pressure and normal-velocity jumps of the 5-point stencil,
// each then compressed as sign(f) log2(1 + |f| / s) with s = SN_FEAT_SCALE:
// linear below s, logarithmic above (6.66 at |f| = 1).  The jumps that matter
// span 1e-4 .. 1; on that range the compression lets a 32-unit ReLU network
// separate the faces far better than the raw jumps do.
//
// Flat stencils.  A face whose compressed features sum (in absolute value) to
// less than SN_FLAT (every jump below ~3e-5) takes the linear flux without
// the network: its density, pressure and normal velocity are constant to
// within FP32 noise of the state, where the trained network decides linear
// as well.
//
// Label.  The characteristic WENO5 of the face (same basis as the flux) gives
// nonlinear weights w_k on both sides for the 5 fields; the deviation is
// max |w_k - d_k| with d = (0.1, 0.6, 0.3), and the face needs WENO when it
// exceeds 0.05.
//
// Network: 15 -> 32 (ReLU) -> 32 (ReLU) -> 1 (sigmoid = probability that the
// face needs WENO).  Parameters (float): W1[32][15] b1[32] W2[32][32] b2[32]
// w3[32] b3.
#pragma once

#include <cuda_runtime.h>

#include "cbns_common.cuh"

namespace cbns {

constexpr int SN_IN = 15, SN_H = 32;
constexpr int SP_W1 = 0, SP_B1 = 480, SP_W2 = 512, SP_B2 = 1536, SP_W3 = 1568, SP_B3 = 1600, SP_N = 1601;
constexpr float SN_DEV_THRESHOLD = 0.05f;
constexpr float SN_FEAT_SCALE = 0.01f;
constexpr float SN_FLAT = 0.0045f;  // sum of |features| below which a stencil is flat

// log2 on the special-function unit; the arguments here are >= 1
__device__ __forceinline__ float lg2_approx(float v) {
  float r;
  asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(v));
  return r;
}

// Compressed feature of a raw difference dlt whose normalised jump is dlt * n,
// with g = n / SN_FEAT_SCALE: sign(dlt) log2(1 + |dlt| g).
__device__ __forceinline__ float feat_of(float dlt, float g) {
  return copysignf(lg2_approx(__fmaf_rn(fabsf(dlt), g, 1.0f)), dlt);
}

// Primitives of one node from its conservative state, as the features use them.
struct NodePrim {
  float r, p, u, v, w;
};

// The feature arithmetic is written with explicit round-to-nearest operations
// (no contraction left to the compiler), so that the per-step sensor and the
// training sampler, which reach a face's stencil in different ways, compute
// bit-identical features.
__device__ __forceinline__ NodePrim node_prim(float q0, float q1, float q2, float q3, float q4, float gam1) {
  NodePrim s;
  const float ir = __frcp_rn(q0);
  s.r = q0;
  s.u = __fmul_rn(q1, ir);
  s.v = __fmul_rn(q2, ir);
  s.w = __fmul_rn(q3, ir);
  const float k = __fmaf_rn(s.w, s.w, __fmaf_rn(s.v, s.v, __fmul_rn(s.u, s.u)));
  s.p = __fmul_rn(gam1, __fsub_rn(q4, __fmul_rn(__fmul_rn(0.5f, q0), k)));
  return s;
}

// Unit face normal from the area vectors of the face's two nodes (FP32 copies).
__device__ __forceinline__ void face_unit_normal(const float a[3], const float b[3], float& x, float& y, float& z) {
  x = __fmul_rn(0.5f, __fadd_rn(a[0], b[0]));
  y = __fmul_rn(0.5f, __fadd_rn(a[1], b[1]));
  z = __fmul_rn(0.5f, __fadd_rn(a[2], b[2]));
  const float in = rsqrtf(__fmaf_rn(z, z, __fmaf_rn(y, y, __fmul_rn(x, x))));
  x = __fmul_rn(x, in);
  y = __fmul_rn(y, in);
  z = __fmul_rn(z, in);
}

// The 15 features of a face from the primitives of its 6 stencil nodes
// (P(q) returns the NodePrim of point q) and the unit face normal.
template <typename PF>
__device__ __forceinline__ void features_of(const PF& P, float ux, float uy, float uz, float gamma, float f[SN_IN]) {
  float r[6], p[6], un[6];
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    const NodePrim s = P(q);
    r[q] = s.r;
    p[q] = s.p;
    un[q] = __fmaf_rn(s.w, uz, __fmaf_rn(s.v, uy, __fmul_rn(s.u, ux)));
  }
  const float rb = __fmul_rn(0.5f, __fadd_rn(r[2], r[3])), pb = __fmul_rn(0.5f, __fadd_rn(p[2], p[3]));
  const float irb = __frcp_rn(rb), ipb = __frcp_rn(pb);
  const float icb = rsqrtf(__fmul_rn(__fmul_rn(gamma, pb), irb));
  const float gr = __fmul_rn(irb, 1.0f / SN_FEAT_SCALE), gp = __fmul_rn(ipb, 1.0f / SN_FEAT_SCALE);
  const float gu = __fmul_rn(icb, 1.0f / SN_FEAT_SCALE);
#pragma unroll
  for (int m = 0; m < 5; ++m) {
    f[m] = feat_of(__fsub_rn(r[m + 1], r[m]), gr);
    f[5 + m] = feat_of(__fsub_rn(p[m + 1], p[m]), gp);
    f[10 + m] = feat_of(__fsub_rn(un[m + 1], un[m]), gu);
  }
}

// Sum of |features| (NaN if any feature is NaN): the flat-stencil test
__device__ __forceinline__ float feature_l1(const float f[SN_IN]) {
  float a = 0.f;
#pragma unroll
  for (int m = 0; m < SN_IN; ++m) a = __fadd_rn(a, fabsf(f[m]));
  return a;
}

// Global face index e -> direction and the low node (i, j, k) of the face:
// i-faces, then j-faces, then k-faces, each in the order of the reference's
// Ep/Fp/Gp arrays (include/Block3d_cuda.h:110-123).  Returns false past the end.
__device__ __forceinline__ bool decode_face(const Dims& d, long e, int& dir, int& i, int& j, int& k) {
  const long ni = (long)(d.IM - 1) * (d.JM - 2) * (d.KM - 2);
  const long nj = (long)(d.IM - 2) * (d.JM - 1) * (d.KM - 2);
  const long nk = (long)(d.IM - 2) * (d.JM - 2) * (d.KM - 1);
  if (e < ni) {
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
  } else if (e < ni + nj + nk) {
    const long r = e - ni - nj;
    dir = 2;
    i = 1 + (int)(r % (d.IM - 2));
    j = 1 + (int)((r / (d.IM - 2)) % (d.JM - 2));
    k = (int)(r / ((long)(d.IM - 2) * (d.JM - 2)));
  } else {
    return false;
  }
  return true;
}

__device__ __forceinline__ long total_faces(const Dims& d) {
  return (long)(d.IM - 1) * (d.JM - 2) * (d.KM - 2) + (long)(d.IM - 2) * (d.JM - 1) * (d.KM - 2) +
         (long)(d.IM - 2) * (d.JM - 2) * (d.KM - 1);
}

// Features of a face from a stencil loader: ld(p, n) = conservative variable n
// at stencil point p.
template <typename LD>
__device__ __forceinline__ void face_features(const LD& ld, float ux, float uy, float uz, float gamma, float gam1,
                                              float f[SN_IN]) {
  auto P = [&](int q) { return node_prim(ld(q, 0), ld(q, 1), ld(q, 2), ld(q, 3), ld(q, 4), gam1); };
  features_of(P, ux, uy, uz, gamma, f);
}

// max |w_k - d_k| of the WENO5-JS weights of one scalar stencil a..e
__device__ __forceinline__ float weno_weight_dev(float a, float b, float c, float d, float e) {
  const float eps = 1.0e-6f;
  const float d1 = a - 2.f * b + c, e1 = a - 4.f * b + 3.f * c;
  const float d2 = b - 2.f * c + d, e2 = b - d;
  const float d3 = c - 2.f * d + e, e3 = 3.f * c - 4.f * d + e;
  const float s1 = (13.f / 12.f) * d1 * d1 + 0.25f * e1 * e1 + eps;
  const float s2 = (13.f / 12.f) * d2 * d2 + 0.25f * e2 * e2 + eps;
  const float s3 = (13.f / 12.f) * d3 * d3 + 0.25f * e3 * e3 + eps;
  const float a1 = 0.1f / (s1 * s1), a2 = 0.6f / (s2 * s2), a3 = 0.3f / (s3 * s3);
  const float is = 1.0f / (a1 + a2 + a3);
  return fmaxf(fmaxf(fabsf(a1 * is - 0.1f), fabsf(a2 * is - 0.6f)), fabsf(a3 * is - 0.3f));
}

// WENO-weight deviation of a face: the characteristic projection of the face
// flux (calc_eigenvectors_roe basis, node states at points 2 and 3) followed by
// the weights of both one-sided reconstructions of all five fields.
template <typename LD>
__device__ __forceinline__ float face_weno_deviation(const LD& ld, float nx, float ny, float nz, float gamma,
                                                     float gam1) {
  const float ra = ld(2, 0), ira = 1.f / ra, rb = ld(3, 0), irb = 1.f / rb;
  const float ua = ld(2, 1) * ira, va = ld(2, 2) * ira, wa = ld(2, 3) * ira;
  const float ub = ld(3, 1) * irb, vb = ld(3, 2) * irb, wb = ld(3, 3) * irb;
  const float pa = gam1 * (ld(2, 4) - 0.5f * ra * (ua * ua + va * va + wa * wa));
  const float pb = gam1 * (ld(3, 4) - 0.5f * rb * (ub * ub + vb * vb + wb * wb));
  float lx = 0.f, ly = nz, lz = -ny, mx, my, mz;
  if (ly * ly + lz * lz > 1.0e-16f) {
    mx = -ny * ny - nz * nz;
    my = nx * ny;
    mz = nx * nz;
  } else {
    lx = -nz;
    ly = 0.f;
    lz = nx;
    mx = nx * ny;
    my = -nx * nx - nz * nz;
    mz = ny * nz;
  }
  const float in = rsqrtf(nx * nx + ny * ny + nz * nz);
  const float ux = nx * in, uy = ny * in, uz = nz * in;
  const float il = rsqrtf(lx * lx + ly * ly + lz * lz), im = rsqrtf(mx * mx + my * my + mz * mz);
  lx *= il; ly *= il; lz *= il;
  mx *= im; my *= im; mz *= im;
  const float Ha = gamma * pa * ira / gam1 + 0.5f * (ua * ua + va * va + wa * wa);
  const float Hb = gamma * pb * irb / gam1 + 0.5f * (ub * ub + vb * vb + wb * wb);
  const float sr = sqrtf(rb * ira), is = 1.f / (1.f + sr);
  const float uu = (ua + sr * ub) * is, vv = (va + sr * vb) * is, ww = (wa + sr * wb) * is;
  const float H = (Ha + sr * Hb) * is, q2 = uu * uu + vv * vv + ww * ww;
  const float c = sqrtf(gam1 * (H - 0.5f * q2)), ic = 1.f / c;
  const float qn = uu * ux + vv * uy + ww * uz, ql = uu * lx + vv * ly + ww * lz, qm = uu * mx + vv * my + ww * mz;
  const float h = 0.5f * ic, K = gam1 * h * ic;
  float W[5][6];
#pragma unroll
  for (int p = 0; p < 6; ++p) {
    const float f0 = ld(p, 0), f1 = ld(p, 1), f2 = ld(p, 2), f3 = ld(p, 3), f4 = ld(p, 4);
    const float A = K * (0.5f * q2 * f0 - (uu * f1 + vv * f2 + ww * f3) + f4);
    const float B = h * (qn * f0 - (ux * f1 + uy * f2 + uz * f3));
    W[0][p] = A + B;
    W[1][p] = f0 - 2.f * A;
    W[2][p] = A - B;
    W[3][p] = lx * f1 + ly * f2 + lz * f3 - ql * f0;
    W[4][p] = mx * f1 + my * f2 + mz * f3 - qm * f0;
  }
  float dev = 0.f;
#pragma unroll
  for (int s = 0; s < 5; ++s) {
    dev = fmaxf(dev, weno_weight_dev(W[s][0], W[s][1], W[s][2], W[s][3], W[s][4]));
    dev = fmaxf(dev, weno_weight_dev(W[s][5], W[s][4], W[s][3], W[s][2], W[s][1]));
  }
  return dev;
}

// FP32 forward pass of the sensor network for one feature vector
__device__ __forceinline__ float mlp_forward(const float* P, const float* x) {
  float h1[SN_H];
#pragma unroll
  for (int c = 0; c < SN_H; ++c) {
    float s = P[SP_B1 + c];
#pragma unroll
    for (int k = 0; k < SN_IN; ++k) s += P[SP_W1 + c * SN_IN + k] * x[k];
    h1[c] = fmaxf(s, 0.f);
  }
  float z = P[SP_B3];
#pragma unroll 4
  for (int c = 0; c < SN_H; ++c) {
    float s = P[SP_B2 + c];
#pragma unroll
    for (int k = 0; k < SN_H; ++k) s += P[SP_W2 + c * SN_H + k] * h1[k];
    z += P[SP_W3 + c] * fmaxf(s, 0.f);
  }
  return z;  // logit
}

}  // namespace cbns
