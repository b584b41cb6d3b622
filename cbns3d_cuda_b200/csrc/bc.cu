// bc.cu - boundary conditions and primitive recovery on the boundary, the
// reference's set_bc_calc_primitive (src/set_bc_calc_primitive.cu:15-47,
// src/primitive_bc_kernel.cu:13-494), as three ordered launches:
//   phase 1  (j,k) interior: i = 0 and i = IM-1 faces, Q and primitives on
//            i = 0,-1,-2 / IM-1,IM,IM+1 from the first interior node with the
//            pressure reset to p_inf (:84-186)
//   phase 2  (i,k), k interior: j = 0 face -- wake-cut average for
//            i < i_begin-1 or wall for i < i_end (unsigned tests, :194-352)
//   phase 3  (a) primitives on j = 0,-1,-2 and on j = JM-1, JM (from Q at
//            JM-1) (:354-413); (b) k = 0 and k = KM-1 faces, zero-gradient
//            copy of Q and primitives for every (i,j) (:417-492); (c) in
//            inviscid runs, the spectral radius of every boundary node for the
//            next time step (the boundary half of src/time_step_kernel.cu).
// With CBNS_BC_FARFIELD (no counterpart in the reference) one kernel replaces
// the three: boundary and ghost nodes keep their Q (a free-stream far field on
// every face), only their primitives and spectral radii are formed; with
// CBNS_BC_CHARACTERISTIC three launches (i, j, k faces) first set every
// boundary node and its ghosts to a characteristic far-field state.  With
// CBNS_BC_OGRID: phase 2 with the wall on every i, the characteristic state on
// j = JM-1, phase 3, then the copies across the periodic seam in i.
// The reference runs these as __syncthreads-separated phases of one kernel, so
// its cross-CTA reads (wake mirror, k-face copies of j-face results) are races;
// separate launches give the program-order result, which is what the reference
// computes whenever those races do not bite.  Primitive arrays are written only
// in viscous runs (inviscid runs recompute primitives from Q where needed).
#include "bc.cuh"

namespace cbns {

namespace {

struct PrimV {
  double r, u, v, w, p;
};

__device__ __forceinline__ PrimV prim_of(const double* q, long o, long VOL, double gam1) {
  PrimV s;
  s.r = q[o];
  s.u = q[VOL + o] / s.r;
  s.v = q[2 * VOL + o] / s.r;
  s.w = q[3 * VOL + o] / s.r;
  s.p = gam1 * (q[4 * VOL + o] - 0.5 * s.r * (s.u * s.u + s.v * s.v + s.w * s.w));
  return s;
}

__device__ __forceinline__ void put_prim(const BCArgs& a, long o, const PrimV& s) {
  a.prim[0][o] = s.r;
  a.prim[1][o] = s.u;
  a.prim[2][o] = s.v;
  a.prim[3][o] = s.w;
  a.prim[4][o] = s.p;
  a.prim[5][o] = a.gM2 * s.p / s.r;
}

// spectral radius sum of time_step_kernel (inviscid form) at node offset o
__device__ __forceinline__ double sigma_inv(const BCArgs& a, long o, const PrimV& s) {
  const double c = sqrt(a.gamma * s.p / s.r);
  double sum = 0.0;
#pragma unroll
  for (int dd = 0; dd < 3; ++dd) {
    const double mx = a.met[3 * dd][o], my = a.met[3 * dd + 1][o], mz = a.met[3 * dd + 2][o];
    sum += fabs(s.u * mx + s.v * my + s.w * mz) + c * sqrt(mx * mx + my * my + mz * mz);
  }
  return sum;
}

// max of two spectral radii that keeps a NaN
__device__ __forceinline__ double smax2(double x, double y) {
  return (x != x || y != y) ? __longlong_as_double(0x7ff8000000000000ll) : fmax(x, y);
}

// Warp max of the per-thread values (has = thread holds a value), one atomic
// per warp.  Every lane of the warp must call this (full-mask shuffles).
__device__ __forceinline__ void warp_sigma_max(const BCArgs& a, double s, bool has) {
  const bool nan = has && (s != s);
  double m = (has && !nan) ? s : 0.0;
  const unsigned anyhas = __ballot_sync(0xffffffffu, has);
  const unsigned anynan = __ballot_sync(0xffffffffu, nan);
#pragma unroll
  for (int k = 16; k > 0; k >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, k));
  if ((threadIdx.x & 31) == 0 && anyhas != 0u)
    atomic_max_sigma(&a.st->sigma_bits, anynan ? __longlong_as_double(0x7ff8000000000000ll) : m);
}

__global__ void bc_phase1(const BCArgs a) {
  if (a.check_done && a.st->done) return;
  const Dims& d = a.d;
  const long n = (long)(d.JM - 2) * (d.KM - 2);
  const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (e >= 2 * n) return;
  const int side = e >= n;
  const long r = side ? e - n : e;
  const int j = 1 + (int)(r % (d.JM - 2)), k = 1 + (int)(r / (d.JM - 2));
  const long VOL = d.VOL;
  const int src = side ? d.IM - 2 : 1;
  const int base = side ? d.IM - 1 : 0;
  const int dir = side ? 1 : -1;
  const long os = node_off(d, src, j, k);
  const double rr = a.q[os], ru = a.q[VOL + os], rv = a.q[2 * VOL + os], rw = a.q[3 * VOL + os];
  const double E = a.p_inf / a.gam1 + 0.5 * (ru * ru + rv * rv + rw * rw) / rr;
  PrimV s;
  s.r = rr;
  s.u = ru / rr;
  s.v = rv / rr;
  s.w = rw / rr;
  s.p = a.gam1 * (E - 0.5 * s.r * (s.u * s.u + s.v * s.v + s.w * s.w));
  for (int l = 0; l <= NG; ++l) {
    const long o = node_off(d, base + dir * l, j, k);
    a.q[o] = rr;
    a.q[VOL + o] = ru;
    a.q[2 * VOL + o] = rv;
    a.q[3 * VOL + o] = rw;
    a.q[4 * VOL + o] = E;
    if (a.viscous) put_prim(a, o, s);
  }
}

__global__ void bc_phase2(const BCArgs a) {
  if (a.check_done && a.st->done) return;
  const Dims& d = a.d;
  const long n = (long)d.IM * (d.KM - 2);
  const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (e >= n) return;
  const int i = (int)(e % d.IM), k = 1 + (int)(e / d.IM);
  const long VOL = d.VOL;
  const double gam1 = a.gam1;
  const unsigned ui = (unsigned)i;
  double* q = a.q;
  if (a.i_begin - 1u > ui) {
    // wake cut: average the primitives of (i,1) and its mirror (IM-1-i,1)
    const int m = d.IM - 1 - i;
    const PrimV x = prim_of(q, node_off(d, i, 1, k), VOL, gam1);
    const PrimV y = prim_of(q, node_off(d, m, 1, k), VOL, gam1);
    const double r = (x.r + y.r) * 0.5, uu = (x.u + y.u) * 0.5, vv = (x.v + y.v) * 0.5, ww = (x.w + y.w) * 0.5,
                 pp = (x.p + y.p) * 0.5;
    const double v5[5] = {r, r * uu, r * vv, r * ww, pp / gam1 + 0.5 * r * (uu * uu + vv * vv + ww * ww)};
    const long o0 = node_off(d, i, 0, k), m0 = node_off(d, m, 0, k);
#pragma unroll
    for (int c = 0; c < NEQ; ++c) {
      q[c * VOL + o0] = v5[c];
      q[c * VOL + m0] = v5[c];
    }
    for (int l = 1; l <= NG; ++l) {
      const long a1 = node_off(d, m, l, k), b1 = node_off(d, i, -l, k);
      const long a2 = node_off(d, i, l, k), b2 = node_off(d, m, -l, k);
#pragma unroll
      for (int c = 0; c < NEQ; ++c) {
        q[c * VOL + b1] = q[c * VOL + a1];
        q[c * VOL + b2] = q[c * VOL + a2];
      }
    }
  } else if (a.i_end > ui) {
    const long o1 = node_off(d, i, 1, k), o0 = node_off(d, i, 0, k);
    if (a.viscous) {
      // adiabatic no-slip wall
      const double rr = q[o1], ru = q[VOL + o1], rv = q[2 * VOL + o1], rw = q[3 * VOL + o1], rE = q[4 * VOL + o1];
      const double pp = gam1 * (rE - 0.5 * (ru * ru + rv * rv + rw * rw) / rr);
      q[o0] = rr;
      q[VOL + o0] = 0.0;
      q[2 * VOL + o0] = 0.0;
      q[3 * VOL + o0] = 0.0;
      q[4 * VOL + o0] = pp / gam1;
      for (int l = 1; l <= NG; ++l) {
        const long s1 = node_off(d, i, l, k), g1 = node_off(d, i, -l, k);
        q[g1] = q[s1];
        q[VOL + g1] = -q[VOL + s1];
        q[2 * VOL + g1] = -q[2 * VOL + s1];
        q[3 * VOL + g1] = -q[3 * VOL + s1];
        q[4 * VOL + g1] = q[4 * VOL + s1];
      }
    } else {
      // slip wall, tangent in the x-y plane
      const PrimV s = prim_of(q, o1, VOL, gam1);
      double tx = a.met[4][o0], ty = -a.met[3][o0];
      const double J = a.met[9][o0];
      tx *= J;
      ty *= J;
      const double tn = sqrt(tx * tx + ty * ty);
      tx /= tn;
      ty /= tn;
      for (int l = 1; l <= NG; ++l) {
        const long s1 = node_off(d, i, l, k), g1 = node_off(d, i, -l, k);
        const double a0 = q[s1], a1 = q[VOL + s1], a2 = q[2 * VOL + s1], a3 = q[3 * VOL + s1], a4 = q[4 * VOL + s1];
        const double vt = a1 * tx + a2 * ty;
        const double b1 = 2 * vt * tx - a1, b2 = 2 * vt * ty - a2;
        q[g1] = a0;
        q[VOL + g1] = b1;
        q[2 * VOL + g1] = b2;
        q[3 * VOL + g1] = a3;
        // the reference's energy expression, sign of the last term included
        q[4 * VOL + g1] = a4 - 0.5 * (a1 * a1 + a2 * a2 - b1 * b1 + b2 * b2) / a0;
      }
      const double vt = s.u * tx + s.v * ty;
      const double uu = vt * tx, vv = vt * ty;
      q[o0] = s.r;
      q[VOL + o0] = s.r * uu;
      q[2 * VOL + o0] = s.r * vv;
      q[3 * VOL + o0] = s.r * s.w;
      q[4 * VOL + o0] = s.p / gam1 + 0.5 * s.r * (uu * uu + vv * vv + s.w * s.w);
    }
  }
}

__global__ void bc_phase3(const BCArgs a) {
  if (a.check_done && a.st->done) return;
  const Dims& d = a.d;
  const long VOL = d.VOL;
  const double gam1 = a.gam1;
  const long nA = (long)d.IM * (d.KM - 2);        // j faces
  const long nB = (long)(d.JM - 2) * (d.KM - 2);  // i faces (sigma only)
  const long nC = (long)d.IM * d.JM;              // k faces
  const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
  double sg = 0.0;
  bool has = false;
  if (e < nA) {
    const int i = (int)(e % d.IM), k = 1 + (int)(e / d.IM);
    if (a.viscous) {
      for (int l = 0; l <= NG; ++l) {
        const long o = node_off(d, i, -l, k);
        put_prim(a, o, prim_of(a.q, o, VOL, gam1));
      }
      const PrimV s = prim_of(a.q, node_off(d, i, d.JM - 1, k), VOL, gam1);
      for (int l = 0; l < NG; ++l) put_prim(a, node_off(d, i, d.JM - 1 + l, k), s);
    } else if (a.sigma) {
      const long o0 = node_off(d, i, 0, k), o1 = node_off(d, i, d.JM - 1, k);
      sg = smax2(sigma_inv(a, o0, prim_of(a.q, o0, VOL, gam1)), sigma_inv(a, o1, prim_of(a.q, o1, VOL, gam1)));
      has = true;
    }
  } else if (e < nA + nB) {
    if (!a.viscous && a.sigma) {
      const long r = e - nA;
      const int j = 1 + (int)(r % (d.JM - 2)), k = 1 + (int)(r / (d.JM - 2));
      const long o0 = node_off(d, 0, j, k), o1 = node_off(d, d.IM - 1, j, k);
      sg = smax2(sigma_inv(a, o0, prim_of(a.q, o0, VOL, gam1)), sigma_inv(a, o1, prim_of(a.q, o1, VOL, gam1)));
      has = true;
    }
  } else if (e < nA + nB + nC) {
    const long r = e - nA - nB;
    const int i = (int)(r % d.IM), j = (int)(r / d.IM);
    for (int side = 0; side < 2; ++side) {
      const int src = side ? d.KM - 2 : 1, base = side ? d.KM - 1 : 0, dir = side ? 1 : -1;
      const long os = node_off(d, i, j, src);
      double v5[NEQ];
#pragma unroll
      for (int c = 0; c < NEQ; ++c) v5[c] = a.q[c * VOL + os];
      for (int l = 0; l <= NG; ++l) {
        const long o = node_off(d, i, j, base + dir * l);
#pragma unroll
        for (int c = 0; c < NEQ; ++c) a.q[c * VOL + o] = v5[c];
      }
      const PrimV s = prim_of(a.q, os, VOL, gam1);
      if (a.viscous) {
        for (int l = 0; l <= NG; ++l) put_prim(a, node_off(d, i, j, base + dir * l), s);
      } else if (a.sigma) {
        const double x = sigma_inv(a, node_off(d, i, j, base), s);
        sg = has ? smax2(sg, x) : x;
        has = true;
      }
    }
  }
  if (!a.viscous && a.sigma) warp_sigma_max(a, sg, has);
}

// Nodes of the ghosted box outside the interior (i, j, k in 1 .. N-2): the
// six k planes of the outer slabs, then per interior k the six outer j rows,
// then per interior (j, k) the six outer i nodes (x fastest where it can be).
__host__ __device__ inline long shell_nodes(const Dims& d) {
  return 6L * d.IG * d.JG + (long)(d.KM - 2) * 6 * d.IG + (long)(d.KM - 2) * (d.JM - 2) * 6;
}
__device__ __forceinline__ void shell_node(const Dims& d, long e, int& i, int& j, int& k) {
  const long A = 6L * d.IG * d.JG, B = (long)(d.KM - 2) * 6 * d.IG;
  if (e < A) {
    const int s = (int)(e / ((long)d.IG * d.JG));
    const long r = e % ((long)d.IG * d.JG);
    i = (int)(r % d.IG) - NG;
    j = (int)(r / d.IG) - NG;
    k = s < 3 ? s - NG : d.KM - 1 + (s - 3);
  } else if (e < A + B) {
    const long e2 = e - A;
    k = 1 + (int)(e2 / (6L * d.IG));
    const int r = (int)(e2 % (6L * d.IG));
    const int s = r / d.IG;
    i = r % d.IG - NG;
    j = s < 3 ? s - NG : d.JM - 1 + (s - 3);
  } else {
    const long e3 = e - A - B;
    const long kj = e3 / 6;
    const int s = (int)(e3 % 6);
    k = 1 + (int)(kj / (d.JM - 2));
    j = 1 + (int)(kj % (d.JM - 2));
    i = s < 3 ? s - NG : d.IM - 1 + (s - 3);
  }
}

// CBNS_BC_FARFIELD: every node of the ghosted box outside the interior keeps
// its Q; its primitives (viscous runs) follow from that Q, and in inviscid
// runs the grid's boundary nodes add their spectral radii for the next dt.
// e: the thread's shell node (shell_node); every lane of the warp calls this.
__device__ __forceinline__ void farfield_body(const BCArgs& a, long e) {
  const Dims& d = a.d;
  double sg = 0.0;
  bool has = false;
  if (e < shell_nodes(d)) {
    int i, j, k;
    shell_node(d, e, i, j, k);
    const long o = node_off(d, i, j, k);
    const PrimV s = prim_of(a.q, o, d.VOL, a.gam1);
    if (a.viscous) {
      put_prim(a, o, s);
    } else if (a.sigma && i >= 0 && i < d.IM && j >= 0 && j < d.JM && k >= 0 && k < d.KM) {
      sg = sigma_inv(a, o, s);
      has = true;
    }
  }
  if (!a.viscous && a.sigma) warp_sigma_max(a, sg, has);
}

__global__ void bc_farfield(const BCArgs a) {
  if (a.check_done && a.st->done) return;
  farfield_body(a, blockIdx.x * (long)blockDim.x + threadIdx.x);
}

// The same for many blocks in one launch: block b owns CTAs cta[b] ..
// cta[b+1]-1 (so a warp's spectral-radius maximum stays within one block);
// args[b] are its BCArgs.
__global__ void bc_farfield_batched(const BCArgs* args, const int* cta, int nblocks) {
  const int lo = block_of_cta(cta, nblocks, (int)blockIdx.x);
  const BCArgs& a = args[lo];
  if (a.check_done && a.st->done) return;
  farfield_body(a, ((long)blockIdx.x - __ldg(cta + lo)) * blockDim.x + threadIdx.x);
}

// CBNS_BC_CHARACTERISTIC, one face direction per launch (dir 0 = i, 1 = j,
// 2 = k; launched in that order).  Boundary node b, its inward neighbour e,
// outward unit normal n = -+grad(xi_dir)/|grad(xi_dir)| at b.  Subsonic: the
// outgoing invariant R+ = qn_e + 2c_e/(g-1) from e, the incoming
// R- = qn_inf - 2c_inf/(g-1) from the free stream, qn_b = (R+ + R-)/2,
// c_b = (g-1)(R+ - R-)/4; entropy p/rho^g and tangential velocity from e when
// qn_b >= 0, from the free stream otherwise.  Supersonic (|qn_e| >= c_e):
// outflow copies e, inflow takes the free stream.  b's two ghosts along dir
// take b's state.  The i faces cover j, k interior, the j faces every i and
// k interior, the k faces every (i, j): every e is an interior node or a
// face node set earlier in the same call, so the state depends on the
// buffer's interior only (not on its history).  Ghosts off those lines keep
// their state.  Dims of at least 4 keep e off the other face.
__global__ void bc_characteristic(const BCArgs a, int dir, int side0, int nsides) {
  if (a.check_done && a.st->done) return;
  const Dims& d = a.d;
  const int n0 = dir == 0 ? d.JM - 2 : d.IM;
  const int n1 = dir == 2 ? d.JM : d.KM - 2;
  const int nf = dir == 0 ? d.IM : dir == 1 ? d.JM : d.KM;
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= (long)nsides * n0 * n1) return;
  const int side = side0 + (int)(t / ((long)n0 * n1));
  const long r = t % ((long)n0 * n1);
  const int f0 = (int)(r % n0), f1 = (int)(r / n0);
  const int lb = side ? nf - 1 : 0;
  const int i = dir == 0 ? lb : f0;
  const int j = dir == 0 ? f0 + 1 : dir == 1 ? lb : f1;
  const int k = dir == 2 ? lb : f1 + 1;
  const long stride = dir == 0 ? 1L : dir == 1 ? d.PX : d.PL;
  const long out = side ? stride : -stride;  // offset of the next node outward
  const long ob = node_off(d, i, j, k), oe = ob - out;
  const long VOL = d.VOL;
  double* q = a.q;
  const double mx = a.met[3 * dir][ob], my = a.met[3 * dir + 1][ob], mz = a.met[3 * dir + 2][ob];
  const double sgn = side ? 1.0 : -1.0;
  const double mn = sgn / sqrt(mx * mx + my * my + mz * mz);
  const double nx = mx * mn, ny = my * mn, nz = mz * mn;
  const PrimV se = prim_of(q, oe, VOL, a.gam1);
  const double ce = sqrt(a.gamma * se.p / se.r);
  const double qne = se.u * nx + se.v * ny + se.w * nz;
  double qb[5];
  if (fabs(qne) >= ce && qne >= 0.0) {
#pragma unroll
    for (int m = 0; m < 5; ++m) qb[m] = q[m * VOL + oe];
  } else {
    double r_b, u_b, v_b, w_b, p_b;
    const double ci = sqrt(a.gamma * a.p_inf);  // rho_inf = 1
    const double qni = a.u_inf * nx + a.v_inf * ny;
    if (fabs(qne) >= ce) {
      r_b = 1.0; u_b = a.u_inf; v_b = a.v_inf; w_b = 0.0; p_b = a.p_inf;
    } else {
      const double rp = qne + 2.0 * ce / a.gam1, rm = qni - 2.0 * ci / a.gam1;
      const double qnb = 0.5 * (rp + rm), cb = 0.25 * a.gam1 * (rp - rm);
      double s, dq;
      if (qnb >= 0.0) {
        s = se.p / pow(se.r, a.gamma);
        dq = qnb - qne;
        u_b = se.u + dq * nx; v_b = se.v + dq * ny; w_b = se.w + dq * nz;
      } else {
        s = a.p_inf;
        dq = qnb - qni;
        u_b = a.u_inf + dq * nx; v_b = a.v_inf + dq * ny; w_b = dq * nz;
      }
      r_b = pow(cb * cb / (a.gamma * s), 1.0 / a.gam1);
      p_b = r_b * cb * cb / a.gamma;
    }
    qb[0] = r_b;
    qb[1] = r_b * u_b;
    qb[2] = r_b * v_b;
    qb[3] = r_b * w_b;
    qb[4] = p_b / a.gam1 + 0.5 * r_b * (u_b * u_b + v_b * v_b + w_b * w_b);
  }
#pragma unroll
  for (int l = 0; l <= NG; ++l)
#pragma unroll
    for (int m = 0; m < 5; ++m) q[m * VOL + ob + l * out] = qb[m];
}

// CBNS_BC_OGRID, last pass: every node with i < wrap or i >= IM - wrap, the
// i ghosts included, over the whole ghosted (j, k) box, takes Q (and in
// viscous runs the primitives) of the node P = IM - 2*wrap away, which lies
// on the stored periodic line and is final by now.
__global__ void bc_wrap(const BCArgs a) {
  if (a.check_done && a.st->done) return;
  const Dims& d = a.d;
  const int W = a.wrap + NG;  // copied positions either side
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= 2L * W * d.JG * d.KG) return;
  const int u = (int)(t % (2 * W));
  const long r = t / (2 * W);
  const int j = (int)(r % d.JG) - NG, k = (int)(r / d.JG) - NG;
  const int P = d.IM - 2 * a.wrap;
  const int i = u < W ? u - NG : d.IM - a.wrap + (u - W);
  const int src = u < W ? i + P : i - P;
  const long o = node_off(d, i, j, k), os = node_off(d, src, j, k);
  const long VOL = d.VOL;
#pragma unroll
  for (int c = 0; c < NEQ; ++c) a.q[c * VOL + o] = a.q[c * VOL + os];
  if (a.viscous) {
#pragma unroll
    for (int m = 0; m < 6; ++m) a.prim[m][o] = a.prim[m][os];
  }
}

// Interior primitives (rho,u,v,w,p,T) from Q, the first part of
// primitive_bc_kernel (:59-79); needed when the primitive arrays do not yet
// describe the buffer the boundary conditions act on.
__global__ void bc_interior_prims(const BCArgs a) {
  const Dims& d = a.d;
  const long n = (long)(d.IM - 2) * (d.JM - 2) * (d.KM - 2);
  const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (e >= n) return;
  const int i = 1 + (int)(e % (d.IM - 2));
  const long r = e / (d.IM - 2);
  const int j = 1 + (int)(r % (d.JM - 2)), k = 1 + (int)(r / (d.JM - 2));
  const long o = node_off(d, i, j, k);
  put_prim(a, o, prim_of(a.q, o, d.VOL, a.gam1));
}

inline unsigned nblk(long n, int b) { return (unsigned)((n + b - 1) / b); }

}  // namespace

cudaError_t launch_bc(const BCArgs& a, bool interior_prims, cudaStream_t s, int* launches) {
  const Dims& d = a.d;
  const int B = 128;
  int nl = 0;
  if (interior_prims && a.viscous) {
    bc_interior_prims<<<nblk((long)(d.IM - 2) * (d.JM - 2) * (d.KM - 2), B), B, 0, s>>>(a);
    ++nl;
  }
  const long n3 = (long)d.IM * (d.KM - 2) + (long)(d.JM - 2) * (d.KM - 2) + (long)d.IM * d.JM;
  if (a.wrap) {
    // O-grid: wall on every i of j = 0, characteristic far field on j = JM-1,
    // the reference's k faces, then the copies across the seam
    BCArgs w = a;
    w.i_begin = 1u;
    w.i_end = (unsigned)d.IM;
    w.sigma = 0;
    bc_phase2<<<nblk((long)d.IM * (d.KM - 2), B), B, 0, s>>>(w);
    bc_characteristic<<<nblk((long)d.IM * (d.KM - 2), B), B, 0, s>>>(w, 1, 1, 1);
    bc_phase3<<<nblk(n3, B), B, 0, s>>>(w);
    bc_wrap<<<nblk(2L * (a.wrap + NG) * d.JG * d.KG, B), B, 0, s>>>(w);
    nl += 4;
    if (launches) *launches += nl;
    return cudaGetLastError();
  }
  if (a.farfield) {
    if (a.characteristic) {
      bc_characteristic<<<nblk(2L * (d.JM - 2) * (d.KM - 2), B), B, 0, s>>>(a, 0, 0, 2);
      bc_characteristic<<<nblk(2L * d.IM * (d.KM - 2), B), B, 0, s>>>(a, 1, 0, 2);
      bc_characteristic<<<nblk(2L * d.IM * d.JM, B), B, 0, s>>>(a, 2, 0, 2);
      nl += 3;
    }
    if (a.viscous || a.sigma) {
      bc_farfield<<<nblk(shell_nodes(d), B), B, 0, s>>>(a);
      ++nl;
    }
    if (launches) *launches += nl;
    return cudaGetLastError();
  }
  bc_phase1<<<nblk(2L * (d.JM - 2) * (d.KM - 2), B), B, 0, s>>>(a);
  ++nl;
  // phase 2 has work only if some i takes the wake or the wall branch
  const bool wake_any = (a.i_begin - 1u) > 0u;  // i = 0 satisfies i_begin-1 > i
  const bool wall_any = a.i_end > 0u;
  if (wake_any || wall_any) {
    bc_phase2<<<nblk((long)d.IM * (d.KM - 2), B), B, 0, s>>>(a);
    ++nl;
  }
  bc_phase3<<<nblk(n3, B), B, 0, s>>>(a);
  ++nl;
  if (launches) *launches += nl;
  return cudaGetLastError();
}

// CTAs of 128 threads the batched far-field kernel gives one block.
int bc_farfield_ctas(const Dims& d) { return (int)nblk(shell_nodes(d), 128); }

cudaError_t launch_bc_farfield_batched(const BCArgs* args, const int* cta, int nblocks, int total_ctas,
                                       cudaStream_t s) {
  if (total_ctas <= 0) return cudaSuccess;
  bc_farfield_batched<<<total_ctas, 128, 0, s>>>(args, cta, nblocks);
  return cudaGetLastError();
}

}  // namespace cbns
