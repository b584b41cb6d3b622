// visc.cu - viscous node fluxes in one kernel.
//
// Replaces the reference's calc_viscous_terms (src/calc_viscous_terms.cu:16-88:
// four gradient_wg_kernel launches, src/gradient_kernel.cu:135-255, and
// viscous_terms_kernel, src/viscous_terms_kernel.cu:13-107) together with the
// node-flux half of calc_viscous_flux_contribution (viscous_flux_kernel,
// src/viscous_flux_kernel.cu:13-112).  Per node of the ghosted box minus its
// outermost layer (the nodes whose fluxes the divergence can reach) it forms
// the computational-space gradients of u, v, w, T with the reference's
// 4th-order stencils (biased at the second layer of the ghosted box), the
// Sutherland viscosity, the stress tensor and heat flux, and the three node
// fluxes E_v, F_v, G_v (momentum and energy components, normals J*grad(xi)).
// None of the 12 gradients, 6 stresses or 3 heat fluxes go to HBM.  In stage 3
// of a step (and at start-up) it also forms the viscous spectral radius of every
// grid node for the next time step (src/time_step_kernel.cu:13-96).
// A second kernel, visc_div_kernel, takes the 4th-order divergence of the node
// fluxes at every interior node (the other half of calc_viscous_flux_contribution,
// viscous_contribution_kernel, src/viscous_contribution_kernel.cu:13-71) into
// four arrays, which the stage kernel reads with one coalesced load each: the
// 48-point stencil runs in a streaming kernel of its own instead of in the
// stage kernel's latency-bound update.
#include "visc.cuh"

namespace cbns {

namespace {

// derivative of a ghosted field along stride s at ghosted index g of n
__device__ __forceinline__ double dg(const double* f, long o, long s, int g, int n) {
  if (g == 1)
    return -5.0 / 6.0 * f[o] - 0.25 * f[o - s] + 1.5 * f[o + s] - 0.5 * f[o + 2 * s] + (1.0 / 12.0) * f[o + 3 * s];
  if (g == n - 2)
    return (5.0 / 6.0) * f[o] - 1.0 / 12.0 * f[o - 3 * s] + 0.5 * f[o - 2 * s] - 1.5 * f[o - s] + 0.25 * f[o + s];
  return (1.0 / 12.0) * f[o - 2 * s] - 2.0 / 3.0 * f[o - s] + (2.0 / 3.0) * f[o + s] - 1.0 / 12.0 * f[o + 2 * s];
}

// Node e of the ghosted box minus its outer layer (i fastest); every lane of
// the warp calls this (the spectral-radius maximum is a warp reduction).
__device__ __forceinline__ void visc_node_body(const ViscArgs& a, long e) {
  const Dims& d = a.d;
  const int VI = d.IG - 2, VJ = d.JG - 2, VK = d.KG - 2;
  double sg = 0.0;
  bool has = false;
  if (e < (long)VI * VJ * VK) {
    const int gi = 1 + (int)(e % VI);
    const long r = e / VI;
    const int gj = 1 + (int)(r % VJ), gk = 1 + (int)(r / VJ);
    const int i = gi - NG, j = gj - NG, k = gk - NG;
    const long o = node_off(d, i, j, k);
    const long sj = d.PX, sk = d.PL;
    const double *U = a.prim[1], *V = a.prim[2], *W = a.prim[3], *T = a.prim[5];
    const double u_x = dg(U, o, 1, gi, d.IG), u_e = dg(U, o, sj, gj, d.JG), u_z = dg(U, o, sk, gk, d.KG);
    const double v_x = dg(V, o, 1, gi, d.IG), v_e = dg(V, o, sj, gj, d.JG), v_z = dg(V, o, sk, gk, d.KG);
    const double w_x = dg(W, o, 1, gi, d.IG), w_e = dg(W, o, sj, gj, d.JG), w_z = dg(W, o, sk, gk, d.KG);
    const double T_x = dg(T, o, 1, gi, d.IG), T_e = dg(T, o, sj, gj, d.JG), T_z = dg(T, o, sk, gk, d.KG);
    double m9[9];
#pragma unroll
    for (int m = 0; m < 9; ++m) m9[m] = a.met[m][o];
    const double J = a.met[9][o];
    const double Tl = T[o];
    double mu = (1.0 + a.C_T_inf) / (Tl + a.C_T_inf) * sqrt(Tl * Tl * Tl);
    a.mu[o] = mu;
    // chain rule: d/dx = xi_x d/dxi + eta_x d/deta + zeta_x d/dzeta, etc.
    const double ux = u_x * m9[0] + u_e * m9[3] + u_z * m9[6];
    const double uy = u_x * m9[1] + u_e * m9[4] + u_z * m9[7];
    const double uz = u_x * m9[2] + u_e * m9[5] + u_z * m9[8];
    const double vx = v_x * m9[0] + v_e * m9[3] + v_z * m9[6];
    const double vy = v_x * m9[1] + v_e * m9[4] + v_z * m9[7];
    const double vz = v_x * m9[2] + v_e * m9[5] + v_z * m9[8];
    const double wx = w_x * m9[0] + w_e * m9[3] + w_z * m9[6];
    const double wy = w_x * m9[1] + w_e * m9[4] + w_z * m9[7];
    const double wz = w_x * m9[2] + w_e * m9[5] + w_z * m9[8];
    const double mr = mu * a.Re_inv;
    const double txx = (2.0 / 3.0) * mr * (2.0 * ux - vy - wz);
    const double tyy = (2.0 / 3.0) * mr * (2.0 * vy - ux - wz);
    const double tzz = (2.0 / 3.0) * mr * (2.0 * wz - ux - vy);
    const double txy = mr * (uy + vx), txz = mr * (uz + wx), tyz = mr * (vz + wy);
    const double kq = mr * a.qc;
    const double qx = kq * (m9[0] * T_x + m9[3] * T_e + m9[6] * T_z);
    const double qy = kq * (m9[1] * T_x + m9[4] * T_e + m9[7] * T_z);
    const double qz = kq * (m9[2] * T_x + m9[5] * T_e + m9[8] * T_z);
    const double uu = U[o], vv = V[o], ww = W[o];
    const double ex = uu * txx + vv * txy + ww * txz - qx;
    const double ey = uu * txy + vv * tyy + ww * tyz - qy;
    const double ez = uu * txz + vv * tyz + ww * tzz - qz;
#pragma unroll
    for (int dd = 0; dd < 3; ++dd) {
      const double nx = m9[3 * dd] * J, ny = m9[3 * dd + 1] * J, nz = m9[3 * dd + 2] * J;
      a.vflux[4 * dd + 0][o] = nx * txx + ny * txy + nz * txz;
      a.vflux[4 * dd + 1][o] = nx * txy + ny * tyy + nz * tyz;
      a.vflux[4 * dd + 2][o] = nx * txz + ny * tyz + nz * tzz;
      a.vflux[4 * dd + 3][o] = nx * ex + ny * ey + nz * ez;
    }
    if (a.sigma && i >= 0 && i < d.IM && j >= 0 && j < d.JM && k >= 0 && k < d.KM) {
      const double rr = a.prim[0][o], pp = a.prim[4][o];
      const double c = sqrt(a.gamma * pp / rr);
      const double fv = a.dt_full ? 2.0 * mu * a.C_dt_v / rr
                                  : 2.0 * mu * a.C_dt_v * sqrt(uu * uu + vv * vv + ww * ww) / c / rr;
      double s = 0.0;
#pragma unroll
      for (int dd = 0; dd < 3; ++dd) {
        const double mx = m9[3 * dd], my = m9[3 * dd + 1], mz = m9[3 * dd + 2];
        const double na = sqrt(mx * mx + my * my + mz * mz);
        s += fabs(uu * mx + vv * my + ww * mz) + c * na + na * na * fv;
      }
      sg = s;
      has = true;
    }
  }
  if (a.sigma) {
    const bool nan = has && (sg != sg);
    double m = (has && !nan) ? sg : 0.0;
    const unsigned anyhas = __ballot_sync(0xffffffffu, has);
    const unsigned anynan = __ballot_sync(0xffffffffu, nan);
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, s));
    if ((threadIdx.x & 31) == 0 && anyhas)
      atomic_max_sigma(&a.st->sigma_bits, anynan ? __longlong_as_double(0x7ff8000000000000ll) : m);
  }
}

// 4th-order central derivative of a node field along a stride, at offset o.
__device__ __forceinline__ double d4(const double* f, long o, long s) {
  return (1.0 / 12.0) * __ldg(f + o - 2 * s) - (2.0 / 3.0) * __ldg(f + o - s) + (2.0 / 3.0) * __ldg(f + o + s) -
         (1.0 / 12.0) * __ldg(f + o + 2 * s);
}

// Interior node e (i fastest): the divergence of the node fluxes; the
// reference takes the i-derivative at (i,j-1,k-1), the j-derivative at
// (i-1,j,k-1), the k-derivative at (i-1,j-1,k) (CBNS_VISDIV_REFERENCE), or
// all three at the node (CBNS_VISDIV_CENTERED).
__device__ __forceinline__ void visc_div_body(const ViscArgs& a, long e) {
  const Dims& d = a.d;
  const int NI = d.IM - 2, NJ = d.JM - 2;
  if (e >= (long)NI * NJ * (d.KM - 2)) return;
  const int i = 1 + (int)(e % NI);
  const long r = e / NI;
  const int j = 1 + (int)(r % NJ), k = 1 + (int)(r / NJ);
  const long o = node_off(d, i, j, k);
  const long sh = a.visdiv == 0 ? 1 : 0;
  const long oi = o - sh * (d.PX + d.PL), oj = o - sh * (1 + d.PL), ok = o - sh * (1 + d.PX);
#pragma unroll
  for (int n = 0; n < 4; ++n)
    a.dfv[n][o] = d4(a.vflux[n], oi, 1) + d4(a.vflux[4 + n], oj, d.PX) + d4(a.vflux[8 + n], ok, d.PL);
}

__global__ void __launch_bounds__(256) visc_div_kernel(const ViscArgs a) {
  if (a.check_done && a.st->done) return;
  visc_div_body(a, blockIdx.x * (long)blockDim.x + threadIdx.x);
}

__global__ void __launch_bounds__(256) visc_div_batched(const ViscArgs* args, const int* cta, int nblocks) {
  int lo = 0, hi = nblocks - 1;  // the last b with cta[b] <= blockIdx.x
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(cta + mid) <= (int)blockIdx.x) lo = mid;
    else hi = mid - 1;
  }
  const ViscArgs& a = args[lo];
  if (a.check_done && a.st->done) return;
  visc_div_body(a, ((long)blockIdx.x - __ldg(cta + lo)) * blockDim.x + threadIdx.x);
}

__global__ void __launch_bounds__(128) visc_node_kernel(const ViscArgs a) {
  if (a.check_done && a.st->done) return;
  visc_node_body(a, blockIdx.x * (long)blockDim.x + threadIdx.x);
}

// Many blocks in one launch: block b owns CTAs cta[b] .. cta[b+1]-1, args[b]
// are its ViscArgs.
__global__ void __launch_bounds__(128) visc_node_batched(const ViscArgs* args, const int* cta, int nblocks) {
  int lo = 0, hi = nblocks - 1;  // the last b with cta[b] <= blockIdx.x
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(cta + mid) <= (int)blockIdx.x) lo = mid;
    else hi = mid - 1;
  }
  const ViscArgs& a = args[lo];
  if (a.check_done && a.st->done) return;
  visc_node_body(a, ((long)blockIdx.x - __ldg(cta + lo)) * blockDim.x + threadIdx.x);
}

}  // namespace

cudaError_t launch_visc(const ViscArgs& a, cudaStream_t s) {
  visc_node_kernel<<<visc_ctas(a.d), 128, 0, s>>>(a);
  visc_div_kernel<<<visc_div_ctas(a.d), 256, 0, s>>>(a);
  return cudaGetLastError();
}

int visc_div_ctas(const Dims& d) {
  const long n = (long)(d.IM - 2) * (d.JM - 2) * (d.KM - 2);
  return (int)((n + 255) / 256);
}

int visc_ctas(const Dims& d) {
  const long n = (long)(d.IG - 2) * (d.JG - 2) * (d.KG - 2);
  return (int)((n + 127) / 128);
}

cudaError_t launch_visc_batched(const ViscArgs* args, const int* cta, int nblocks, int total_ctas,
                                const int* dcta, int dtotal, cudaStream_t s) {
  if (total_ctas <= 0) return cudaSuccess;
  visc_node_batched<<<total_ctas, 128, 0, s>>>(args, cta, nblocks);
  visc_div_batched<<<dtotal, 256, 0, s>>>(args, dcta, nblocks);
  return cudaGetLastError();
}

}  // namespace cbns
