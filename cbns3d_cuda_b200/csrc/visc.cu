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

// Tiles of the node kernel: 32 x 8 nodes of the box (i fastest, one warp per
// row), marched through a chunk of k planes.  Shared memory holds the plane
// being computed with a 3-node halo in i and j (the stencils reach 2 nodes, the
// one-sided ones at the box edges 3) and a ring of the tile's own nodes on the
// planes k-2 .. k+2 (the k stencils), for the four differentiated fields u, v,
// w, T.  Each thread holds the next plane's values for the ring (plane k+3)
// and the halo (plane k+1) in registers: their loads are issued before the
// plane's arithmetic and stored to shared memory after it.
constexpr int VTI = 32, VTJ = 8, VH = 3, VT = VTI * VTJ, VR = 5;
constexpr int CW = VTI + 2 * VH, CJ = VTJ + 2 * VH;
constexpr int VHALO = 2 * VH * VTJ + 2 * VH * VTI;  // 240 halo nodes: i strips, then j strips
static_assert(VHALO <= VT, "one halo node per thread");

// T: the node arithmetic and the staged fields (double for the plain path,
// float for the FP32-flux precisions)
template <typename T>
struct ViscSmem {
  T c[4][CJ][CW];            // plane k with its halo (corners unused)
  T ring[VR][4][VTJ][VTI];   // the tile on planes k-2 .. k+2, slot = plane mod 5
};

// derivative from the values v(-3) .. v(+3) along the axis (only those the
// stencil uses are read), at ghosted index g of n: the reference's 4th-order
// stencils, one-sided at g = 1 and g = n - 2 (src/gradient_kernel.cu:135-255)
template <typename T, typename A>
__device__ __forceinline__ T dgv(const A& v, int g, int n) {
  if (g == 1) return T(-5.0 / 6.0) * v(0) - T(0.25) * v(-1) + T(1.5) * v(1) - T(0.5) * v(2) + T(1.0 / 12.0) * v(3);
  if (g == n - 2)
    return T(5.0 / 6.0) * v(0) - T(1.0 / 12.0) * v(-3) + T(0.5) * v(-2) - T(1.5) * v(-1) + T(0.25) * v(1);
  return T(1.0 / 12.0) * v(-2) - T(2.0 / 3.0) * v(-1) + T(2.0 / 3.0) * v(1) - T(1.0 / 12.0) * v(2);
}

// halo node h of the tile at (i0, j0): ghosted (gi, gj) and its place in c
__device__ __forceinline__ void halo_node(int h, int i0, int j0, int& gi, int& gj, int& cy, int& cx) {
  if (h < 2 * VH * VTJ) {  // i strips: 3 columns x 8 rows each side
    const int side = h / (VH * VTJ), r = h % (VH * VTJ), col = r % VH, row = r / VH;
    cx = side ? VH + VTI + col : col;
    cy = VH + row;
    gi = side ? i0 + VTI + col : i0 - VH + col;
    gj = j0 + row;
  } else {  // j strips: 32 columns x 3 rows each side
    const int h2 = h - 2 * VH * VTJ, side = h2 / (VH * VTI), r = h2 % (VH * VTI), col = r % VTI, row = r / VTI;
    cx = VH + col;
    cy = side ? VH + VTJ + row : row;
    gi = i0 + col;
    gj = side ? j0 + VTJ + row : j0 - VH + row;
  }
}

// CTA `cta` of one block's node-kernel grid (tiles in i, then j, then k chunks).
// Every thread of the CTA calls this (block-wide barriers; the spectral-radius
// maximum is a warp reduction).
template <typename V>
__device__ __forceinline__ void visc_node_tile(const ViscArgs& a, int cta, ViscSmem<V>& sm) {
  using T = V;  // the arithmetic follows the storage
  const Dims& d = a.d;
  const int IG = d.IG, JG = d.JG, KG = d.KG;
  const int nti = (IG - 2 + VTI - 1) / VTI, ntj = (JG - 2 + VTJ - 1) / VTJ;
  const int ti = cta % nti, tj = (cta / nti) % ntj, kc = cta / (nti * ntj);
  const int i0 = 1 + ti * VTI, j0 = 1 + tj * VTJ;
  const int kb = 1 + kc * a.kc, ke = min(KG - 1, kb + a.kc);  // planes kb .. ke-1 of 1 .. KG-2
  const int t = threadIdx.x, tx = t % VTI, ty = t / VTI;
  const int gi = i0 + tx, gj = j0 + ty;
  const bool own = gi <= IG - 1 && gj <= JG - 1;        // a node of the ghosted box: kept in the ring
  const bool valid = gi <= IG - 2 && gj <= JG - 2;      // a node whose fluxes this thread forms
  const long sk = d.PL;
  const double* F[4] = {a.prim[1], a.prim[2], a.prim[3], a.prim[5]};
  const long o_own = node_off(d, gi - NG, gj - NG, -NG);  // plane 0 of this thread's column
  int hgi = 0, hgj = 0, hcy = 0, hcx = 0;
  const bool hal = t < VHALO;
  if (hal) halo_node(t, i0, j0, hgi, hgj, hcy, hcx);
  const bool hin = hal && hgi >= 0 && hgi <= IG - 1 && hgj >= 0 && hgj <= JG - 1;
  const long o_hal = hin ? node_off(d, hgi - NG, hgj - NG, -NG) : 0;

  T rn[4], hn[4];
  auto load_ring = [&](int p, T v[4]) {
    if (own && p >= 0 && p <= KG - 1) {
#pragma unroll
      for (int f = 0; f < 4; ++f) v[f] = (T)__ldg(F[f] + o_own + p * sk);
    }
  };
  auto load_halo = [&](int p, T v[4]) {
    if (hin) {
#pragma unroll
      for (int f = 0; f < 4; ++f) v[f] = (T)__ldg(F[f] + o_hal + p * sk);
    }
  };
  auto put_ring = [&](int p, const T v[4]) {
    if (own && p >= 0 && p <= KG - 1) {
#pragma unroll
      for (int f = 0; f < 4; ++f) sm.ring[p % VR][f][ty][tx] = v[f];
    }
  };
  auto put_plane = [&](int p, const T h[4]) {  // c <- plane p: halo from h, the tile from the ring
    if (hin) {
#pragma unroll
      for (int f = 0; f < 4; ++f) sm.c[f][hcy][hcx] = h[f];
    }
    if (own) {
#pragma unroll
      for (int f = 0; f < 4; ++f) sm.c[f][VH + ty][VH + tx] = sm.ring[p % VR][f][ty][tx];
    }
  };

  // warm-up: the ring on planes kb-2 .. kb+2, plane kb in c
  for (int p = kb - 2; p <= kb + 2; ++p) {
    load_ring(p, rn);
    put_ring(p, rn);
  }
  load_halo(kb, hn);
  put_plane(kb, hn);
  __syncthreads();

  double sg = 0.0;  // the thread's largest spectral radius (grid nodes only)
  bool has = false, nanseen = false;
  for (int k = kb; k < ke; ++k) {
    const bool more = k + 1 < ke;
    if (more) {
      load_ring(k + 3, rn);
      load_halo(k + 1, hn);
    }
    if (valid) {
      const long o = o_own + k * sk;
      T m9[9];
#pragma unroll
      for (int m = 0; m < 9; ++m) m9[m] = (T)__ldg(a.met[m] + o);
      const T J = (T)__ldg(a.met[9] + o);
      T gx[4], ge[4], gz[4];
      const int s0 = (k + VR - 2) % VR, s1 = (k + VR - 1) % VR, s3 = (k + 1) % VR, s4 = (k + 2) % VR;
#pragma unroll
      for (int f = 0; f < 4; ++f) {
        const T (*cp)[CW] = sm.c[f];
        const int y = VH + ty, x = VH + tx;
        gx[f] = dgv<T>([&](int q) { return cp[y][x + q]; }, gi, IG);
        ge[f] = dgv<T>([&](int q) { return cp[y + q][x]; }, gj, JG);
        // along k: the ring; the one-sided stencils of planes 1 and KG-2 reach
        // a third plane (4 and KG-5), read from global memory
        gz[f] = dgv<T>(
            [&](int q) -> T {
              switch (q) {
                case -2: return sm.ring[s0][f][ty][tx];
                case -1: return sm.ring[s1][f][ty][tx];
                case 0: return cp[y][x];
                case 1: return sm.ring[s3][f][ty][tx];
                case 2: return sm.ring[s4][f][ty][tx];
                default: return (T)__ldg(F[f] + o + q * sk);
              }
            },
            k, KG);
      }
      const T uu = sm.c[0][VH + ty][VH + tx], vv = sm.c[1][VH + ty][VH + tx], ww = sm.c[2][VH + ty][VH + tx];
      const T Tl = sm.c[3][VH + ty][VH + tx];
      const T CT = (T)a.C_T_inf;
      const T mu = (T(1) + CT) / (Tl + CT) * sqrt(Tl * Tl * Tl);
      a.mu[o] = (double)mu;
      // chain rule: d/dx = xi_x d/dxi + eta_x d/deta + zeta_x d/dzeta, etc.
      const T ux = gx[0] * m9[0] + ge[0] * m9[3] + gz[0] * m9[6];
      const T uy = gx[0] * m9[1] + ge[0] * m9[4] + gz[0] * m9[7];
      const T uz = gx[0] * m9[2] + ge[0] * m9[5] + gz[0] * m9[8];
      const T vx = gx[1] * m9[0] + ge[1] * m9[3] + gz[1] * m9[6];
      const T vy = gx[1] * m9[1] + ge[1] * m9[4] + gz[1] * m9[7];
      const T vz = gx[1] * m9[2] + ge[1] * m9[5] + gz[1] * m9[8];
      const T wx = gx[2] * m9[0] + ge[2] * m9[3] + gz[2] * m9[6];
      const T wy = gx[2] * m9[1] + ge[2] * m9[4] + gz[2] * m9[7];
      const T wz = gx[2] * m9[2] + ge[2] * m9[5] + gz[2] * m9[8];
      const T mr = mu * (T)a.Re_inv;
      const T txx = T(2.0 / 3.0) * mr * (T(2) * ux - vy - wz);
      const T tyy = T(2.0 / 3.0) * mr * (T(2) * vy - ux - wz);
      const T tzz = T(2.0 / 3.0) * mr * (T(2) * wz - ux - vy);
      const T txy = mr * (uy + vx), txz = mr * (uz + wx), tyz = mr * (vz + wy);
      const T kq = mr * (T)a.qc;
      const T qx = kq * (m9[0] * gx[3] + m9[3] * ge[3] + m9[6] * gz[3]);
      const T qy = kq * (m9[1] * gx[3] + m9[4] * ge[3] + m9[7] * gz[3]);
      const T qz = kq * (m9[2] * gx[3] + m9[5] * ge[3] + m9[8] * gz[3]);
      const T ex = uu * txx + vv * txy + ww * txz - qx;
      const T ey = uu * txy + vv * tyy + ww * tyz - qy;
      const T ez = uu * txz + vv * tyz + ww * tzz - qz;
#pragma unroll
      for (int dd = 0; dd < 3; ++dd) {
        const T nx = m9[3 * dd] * J, ny = m9[3 * dd + 1] * J, nz = m9[3 * dd + 2] * J;
        reinterpret_cast<V*>(a.vflux[4 * dd + 0])[o] = nx * txx + ny * txy + nz * txz;
        reinterpret_cast<V*>(a.vflux[4 * dd + 1])[o] = nx * txy + ny * tyy + nz * tyz;
        reinterpret_cast<V*>(a.vflux[4 * dd + 2])[o] = nx * txz + ny * tyz + nz * tzz;
        reinterpret_cast<V*>(a.vflux[4 * dd + 3])[o] = nx * ex + ny * ey + nz * ez;
      }
      const int i = gi - NG, j = gj - NG, kk = k - NG;
      if (a.sigma && i >= 0 && i < d.IM && j >= 0 && j < d.JM && kk >= 0 && kk < d.KM) {
        // the spectral radius for the next dt, in FP64 from the FP64 fields
        // whatever T is (src/time_step_kernel.cu:13-96)
        const double rr = __ldg(a.prim[0] + o), pp = __ldg(a.prim[4] + o);
        const bool t64 = sizeof(T) == 8;
        const double ud = t64 ? (double)uu : __ldg(a.prim[1] + o), vd = t64 ? (double)vv : __ldg(a.prim[2] + o),
                     wd = t64 ? (double)ww : __ldg(a.prim[3] + o), Td = t64 ? (double)Tl : __ldg(a.prim[5] + o);
        const double mud = t64 ? (double)mu : (1.0 + a.C_T_inf) / (Td + a.C_T_inf) * sqrt(Td * Td * Td);
        const double c = sqrt(a.gamma * pp / rr);
        const double fv = a.dt_full ? 2.0 * mud * a.C_dt_v / rr
                                    : 2.0 * mud * a.C_dt_v * sqrt(ud * ud + vd * vd + wd * wd) / c / rr;
        double s = 0.0;
#pragma unroll
        for (int dd = 0; dd < 3; ++dd) {
          const double mx = t64 ? (double)m9[3 * dd] : __ldg(a.met[3 * dd] + o);
          const double my = t64 ? (double)m9[3 * dd + 1] : __ldg(a.met[3 * dd + 1] + o);
          const double mz = t64 ? (double)m9[3 * dd + 2] : __ldg(a.met[3 * dd + 2] + o);
          const double na = sqrt(mx * mx + my * my + mz * mz);
          s += fabs(ud * mx + vd * my + wd * mz) + c * na + na * na * fv;
        }
        if (s != s) nanseen = true;
        else if (!has || s > sg) sg = s;
        has = true;
      }
    }
    __syncthreads();  // plane k and ring slot k-2 are no longer read
    if (more) {
      put_ring(k + 3, rn);
      put_plane(k + 1, hn);
    }
    __syncthreads();
  }
  if (a.sigma) {
    const bool nan = nanseen;
    double m = (has && !nan) ? sg : 0.0;
    const unsigned anyhas = __ballot_sync(0xffffffffu, has);
    const unsigned anynan = __ballot_sync(0xffffffffu, nan);
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, s));
    if ((threadIdx.x & 31) == 0 && anyhas)
      atomic_max_sigma(&a.st->sigma_bits, anynan ? __longlong_as_double(0x7ff8000000000000ll) : m);
  }
}

// 4th-order central derivative of a node field along a stride, at offset o
// (in the storage type V).
template <typename V>
__device__ __forceinline__ V d4(const double* fd, long o, long s) {
  const V* f = reinterpret_cast<const V*>(fd);
  return V(1.0 / 12.0) * __ldg(f + o - 2 * s) - V(2.0 / 3.0) * __ldg(f + o - s) + V(2.0 / 3.0) * __ldg(f + o + s) -
         V(1.0 / 12.0) * __ldg(f + o + 2 * s);
}

// Interior node e (i fastest): the divergence of the node fluxes; the
// reference takes the i-derivative at (i,j-1,k-1), the j-derivative at
// (i-1,j,k-1), the k-derivative at (i-1,j-1,k) (CBNS_VISDIV_REFERENCE), or
// all three at the node (CBNS_VISDIV_CENTERED).
template <typename V>
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
    reinterpret_cast<V*>(a.dfv[n])[o] =
        d4<V>(a.vflux[n], oi, 1) + d4<V>(a.vflux[4 + n], oj, d.PX) + d4<V>(a.vflux[8 + n], ok, d.PL);
}

template <typename V>
__global__ void __launch_bounds__(256) visc_div_kernel(const ViscArgs a) {
  if (a.check_done && a.st->done) return;
  visc_div_body<V>(a, blockIdx.x * (long)blockDim.x + threadIdx.x);
}

template <typename V>
__global__ void __launch_bounds__(256) visc_div_batched(const ViscArgs* args, const int* cta, int nblocks) {
  const int lo = block_of_cta(cta, nblocks, (int)blockIdx.x);
  const ViscArgs& a = args[lo];
  if (a.check_done && a.st->done) return;
  visc_div_body<V>(a, ((long)blockIdx.x - __ldg(cta + lo)) * blockDim.x + threadIdx.x);
}

template <typename V>
__global__ void __launch_bounds__(VT, sizeof(V) == 4 ? 3 : 2) visc_node_kernel(const ViscArgs a) {
  if (a.check_done && a.st->done) return;
  extern __shared__ __align__(16) unsigned char vraw[];
  visc_node_tile<V>(a, blockIdx.x, *reinterpret_cast<ViscSmem<V>*>(vraw));
}

// Many blocks in one launch: block b owns CTAs cta[b] .. cta[b+1]-1, args[b]
// are its ViscArgs.
template <typename V>
__global__ void __launch_bounds__(VT, sizeof(V) == 4 ? 3 : 2) visc_node_batched(const ViscArgs* args, const int* cta,
                                                                               int nblocks) {
  const int lo = block_of_cta(cta, nblocks, (int)blockIdx.x);
  const ViscArgs& a = args[lo];
  if (a.check_done && a.st->done) return;
  extern __shared__ __align__(16) unsigned char vraw[];
  visc_node_tile<V>(a, (int)blockIdx.x - __ldg(cta + lo), *reinterpret_cast<ViscSmem<V>*>(vraw));
}

cudaError_t visc_prepare() {
  static bool done = false;
  if (done) return cudaSuccess;
  const int s64 = (int)sizeof(ViscSmem<double>), s32 = (int)sizeof(ViscSmem<float>);
  cudaError_t e = cudaFuncSetAttribute(visc_node_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, s64);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(visc_node_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, s32);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(visc_node_batched<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, s64);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(visc_node_batched<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, s32);
  done = e == cudaSuccess;
  return e;
}

}  // namespace

cudaError_t launch_visc(const ViscArgs& a, cudaStream_t s) {
  cudaError_t e = visc_prepare();
  if (e != cudaSuccess) return e;
  if (a.f32) {
    visc_node_kernel<float><<<visc_ctas(a), VT, sizeof(ViscSmem<float>), s>>>(a);
    visc_div_kernel<float><<<visc_div_ctas(a.d), 256, 0, s>>>(a);
  } else {
    visc_node_kernel<double><<<visc_ctas(a), VT, sizeof(ViscSmem<double>), s>>>(a);
    visc_div_kernel<double><<<visc_div_ctas(a.d), 256, 0, s>>>(a);
  }
  return cudaGetLastError();
}

int visc_div_ctas(const Dims& d) {
  const long n = (long)(d.IM - 2) * (d.JM - 2) * (d.KM - 2);
  return (int)((n + 255) / 256);
}

int visc_kchunk(const Dims& d, int nsm) {
  // chunks enough for about four waves of 2 CTAs per SM, at least 16 planes
  // each (each chunk loads 5 planes ahead of its first)
  const int VK = d.KG - 2;
  const long tiles = (long)((d.IG - 2 + VTI - 1) / VTI) * ((d.JG - 2 + VTJ - 1) / VTJ);
  const long want = (8L * nsm + tiles - 1) / tiles;
  int kc = (int)((VK + want - 1) / want);
  if (kc < 16) kc = 16;
  return kc < VK ? kc : VK;
}

int visc_ctas(const ViscArgs& a) {
  const Dims& d = a.d;
  const int VK = d.KG - 2;
  return ((d.IG - 2 + VTI - 1) / VTI) * ((d.JG - 2 + VTJ - 1) / VTJ) * ((VK + a.kc - 1) / a.kc);
}

cudaError_t launch_visc_batched(const ViscArgs* args, const int* cta, int nblocks, int total_ctas,
                                const int* dcta, int dtotal, bool f32, cudaStream_t s) {
  if (total_ctas <= 0) return cudaSuccess;
  cudaError_t e = visc_prepare();
  if (e != cudaSuccess) return e;
  if (f32) {
    visc_node_batched<float><<<total_ctas, VT, sizeof(ViscSmem<float>), s>>>(args, cta, nblocks);
    visc_div_batched<float><<<dtotal, 256, 0, s>>>(args, dcta, nblocks);
  } else {
    visc_node_batched<double><<<total_ctas, VT, sizeof(ViscSmem<double>), s>>>(args, cta, nblocks);
    visc_div_batched<double><<<dtotal, 256, 0, s>>>(args, dcta, nblocks);
  }
  return cudaGetLastError();
}

}  // namespace cbns
