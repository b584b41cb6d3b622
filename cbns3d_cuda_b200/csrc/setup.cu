// setup.cu - one-time and I/O kernels: metrics (FP64), initial condition,
// primitive <-> conservative conversion, the AoS <-> SoA transposes that keep the
// reference's host/checkpoint layout at the boundary, and gathers for getters.
#include "setup.cuh"

namespace cbns {

namespace {

// 4th-order first derivative along one axis, the stencils of
// src/gradient_kernel.cu:41-63 (one-sided at the two ends, biased next to
// them, central inside).  Axes shorter than 5 points, where those stencils
// index outside the array, use 2nd-order differences.
__device__ __forceinline__ double dax(const double* f, long s, int g, int n) {
  if (n < 5) {
    if (n == 1) return 0.0;
    if (g == 0) return n >= 3 ? 0.5 * (-3.0 * f[0] + 4.0 * f[s] - f[2 * s]) : f[s] - f[0];
    if (g == n - 1) return n >= 3 ? 0.5 * (3.0 * f[0] - 4.0 * f[-s] + f[-2 * s]) : f[0] - f[-s];
    return 0.5 * (f[s] - f[-s]);
  }
  if (g == 0)
    return -25.0 / 12.0 * f[0] + 4.0 * f[s] - 3.0 * f[2 * s] + (4.0 / 3.0) * f[3 * s] - 0.25 * f[4 * s];
  if (g == 1)
    return -5.0 / 6.0 * f[0] - 0.25 * f[-s] + 1.5 * f[s] - 0.5 * f[2 * s] + (1.0 / 12.0) * f[3 * s];
  if (g == n - 2)
    return (5.0 / 6.0) * f[0] - 1.0 / 12.0 * f[-3 * s] + 0.5 * f[-2 * s] - 1.5 * f[-s] + 0.25 * f[s];
  if (g == n - 1)
    return (25.0 / 12.0) * f[0] + 0.25 * f[-4 * s] - 4.0 / 3.0 * f[-3 * s] + 3.0 * f[-2 * s] - 4.0 * f[-s];
  return (1.0 / 12.0) * f[-2 * s] - 2.0 / 3.0 * f[-s] + (2.0 / 3.0) * f[s] - 1.0 / 12.0 * f[2 * s];
}

struct Met {
  double* m[10];
};

// x_xi .. z_zeta by the stencils above, J by the cofactor determinant and the
// nine inverse metrics by cofactor / J (src/metrics_kernel.cu:55-70).
__global__ void metrics_nodes(Dims d, const double* x, const double* y, const double* z, Met M) {
  const long N = (long)d.IM * d.JM * d.KM;
  const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (e >= N) return;
  const int i = (int)(e % d.IM);
  const long r = e / d.IM;
  const int j = (int)(r % d.JM), k = (int)(r / d.JM);
  const long sj = d.IM, sk = (long)d.IM * d.JM;
  const double xx = dax(x + e, 1, i, d.IM), xe = dax(x + e, sj, j, d.JM), xz = dax(x + e, sk, k, d.KM);
  const double yx = dax(y + e, 1, i, d.IM), ye = dax(y + e, sj, j, d.JM), yz = dax(y + e, sk, k, d.KM);
  const double zx = dax(z + e, 1, i, d.IM), ze = dax(z + e, sj, j, d.JM), zz = dax(z + e, sk, k, d.KM);
  const double J = -xe * yx * zz + xe * yz * zx + xx * ye * zz - xx * yz * ze - xz * ye * zx + xz * yx * ze;
  const long o = node_off(d, i, j, k);
  M.m[9][o] = J;
  M.m[0][o] = (ye * zz - yz * ze) / J;
  M.m[1][o] = (-xe * zz + xz * ze) / J;
  M.m[2][o] = (xe * yz - xz * ye) / J;
  M.m[3][o] = (-yx * zz + yz * zx) / J;
  M.m[4][o] = (xx * zz - xz * zx) / J;
  M.m[5][o] = (-xx * yz + xz * yx) / J;
  M.m[6][o] = (-ye * zx + yx * ze) / J;
  M.m[7][o] = (xe * zx - xx * ze) / J;
  M.m[8][o] = (-xe * yx + xx * ye) / J;
}

// O-grid: the stored copies of the points across the seam (i < wrap and
// i >= IM - wrap) take the metrics of the points they copy, P = IM - 2*wrap
// away, whose stencils all lie on the stored periodic line.
__global__ void metrics_wrap(Dims d, Met M, int wrap) {
  const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (e >= 2L * wrap * d.JM * d.KM) return;
  const int t = (int)(e % (2 * wrap));
  const long r = e / (2 * wrap);
  const int j = (int)(r % d.JM), k = (int)(r / d.JM);
  const int P = d.IM - 2 * wrap;
  const int i = t < wrap ? t : d.IM - 2 * wrap + t;
  const int src = t < wrap ? i + P : i - P;
  const long o = node_off(d, i, j, k), c = node_off(d, src, j, k);
#pragma unroll
  for (int m = 0; m < 10; ++m) M.m[m][o] = M.m[m][c];
}

// Ghost faces, edges and corners take the value of the nearest boundary node
// (the clamped index), which is what metrics_kernel.cu:72-560 writes.
__global__ void metrics_ghosts(Dims d, Met M) {
  const long NGt = (long)d.IG * d.JG * d.KG;
  const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (e >= NGt) return;
  const int i = (int)(e % d.IG) - NG;
  const long r = e / d.IG;
  const int j = (int)(r % d.JG) - NG, k = (int)(r / d.JG) - NG;
  if (i >= 0 && i < d.IM && j >= 0 && j < d.JM && k >= 0 && k < d.KM) return;
  const int ci = min(max(i, 0), d.IM - 1), cj = min(max(j, 0), d.JM - 1), ck = min(max(k, 0), d.KM - 1);
  const long o = node_off(d, i, j, k), c = node_off(d, ci, cj, ck);
#pragma unroll
  for (int m = 0; m < 10; ++m) M.m[m][o] = M.m[m][c];
}

// Node area vectors J*grad(xi), J*grad(eta), J*grad(zeta) and 1/J over the
// ghosted box: the face normal of the reference is the mean of the two nodes'
// J*grad(xi) (src/rec_riemann_kernel.cu:44-49), so it is formed once here.
// The FP32 kernels stage FP32 copies of J*grad(xi) and J*grad(eta) (A32, may
// be absent).
struct Area32 {
  float* m[6];
};

__global__ void area_kernel(Dims d, Met M, Met A, Area32 A32) {
  const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (e >= (long)d.IG * d.JG * d.KG) return;
  const int i = (int)(e % d.IG) - NG;
  const long r = e / d.IG;
  const long o = node_off(d, i, (int)(r % d.JG) - NG, (int)(r / d.JG) - NG);
  const double J = M.m[9][o];
#pragma unroll
  for (int m = 0; m < 9; ++m) A.m[m][o] = M.m[m][o] * J;
  A.m[9][o] = 1.0 / J;
  if (A32.m[0]) {
#pragma unroll
    for (int m = 0; m < 6; ++m) A32.m[m][o] = (float)A.m[m][o];
  }
}

struct Prims {
  double* p[6];
};

__device__ __forceinline__ bool ghosted_node(const Dims& d, long e, int& i, int& j, int& k) {
  if (e >= (long)d.IG * d.JG * d.KG) return false;
  i = (int)(e % d.IG) - NG;
  const long r = e / d.IG;
  j = (int)(r % d.JG) - NG;
  k = (int)(r / d.JG) - NG;
  return true;
}

// src/initial_condition_kernel.cu:13-47: uniform free stream at the angle of attack.
__global__ void ic_kernel(Dims d, Prims P, double cu, double sv, double p_inf, int viscous) {
  int i, j, k;
  if (!ghosted_node(d, blockIdx.x * (long)blockDim.x + threadIdx.x, i, j, k)) return;
  const long o = node_off(d, i, j, k);
  P.p[0][o] = 1.0;
  P.p[1][o] = cu;
  P.p[2][o] = sv;
  P.p[3][o] = 0.0;
  P.p[4][o] = p_inf;
  if (viscous) P.p[5][o] = 1.0;
}

// src/conservative_kernel.cu:13-48 over the whole ghosted box.
__global__ void conservative_kernel(Dims d, Prims P, double* q, double gam1) {
  int i, j, k;
  if (!ghosted_node(d, blockIdx.x * (long)blockDim.x + threadIdx.x, i, j, k)) return;
  const long o = node_off(d, i, j, k), V = d.VOL;
  const double r = P.p[0][o], uu = P.p[1][o], vv = P.p[2][o], ww = P.p[3][o], pp = P.p[4][o];
  q[o] = r;
  q[V + o] = r * uu;
  q[2 * V + o] = r * vv;
  q[3 * V + o] = r * ww;
  q[4 * V + o] = pp / gam1 + 0.5 * r * (uu * uu + vv * vv + ww * ww);
}

// src/primitive_kernel.cu:13-51 over the whole ghosted box (with T).
__global__ void primitive_kernel(Dims d, const double* q, Prims P, double gam1, double gM2) {
  int i, j, k;
  if (!ghosted_node(d, blockIdx.x * (long)blockDim.x + threadIdx.x, i, j, k)) return;
  const long o = node_off(d, i, j, k), V = d.VOL;
  const double r = q[o], uu = q[V + o] / r, vv = q[2 * V + o] / r, ww = q[3 * V + o] / r;
  const double pp = gam1 * (q[4 * V + o] - 0.5 * r * (uu * uu + vv * vv + ww * ww));
  P.p[0][o] = r;
  P.p[1][o] = uu;
  P.p[2][o] = vv;
  P.p[3][o] = ww;
  P.p[4][o] = pp;
  P.p[5][o] = gM2 * pp / r;
}

// dense AoS ghosted (n + 5*(i + IM_G*(j + JM_G*k))) <-> SoA padded
__global__ void aos_to_soa(Dims d, const double* aos, double* q) {
  const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
  int i, j, k;
  if (!ghosted_node(d, e, i, j, k)) return;
  const long o = node_off(d, i, j, k);
#pragma unroll
  for (int n = 0; n < NEQ; ++n) q[n * d.VOL + o] = aos[5 * e + n];
}
__global__ void soa_to_aos(Dims d, const double* q, double* aos) {
  const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
  int i, j, k;
  if (!ghosted_node(d, e, i, j, k)) return;
  const long o = node_off(d, i, j, k);
#pragma unroll
  for (int n = 0; n < NEQ; ++n) aos[5 * e + n] = q[n * d.VOL + o];
}

// field over the N nodes -> dense IM*JM*KM
__global__ void gather_nodes(Dims d, const double* f, double* out) {
  const long N = (long)d.IM * d.JM * d.KM;
  const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (e >= N) return;
  const int i = (int)(e % d.IM);
  const long r = e / d.IM;
  out[e] = f[node_off(d, i, (int)(r % d.JM), (int)(r / d.JM))];
}
// field over the ghosted box -> dense IM_G*JM_G*KM_G
__global__ void gather_ghosted(Dims d, const double* f, double* out) {
  const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
  int i, j, k;
  if (!ghosted_node(d, e, i, j, k)) return;
  out[e] = f[node_off(d, i, j, k)];
}

// stand-alone gradient of a dense field (src/calc_gradient.cu, gradient_kernel)
__global__ void gradient_dense(int IM, int JM, int KM, const double* f, double* fx, double* fy, double* fz) {
  const long N = (long)IM * JM * KM;
  const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (e >= N) return;
  const int i = (int)(e % IM);
  const long r = e / IM;
  const int j = (int)(r % JM), k = (int)(r / JM);
  fx[e] = dax(f + e, 1, i, IM);
  fy[e] = dax(f + e, IM, j, JM);
  fz[e] = dax(f + e, (long)IM * JM, k, KM);
}

// Case initialisation on the device (no counterpart in the reference, whose
// driver reads a checkpoint or starts from the free stream).  The grid's
// coordinates are extended into the ghost layers by odd reflection, axis by
// axis in the order k, j, i (x(-l) = 2 x(0) - x(l)), and the configurations'
// initial states are formed on the whole ghosted box in the reference's units.
struct CaseParams {
  double v[8];
};

// coordinate f (IM x JM x KM, i fastest) at ghosted node (i, j, k)
__device__ __forceinline__ double coord_ext(const Dims& d, const double* f, int i, int j, int k) {
  auto at = [&](int ii, int jj, int kk) -> double { return f[ii + (long)d.IM * (jj + (long)d.JM * kk)]; };
  auto ek = [&](int ii, int jj) -> double {  // along k
    if (k < 0) return 2.0 * at(ii, jj, 0) - at(ii, jj, -k);
    if (k > d.KM - 1) return 2.0 * at(ii, jj, d.KM - 1) - at(ii, jj, 2 * (d.KM - 1) - k);
    return at(ii, jj, k);
  };
  auto ejk = [&](int ii) -> double {  // along j, on the k-extended values
    if (j < 0) return 2.0 * ek(ii, 0) - ek(ii, -j);
    if (j > d.JM - 1) return 2.0 * ek(ii, d.JM - 1) - ek(ii, 2 * (d.JM - 1) - j);
    return ek(ii, j);
  };
  if (i < 0) return 2.0 * ejk(0) - ejk(-i);  // along i, on the (k, j)-extended values
  if (i > d.IM - 1) return 2.0 * ejk(d.IM - 1) - ejk(2 * (d.IM - 1) - i);
  return ejk(i);
}

__global__ void case_ic_kernel(Dims d, const double* x, const double* y, const double* z, int kind, CaseParams cp,
                               double g, double* q) {
  const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (e >= (long)d.IG * d.JG * d.KG) return;
  const int i = (int)(e % d.IG) - NG;
  const long r = e / d.IG;
  const int j = (int)(r % d.JG) - NG, k = (int)(r / d.JG) - NG;
  const double xg = coord_ext(d, x, i, j, k), yg = coord_ext(d, y, i, j, k);
  const double PI = 3.14159265358979323846;
  double rho, u, v, w = 0.0, p;
  if (kind == CBNS_CASE_VORTEX) {
    // isentropic vortex of strength beta (free-stream sound-speed units) and
    // Gaussian radius R in a free stream of Mach number M along (dirx, diry)
    const double M = cp.v[0], beta = cp.v[1], xc = cp.v[2], yc = cp.v[3], R = cp.v[4], dirx = cp.v[5],
                 diry = cp.v[6];
    const double dx = (xg - xc) / R, dy = (yg - yc) / R;
    const double r2 = dx * dx + dy * dy;
    const double f = exp(0.5 * (1.0 - r2));
    const double U = M * sqrt(g);
    const double ua = U * dirx - beta / (2.0 * PI) * dy * f;
    const double va = U * diry + beta / (2.0 * PI) * dx * f;
    const double T = 1.0 - (g - 1.0) * (beta * beta) / (8.0 * g * (PI * PI)) * exp(1.0 - r2);
    rho = pow(T, 1.0 / (g - 1.0));
    u = ua / U;
    v = va / U;
    p = rho * T / (U * U);
  } else if (kind == CBNS_CASE_BLAST) {
    // pressure p_in where x^2 + y^2 + z^2 < r2_in, p_out elsewhere, unit
    // density, at rest
    const double zg = coord_ext(d, z, i, j, k);
    const double r2 = xg * xg + yg * yg + zg * zg;
    rho = 1.0;
    u = v = 0.0;
    p = r2 < cp.v[0] ? cp.v[1] : cp.v[2];
  } else {
    // stationary normal shock of Mach Ms at x = xs; upstream (rho, u, p) =
    // (1, 1, 1/(g Ms^2)) with a vortex (strength eps, radius rc, centre
    // (xc, yc), u_theta = eps c1 tau exp(a (1 - tau^2)), a = 0.204)
    const double Ms = cp.v[0], eps = cp.v[1], rc = cp.v[2], xc = cp.v[3], yc = cp.v[4], xs = cp.v[5];
    const double a = 0.204;
    const double p1 = 1.0 / (g * Ms * Ms);
    if (xg < xs) {
      const double dx = xg - xc, dy = yg - yc;
      const double rr = sqrt(dx * dx + dy * dy);
      const double tau = rr / rc;
      const double c1 = sqrt(g * p1 / 1.0);
      const double ut = eps * c1 * tau * exp(a * (1.0 - tau * tau));
      const double sn = rr > 0.0 ? dy / rr : 0.0, cs = rr > 0.0 ? dx / rr : 0.0;
      const double T1 = p1 / 1.0;
      const double T = T1 - (g - 1.0) * ((eps * c1) * (eps * c1)) / (4.0 * a * g) * exp(2.0 * a * (1.0 - tau * tau)) *
                                (1.0 / 1.0);
      rho = pow(T / T1, 1.0 / (g - 1.0));
      u = 1.0 - ut * sn;
      v = ut * cs;
      p = p1 * pow(T / T1, g / (g - 1.0));
    } else {
      const double r21 = ((g + 1.0) * Ms * Ms) / ((g - 1.0) * Ms * Ms + 2.0);
      const double p21 = 1.0 + 2.0 * g / (g + 1.0) * (Ms * Ms - 1.0);
      rho = r21;
      u = 1.0 / r21;
      v = 0.0;
      p = p1 * p21;
    }
  }
  const long o = node_off(d, i, j, k), VOL = d.VOL;
  q[o] = rho;
  q[VOL + o] = rho * u;
  q[2 * VOL + o] = rho * v;
  q[3 * VOL + o] = rho * w;
  q[4 * VOL + o] = p / (g - 1.0) + 0.5 * rho * (u * u + v * v + w * w);
}

inline unsigned nb(long n) { return (unsigned)((n + 255) / 256); }

}  // namespace

cudaError_t launch_metrics(const Dims& d, const double* x, const double* y, const double* z, double* const met[10],
                           double* const area[10], float* const area32[6], int wrap, cudaStream_t s) {
  Met M, A;
  Area32 A32;
  for (int m = 0; m < 10; ++m) {
    M.m[m] = met[m];
    A.m[m] = area[m];
  }
  for (int m = 0; m < 6; ++m) A32.m[m] = area32 ? area32[m] : nullptr;
  metrics_nodes<<<nb((long)d.IM * d.JM * d.KM), 256, 0, s>>>(d, x, y, z, M);
  if (wrap > 0) metrics_wrap<<<nb(2L * wrap * d.JM * d.KM), 256, 0, s>>>(d, M, wrap);
  metrics_ghosts<<<nb((long)d.IG * d.JG * d.KG), 256, 0, s>>>(d, M);
  area_kernel<<<nb((long)d.IG * d.JG * d.KG), 256, 0, s>>>(d, M, A, A32);
  return cudaGetLastError();
}

cudaError_t launch_ic(const Dims& d, double* const prim[6], double angle_deg, double p_inf, int viscous,
                      cudaStream_t s) {
  Prims P;
  for (int m = 0; m < 6; ++m) P.p[m] = prim[m];
  const double PI = 3.14159265358979323846;
  const double AoA = angle_deg * PI / 180.0;
  ic_kernel<<<nb((long)d.IG * d.JG * d.KG), 256, 0, s>>>(d, P, cos(AoA), sin(AoA), p_inf, viscous);
  return cudaGetLastError();
}

cudaError_t launch_case_ic(const Dims& d, const double* x, const double* y, const double* z, int kind,
                           const double* prm, int nprm, double gamma, double* q, cudaStream_t s) {
  CaseParams cp;
  for (int m = 0; m < 8; ++m) cp.v[m] = m < nprm ? prm[m] : 0.0;
  case_ic_kernel<<<nb((long)d.IG * d.JG * d.KG), 256, 0, s>>>(d, x, y, z, kind, cp, gamma, q);
  return cudaGetLastError();
}

cudaError_t launch_conservative(const Dims& d, double* const prim[6], double* q, double gam1, cudaStream_t s) {
  Prims P;
  for (int m = 0; m < 6; ++m) P.p[m] = prim[m];
  conservative_kernel<<<nb((long)d.IG * d.JG * d.KG), 256, 0, s>>>(d, P, q, gam1);
  return cudaGetLastError();
}

cudaError_t launch_primitive(const Dims& d, const double* q, double* const prim[6], double gam1, double gM2,
                             cudaStream_t s) {
  Prims P;
  for (int m = 0; m < 6; ++m) P.p[m] = prim[m];
  primitive_kernel<<<nb((long)d.IG * d.JG * d.KG), 256, 0, s>>>(d, q, P, gam1, gM2);
  return cudaGetLastError();
}

cudaError_t launch_aos_to_soa(const Dims& d, const double* aos, double* q, cudaStream_t s) {
  aos_to_soa<<<nb((long)d.IG * d.JG * d.KG), 256, 0, s>>>(d, aos, q);
  return cudaGetLastError();
}

cudaError_t launch_soa_to_aos(const Dims& d, const double* q, double* aos, cudaStream_t s) {
  soa_to_aos<<<nb((long)d.IG * d.JG * d.KG), 256, 0, s>>>(d, q, aos);
  return cudaGetLastError();
}

cudaError_t launch_gather_nodes(const Dims& d, const double* f, double* out, cudaStream_t s) {
  gather_nodes<<<nb((long)d.IM * d.JM * d.KM), 256, 0, s>>>(d, f, out);
  return cudaGetLastError();
}

cudaError_t launch_gather_ghosted(const Dims& d, const double* f, double* out, cudaStream_t s) {
  gather_ghosted<<<nb((long)d.IG * d.JG * d.KG), 256, 0, s>>>(d, f, out);
  return cudaGetLastError();
}

cudaError_t launch_gradient_dense(int IM, int JM, int KM, const double* f, double* fx, double* fy, double* fz,
                                  cudaStream_t s) {
  gradient_dense<<<nb((long)IM * JM * KM), 256, 0, s>>>(IM, JM, KM, f, fx, fy, fz);
  return cudaGetLastError();
}

}  // namespace cbns
