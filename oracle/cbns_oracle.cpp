// cbns_oracle.cpp -- CPU FP64 restatement of the cbns3d_cuda RK3 right-hand-side path.
//
// TEST INFRASTRUCTURE, NOT PRODUCT CODE.  Only tests/, __graft_entry__.smoke()
// and bench.py's cpu_baseline leg load this library, and only as the checker
// (or as the timed CPU baseline).  The B200 library never calls it.
//
// Every function restates one reference kernel or host routine (paths inside
// the reference project chenbei102/cbns3d_cuda are cited per function) with the
// reference's own data layout: AoS conservative state Q[n + 5*node], ghosted
// node arrays with NG = 2 ghost layers, face-flux arrays Ep/Fp/Gp and the
// viscous arrays Ev/Fv/Gv/dfv.  Kernels whose GPU threads race in the reference
// (primitive_bc_kernel, see the phase notes below) are restated with their
// phases in program order, which is what the reference computes whenever its
// racing branches are not taken.  Loops run with OpenMP over the outermost
// index; every loop body writes disjoint cells, so the result does not depend
// on the thread count.
//
// Dimensions below 5 points: the reference's one-sided 4th-order stencils
// (src/gradient_kernel.cu:41-63) index outside the array when a dimension has
// fewer than 5 points.  Here (and in the B200 library) such a dimension uses
// 2nd-order differences instead; the reference itself cannot run that case.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../include/cbns_b200.h"

namespace {

constexpr int NEQ = 5;
constexpr int NG = 2;
constexpr double PI = 3.14159265358979323846;

struct Derived {
  double Mach2, gM2, Re_inv, p_inf, gam1, gam1_inv, Pr_inv, Pr_t_inv, gPr, C_T_inf, C_dt_v;
};

// Derived parameters, src/Block3d.cpp:99-113.
Derived derive(const cbns_params& p) {
  Derived d;
  d.Mach2 = p.Mach * p.Mach;
  d.Re_inv = 1.0 / p.Re;
  d.Pr_inv = 1.0 / p.Pr;
  d.Pr_t_inv = 1.0 / p.Pr_t;
  d.gam1 = p.gamma - 1.0;
  d.gM2 = p.gamma * d.Mach2;
  d.gam1_inv = 1.0 / d.gam1;
  d.gPr = p.gamma / p.Pr;
  d.p_inf = 1.0 / d.gM2;
  d.C_T_inf = 110.5 / p.T_inf;
  d.C_dt_v = std::max(4.0 / 3.0, p.gamma * d.Pr_inv) * d.Re_inv;
  return d;
}

// 4th-order first derivative along one axis at index g of n points; s is the
// element stride of that axis.  Stencils of src/gradient_kernel.cu:41-63
// (one-sided at g=0 and n-1, biased at g=1 and n-2, central elsewhere).
inline double d_axis(const double* f, long s, long g, long n) {
  if (n < 5) {  // extension for short dimensions (see file header)
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

// Gradient of an n0 x n1 x n2 array (i fastest), src/gradient_kernel.cu:13-133
// (unghosted) and :135-255 (ghosted; same stencils over the whole ghosted box).
void gradient3(const double* f, long n0, long n1, long n2, double* f0, double* f1, double* f2) {
#pragma omp parallel for schedule(static)
  for (long k = 0; k < n2; ++k)
    for (long j = 0; j < n1; ++j)
      for (long i = 0; i < n0; ++i) {
        const long id = i + n0 * (j + n1 * k);
        f0[id] = d_axis(f + id, 1, i, n0);
        f1[id] = d_axis(f + id, n0, j, n1);
        f2[id] = d_axis(f + id, n0 * n1, k, n2);
      }
}

struct Prim {
  double r, u, v, w, p;
};

// Conservative -> primitive, the formula used throughout primitive_bc_kernel
// (src/primitive_bc_kernel.cu:63-67).
inline Prim to_prim(const double* q, double gam1) {
  Prim s;
  s.r = q[0];
  s.u = q[1] / s.r;
  s.v = q[2] / s.r;
  s.w = q[3] / s.r;
  s.p = gam1 * (q[4] - 0.5 * s.r * (s.u * s.u + s.v * s.v + s.w * s.w));
  return s;
}

// WENO5-JS reconstruction of one scalar at the i+1/2 side of U0 from
// Um2..Up2, src/weno.cu:13-44 (eps = 1e-6 added inside beta before squaring).
inline double weno5(double Um2, double Um1, double U0, double Up1, double Up2) {
  const double eps = 1.0e-6;
  const double a1 = Um2 - 2.0 * Um1 + U0, b1 = Um2 - 4.0 * Um1 + 3.0 * U0;
  const double a2 = Um1 - 2.0 * U0 + Up1, b2 = Um1 - Up1;
  const double a3 = U0 - 2.0 * Up1 + Up2, b3 = 3.0 * U0 - 4.0 * Up1 + Up2;
  const double s1 = (13.0 / 12.0) * a1 * a1 + 0.25 * b1 * b1 + eps;
  const double s2 = (13.0 / 12.0) * a2 * a2 + 0.25 * b2 * b2 + eps;
  const double s3 = (13.0 / 12.0) * a3 * a3 + 0.25 * b3 * b3 + eps;
  const double w1 = 0.1 / (s1 * s1), w2 = 0.6 / (s2 * s2), w3 = 0.3 / (s3 * s3);
  const double p1 = (2.0 * Um2 - 7.0 * Um1 + 11.0 * U0) / 6.0;
  const double p2 = (-Um1 + 5.0 * U0 + 2.0 * Up1) / 6.0;
  const double p3 = (2.0 * U0 + 5.0 * Up1 - Up2) / 6.0;
  return (w1 * p1 + w2 * p2 + w3 * p3) / (w1 + w2 + w3);
}

// Roe-averaged right (R) and left (L) eigenvectors for face normal n,
// src/calc_eigenvectors_roe.cu:13-152.  a = node on the low side, b = high side.
void roe_eigen(const Prim& a, const Prim& b, double nx, double ny, double nz, double gamma,
               double gam1, double R[5][5], double L[5][5]) {
  // tangent l = (0, nz, -ny) unless degenerate, then (-nz, 0, nx); m by cross-construction
  double lx = 0.0, ly = nz, lz = -ny, mx, my, mz;
  double nrm = std::sqrt(lx * lx + ly * ly + lz * lz);
  if (nrm > 1.0e-8) {
    mx = -ny * ny - nz * nz;
    my = nx * ny;
    mz = nx * nz;
  } else {
    lx = -nz;
    ly = 0.0;
    lz = nx;
    mx = nx * ny;
    my = -nx * nx - nz * nz;
    mz = ny * nz;
  }
  nrm = std::sqrt(nx * nx + ny * ny + nz * nz);
  nx /= nrm; ny /= nrm; nz /= nrm;
  nrm = std::sqrt(lx * lx + ly * ly + lz * lz);
  lx /= nrm; ly /= nrm; lz /= nrm;
  nrm = std::sqrt(mx * mx + my * my + mz * mz);
  mx /= nrm; my /= nrm; mz /= nrm;

  const double ca = std::sqrt(gamma * a.p / a.r);
  const double Ha = ca * ca / gam1 + 0.5 * (a.u * a.u + a.v * a.v + a.w * a.w);
  const double cb = std::sqrt(gamma * b.p / b.r);
  const double Hb = cb * cb / gam1 + 0.5 * (b.u * b.u + b.v * b.v + b.w * b.w);
  const double sr = std::sqrt(b.r / a.r);
  const double uu = (a.u + sr * b.u) / (1.0 + sr);
  const double vv = (a.v + sr * b.v) / (1.0 + sr);
  const double ww = (a.w + sr * b.w) / (1.0 + sr);
  const double H = (Ha + sr * Hb) / (1.0 + sr);
  const double q2 = uu * uu + vv * vv + ww * ww;
  const double c = std::sqrt(gam1 * (H - 0.5 * q2));
  const double qn = uu * nx + vv * ny + ww * nz;
  const double ql = uu * lx + vv * ly + ww * lz;
  const double qm = uu * mx + vv * my + ww * mz;

  // columns: acoustic (-), entropy, acoustic (+), shear l, shear m
  const double col[5][5] = {{1.0, uu - c * nx, vv - c * ny, ww - c * nz, H - qn * c},
                            {1.0, uu, vv, ww, 0.5 * q2},
                            {1.0, uu + c * nx, vv + c * ny, ww + c * nz, H + qn * c},
                            {0.0, lx, ly, lz, ql},
                            {0.0, mx, my, mz, qm}};
  for (int r = 0; r < 5; ++r)
    for (int s = 0; s < 5; ++s) R[r][s] = col[s][r];

  const double K = gam1 / (2.0 * c * c);
  const double h = 0.5 / c;
  const double rows[5][5] = {
      {0.5 * K * q2 + h * qn, -(K * uu + h * nx), -(K * vv + h * ny), -(K * ww + h * nz), K},
      {1.0 - K * q2, 2.0 * K * uu, 2.0 * K * vv, 2.0 * K * ww, -2.0 * K},
      {0.5 * K * q2 - h * qn, -(K * uu - h * nx), -(K * vv - h * ny), -(K * ww - h * nz), K},
      {-ql, lx, ly, lz, 0.0},
      {-qm, mx, my, mz, 0.0}};
  std::memcpy(L, rows, sizeof(rows));
}

// Characteristic-wise WENO5 of five stencil states, back to primitives,
// src/weno.cu:46-120.  st[p] points at the 5 conservative values of stencil point p.
Prim rec_weno5(const double* const st[5], const double R[5][5], const double L[5][5], double gam1) {
  double w[5];
  for (int s = 0; s < 5; ++s) {
    double c[5];
    for (int p = 0; p < 5; ++p) {
      double acc = 0.0;
      for (int n = 0; n < 5; ++n) acc += L[s][n] * st[p][n];
      c[p] = acc;
    }
    w[s] = weno5(c[0], c[1], c[2], c[3], c[4]);
  }
  double q[5];
  for (int n = 0; n < 5; ++n) {
    double acc = 0.0;
    for (int s = 0; s < 5; ++s) acc += R[n][s] * w[s];
    q[n] = acc;
  }
  return to_prim(q, gam1);
}

// Local Lax-Friedrichs flux with the reference's Cartesian wave-speed bound,
// src/lf_flux.cu:13-80.  hi = state reconstructed from the high side (the
// reference's "R"), lo = from the low side ("L"); n is the area vector.
void lf_flux(const Prim& hi, const Prim& lo, double nx, double ny, double nz, double gamma,
             double gam1, double* flux) {
  const double cH = std::sqrt(gamma * hi.p / hi.r);
  const double kH = hi.u * hi.u + hi.v * hi.v + hi.w * hi.w;
  const double HH = cH * cH / gam1 + 0.5 * kH;
  const double EH = hi.p / gam1 + 0.5 * hi.r * kH;
  const double cL = std::sqrt(gamma * lo.p / lo.r);
  const double kL = lo.u * lo.u + lo.v * lo.v + lo.w * lo.w;
  const double HL = cL * cL / gam1 + 0.5 * kL;
  const double EL = lo.p / gam1 + 0.5 * lo.r * kL;
  const double qH = hi.u * nx + hi.v * ny + hi.w * nz;
  const double qL = lo.u * nx + lo.v * ny + lo.w * nz;
  const double sx = std::max(std::abs(hi.u) + cH, std::abs(lo.u) + cL);
  const double sy = std::max(std::abs(hi.v) + cH, std::abs(lo.v) + cL);
  const double sz = std::max(std::abs(hi.w) + cH, std::abs(lo.w) + cL);
  const double ws = std::abs(sx * nx + sy * ny + sz * nz);
  const double dU[5] = {hi.r - lo.r, hi.r * hi.u - lo.r * lo.u, hi.r * hi.v - lo.r * lo.v,
                        hi.r * hi.w - lo.r * lo.w, EH - EL};
  const double FL[5] = {lo.r * qL, lo.r * qL * lo.u + lo.p * nx, lo.r * qL * lo.v + lo.p * ny,
                        lo.r * qL * lo.w + lo.p * nz, lo.r * qL * HL};
  const double FH[5] = {hi.r * qH, hi.r * qH * hi.u + hi.p * nx, hi.r * qH * hi.v + hi.p * ny,
                        hi.r * qH * hi.w + hi.p * nz, hi.r * qH * HH};
  for (int n = 0; n < 5; ++n) flux[n] = 0.5 * (FL[n] + FH[n] - ws * dU[n]);
}

struct Oracle {
  cbns_params P;
  Derived D;
  long IM, JM, KM, IG, JG, KG, NGt;
  std::vector<double> met[10];  // xi_x..zeta_z, Jac (ghosted)
  std::vector<double> Qa, Qb;   // block_data->Q, block_data->Q_p (AoS, ghosted)
  std::vector<double> rho, u, v, w, p, T, mu;
  std::vector<double> grad[12];  // u_xi,u_eta,u_zeta, v.., w.., T..
  std::vector<double> tau[6];    // xx, yy, zz, xy, xz, yz
  std::vector<double> qf[3];
  std::vector<double> Ev, Fv, Gv, dfv, Ep, Fp, Gp, dtn;
  std::vector<unsigned char> hmask;  // hybrid flux decisions (1 = WENO5); empty = WENO5 everywhere
  bool have_metrics = false;

  explicit Oracle(const cbns_params& p) : P(p), D(derive(p)) {
    IM = p.IM; JM = p.JM; KM = p.KM;
    IG = IM + 2 * NG; JG = JM + 2 * NG; KG = KM + 2 * NG;
    NGt = IG * JG * KG;
    for (auto& m : met) m.assign(NGt, 0.0);
    Qa.assign(NEQ * NGt, 0.0);
    Qb.assign(NEQ * NGt, 0.0);
    for (auto* a : {&rho, &u, &v, &w, &p_(), &T, &mu}) a->assign(NGt, 0.0);
    if (P.viscous) {
      for (auto& g : grad) g.assign(NGt, 0.0);
      for (auto& t : tau) t.assign(NGt, 0.0);
      for (auto& q : qf) q.assign(NGt, 0.0);
      const long nv = (NEQ - 1) * (IG - 2) * (JG - 2) * (KG - 2);
      Ev.assign(nv, 0.0); Fv.assign(nv, 0.0); Gv.assign(nv, 0.0);
      dfv.assign((NEQ - 1) * (IM - 2) * (JM - 2) * (KM - 2), 0.0);
    }
    Ep.assign(NEQ * (IM - 1) * (JM - 2) * (KM - 2), 0.0);
    Fp.assign(NEQ * (IM - 2) * (JM - 1) * (KM - 2), 0.0);
    Gp.assign(NEQ * (IM - 2) * (JM - 2) * (KM - 1), 0.0);
    dtn.assign(IM * JM * KM, 0.0);
  }
  std::vector<double>& p_() { return p; }

  // node (i,j,k) with i in [-NG, IM+NG) -> ghosted flat index (include/Block3d_cuda.h:96-98)
  long g(long i, long j, long k) const { return (NG + i) + IG * ((NG + j) + JG * (NG + k)); }
  std::vector<double>& buf(int which) { return which == CBNS_QP ? Qb : Qa; }

  // ---------------------------------------------------------------------------
  // calc_metrics: src/calc_metrics.cu:16-111 + src/metrics_kernel.cu:13-562.
  void calc_metrics(const double* x, const double* y, const double* z) {
    const long N = IM * JM * KM;
    std::vector<double> d[9];  // x_xi x_eta x_zeta y_xi ... z_zeta
    for (auto& a : d) a.resize(N);
    gradient3(x, IM, JM, KM, d[0].data(), d[1].data(), d[2].data());
    gradient3(y, IM, JM, KM, d[3].data(), d[4].data(), d[5].data());
    gradient3(z, IM, JM, KM, d[6].data(), d[7].data(), d[8].data());
#pragma omp parallel for schedule(static)
    for (long k = 0; k < KM; ++k)
      for (long j = 0; j < JM; ++j)
        for (long i = 0; i < IM; ++i) {
          const long s = i + IM * (j + JM * k), t = g(i, j, k);
          const double xx = d[0][s], xe = d[1][s], xz = d[2][s];
          const double yx = d[3][s], ye = d[4][s], yz = d[5][s];
          const double zx = d[6][s], ze = d[7][s], zz = d[8][s];
          const double J = -xe * yx * zz + xe * yz * zx + xx * ye * zz - xx * yz * ze - xz * ye * zx +
                           xz * yx * ze;
          met[9][t] = J;
          met[0][t] = (ye * zz - yz * ze) / J;
          met[1][t] = (-xe * zz + xz * ze) / J;
          met[2][t] = (xe * yz - xz * ye) / J;
          met[3][t] = (-yx * zz + yz * zx) / J;
          met[4][t] = (xx * zz - xz * zx) / J;
          met[5][t] = (-xx * yz + xz * yx) / J;
          met[6][t] = (-ye * zx + yx * ze) / J;
          met[7][t] = (xe * zx - xx * ze) / J;
          met[8][t] = (-xe * yx + xx * ye) / J;
        }
    // CBNS_BC_OGRID (no counterpart in the reference): the stored copies of
    // the points across the seam take the metrics of the points they copy.
    if (P.bc_mode == CBNS_BC_OGRID) {
      const long W = CBNS_OGRID_WRAP, Pw = IM - 2 * W;
      for (long k = 0; k < KM; ++k)
        for (long j = 0; j < JM; ++j)
          for (long i = 0; i < IM; ++i) {
            if (i >= W && i < IM - W) continue;
            const long src = i < W ? i + Pw : i - Pw;
            for (auto& m : met) m[g(i, j, k)] = m[g(src, j, k)];
          }
    }
    // Ghost faces, edges and corners take the value of the nearest boundary
    // node (metrics_kernel.cu:72-560 writes exactly the clamped-index copy).
#pragma omp parallel for schedule(static)
    for (long k = -NG; k < KM + NG; ++k)
      for (long j = -NG; j < JM + NG; ++j)
        for (long i = -NG; i < IM + NG; ++i) {
          if (i >= 0 && i < IM && j >= 0 && j < JM && k >= 0 && k < KM) continue;
          const long ci = std::min(std::max(i, 0L), IM - 1);
          const long cj = std::min(std::max(j, 0L), JM - 1);
          const long ck = std::min(std::max(k, 0L), KM - 1);
          for (auto& m : met) m[g(i, j, k)] = m[g(ci, cj, ck)];
        }
    have_metrics = true;
  }

  // ---------------------------------------------------------------------------
  // initial_condition: src/initial_condition_kernel.cu:13-47 (whole ghosted box).
  void initial_condition() {
    const double AoA = P.angle_attack * PI / 180.0;
    const double cu = std::cos(AoA), sv = std::sin(AoA);
    for (long t = 0; t < NGt; ++t) {
      rho[t] = 1.0; u[t] = cu; v[t] = sv; w[t] = 0.0; p[t] = D.p_inf;
      if (P.viscous) T[t] = 1.0;
    }
  }

  // calc_conservative: src/conservative_kernel.cu:13-48, src/calc_conservative.cu:15-40
  // (fills the given buffer from the primitives, then copies Q into Q_p).
  void calc_conservative(int which) {
    auto& Q = buf(which);
    for (long t = 0; t < NGt; ++t) {
      const double r = rho[t], uu = u[t], vv = v[t], ww = w[t], pp = p[t];
      Q[5 * t + 0] = r;
      Q[5 * t + 1] = r * uu;
      Q[5 * t + 2] = r * vv;
      Q[5 * t + 3] = r * ww;
      Q[5 * t + 4] = pp / D.gam1 + 0.5 * r * (uu * uu + vv * vv + ww * ww);
    }
    Qb = Qa;
  }

  // calc_primitive: src/primitive_kernel.cu:13-51 (whole ghosted box, with T).
  void calc_primitive(int which) {
    const auto& Q = buf(which);
#pragma omp parallel for schedule(static)
    for (long t = 0; t < NGt; ++t) {
      const Prim s = to_prim(&Q[5 * t], D.gam1);
      rho[t] = s.r; u[t] = s.u; v[t] = s.v; w[t] = s.w; p[t] = s.p;
      T[t] = D.gM2 * s.p / s.r;
    }
  }

  void put_prim(long t, const Prim& s) {
    rho[t] = s.r; u[t] = s.u; v[t] = s.v; w[t] = s.w; p[t] = s.p;
    if (P.viscous) T[t] = D.gM2 * s.p / s.r;
  }

  // ---------------------------------------------------------------------------
  // CBNS_BC_CHARACTERISTIC (no counterpart in the reference), one face
  // direction: every node of the dir = 0 / IM-1 (resp. JM-1, KM-1) faces takes
  // the Riemann-invariant far-field state built from its inward neighbour and
  // the free stream along the outward unit normal; its two ghosts copy it.
  // i faces over j, k interior, j faces over all i and k interior, k faces
  // over all (i, j), so each neighbour is interior or set earlier in the call.
  void bc_characteristic(std::vector<double>& Q, int dir, int side0 = 0, int nsides = 2) {
    const double gamma = P.gamma, gam1 = D.gam1, p_inf = D.p_inf;
    const double AoA = P.angle_attack * PI / 180.0;
    const double u_inf = std::cos(AoA), v_inf = std::sin(AoA);
    const long n0 = dir == 0 ? JM - 2 : IM, n1 = dir == 2 ? JM : KM - 2, nf = dir == 0 ? IM : dir == 1 ? JM : KM;
    for (int side = side0; side < side0 + nsides; ++side)
#pragma omp parallel for schedule(static)
      for (long f1 = 0; f1 < n1; ++f1)
        for (long f0 = 0; f0 < n0; ++f0) {
          const long lb = side ? nf - 1 : 0, st = side ? 1 : -1;
          long ijk[3] = {dir == 0 ? lb : f0, dir == 0 ? f0 + 1 : dir == 1 ? lb : f1, dir == 2 ? lb : f1 + 1};
          const long tb = g(ijk[0], ijk[1], ijk[2]);
          ijk[dir] -= st;
          const long te = g(ijk[0], ijk[1], ijk[2]);
          const double mx = met[3 * dir][tb], my = met[3 * dir + 1][tb], mz = met[3 * dir + 2][tb];
          const double mn = (side ? 1.0 : -1.0) / std::sqrt(mx * mx + my * my + mz * mz);
          const double nx = mx * mn, ny = my * mn, nz = mz * mn;
          const Prim se = to_prim(&Q[5 * te], gam1);
          const double ce = std::sqrt(gamma * se.p / se.r);
          const double qne = se.u * nx + se.v * ny + se.w * nz;
          double qb[5];
          if (std::fabs(qne) >= ce && qne >= 0.0) {  // supersonic outflow
            for (int m = 0; m < 5; ++m) qb[m] = Q[5 * te + m];
          } else {
            Prim b;
            if (std::fabs(qne) >= ce) {  // supersonic inflow
              b.r = 1.0; b.u = u_inf; b.v = v_inf; b.w = 0.0; b.p = p_inf;
            } else {
              const double ci = std::sqrt(gamma * p_inf);
              const double qni = u_inf * nx + v_inf * ny;
              const double rp = qne + 2.0 * ce / gam1, rm = qni - 2.0 * ci / gam1;
              const double qnb = 0.5 * (rp + rm), cb = 0.25 * gam1 * (rp - rm);
              double s;
              if (qnb >= 0.0) {
                s = se.p / std::pow(se.r, gamma);
                const double dq = qnb - qne;
                b.u = se.u + dq * nx; b.v = se.v + dq * ny; b.w = se.w + dq * nz;
              } else {
                s = p_inf;
                const double dq = qnb - qni;
                b.u = u_inf + dq * nx; b.v = v_inf + dq * ny; b.w = dq * nz;
              }
              b.r = std::pow(cb * cb / (gamma * s), 1.0 / gam1);
              b.p = b.r * cb * cb / gamma;
            }
            qb[0] = b.r; qb[1] = b.r * b.u; qb[2] = b.r * b.v; qb[3] = b.r * b.w;
            qb[4] = b.p / gam1 + 0.5 * b.r * (b.u * b.u + b.v * b.v + b.w * b.w);
          }
          ijk[dir] += st;
          for (long l = 0; l <= NG; ++l) {
            const long t = g(ijk[0], ijk[1], ijk[2]);
            for (int m = 0; m < 5; ++m) Q[5 * t + m] = qb[m];
            ijk[dir] += st;
          }
        }
  }

  // ---------------------------------------------------------------------------
  // set_bc_calc_primitive: src/primitive_bc_kernel.cu:13-494.  The kernel's
  // three __syncthreads-separated phases run here in order over the whole grid:
  //   1. interior primitives; i=0 and i=IM-1 faces (pressure reset to p_inf)
  //   2a. j=0 face: wake-cut average (i < i_begin-1) or wall (i < i_end)
  //   2b. primitives on j=0..-2 and on j=JM-1, JM (from Q at JM-1)
  //   3. k=0 and k=KM-1 faces (zero-gradient copy of Q and primitives)
  void set_bc_calc_primitive(int which) {
    auto& Q = buf(which);
    const double gam1 = D.gam1, p_inf = D.p_inf;
    // phase 1a: interior primitives (:59-79)
#pragma omp parallel for schedule(static)
    for (long k = 1; k < KM - 1; ++k)
      for (long j = 1; j < JM - 1; ++j)
        for (long i = 1; i < IM - 1; ++i) put_prim(g(i, j, k), to_prim(&Q[5 * g(i, j, k)], gam1));
    if (P.bc_mode == CBNS_BC_FARFIELD || P.bc_mode == CBNS_BC_CHARACTERISTIC) {
      // no counterpart in the reference: boundary and ghost nodes keep their Q
      // (or first take the characteristic state), their primitives follow from it
      if (P.bc_mode == CBNS_BC_CHARACTERISTIC)
        for (int dir = 0; dir < 3; ++dir) bc_characteristic(Q, dir);
#pragma omp parallel for schedule(static)
      for (long k = -NG; k < KM + NG; ++k)
        for (long j = -NG; j < JM + NG; ++j)
          for (long i = -NG; i < IM + NG; ++i) {
            if (i >= 1 && i < IM - 1 && j >= 1 && j < JM - 1 && k >= 1 && k < KM - 1) continue;
            put_prim(g(i, j, k), to_prim(&Q[5 * g(i, j, k)], gam1));
          }
      return;
    }
    // CBNS_BC_OGRID (no counterpart in the reference): no i-face pass, the
    // wall on every i of j = 0, the characteristic far field on j = JM-1, and
    // after phase 3 the copies across the periodic seam
    const bool og = P.bc_mode == CBNS_BC_OGRID;
    const long k1b = og ? 1 : KM - 1;
    // phase 1b: i faces (:84-186)
#pragma omp parallel for schedule(static)
    for (long k = 1; k < k1b; ++k)
      for (long j = 1; j < JM - 1; ++j) {
        for (int side = 0; side < 2; ++side) {
          const long src = side == 0 ? 1 : IM - 2;
          const long base = side == 0 ? 0 : IM - 1;
          const long dir = side == 0 ? -1 : 1;
          const double* q = &Q[5 * g(src, j, k)];
          const double r = q[0], ru = q[1], rv = q[2], rw = q[3];
          const double E = p_inf / gam1 + 0.5 * (ru * ru + rv * rv + rw * rw) / r;
          Prim s;
          s.r = r; s.u = ru / r; s.v = rv / r; s.w = rw / r;
          s.p = gam1 * (E - 0.5 * s.r * (s.u * s.u + s.v * s.v + s.w * s.w));
          for (long l = 0; l <= NG; ++l) {
            const long t = g(base + dir * l, j, k);
            double* o = &Q[5 * t];
            o[0] = r; o[1] = ru; o[2] = rv; o[3] = rw; o[4] = E;
            put_prim(t, s);
          }
        }
      }
    // phase 2a: j = 0 face, Q part (:190-352)
    const unsigned ib1 = og ? 0u : P.i_begin - 1u;  // unsigned, as in the reference
    const unsigned iend = og ? (unsigned)IM : (unsigned)P.i_end;
#pragma omp parallel for schedule(static)
    for (long k = 1; k < KM - 1; ++k)
      for (long i = 0; i < IM; ++i) {
        const unsigned ui = (unsigned)i;
        if (ib1 > ui) {  // wake cut: average with the mirror point across the cut
          const long m = IM - 1 - i;
          const Prim a = to_prim(&Q[5 * g(i, 1, k)], gam1);
          const Prim b = to_prim(&Q[5 * g(m, 1, k)], gam1);
          const double r = 0.5 * (a.r + b.r), uu = 0.5 * (a.u + b.u), vv = 0.5 * (a.v + b.v),
                       ww = 0.5 * (a.w + b.w), pp = 0.5 * (a.p + b.p);
          double* o = &Q[5 * g(i, 0, k)];
          o[0] = r; o[1] = r * uu; o[2] = r * vv; o[3] = r * ww;
          o[4] = pp / gam1 + 0.5 * r * (uu * uu + vv * vv + ww * ww);
          std::memcpy(&Q[5 * g(m, 0, k)], o, 5 * sizeof(double));
          for (long l = 1; l <= NG; ++l) {
            std::memcpy(&Q[5 * g(i, -l, k)], &Q[5 * g(m, l, k)], 5 * sizeof(double));
            std::memcpy(&Q[5 * g(m, -l, k)], &Q[5 * g(i, l, k)], 5 * sizeof(double));
          }
        } else if (iend > ui) {
          if (P.viscous) {  // adiabatic no-slip wall (:263-295)
            const double* q = &Q[5 * g(i, 1, k)];
            const double r = q[0], ru = q[1], rv = q[2], rw = q[3], rE = q[4];
            const double pp = gam1 * (rE - 0.5 * (ru * ru + rv * rv + rw * rw) / r);
            double* o = &Q[5 * g(i, 0, k)];
            o[0] = r; o[1] = 0.0; o[2] = 0.0; o[3] = 0.0; o[4] = pp / gam1;
            for (long l = 1; l <= NG; ++l) {
              const double* a = &Q[5 * g(i, l, k)];
              double* b = &Q[5 * g(i, -l, k)];
              b[0] = a[0]; b[1] = -a[1]; b[2] = -a[2]; b[3] = -a[3]; b[4] = a[4];
            }
          } else {  // inviscid slip wall in the x-y plane (:296-350)
            const Prim s = to_prim(&Q[5 * g(i, 1, k)], gam1);
            const long t0 = g(i, 0, k);
            double tx = met[4][t0], ty = -met[3][t0], J = met[9][t0];
            tx *= J; ty *= J;
            const double tn = std::sqrt(tx * tx + ty * ty);
            tx /= tn; ty /= tn;
            for (long l = 1; l <= NG; ++l) {
              const double* a = &Q[5 * g(i, l, k)];
              double* b = &Q[5 * g(i, -l, k)];
              const double vt = a[1] * tx + a[2] * ty;
              b[0] = a[0];
              b[1] = 2 * vt * tx - a[1];
              b[2] = 2 * vt * ty - a[2];
              b[3] = a[3];
              // the reference's expression, sign of the last term included (:331-333)
              b[4] = a[4] - 0.5 * (a[1] * a[1] + a[2] * a[2] - b[1] * b[1] + b[2] * b[2]) / b[0];
            }
            const double vt = s.u * tx + s.v * ty;
            const double uu = vt * tx, vv = vt * ty;
            double* o = &Q[5 * t0];
            o[0] = s.r; o[1] = s.r * uu; o[2] = s.r * vv; o[3] = s.r * s.w;
            o[4] = s.p / gam1 + 0.5 * s.r * (uu * uu + vv * vv + s.w * s.w);
          }
        }
      }
    if (og) bc_characteristic(Q, 1, 1, 1);
    // phase 2b: primitives on the j faces (:354-413)
#pragma omp parallel for schedule(static)
    for (long k = 1; k < KM - 1; ++k)
      for (long i = 0; i < IM; ++i) {
        for (long l = 0; l <= NG; ++l) put_prim(g(i, -l, k), to_prim(&Q[5 * g(i, -l, k)], gam1));
        const Prim s = to_prim(&Q[5 * g(i, JM - 1, k)], gam1);
        for (long l = 0; l < NG; ++l) put_prim(g(i, JM - 1 + l, k), s);
      }
    // phase 3: k faces (:417-492)
#pragma omp parallel for schedule(static)
    for (long j = 0; j < JM; ++j)
      for (long i = 0; i < IM; ++i) {
        for (int side = 0; side < 2; ++side) {
          const long src = side == 0 ? 1 : KM - 2;
          const long base = side == 0 ? 0 : KM - 1;
          const long dir = side == 0 ? -1 : 1;
          const long ts = g(i, j, src);
          for (long l = 0; l <= NG; ++l)
            std::memcpy(&Q[5 * g(i, j, base + dir * l)], &Q[5 * ts], 5 * sizeof(double));
          const Prim s = to_prim(&Q[5 * ts], gam1);
          for (long l = 0; l <= NG; ++l) put_prim(g(i, j, base + dir * l), s);
        }
      }
    if (og) {  // i < W and i >= IM - W, ghosts included, over the ghosted (j, k) box
      const long W = CBNS_OGRID_WRAP, Pw = IM - 2 * W;
#pragma omp parallel for schedule(static)
      for (long k = -NG; k < KM + NG; ++k)
        for (long j = -NG; j < JM + NG; ++j)
          for (long i = -NG; i < IM + NG; ++i) {
            if (i >= W && i < IM - W) continue;
            const long t = g(i, j, k), ts = g(i < W ? i + Pw : i - Pw, j, k);
            std::memcpy(&Q[5 * t], &Q[5 * ts], 5 * sizeof(double));
            rho[t] = rho[ts]; u[t] = u[ts]; v[t] = v[ts]; w[t] = w[ts]; p[t] = p[ts];
            if (P.viscous) T[t] = T[ts];
          }
    }
  }

  // ---------------------------------------------------------------------------
  // One face of rec_riemann_{xi,eta,zeta}_kernel (src/rec_riemann_kernel.cu:15-247):
  // nodes a (low) and b (high) along direction with stride sd, metric arrays mx,my,mz.
  // Linear upwind-5 face flux of the hybrid scheme (no counterpart in the
  // reference): each conservative component reconstructed with the WENO5
  // optimal weights frozen, (2a - 13b + 47c + 27d - 3e) / 60 on both sides,
  // then the same Lax-Friedrichs flux as the WENO5 face.
  void face_linear(const std::vector<double>& Q, long ta, long sd, int mdir, double* out) const {
    const long tb = ta + sd;
    const double Ja = met[9][ta], Jb = met[9][tb];
    const double nx = 0.5 * (met[3 * mdir + 0][ta] * Ja + met[3 * mdir + 0][tb] * Jb);
    const double ny = 0.5 * (met[3 * mdir + 1][ta] * Ja + met[3 * mdir + 1][tb] * Jb);
    const double nz = 0.5 * (met[3 * mdir + 2][ta] * Ja + met[3 * mdir + 2][tb] * Jb);
    double ql[5], qh[5];
    for (int n = 0; n < 5; ++n) {
      const double f0 = Q[5 * (ta - 2 * sd) + n], f1 = Q[5 * (ta - sd) + n], f2 = Q[5 * ta + n];
      const double f3 = Q[5 * tb + n], f4 = Q[5 * (tb + sd) + n], f5 = Q[5 * (tb + 2 * sd) + n];
      ql[n] = (2.0 * f0 - 13.0 * f1 + 47.0 * f2 + 27.0 * f3 - 3.0 * f4) / 60.0;
      qh[n] = (2.0 * f5 - 13.0 * f4 + 47.0 * f3 + 27.0 * f2 - 3.0 * f1) / 60.0;
    }
    lf_flux(to_prim(qh, D.gam1), to_prim(ql, D.gam1), nx, ny, nz, P.gamma, D.gam1, out);
  }

  // Face flux under the hybrid mask (empty mask: WENO5 everywhere).
  void face_h(const std::vector<double>& Q, long e, long ta, long sd, int mdir, double* out) const {
    if (!hmask.empty() && hmask[e] == 0) face_linear(Q, ta, sd, mdir, out);
    else face(Q, ta, sd, mdir, out);
  }

  void face(const std::vector<double>& Q, long ta, long sd, int mdir, double* out) const {
    const long tb = ta + sd;
    const double Ja = met[9][ta], Jb = met[9][tb];
    const double nx = 0.5 * (met[3 * mdir + 0][ta] * Ja + met[3 * mdir + 0][tb] * Jb);
    const double ny = 0.5 * (met[3 * mdir + 1][ta] * Ja + met[3 * mdir + 1][tb] * Jb);
    const double nz = 0.5 * (met[3 * mdir + 2][ta] * Ja + met[3 * mdir + 2][tb] * Jb);
    const Prim a{rho[ta], u[ta], v[ta], w[ta], p[ta]};
    const Prim b{rho[tb], u[tb], v[tb], w[tb], p[tb]};
    double R[5][5], L[5][5];
    roe_eigen(a, b, nx, ny, nz, P.gamma, D.gam1, R, L);
    const double* lo[5] = {&Q[5 * (ta - 2 * sd)], &Q[5 * (ta - sd)], &Q[5 * ta], &Q[5 * tb],
                           &Q[5 * (tb + sd)]};
    const double* hi[5] = {&Q[5 * (tb + 2 * sd)], &Q[5 * (tb + sd)], &Q[5 * tb], &Q[5 * ta],
                           &Q[5 * (ta - sd)]};
    const Prim sl = rec_weno5(lo, R, L, D.gam1);
    const Prim sh = rec_weno5(hi, R, L, D.gam1);
    lf_flux(sh, sl, nx, ny, nz, P.gamma, D.gam1, out);
  }

  // calc_numerical_flux: src/calc_numerical_flux.cu:15-74.
  // With a hybrid mask set, faces whose mask byte is 0 take face_linear;
  // mask index: i-faces, then j-faces, then k-faces, each in Ep/Fp/Gp order.
  void calc_numerical_flux(int which) {
    const auto& Q = buf(which);
    const long sI = 1, sJ = IG, sK = IG * JG;
    const long ni = (IM - 1) * (JM - 2) * (KM - 2), nj = (IM - 2) * (JM - 1) * (KM - 2);
#pragma omp parallel for schedule(dynamic, 1)
    for (long k = 0; k < KM - 2; ++k)
      for (long j = 0; j < JM - 2; ++j)
        for (long i = 0; i < IM - 1; ++i) {
          const long e = i + (IM - 1) * (j + (JM - 2) * k);
          face_h(Q, e, g(i, j + 1, k + 1), sI, 0, &Ep[NEQ * e]);
        }
#pragma omp parallel for schedule(dynamic, 1)
    for (long k = 0; k < KM - 2; ++k)
      for (long j = 0; j < JM - 1; ++j)
        for (long i = 0; i < IM - 2; ++i) {
          const long e = i + (IM - 2) * (j + (JM - 1) * k);
          face_h(Q, ni + e, g(i + 1, j, k + 1), sJ, 1, &Fp[NEQ * e]);
        }
#pragma omp parallel for schedule(dynamic, 1)
    for (long k = 0; k < KM - 1; ++k)
      for (long j = 0; j < JM - 2; ++j)
        for (long i = 0; i < IM - 2; ++i) {
          const long e = i + (IM - 2) * (j + (JM - 2) * k);
          face_h(Q, ni + nj + e, g(i + 1, j + 1, k), sK, 2, &Gp[NEQ * e]);
        }
  }

  // Flux difference + viscous contribution over J at interior node (i,j,k),
  // src/runge_kutta_kernel.cu:45-66.
  void df_at(long i, long j, long k, double* df) const {
    const double J = met[9][g(i, j, k)];
    for (int n = 0; n < NEQ; ++n) {
      double d = Ep[n + NEQ * (i + (IM - 1) * ((j - 1) + (JM - 2) * (k - 1)))] -
                 Ep[n + NEQ * ((i - 1) + (IM - 1) * ((j - 1) + (JM - 2) * (k - 1)))];
      d += Fp[n + NEQ * ((i - 1) + (IM - 2) * (j + (JM - 1) * (k - 1)))] -
           Fp[n + NEQ * ((i - 1) + (IM - 2) * ((j - 1) + (JM - 1) * (k - 1)))];
      d += Gp[n + NEQ * ((i - 1) + (IM - 2) * ((j - 1) + (JM - 2) * k))] -
           Gp[n + NEQ * ((i - 1) + (IM - 2) * ((j - 1) + (JM - 2) * (k - 1)))];
      if (P.viscous && n > 0) d -= dfv[(n - 1) + (NEQ - 1) * ((i - 1) + (IM - 2) * ((j - 1) + (JM - 2) * (k - 1)))];
      df[n] = d / J;
    }
  }

  // update_rk3: src/time_integration.cu:15-40, src/runge_kutta_kernel.cu:13-80.
  void update_rk3(double dt, unsigned stage) {
#pragma omp parallel for schedule(static)
    for (long k = 1; k < KM - 1; ++k)
      for (long j = 1; j < JM - 1; ++j)
        for (long i = 1; i < IM - 1; ++i) {
          double df[NEQ];
          df_at(i, j, k, df);
          const long t = g(i, j, k);
          for (int n = 0; n < NEQ; ++n) {
            const long e = 5 * t + n;
            if (stage == 1) Qb[e] = Qa[e] - dt * df[n];
            else if (stage == 2) Qb[e] = 0.75 * Qa[e] + 0.25 * (Qb[e] - dt * df[n]);
            else if (stage == 3) Qa[e] = (Qa[e] + 2.0 * (Qb[e] - dt * df[n])) / 3.0;
          }
        }
  }

  // ---------------------------------------------------------------------------
  // calc_dt: src/calc_dt.cu:18-62 + src/time_step_kernel.cu:13-96.  Returns
  // CFL / max(sigma); a NaN sigma anywhere makes the result NaN.
  double calc_dt() {
    double smax = 0.0;
    bool nan = false;
#pragma omp parallel for schedule(static) reduction(max : smax) reduction(|| : nan)
    for (long k = 0; k < KM; ++k)
      for (long j = 0; j < JM; ++j)
        for (long i = 0; i < IM; ++i) {
          const long t = g(i, j, k);
          const double r = rho[t], uu = u[t], vv = v[t], ww = w[t], pp = p[t];
          const double c = std::sqrt(P.gamma * pp / r);
          double fv = 0.0;
          // dt_viscous = 1 (CBNS_DTV_FULL) drops the local-Mach factor |u|/c
          if (P.viscous)
            fv = P.dt_viscous == 1 ? 2.0 * mu[t] * D.C_dt_v / r
                                   : 2.0 * mu[t] * D.C_dt_v * std::sqrt(uu * uu + vv * vv + ww * ww) / c / r;
          double s = 0.0;
          for (int d = 0; d < 3; ++d) {
            const double nx = met[3 * d][t], ny = met[3 * d + 1][t], nz = met[3 * d + 2][t];
            const double qn = uu * nx + vv * ny + ww * nz;
            const double na = std::sqrt(nx * nx + ny * ny + nz * nz);
            double sd = std::abs(qn) + c * na;
            if (P.viscous) sd += na * na * fv;
            s += sd;
          }
          dtn[i + IM * (j + JM * k)] = s;
          if (std::isnan(s)) nan = true;
          else smax = std::max(smax, s);
        }
    if (nan) return std::nan("");
    return P.CFL / smax;
  }

  // ---------------------------------------------------------------------------
  // calc_viscous_terms: src/calc_viscous_terms.cu:16-88 with gradient_wg_kernel
  // (src/gradient_kernel.cu:135-255) and src/viscous_terms_kernel.cu:13-107.
  void calc_viscous_terms() {
    gradient3(u.data(), IG, JG, KG, grad[0].data(), grad[1].data(), grad[2].data());
    gradient3(v.data(), IG, JG, KG, grad[3].data(), grad[4].data(), grad[5].data());
    gradient3(w.data(), IG, JG, KG, grad[6].data(), grad[7].data(), grad[8].data());
    gradient3(T.data(), IG, JG, KG, grad[9].data(), grad[10].data(), grad[11].data());
    const double qc = -D.Pr_inv * D.gam1_inv / D.Mach2;
#pragma omp parallel for schedule(static)
    for (long t = 0; t < NGt; ++t) {
      const double Tl = T[t];
      double m = (1.0 + D.C_T_inf) / (Tl + D.C_T_inf) * std::sqrt(Tl * Tl * Tl);
      mu[t] = m;
      const double xx = met[0][t], xy = met[1][t], xz = met[2][t];
      const double ex = met[3][t], ey = met[4][t], ez = met[5][t];
      const double zx = met[6][t], zy = met[7][t], zz = met[8][t];
      // velocity gradient in physical space by the chain rule
      const double ux = grad[0][t] * xx + grad[1][t] * ex + grad[2][t] * zx;
      const double uy = grad[0][t] * xy + grad[1][t] * ey + grad[2][t] * zy;
      const double uz = grad[0][t] * xz + grad[1][t] * ez + grad[2][t] * zz;
      const double vx = grad[3][t] * xx + grad[4][t] * ex + grad[5][t] * zx;
      const double vy = grad[3][t] * xy + grad[4][t] * ey + grad[5][t] * zy;
      const double vz = grad[3][t] * xz + grad[4][t] * ez + grad[5][t] * zz;
      const double wx = grad[6][t] * xx + grad[7][t] * ex + grad[8][t] * zx;
      const double wy = grad[6][t] * xy + grad[7][t] * ey + grad[8][t] * zy;
      const double wz = grad[6][t] * xz + grad[7][t] * ez + grad[8][t] * zz;
      m *= D.Re_inv;
      tau[0][t] = (2.0 / 3.0) * m * (2.0 * ux - vy - wz);
      tau[1][t] = (2.0 / 3.0) * m * (2.0 * vy - ux - wz);
      tau[2][t] = (2.0 / 3.0) * m * (2.0 * wz - ux - vy);
      tau[3][t] = m * (uy + vx);
      tau[4][t] = m * (uz + wx);
      tau[5][t] = m * (vz + wy);
      const double k = m * qc;
      qf[0][t] = k * (xx * grad[9][t] + ex * grad[10][t] + zx * grad[11][t]);
      qf[1][t] = k * (xy * grad[9][t] + ey * grad[10][t] + zy * grad[11][t]);
      qf[2][t] = k * (xz * grad[9][t] + ez * grad[10][t] + zz * grad[11][t]);
    }
  }

  // calc_viscous_flux_contribution: src/calc_viscous_flux_contribution.cu:16-69,
  // src/viscous_flux_kernel.cu:13-112 and src/viscous_contribution_kernel.cu:13-71.
  void calc_viscous_flux_contribution() {
    const long VI = IG - 2, VJ = JG - 2, VK = KG - 2;
    auto ev = [&](long a, long b, long c) { return (NEQ - 1) * (a + VI * (b + VJ * c)); };
#pragma omp parallel for schedule(static)
    for (long c = 0; c < VK; ++c)
      for (long b = 0; b < VJ; ++b)
        for (long a = 0; a < VI; ++a) {
          const long t = g(a - 1, b - 1, c - 1);  // node of flux entry (a,b,c)
          const double J = met[9][t];
          const double uu = u[t], vv = v[t], ww = w[t];
          const double txx = tau[0][t], tyy = tau[1][t], tzz = tau[2][t];
          const double txy = tau[3][t], txz = tau[4][t], tyz = tau[5][t];
          const double ex = uu * txx + vv * txy + ww * txz - qf[0][t];
          const double ey = uu * txy + vv * tyy + ww * tyz - qf[1][t];
          const double ez = uu * txz + vv * tyz + ww * tzz - qf[2][t];
          std::vector<double>* outs[3] = {&Ev, &Fv, &Gv};
          for (int d = 0; d < 3; ++d) {
            const double nx = met[3 * d][t] * J, ny = met[3 * d + 1][t] * J, nz = met[3 * d + 2][t] * J;
            double* o = &(*outs[d])[ev(a, b, c)];
            o[0] = nx * txx + ny * txy + nz * txz;
            o[1] = nx * txy + ny * tyy + nz * tyz;
            o[2] = nx * txz + ny * tyz + nz * tzz;
            o[3] = nx * ex + ny * ey + nz * ez;
          }
        }
    // 4th-order central divergence.  With CBNS_VISDIV_REFERENCE each
    // directional derivative is taken where viscous_contribution_kernel.cu:269-288
    // takes it: flux entry (i+NG-3.., j, k) is node (i-2.., j-1, k-1), i.e. the
    // i-derivative at node (i, j-1, k-1), the j-derivative at (i-1, j, k-1) and
    // the k-derivative at (i-1, j-1, k).
    const bool ref = P.vis_divergence == CBNS_VISDIV_REFERENCE;
    const long sh = ref ? 1 : 0;
#pragma omp parallel for schedule(static)
    for (long k = 1; k < KM - 1; ++k)
      for (long j = 1; j < JM - 1; ++j)
        for (long i = 1; i < IM - 1; ++i) {
          for (int n = 0; n < NEQ - 1; ++n) {
            auto D4 = [&](const std::vector<double>& F, long a, long b, long c, long da, long db, long dc) {
              // entry index of node (x,y,z) is (x+1, y+1, z+1)
              auto at = [&](long s) { return F[n + ev(a + 1 + s * da, b + 1 + s * db, c + 1 + s * dc)]; };
              return (1.0 / 12.0) * at(-2) + (-2.0 / 3.0) * at(-1) - (-2.0 / 3.0) * at(1) - (1.0 / 12.0) * at(2);
            };
            double d = D4(Ev, i, j - sh, k - sh, 1, 0, 0);
            d += D4(Fv, i - sh, j, k - sh, 0, 1, 0);
            d += D4(Gv, i - sh, j - sh, k, 0, 0, 1);
            dfv[n + (NEQ - 1) * ((i - 1) + (IM - 2) * ((j - 1) + (JM - 2) * (k - 1)))] = d;
          }
        }
  }

  // The time loop of Block3d::solve (src/Block3d.cpp:237-293) without I/O.
  // Returns 0, or CBNS_ERR_NAN_DT when calc_dt yields NaN (src/calc_dt.cu:56-58).
  int solve(unsigned nstep_max, double t_end, double* t_cur, unsigned* steps_done) {
    unsigned n = 0;
    for (; n < nstep_max; ++n) {
      if (*t_cur + 1.0e-8 > t_end) break;
      double dt = calc_dt();
      if (std::isnan(dt)) {
        if (steps_done) *steps_done = n;
        return CBNS_ERR_NAN_DT;
      }
      if (t_end - *t_cur < dt) dt = t_end - *t_cur;
      *t_cur += dt;
      for (unsigned s = 1; s <= 3; ++s) {
        calc_numerical_flux(s == 1 ? CBNS_Q : CBNS_QP);
        if (P.viscous) calc_viscous_flux_contribution();
        update_rk3(dt, s);
        set_bc_calc_primitive(s == 3 ? CBNS_Q : CBNS_QP);
        if (P.viscous) calc_viscous_terms();
      }
    }
    if (steps_done) *steps_done = n;
    return 0;
  }
};

// AoS <-> per-array helpers for the ghosted-array getters.
void copy_interior(const Oracle& o, const std::vector<double>& src, double* dst) {
  for (long k = 0; k < o.KM; ++k)
    for (long j = 0; j < o.JM; ++j)
      for (long i = 0; i < o.IM; ++i) dst[i + o.IM * (j + o.JM * k)] = src[o.g(i, j, k)];
}

}  // namespace

// ----------------------------------------------------------------------------
// extern "C" surface used by the Python tests (ctypes).
extern "C" {

void* orc_create(const cbns_params* p) {
  if (!p || p->IM < 4 || p->JM < 4 || p->KM < 4) return nullptr;
  return new Oracle(*p);
}
void orc_destroy(void* h) { delete static_cast<Oracle*>(h); }
void orc_calc_metrics(void* h, const double* x, const double* y, const double* z) {
  static_cast<Oracle*>(h)->calc_metrics(x, y, z);
}
// 10 ghosted arrays (xi_x..zeta_z, Jac), each IM_G*JM_G*KM_G, concatenated.
void orc_get_metrics_ghosted(void* h, double* out) {
  auto* o = static_cast<Oracle*>(h);
  for (int m = 0; m < 10; ++m) std::memcpy(out + m * o->NGt, o->met[m].data(), o->NGt * sizeof(double));
}
// get_metrics (src/get_metrics.cu:6-67): the 10 metric arrays on the IM*JM*KM nodes.
void orc_get_metrics(void* h, double* out) {
  auto* o = static_cast<Oracle*>(h);
  const long N = o->IM * o->JM * o->KM;
  for (int m = 0; m < 10; ++m) copy_interior(*o, o->met[m], out + m * N);
}
void orc_initial_condition(void* h) { static_cast<Oracle*>(h)->initial_condition(); }
void orc_calc_conservative(void* h, int which) { static_cast<Oracle*>(h)->calc_conservative(which); }
// set_conservative (src/set_conservative.cu): Q from the host, then Q_p = Q.
void orc_set_conservative(void* h, const double* Q) {
  auto* o = static_cast<Oracle*>(h);
  std::memcpy(o->Qa.data(), Q, o->Qa.size() * sizeof(double));
  o->Qb = o->Qa;
}
void orc_get_conservative(void* h, int which, double* Q) {
  auto* o = static_cast<Oracle*>(h);
  const auto& b = o->buf(which);
  std::memcpy(Q, b.data(), b.size() * sizeof(double));
}
// rho,u,v,w,p,T,mu ghosted arrays concatenated (7 * IM_G*JM_G*KM_G).
void orc_get_primitive(void* h, double* out) {
  auto* o = static_cast<Oracle*>(h);
  const std::vector<double>* a[7] = {&o->rho, &o->u, &o->v, &o->w, &o->p, &o->T, &o->mu};
  for (int m = 0; m < 7; ++m) std::memcpy(out + m * o->NGt, a[m]->data(), o->NGt * sizeof(double));
}
void orc_calc_primitive(void* h, int which) { static_cast<Oracle*>(h)->calc_primitive(which); }
void orc_set_bc_calc_primitive(void* h, int which) { static_cast<Oracle*>(h)->set_bc_calc_primitive(which); }
void orc_calc_numerical_flux(void* h, int which) { static_cast<Oracle*>(h)->calc_numerical_flux(which); }
void orc_get_face_fluxes(void* h, double* Ep, double* Fp, double* Gp) {
  auto* o = static_cast<Oracle*>(h);
  std::memcpy(Ep, o->Ep.data(), o->Ep.size() * sizeof(double));
  std::memcpy(Fp, o->Fp.data(), o->Fp.size() * sizeof(double));
  std::memcpy(Gp, o->Gp.data(), o->Gp.size() * sizeof(double));
}
void orc_calc_viscous_terms(void* h) { static_cast<Oracle*>(h)->calc_viscous_terms(); }
void orc_calc_viscous_flux_contribution(void* h) { static_cast<Oracle*>(h)->calc_viscous_flux_contribution(); }
void orc_update_rk3(void* h, double dt, unsigned stage) { static_cast<Oracle*>(h)->update_rk3(dt, stage); }
double orc_calc_dt(void* h) { return static_cast<Oracle*>(h)->calc_dt(); }
int orc_solve(void* h, unsigned nstep_max, double t_end, double* t_cur, unsigned* steps_done) {
  return static_cast<Oracle*>(h)->solve(nstep_max, t_end, t_cur, steps_done);
}
// One RHS evaluation (flux + viscous contribution, then df/J as rk3_kernel forms it)
// for the given buffer; boundary conditions (and viscous terms) must be current.
void orc_eval_rhs(void* h, int which, double* rhs) {
  auto* o = static_cast<Oracle*>(h);
  o->calc_numerical_flux(which);
  if (o->P.viscous) o->calc_viscous_flux_contribution();
  const long I2 = o->IM - 2, J2 = o->JM - 2, K2 = o->KM - 2;
#pragma omp parallel for schedule(static)
  for (long k = 1; k <= K2; ++k)
    for (long j = 1; j <= J2; ++j)
      for (long i = 1; i <= I2; ++i) o->df_at(i, j, k, &rhs[5 * ((i - 1) + I2 * ((j - 1) + J2 * (k - 1)))]);
}
// Hybrid flux decisions for the following flux evaluations: n bytes in global
// face index order (1 = WENO5, 0 = linear upwind-5); n = 0 clears the mask.
void orc_set_face_mask(void* h, const unsigned char* mask, long n) {
  auto* o = static_cast<Oracle*>(h);
  if (n <= 0 || !mask) o->hmask.clear();
  else o->hmask.assign(mask, mask + n);
}

// Sensor features and WENO-weight deviation of every grid face, in the order
// i-faces, j-faces, k-faces (each i fastest), for the learned shock sensor
// (no counterpart in the reference).  Restates the definitions of the
// library's sensor.cuh in FP64: 15 normalised (then log-compressed) jumps of density, pressure and
// normal velocity; deviation = max |w_k - d_k| of the characteristic WENO5
// weights (basis and Roe average of the flux) on both sides of all 5 fields.
void orc_sensor_faces(void* h, int which, float* feat, float* dev) {
  // each jump compressed as sign(f) log2(1 + |f| / 0.01)
  auto compress = [](double f) { return std::copysign(std::log2(1.0 + std::abs(f) / 0.01), f); };
  auto* o = static_cast<Oracle*>(h);
  const auto& Q = o->buf(which);
  const long IM = o->IM, JM = o->JM, KM = o->KM;
  const long ni = (IM - 1) * (JM - 2) * (KM - 2), nj = (IM - 2) * (JM - 1) * (KM - 2), nk = (IM - 2) * (JM - 2) * (KM - 1);
  const double gam1 = o->D.gam1, gamma = o->P.gamma;
#pragma omp parallel for schedule(static)
  for (long e = 0; e < ni + nj + nk; ++e) {
    int dir;
    long i, j, k;
    if (e < ni) { dir = 0; i = e % (IM - 1); j = 1 + (e / (IM - 1)) % (JM - 2); k = 1 + e / ((IM - 1) * (JM - 2)); }
    else if (e < ni + nj) { const long r = e - ni; dir = 1; i = 1 + r % (IM - 2); j = (r / (IM - 2)) % (JM - 1); k = 1 + r / ((IM - 2) * (JM - 1)); }
    else { const long r = e - ni - nj; dir = 2; i = 1 + r % (IM - 2); j = 1 + (r / (IM - 2)) % (JM - 2); k = r / ((IM - 2) * (JM - 2)); }
    const long sd = dir == 0 ? 1 : (dir == 1 ? o->IG : o->IG * o->JG);
    const long ta = o->g(i, j, k), tb = ta + sd;
    const double Ja = o->met[9][ta], Jb = o->met[9][tb];
    const double nx = 0.5 * (o->met[3 * dir][ta] * Ja + o->met[3 * dir][tb] * Jb);
    const double ny = 0.5 * (o->met[3 * dir + 1][ta] * Ja + o->met[3 * dir + 1][tb] * Jb);
    const double nz = 0.5 * (o->met[3 * dir + 2][ta] * Ja + o->met[3 * dir + 2][tb] * Jb);
    const double nn = std::sqrt(nx * nx + ny * ny + nz * nz);
    double r[6], pr[6], un[6];
    for (int q = 0; q < 6; ++q) {
      const Prim s = to_prim(&Q[5 * (ta + (q - 2) * sd)], gam1);
      r[q] = s.r; pr[q] = s.p; un[q] = (s.u * nx + s.v * ny + s.w * nz) / nn;
    }
    const double rb = 0.5 * (r[2] + r[3]), pb = 0.5 * (pr[2] + pr[3]), cb = std::sqrt(gamma * pb / rb);
    for (int m = 0; m < 5; ++m) {
      feat[15 * e + m] = (float)compress((r[m + 1] - r[m]) / rb);
      feat[15 * e + 5 + m] = (float)compress((pr[m + 1] - pr[m]) / pb);
      feat[15 * e + 10 + m] = (float)compress((un[m + 1] - un[m]) / cb);
    }
    const Prim a = to_prim(&Q[5 * ta], gam1), b = to_prim(&Q[5 * tb], gam1);
    double R[5][5], L[5][5];
    roe_eigen(a, b, nx, ny, nz, gamma, gam1, R, L);
    double W[5][6];
    for (int q = 0; q < 6; ++q)
      for (int s = 0; s < 5; ++s) {
        double acc = 0.0;
        for (int n = 0; n < 5; ++n) acc += L[s][n] * Q[5 * (ta + (q - 2) * sd) + n];
        W[s][q] = acc;
      }
    auto wdev = [](double A, double B, double Cc, double Dd, double E) {
      const double eps = 1.0e-6;
      const double s1 = (13.0 / 12.0) * (A - 2 * B + Cc) * (A - 2 * B + Cc) + 0.25 * (A - 4 * B + 3 * Cc) * (A - 4 * B + 3 * Cc) + eps;
      const double s2 = (13.0 / 12.0) * (B - 2 * Cc + Dd) * (B - 2 * Cc + Dd) + 0.25 * (B - Dd) * (B - Dd) + eps;
      const double s3 = (13.0 / 12.0) * (Cc - 2 * Dd + E) * (Cc - 2 * Dd + E) + 0.25 * (3 * Cc - 4 * Dd + E) * (3 * Cc - 4 * Dd + E) + eps;
      const double a1 = 0.1 / (s1 * s1), a2 = 0.6 / (s2 * s2), a3 = 0.3 / (s3 * s3), t = a1 + a2 + a3;
      return std::max(std::max(std::abs(a1 / t - 0.1), std::abs(a2 / t - 0.6)), std::abs(a3 / t - 0.3));
    };
    double dv = 0.0;
    for (int s = 0; s < 5; ++s) {
      dv = std::max(dv, wdev(W[s][0], W[s][1], W[s][2], W[s][3], W[s][4]));
      dv = std::max(dv, wdev(W[s][5], W[s][4], W[s][3], W[s][2], W[s][1]));
    }
    dev[e] = (float)dv;
  }
}

// calc_gradient (src/calc_gradient.cu:17-51): gradient of an unghosted field.
void orc_calc_gradient(unsigned IM, unsigned JM, unsigned KM, const double* f, double* fx, double* fy,
                       double* fz) {
  gradient3(f, IM, JM, KM, fx, fy, fz);
}

}  // extern "C"
