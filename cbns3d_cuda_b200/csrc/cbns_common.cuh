// cbns_common.cuh - data layout, run parameters and small device helpers shared
// by every kernel of the B200 RK3 right-hand-side library.
//
// HBM layout (structure of arrays).  Every node field (each conservative
// variable, each metric, each primitive, each viscous flux component) is one
// FP64 array over the ghosted box of IM_G x JM_G x KM_G nodes (NG = 2 ghost
// layers, as include/Block3d_cuda.h:40-49 of the reference).  Node (i,j,k),
// i in [-2, IM+2), sits at element
//     LP + (i+2) + PX*((j+2) + JG*(k+2))
// where LP = 13 leading pad elements make interior node i = 1 (ghosted index 3)
// start on a 128-byte boundary, and the row pitch PX (a multiple of 16 elements)
// keeps every row 128-byte aligned.  A conservative state buffer holds its five
// variables back to back, VOL elements apart (VOL a multiple of 32 elements).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace cbns {

constexpr int NEQ = 5;
constexpr int NG = 2;
constexpr long LP = 13;

struct Dims {
  int IM, JM, KM;  // grid points
  int IG, JG, KG;  // ghosted extents
  long PX;         // row pitch (elements)
  long PL;         // plane pitch = PX * JG
  long VOL;        // one field, padded
};

__host__ __device__ inline long node_off(const Dims& d, int i, int j, int k) {
  return LP + (long)(i + NG) + d.PX * ((long)(j + NG) + (long)d.JG * (long)(k + NG));
}

// Physical parameters after the derivation of src/Block3d.cpp:99-113.
struct Phys {
  double gamma, gam1, gam1_inv, gM2, Mach2, p_inf, CFL, Re_inv, Pr_inv, C_T_inf, C_dt_v;
  double angle_attack;
  unsigned i_begin, i_end;
  int viscous, visdiv, precision;
};

// Device pointers of one context.  Q buffers hold 5 fields each.
struct Fields {
  double* met[10];   // xi_x, xi_y, xi_z, eta_x, eta_y, eta_z, zeta_x, zeta_y, zeta_z, Jac
  double* area[10];  // J*grad(xi) (3), J*grad(eta) (3), J*grad(zeta) (3), 1/J
  float* area32[6];  // FP32 and hybrid contexts: J*grad(xi), J*grad(eta) rounded to FP32
  double* prim[7];   // rho, u, v, w, p, T, mu (viscous upkeep; on-demand otherwise)
  double* vflux[12]; // E0..E3, F0..F3, G0..G3 (viscous node fluxes, times J-scaled normals)
  double* dfv[4];    // divergence of the viscous node fluxes at the interior nodes (momentum 3, energy)
};

// Per-run scalars kept on the device so a whole step can be replayed from a graph.
struct StepState {
  unsigned long long sigma_bits;  // max spectral radius (bit pattern of a positive double)
  double dt;                      // time step of the current step
  double t_cur;                   // simulated time
  double t_end;
  unsigned steps;                 // steps taken
  int done;                       // time loop finished: kernels return immediately
  int nan_dt;                     // CFL/max(sigma) was NaN
  int force_weno;                 // hybrid: the audit rejected this step's sensor decisions
  unsigned audit_fail_steps;      // hybrid: steps whose sensor decisions the audit rejected
  unsigned long long weno_faces;  // hybrid: faces sent to WENO5 (summed over steps)
  unsigned long long weno_last;   // hybrid: faces the last widening sent to WENO5 (the held steps' count)
  unsigned long long audit_faces; // hybrid: faces the audit re-evaluated
  float audit_max;                // hybrid: largest relative flux difference the audit saw
  int sensor_fail;                // hybrid: a tensor-core wait timed out
  unsigned weno_listed[3];        // hybrid: lengths of the step's lists of WENO5 i-, j- and k-faces
  int stage_fail;                 // a stage kernel's TMA wait timed out (the state is not valid)
};

// Batched launches of per-block kernels: block b of a batch owns the CTAs
// cta[b] .. cta[b+1]-1 of the grid.  Returns the block of CTA x (the last b
// with cta[b] <= x; blocks that own no CTA are never returned).
__device__ __forceinline__ int block_of_cta(const int* cta, int nblocks, int x) {
  int lo = 0, hi = nblocks - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(cta + mid) <= x) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Positive doubles order like their bit patterns; a NaN (either sign) compares
// above every finite value, so a max over bit patterns propagates NaN.
__device__ inline void atomic_max_sigma(unsigned long long* a, double s) {
  unsigned long long b = (unsigned long long)__double_as_longlong(s);
  if (s != s) b = 0x7ff8000000000000ull;  // canonical NaN, above +inf
  atomicMax(a, b);
}

}  // namespace cbns
