// visc.cuh - launch interface of the viscous node-flux kernel (visc.cu).
#pragma once

#include "cbns_common.cuh"

namespace cbns {

struct ViscArgs {
  Dims d;
  double gamma, Re_inv, C_T_inf, C_dt_v;
  int dt_full;               // viscous spectral radius without the |u|/c factor (CBNS_DTV_FULL)
  double qc;                 // -1/(Pr (gamma-1) M^2): heat-flux factor before mu/Re
  const double* prim[6];     // rho,u,v,w,p,T
  const double* met[10];
  double* vflux[12];         // E0..E3, F0..F3, G0..G3 (FP32 elements when f32)
  double* dfv[4];            // their divergence at the interior nodes (FP32 elements when f32)
  int f32;                   // FP32-flux precisions: node fluxes and divergence stored (and differenced) in FP32
  int visdiv;                // CBNS_VISDIV_*
  double* mu;
  StepState* st;
  int check_done;
  int sigma;                 // accumulate the spectral-radius max over the grid nodes
  int kc;                    // node kernel: k planes per CTA (visc_kchunk)
};

// The node fluxes, then their divergence (two kernels).
cudaError_t launch_visc(const ViscArgs& a, cudaStream_t s);
// k planes per CTA of the node kernel for a block on a device of nsm SMs.
int visc_kchunk(const Dims& d, int nsm);
// The same for many blocks in one launch: args and cta are device tables,
// block b owning CTAs cta[b] .. cta[b+1]-1, cta[b+1] - cta[b] = visc_ctas(its args).
int visc_ctas(const ViscArgs& a);
// The divergence kernel's CTAs for one block (cta tables of the batched divergence launch).
int visc_div_ctas(const Dims& d);
cudaError_t launch_visc_batched(const ViscArgs* args, const int* cta, int nblocks, int total_ctas,
                                const int* dcta, int dtotal, bool f32, cudaStream_t s);

}  // namespace cbns
