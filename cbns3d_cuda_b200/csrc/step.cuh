// step.cuh - launch interface of the time-step bookkeeping kernels (step.cu).
#pragma once

#include "cbns_common.cuh"

namespace cbns {

struct SigmaArgs {
  Dims d;
  double gamma, gam1, C_dt_v;
  int viscous;
  int dt_full;            // viscous spectral radius without the |u|/c factor (CBNS_DTV_FULL)
  const double* q;        // inviscid: primitives recomputed from this buffer
  const double* prim[6];  // viscous: rho,u,v,w,p,T
  const double* mu;       // viscous
  const double* met[10];
  StepState* st;
};

// Zero the accumulator and reduce the spectral radius over all grid nodes.
cudaError_t launch_sigma_nodes(const SigmaArgs& a, cudaStream_t s);
cudaError_t launch_step_prologue(StepState* st, double CFL, cudaStream_t s);
// the prologues of n blocks in one launch (device tables st[n], CFL[n])
cudaError_t launch_step_prologue_batched(StepState* const* st, const double* CFL, int n, cudaStream_t s);
// new_step: count a step (per-call stage 1); restart: the count starts over first
cudaError_t launch_set_dt(StepState* st, double dt, bool new_step, bool restart, cudaStream_t s);

}  // namespace cbns
