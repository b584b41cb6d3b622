// stage.cuh - launch interface of the fused RK3 stage kernel (stage.cu).
#pragma once

#include <cuda.h>

#include "cbns_common.cuh"

namespace cbns {

// TMA tensor maps of the stage kernels' plane staging (tma.cuh), 4-D: x,
// rows, planes, fields.  FP32 kernels: q_a the stage input's i-side halo box
// (4 x 15 x 1 x 5, FP64), q_b its j-side halo box (16 x 3 x 1 x 5), xi / eta
// the FP32 face-node area vectors (the 6 area32 components; 24 x 15 x 1 x 3
// and 16 x 17 x 1 x 3).  FP64 TMA kernel: q_a the ring column box (16 x 15 x
// 1 x 5), q_b the plane-with-halo box (24 x 21 x 1 x 5), xi / eta the FP64
// area vectors (the 10 area components; the same boxes).
struct StageMaps {
  CUtensorMap q_a, q_b, xi, eta;
};

struct StageArgs {
  StageMaps tm;        // FP32 kernels: TMA maps for src and area32
  Dims d;
  double gamma, gam1, gam1_inv, gM2;
  const double* src;   // stage input (stencil source), 5 fields
  const double* q0;    // the reference's Q at the node (RK base)
  const double* qp;    // the reference's Q_p at the node (stages 2, 3)
  double* out;         // stage output (5 fields), or the dense RHS array in mode 0
  const double* met[10];
  const double* area[10];  // J*grad(xi|eta|zeta) per node, then 1/J
  const double* dfv[4];    // viscous: the divergence of the node fluxes (visc.cu; FP32 elements in the FP32 kernels)
  double* prim[6];     // viscous: rho,u,v,w,p,T of the new interior state
  StepState* st;       // dt, done flag, spectral-radius max
  const unsigned char* mask;  // hybrid: per-face sensor decision (null: plain flux everywhere)
  float* wflux;        // hybrid: WENO5 flux of each WENO5 face (8 floats per face, 5 used)
  const float* area32[6];  // FP32 kernels: J*grad(xi), J*grad(eta) per node in FP32
  int q0_is_src, qp_is_src;  // RK operands that equal the stage input (read from the ring)
  int ntile_i, ntile_j, kchunk;
  int visdiv;          // CBNS_VISDIV_*
  int sigma;           // accumulate the interior spectral-radius max (inviscid stage 3)
};

// Many blocks in one launch (a persistent work queue): args[b] are the
// StageArgs of block b, its work items (tile, k chunk) are numbered
// start[b] .. start[b+1]-1 of total, and *counter (zeroed before the launch)
// hands them out.
struct BatchStage {
  const StageArgs* args;  // device, nblocks entries
  const int* start;       // device, nblocks + 1 entries
  int nblocks, total;
  unsigned* counter;      // device
};

// mode 0: dense RHS output; 1..3: RK stage.  fp32: split-precision flux arithmetic.
// variant: a compiled occupancy variant, 0 .. stage_variants(fp32)-1.
cudaError_t launch_stage(const StageArgs& a, int mode, bool visc, bool fp32, int variant, cudaStream_t s);
int stage_variants(bool fp32, bool hybrid);
// Hybrid: list the faces whose decision byte is set (once per step, after the
// decisions are final; each face kind in its own list, st->weno_listed[kind]
// receiving its length) ...
cudaError_t launch_weno_list(const Dims& d, const unsigned char* mask, long nfaces, StepState* st, int2* list,
                             bool check_done, unsigned every, cudaStream_t s);
// ... and evaluate the listed faces (every face while force_weno is set) into
// a.wflux, where the stage kernel reads them: before each hybrid stage-kernel
// launch, on the same input.
cudaError_t launch_weno_faces(const StageArgs& a, int mode, long nfaces, const int2* list, cudaStream_t s);
// Size the evaluation kernel's grid (once, outside any stream capture).
cudaError_t weno_prepare();
// The lists of many blocks in one launch (after zeroing each block's count):
// block b owns CTAs cta[b] .. cta[b+1]-1 of total, weno_list_ctas(its Dims) of them.
struct ListArgs {
  Dims d;
  const unsigned char* mask;
  long nf;
  StepState* st;
  int2* list;
  int check_done;
  unsigned every;  // the network's interval (MaskArgs::every): the lists are rebuilt on its steps only
};
int weno_list_ctas(const Dims& d);
cudaError_t launch_weno_list_batched(const ListArgs* args, const int* cta, int nblocks, int total, cudaStream_t s);
// modes 1..3 only; hybrid: the StageArgs carry decision masks.
cudaError_t launch_stage_batched(const BatchStage& b, int mode, bool visc, bool fp32, bool hybrid, cudaStream_t s);
void stage_tiles(const Dims& d, int* ntile_i, int* ntile_j);

}  // namespace cbns
