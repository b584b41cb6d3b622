// bc.cuh - launch interface of the boundary-condition kernels (bc.cu).
#pragma once

#include "cbns_common.cuh"

namespace cbns {

struct BCArgs {
  Dims d;
  double gamma, gam1, gM2, p_inf;
  unsigned i_begin, i_end;
  int viscous;
  double* q;             // the buffer the boundary conditions act on (5 fields)
  const double* met[10];
  double* prim[6];       // rho,u,v,w,p,T (viscous runs)
  StepState* st;
  int check_done;        // return at once when st->done is set (graph-replayed steps)
  int sigma;             // inviscid: accumulate boundary-node spectral radii
  int farfield;          // boundary and ghost nodes hold their state (FARFIELD), or take the
                         // characteristic far-field state (CHARACTERISTIC); primitives from Q
  int characteristic;    // CBNS_BC_CHARACTERISTIC
  double u_inf, v_inf;   // free-stream velocity (cos, sin of the angle of attack)
  int wrap;              // CBNS_BC_OGRID: number of copied points either side of the seam, else 0
};

// interior_prims: also recompute interior primitives (viscous runs), when the
// primitive arrays do not describe this buffer.  *launches += kernels launched.
cudaError_t launch_bc(const BCArgs& a, bool interior_prims, cudaStream_t s, int* launches);

// CBNS_BC_FARFIELD for many blocks in one launch (the batched form): args and
// cta are device tables, block b owning CTAs cta[b] .. cta[b+1]-1 (cta has
// nblocks + 1 entries, cta[b+1] - cta[b] = bc_farfield_ctas(its Dims)).
int bc_farfield_ctas(const Dims& d);
cudaError_t launch_bc_farfield_batched(const BCArgs* args, const int* cta, int nblocks, int total_ctas,
                                       cudaStream_t s);

}  // namespace cbns
