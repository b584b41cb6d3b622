// setup.cuh - launch interface of the setup and I/O kernels (setup.cu).
#pragma once

#include "cbns_common.cuh"
#include "../../include/cbns_b200.h"

namespace cbns {

// metrics, their ghost extension, and the node area vectors / 1/J (area32,
// may be null: FP32 copies of the xi and eta area vectors).  wrap > 0 (O-grid):
// the nodes i < wrap and i >= IM - wrap take the metrics of the nodes
// IM - 2*wrap away, before the ghost extension.
cudaError_t launch_metrics(const Dims& d, const double* x, const double* y, const double* z, double* const met[10],
                           double* const area[10], float* const area32[6], int wrap, cudaStream_t s);
cudaError_t launch_ic(const Dims& d, double* const prim[6], double angle_deg, double p_inf, int viscous,
                      cudaStream_t s);
// Case initial states on the ghosted box (kind CBNS_CASE_*, prm as in
// cbns_init_case) from the grid coordinates x, y, z (device, IM*JM*KM).
cudaError_t launch_case_ic(const Dims& d, const double* x, const double* y, const double* z, int kind,
                           const double* prm, int nprm, double gamma, double* q, cudaStream_t s);
cudaError_t launch_conservative(const Dims& d, double* const prim[6], double* q, double gam1, cudaStream_t s);
cudaError_t launch_primitive(const Dims& d, const double* q, double* const prim[6], double gam1, double gM2,
                             cudaStream_t s);
cudaError_t launch_aos_to_soa(const Dims& d, const double* aos, double* q, cudaStream_t s);
cudaError_t launch_soa_to_aos(const Dims& d, const double* q, double* aos, cudaStream_t s);
cudaError_t launch_gather_nodes(const Dims& d, const double* f, double* out, cudaStream_t s);
cudaError_t launch_gather_ghosted(const Dims& d, const double* f, double* out, cudaStream_t s);
cudaError_t launch_gradient_dense(int IM, int JM, int KM, const double* f, double* fx, double* fy, double* fz,
                                  cudaStream_t s);

}  // namespace cbns
