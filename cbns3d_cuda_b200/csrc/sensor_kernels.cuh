// sensor_kernels.cuh - launch interface of the sensor training kernels
// (sensor.cu) and the tensor-core inference (sensor_tc.cu).
#pragma once

#include "cbns_common.cuh"

namespace cbns {

struct SampleArgs {
  Dims d;
  float gamma, gam1;
  const double* q;          // state buffer (5 fields)
  const double* area[10];   // node area vectors
  unsigned stride, offset;  // faces with (global face index % stride) == offset
  float* feat;              // capacity x 15
  unsigned char* label;     // capacity
  float* dev;               // capacity (may be null): WENO-weight deviation
  unsigned* index;          // capacity (may be null): global face index of each sample
  unsigned capacity;
  unsigned* count;          // device counter, incremented per sampled face
};

// Per-step decision of the hybrid flux: features of every face of q, the
// network on the tensor cores, mask[e] = 1 (WENO5) where p >= tau else 0.
struct MaskArgs {
  Dims d;
  float gamma, gam1;
  const double* q;
  const double* area[10];
  const float* params;      // CBNS_SENSOR_NPARAM floats (device)
  float tau;
  unsigned char* mask;      // one byte per face
  StepState* st;            // statistics, failure flag, done flag
  int check_done;
};

// Audit of the decisions: on the faces with e % stride == steps % stride that
// the sensor sent to the linear flux, recompute the WENO5 flux; a relative
// difference above bound sets st->force_weno for the step.
struct AuditArgs {
  Dims d;
  float gamma, gam1, gam1_inv;
  const double* q;
  const double* area[10];
  const unsigned char* mask;
  unsigned stride;
  float bound;
  StepState* st;
  int check_done;
};

cudaError_t launch_sample_faces(const SampleArgs& a, cudaStream_t s);
cudaError_t launch_sensor_mask(const MaskArgs& a, cudaStream_t s);
cudaError_t launch_sensor_audit(const AuditArgs& a, cudaStream_t s);
cudaError_t launch_mlp_grad(const float* P, const float* X, const unsigned char* Y, unsigned n, float pos_w, float* G,
                            float* loss, cudaStream_t s);
cudaError_t launch_adam(float* P, const float* G, float* M, float* V, unsigned step, float lr, cudaStream_t s);
cudaError_t launch_mlp_predict(const float* P, const float* X, unsigned n, float* out, cudaStream_t s);

}  // namespace cbns
