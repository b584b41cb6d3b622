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
  unsigned every;           // evaluate on steps with steps % every == 1 % every (1: always)
  unsigned char* mask;      // one byte per face
  StepState* st;            // statistics, failure flag, done flag
  int check_done;
};

// Widening of the decisions: a face takes WENO5 when the sensor chose WENO5
// for a face of the same direction within SN_DILATE_ALONG faces along its own
// grid line or SN_DILATE_ACROSS faces in the two other index directions.  A
// discontinuity moves less than a cell per time step (CFL <= 1): along a line
// it reaches at most one more node of the 6-node stencils near it, and a
// curved front (a blast) reaches grid lines next to those it crossed at the
// step's start, so those faces stay on WENO5 for the step's three stages.
// Three separable passes (one per index direction); the last one counts the
// WENO5 faces.  When the network runs only every n-th step, its decisions
// must hold for n steps: widths 1 + n along and n across.
struct DilateArgs {
  Dims d;
  const unsigned char* in;
  unsigned char* out;
  int dim;                 // index direction of this pass: 0 = i, 1 = j, 2 = k
  int along, across;       // widening widths (faces)
  StepState* st;           // WENO5 faces are counted when count != 0
  int count;
  unsigned every;          // as MaskArgs::every; the count is kept every step
  int hold;                // the decisions hold this step: count only (per-call path)
  int check_done;
};

// true when the sensor is evaluated in the current step (steps counts from 1)
__device__ __forceinline__ bool sensor_step(const StepState* st, unsigned every) {
  return every <= 1 || st->steps % every == 1;
}

// Audit of the decisions: on the runs of 128 consecutive faces with
// (e / 128) % stride == steps % stride, the faces the sensor sent to the linear
// flux are recomputed with WENO5; a relative difference above bound sets
// st->force_weno for the step.
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
cudaError_t launch_sensor_dilate(const DilateArgs& a, cudaStream_t s);
// Batched forms (many blocks in one launch): args and cta are device tables,
// block b owning CTAs cta[b] .. cta[b+1]-1 of total, cta[b+1] - cta[b] the
// block's count below.  Mask: ipre[b] .. ipre[b+1]-1 are block b's work items
// of each kind (sensor_mask_items); every block's MaskArgs::params must hold
// the same network (it is loaded once per CTA, from args[0]).
int sensor_dilate_ctas(const Dims& d, int dim);  // pass dim's grid
int sensor_audit_ctas(const AuditArgs& a);
void sensor_mask_items(const Dims& d, long* items0, long* items1);
cudaError_t launch_sensor_dilate_batched(const DilateArgs* args, const int* cta, int nblocks, int total,
                                         cudaStream_t s);
cudaError_t launch_sensor_audit_batched(const AuditArgs* args, const int* cta, int nblocks, int total,
                                        cudaStream_t s);
cudaError_t launch_sensor_mask_batched(const MaskArgs* args, const long* ipre0, const long* ipre1, long total0,
                                       long total1, int nblocks, cudaStream_t s);
cudaError_t launch_mlp_grad(const float* P, const float* X, const unsigned char* Y, unsigned n, float pos_w, float* G,
                            float* loss, cudaStream_t s);
cudaError_t launch_adam(float* P, const float* G, float* M, float* V, unsigned step, float lr, cudaStream_t s);
cudaError_t launch_mlp_predict(const float* P, const float* X, unsigned n, float* out, cudaStream_t s);

}  // namespace cbns
