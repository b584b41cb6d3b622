// step.cu - time-step bookkeeping kept on the device.
//
// The reference computes dt on the host every step: time_step_kernel writes a
// per-node spectral radius to HBM, thrust::max_element reduces it and the host
// reads the maximum back (src/calc_dt.cu:18-62), then Block3d::solve clamps dt
// to t_end and advances t_cur (src/Block3d.cpp:239-247).  Here the per-node
// spectral radius is reduced with warp shuffles into one 64-bit atomic max
// (inside the stage-3 and boundary kernels during a step, or by sigma_nodes
// below at start-up), and step_prologue forms dt, applies the clamp and the
// finish test and zeroes the accumulator for the next step, so whole steps
// replay from a CUDA graph without a host round trip.
#include "step.cuh"

namespace cbns {

namespace {

__global__ void sigma_nodes(const SigmaArgs a) {
  const Dims& d = a.d;
  const long N = (long)d.IM * d.JM * d.KM;
  const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
  double sg = 0.0;
  bool has = false;
  if (e < N) {
    const int i = (int)(e % d.IM);
    const long r = e / d.IM;
    const int j = (int)(r % d.JM), k = (int)(r / d.JM);
    const long o = node_off(d, i, j, k);
    double rr, uu, vv, ww, pp;
    if (a.viscous) {
      rr = a.prim[0][o];
      uu = a.prim[1][o];
      vv = a.prim[2][o];
      ww = a.prim[3][o];
      pp = a.prim[4][o];
    } else {
      const long V = d.VOL;
      rr = a.q[o];
      uu = a.q[V + o] / rr;
      vv = a.q[2 * V + o] / rr;
      ww = a.q[3 * V + o] / rr;
      pp = a.gam1 * (a.q[4 * V + o] - 0.5 * rr * (uu * uu + vv * vv + ww * ww));
    }
    const double c = sqrt(a.gamma * pp / rr);
    double fv = 0.0;
    if (a.viscous)
      fv = a.dt_full ? 2.0 * a.mu[o] * a.C_dt_v / rr
                     : 2.0 * a.mu[o] * a.C_dt_v * sqrt(uu * uu + vv * vv + ww * ww) / c / rr;
    double s = 0.0;
#pragma unroll
    for (int dd = 0; dd < 3; ++dd) {
      const double mx = a.met[3 * dd][o], my = a.met[3 * dd + 1][o], mz = a.met[3 * dd + 2][o];
      const double na = sqrt(mx * mx + my * my + mz * mz);
      double t = fabs(uu * mx + vv * my + ww * mz) + c * na;
      if (a.viscous) t += na * na * fv;
      s += t;
    }
    sg = s;
    has = true;
  }
  const bool nan = has && (sg != sg);
  double m = (has && !nan) ? sg : 0.0;
  const unsigned anyhas = __ballot_sync(0xffffffffu, has);
  const unsigned anynan = __ballot_sync(0xffffffffu, nan);
#pragma unroll
  for (int s = 16; s > 0; s >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, s));
  if ((threadIdx.x & 31) == 0 && anyhas)
    atomic_max_sigma(&a.st->sigma_bits, anynan ? __longlong_as_double(0x7ff8000000000000ll) : m);
}

// One thread: the host-side prologue of a time step of Block3d::solve.
__device__ __forceinline__ void prologue_body(StepState* st, double CFL) {
  if (st->done) return;
  const double t_cur = st->t_cur, t_end = st->t_end;
  if (t_cur + 1.0e-8 > t_end) {  // is_finished (src/Block3d.cpp:476-488)
    st->done = 1;
    return;
  }
  const double smax = __longlong_as_double((long long)st->sigma_bits);
  double dt = CFL / smax;
  if (dt != dt) {  // calc_dt throws on NaN (src/calc_dt.cu:56-58)
    st->nan_dt = 1;
    st->done = 1;
    return;
  }
  if (t_end - t_cur < dt) dt = t_end - t_cur;
  st->dt = dt;
  st->t_cur = t_cur + dt;
  st->sigma_bits = 0ull;  // stage 3 of this step accumulates the next maximum
  st->force_weno = 0;     // the hybrid's audit decides afresh for every step
  st->steps += 1;
}

__global__ void step_prologue(StepState* st, double CFL) { prologue_body(st, CFL); }

// The prologues of many blocks, one thread each.
__global__ void step_prologue_batched(StepState* const* st, const double* CFL, int n) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b < n) prologue_body(st[b], CFL[b]);
}

// The per-call path's dt for the stages that follow; new_step (stage 1) also
// counts the step, as step_prologue does (restart: the count starts over), so
// the audit's rotating sample advances as in a run.
__global__ void set_dt_kernel(StepState* st, double dt, int new_step, int restart) {
  st->dt = dt;
  st->done = 0;
  if (restart) st->steps = 0;
  if (new_step) st->steps += 1;
}

}  // namespace

cudaError_t launch_sigma_nodes(const SigmaArgs& a, cudaStream_t s) {
  const long N = (long)a.d.IM * a.d.JM * a.d.KM;
  cudaError_t e = cudaMemsetAsync(&a.st->sigma_bits, 0, sizeof(unsigned long long), s);
  if (e != cudaSuccess) return e;
  sigma_nodes<<<(unsigned)((N + 255) / 256), 256, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_step_prologue(StepState* st, double CFL, cudaStream_t s) {
  step_prologue<<<1, 1, 0, s>>>(st, CFL);
  return cudaGetLastError();
}

cudaError_t launch_step_prologue_batched(StepState* const* st, const double* CFL, int n, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  step_prologue_batched<<<(n + 63) / 64, 64, 0, s>>>(st, CFL, n);
  return cudaGetLastError();
}

cudaError_t launch_set_dt(StepState* st, double dt, bool new_step, bool restart, cudaStream_t s) {
  set_dt_kernel<<<1, 1, 0, s>>>(st, dt, new_step, restart);
  return cudaGetLastError();
}

}  // namespace cbns
