// abi.cu - the extern "C" entry points declared in include/cbns_b200.h.
//
// State buffers.  The reference keeps two conservative arrays, Q and Q_p, and
// updates Q_p in place in stage 2 (src/runge_kutta_kernel.cu:72-73), which a
// fused stencil+update kernel cannot do.  The context therefore owns three
// physical buffers and maps the reference's logical Q and Q_p (and a spare) onto
// them; a stage whose output would overwrite its own stencil source writes the
// spare and the two roles swap.  Cells that no kernel ever writes (far-field
// ghosts held at their initial values) are identical in all three buffers
// because every state upload or initialisation fills all three.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <utility>
#include <vector>

#include "../../include/cbns_b200.h"
#include "bc.cuh"
#include "cbns_common.cuh"
#include "setup.cuh"
#include "stage.cuh"
#include "step.cuh"
#include "tma.cuh"
#include "visc.cuh"
#include "sensor_kernels.cuh"

using namespace cbns;

namespace cbns {
cudaError_t launch_mlp_predict_tc(const float* P, const float* X, unsigned n, float* out, int* fail, cudaStream_t s);
}

namespace cbns {
void stage_prepare();
}

enum { PK_STAGE = 0, PK_BC = 1, PK_VISC = 2, PK_STEP = 3, PK_SENSOR = 4, PK_AUDIT = 5, PK_WENO = 6, PK_N = 7 };

struct cbns_ctx {
  cbns_params prm;
  Phys ph;
  Dims d;
  cudaStream_t own = nullptr, stream = nullptr;
  double* qb[3] = {nullptr, nullptr, nullptr};
  int lq = 0, lp = 1, ls = 2;  // physical index of logical Q, Q_p, spare
  Fields f;
  double* staging = nullptr;
  size_t staging_elems = 0;
  StepState* st = nullptr;
  unsigned* counter = nullptr;  // device counter for face sampling
  bool have_metrics = false, sigma_valid = false;
  bool sigma_pending = false;  // per-call path: stage 3 accumulated the interior spectral radii
  unsigned percall_hold = 0;   // per-call path: steps the current decisions still hold
  bool percall_restart = true; // per-call path: the next stage 1 starts a new sequence of steps
  int prims_of = -1;     // physical buffer whose interior primitives the arrays hold
  int pending_src = -1;  // buffer given to calc_numerical_flux, consumed by update_rk3
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  // bumped whenever a captured step of this context goes stale (a setting its
  // kernels were captured with changed): a batch holding it captures anew
  unsigned long long graph_gen = 0;
  int g_q = -1, g_p = -1, g_s = -1;
  int ntile_i = 1, ntile_j = 1, kchunk = 1;
  int stage_variant = 0;  // compiled variant of the stage kernel (set in cbns_create, cbns_autotune)
  int nsm = 148;          // SMs of the device
  StageMaps tm[3];        // FP32 precisions: TMA maps of the stage kernel, per state buffer
  // hybrid flux: the learned sensor's parameters and per-face decisions
  float* sensor_params = nullptr;  // device, CBNS_SENSOR_NPARAM floats
  unsigned char* mask = nullptr;   // device, one byte per face: the decisions the fluxes use
  unsigned char* mask_raw = nullptr;  // device: the network's decisions before widening
  float* wflux = nullptr;  // device, 8 floats per face: WENO5 fluxes of the stage's WENO5 faces
  int2* wlist = nullptr;   // device, up to one entry per face: the step's WENO5 faces
  long nfaces = 0;
  float sensor_tau = 0.5f;
  unsigned audit_stride = 97;
  unsigned sensor_every = 3;  // network evaluated every n-th step of cbns_run
  float audit_bound = 1.0e-2f;
  bool sensor_loaded = false;
  bool prof = false;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev[PK_N];
  std::vector<cudaEvent_t> ev_pool;
  unsigned long long launches = 0;
  int launches_per_step = 0;
  std::vector<void*> allocs;
};

namespace {

thread_local std::string g_last;

#define CK(call)                                                                    \
  do {                                                                              \
    cudaError_t e_ = (call);                                                        \
    if (e_ != cudaSuccess) {                                                        \
      g_last = std::string(#call) + ": " + cudaGetErrorString(e_);                  \
      return CBNS_ERR_CUDA;                                                         \
    }                                                                               \
  } while (0)

}  // namespace

namespace cbns {
// The last error text of this thread, for entry points in other files.
void set_last_error(const char* what, cudaError_t e) { g_last = std::string(what) + ": " + cudaGetErrorString(e); }
}  // namespace cbns

namespace {

int dalloc(cbns_ctx* c, double** p, size_t elems) {
  void* q = nullptr;
  if (cudaMalloc(&q, elems * sizeof(double)) != cudaSuccess) {
    cudaGetLastError();
    g_last = "device allocation failed";
    return CBNS_ERR_NOMEM;
  }
  c->allocs.push_back(q);
  *p = static_cast<double*>(q);
  return CBNS_OK;
}

inline long round_up(long x, long m) { return (x + m - 1) / m * m; }

// k planes per CTA of the stage kernel.  The CTAs (tiles x k chunks) run in
// waves of `slots` (SMs x CTAs per SM); a chunk costs its planes plus some
// warm-up (the ring's first planes and the first k-face), `warm` planes'
// worth.  The chunk count whose waves x (planes + warm) is least, keeping
// chunks of at least 8 planes.
int kchunk_by_waves(int ntiles, int nint, int slots, double warm) {
  const int maxchunk = std::max(1, nint / 8);
  double best = 1e300;
  int best_k = nint;
  for (int nchunk = 1; nchunk <= maxchunk; ++nchunk) {
    const int kc = (nint + nchunk - 1) / nchunk;
    const long items = (long)ntiles * ((nint + kc - 1) / kc);
    const long waves = (items + slots - 1) / slots;
    const double cost = (double)waves * (kc + warm);
    if (cost < best - 1e-9) {
      best = cost;
      best_k = kc;
    }
  }
  return best_k;
}

// The chunk for about `waves` waves of `slots` CTAs, chunks of at least 8 planes.
// Many short waves balance CTAs of unequal cost (tiles cut by the grid's edge,
// WENO5 faces gathered unevenly): on a 256 x 256 x 128 grid the FP64 kernel
// runs fastest at about 9 waves (13-plane chunks), 3.5% faster than at 4.6
// waves (26-plane chunks) and 10% faster than in one wave.
int kchunk_for_waves(int ntiles, int nint, int slots, double waves) {
  const int want = (int)std::ceil(waves * slots / ntiles);
  const int nchunk = std::max(1, std::min(want, nint / 8));
  return (nint + nchunk - 1) / nchunk;
}

// The default: about four CTAs per slot of 2 CTAs per SM, chunks of at least 8 planes.
int kchunk_default(int ntiles, int nint, int nsm) {
  const int nchunk = std::max(1, std::min((4 * 2 * nsm + ntiles - 1) / ntiles, nint / 8));
  return (nint + nchunk - 1) / nchunk;
}

// Candidate chunkings for cbns_autotune at `per_sm` CTAs per SM (distinct values).
std::vector<int> kchunk_candidates(const cbns_ctx* c, int per_sm) {
  const int ntiles = c->ntile_i * c->ntile_j, nint = c->d.KM - 2, slots = c->nsm * per_sm;
  std::vector<int> v = {kchunk_default(ntiles, nint, c->nsm)};
  auto add = [&v](int kc) {
    if (std::find(v.begin(), v.end(), kc) == v.end()) v.push_back(kc);
  };
  for (double warm : {0.5, 2.0}) add(kchunk_by_waves(ntiles, nint, slots, warm));
  for (double waves : {4.0, 6.0, 9.0, 12.0}) add(kchunk_for_waves(ntiles, nint, slots, waves));
  return v;
}

cudaEvent_t take_event(cbns_ctx* c) {
  cudaEvent_t e;
  if (!c->ev_pool.empty()) {
    e = c->ev_pool.back();
    c->ev_pool.pop_back();
  } else {
    cudaEventCreate(&e);
  }
  return e;
}

// wraps one group of launches with timing events when profiling is on
struct Prof {
  cbns_ctx* c;
  int id;
  cudaEvent_t a = nullptr;
  Prof(cbns_ctx* c_, int id_) : c(c_), id(id_) {
    if (c->prof) {
      a = take_event(c);
      cudaEventRecord(a, c->stream);
    }
  }
  ~Prof() {
    if (c->prof) {
      cudaEvent_t b = take_event(c);
      cudaEventRecord(b, c->stream);
      c->ev[id].push_back({a, b});
    }
  }
};

double* buf(cbns_ctx* c, int logical) { return c->qb[logical == CBNS_QP ? c->lp : c->lq]; }
int phys(cbns_ctx* c, int logical) { return logical == CBNS_QP ? c->lp : c->lq; }

void fill_met(const cbns_ctx* c, const double* out[10]) {
  for (int m = 0; m < 10; ++m) out[m] = c->f.met[m];
}

BCArgs bc_args(cbns_ctx* c, double* q, bool check_done, bool sigma) {
  BCArgs a;
  a.d = c->d;
  a.gamma = c->ph.gamma;
  a.gam1 = c->ph.gam1;
  a.gM2 = c->ph.gM2;
  a.p_inf = c->ph.p_inf;
  a.i_begin = c->ph.i_begin;
  a.i_end = c->ph.i_end;
  a.viscous = c->ph.viscous;
  a.q = q;
  fill_met(c, a.met);
  for (int m = 0; m < 6; ++m) a.prim[m] = c->f.prim[m];
  a.st = c->st;
  a.check_done = check_done;
  a.sigma = sigma;
  a.farfield = c->prm.bc_mode == CBNS_BC_FARFIELD || c->prm.bc_mode == CBNS_BC_CHARACTERISTIC;
  a.characteristic = c->prm.bc_mode == CBNS_BC_CHARACTERISTIC;
  a.wrap = c->prm.bc_mode == CBNS_BC_OGRID ? CBNS_OGRID_WRAP : 0;
  const double aoa = c->ph.angle_attack * 3.14159265358979323846 / 180.0;
  a.u_inf = std::cos(aoa);
  a.v_inf = std::sin(aoa);
  return a;
}

ViscArgs visc_args(cbns_ctx* c, bool check_done, bool sigma) {
  ViscArgs a;
  a.d = c->d;
  a.gamma = c->ph.gamma;
  a.Re_inv = c->ph.Re_inv;
  a.C_T_inf = c->ph.C_T_inf;
  a.C_dt_v = c->ph.C_dt_v;
  a.dt_full = c->prm.dt_viscous == CBNS_DTV_FULL;
  a.qc = -c->ph.Pr_inv * c->ph.gam1_inv / c->ph.Mach2;
  for (int m = 0; m < 6; ++m) a.prim[m] = c->f.prim[m];
  fill_met(c, a.met);
  for (int m = 0; m < 12; ++m) a.vflux[m] = c->f.vflux[m];
  for (int m = 0; m < 4; ++m) a.dfv[m] = c->f.dfv[m];
  a.f32 = c->ph.precision != CBNS_PREC_FP64;
  a.visdiv = c->ph.visdiv;
  a.mu = c->f.prim[6];
  a.st = c->st;
  a.check_done = check_done;
  a.sigma = sigma;
  a.kc = visc_kchunk(c->d, c->nsm);
  return a;
}

StageArgs stage_args(cbns_ctx* c, const double* src, const double* q0, const double* qp, double* out, bool sigma) {
  StageArgs a;
  a.d = c->d;
  a.gamma = c->ph.gamma;
  a.gam1 = c->ph.gam1;
  a.gam1_inv = c->ph.gam1_inv;
  a.gM2 = c->ph.gM2;
  a.src = src;
  a.q0 = q0;
  a.qp = qp;
  a.out = out;
  fill_met(c, a.met);
  for (int m = 0; m < 10; ++m) a.area[m] = c->f.area[m];
  for (int m = 0; m < 4; ++m) a.dfv[m] = c->f.dfv[m];
  for (int m = 0; m < 6; ++m) a.prim[m] = c->f.prim[m];
  a.st = c->st;
  a.q0_is_src = q0 == src;
  a.qp_is_src = qp == src;
  a.ntile_i = c->ntile_i;
  a.ntile_j = c->ntile_j;
  a.kchunk = c->kchunk;
  a.visdiv = c->ph.visdiv;
  a.sigma = sigma;
  a.mask = c->ph.precision == CBNS_PREC_HYBRID ? c->mask : nullptr;
  a.wflux = c->wflux;
  a.tm = c->tm[0];  // src is always one of the three state buffers
  for (int b = 0; b < 3; ++b)
    if (src == c->qb[b]) a.tm = c->tm[b];
  for (int m = 0; m < 6; ++m) a.area32[m] = c->f.area32[m];
  return a;
}

int stage_launch(cbns_ctx* c, const StageArgs& a, int mode) {
  if (a.mask) {
    Prof p(c, PK_WENO);
    CK(launch_weno_faces(a, mode, c->nfaces, c->wlist, c->stream));
    c->launches += 1;
  }
  Prof p(c, PK_STAGE);
  CK(launch_stage(a, mode, c->ph.viscous != 0, c->ph.precision != CBNS_PREC_FP64, c->stage_variant, c->stream));
  c->launches += 1;
  return CBNS_OK;
}

int bc_launch(cbns_ctx* c, const BCArgs& a, bool interior_prims) {
  Prof p(c, PK_BC);
  int n = 0;
  CK(launch_bc(a, interior_prims, c->stream, &n));
  c->launches += n;
  return CBNS_OK;
}

int visc_launch(cbns_ctx* c, const ViscArgs& a) {
  Prof p(c, PK_VISC);
  CK(launch_visc(a, c->stream));
  c->launches += 2;  // node fluxes, their divergence
  return CBNS_OK;
}

int sigma_launch(cbns_ctx* c) {
  SigmaArgs a;
  a.d = c->d;
  a.gamma = c->ph.gamma;
  a.gam1 = c->ph.gam1;
  a.C_dt_v = c->ph.C_dt_v;
  a.dt_full = c->prm.dt_viscous == CBNS_DTV_FULL;
  a.viscous = c->ph.viscous;
  a.q = c->qb[c->lq];
  for (int m = 0; m < 6; ++m) a.prim[m] = c->f.prim[m];
  a.mu = c->f.prim[6];
  fill_met(c, a.met);
  a.st = c->st;
  Prof p(c, PK_STEP);
  CK(launch_sigma_nodes(a, c->stream));
  c->launches += 1;
  return CBNS_OK;
}

#define RET(x)                 \
  do {                         \
    int r_ = (x);              \
    if (r_ != CBNS_OK) return r_; \
  } while (0)

int sync(cbns_ctx* c) {
  CK(cudaStreamSynchronize(c->stream));
  return CBNS_OK;
}

// Copy the logical Q buffer into the other two (set_conservative / calc_conservative
// copy Q into Q_p, src/set_conservative.cu, src/calc_conservative.cu:39).
int replicate_q(cbns_ctx* c) {
  const size_t bytes = (size_t)NEQ * c->d.VOL * sizeof(double);
  for (int b = 0; b < 3; ++b)
    if (b != c->lq) CK(cudaMemcpyAsync(c->qb[b], c->qb[c->lq], bytes, cudaMemcpyDeviceToDevice, c->stream));
  return CBNS_OK;
}

void drop_graph(cbns_ctx* c) {
  if (c->gexec) cudaGraphExecDestroy(c->gexec);
  if (c->graph) cudaGraphDestroy(c->graph);
  c->gexec = nullptr;
  c->graph = nullptr;
  ++c->graph_gen;
}

// The arguments of one context's sensor kernels (sensor_launch, and the
// batched launches of a batch).
struct SensorSet {
  MaskArgs m;
  DilateArgs w[3];  // widening in i, j, k: raw -> mask -> raw -> mask
  AuditArgs au;
  ListArgs li;
};

SensorSet sensor_set(cbns_ctx* c, const double* q, bool check_done, bool every_step, unsigned widen, bool hold) {
  const unsigned every = every_step ? 1u : c->sensor_every;
  const unsigned wn = widen ? widen : every;
  SensorSet ss;
  MaskArgs& m = ss.m;
  m.d = c->d;
  m.gamma = (float)c->ph.gamma;
  m.gam1 = (float)c->ph.gam1;
  m.q = q;
  for (int k = 0; k < 10; ++k) m.area[k] = c->f.area[k];
  m.params = c->sensor_params;
  m.tau = c->sensor_tau;
  m.every = every;
  m.mask = c->mask_raw;
  m.st = c->st;
  m.check_done = check_done;
  unsigned char* bufs[4] = {c->mask_raw, c->mask, c->mask_raw, c->mask};
  for (int dim = 0; dim < 3; ++dim) {
    DilateArgs& w = ss.w[dim];
    w.d = c->d;
    w.in = bufs[dim];
    w.out = bufs[dim + 1];
    w.dim = dim;
    w.along = 1 + (int)wn;
    w.across = (int)wn;
    w.st = c->st;
    w.count = dim == 2;
    w.every = every;
    w.hold = hold;
    w.check_done = check_done;
  }
  AuditArgs& a = ss.au;
  a.d = c->d;
  a.gamma = (float)c->ph.gamma;
  a.gam1 = (float)c->ph.gam1;
  a.gam1_inv = (float)c->ph.gam1_inv;
  a.q = q;
  for (int k = 0; k < 10; ++k) a.area[k] = c->f.area[k];
  a.mask = c->mask;
  a.stride = c->audit_stride;
  a.bound = c->audit_bound;
  a.st = c->st;
  a.check_done = check_done;
  ListArgs& l = ss.li;
  l.d = c->d;
  l.mask = c->mask;
  l.nf = c->nfaces;
  l.st = c->st;
  l.list = c->wlist;
  l.check_done = check_done;
  l.every = every;
  return ss;
}

// The hybrid flux's decisions for the state q: the sensor network on every
// face (tensor cores), then the audit of a rotating sample of its linear-flux
// faces against WENO5 (which forces WENO5 for the step on a violation).
// every_step: evaluate the network now instead of on every sensor_every-th
// step of a run; widen: widening interval (0: that of the evaluation
// schedule).  hold: the per-call path's steps between evaluations — only the
// audit and the WENO5-face count run, the decisions (and their list) stand.
int sensor_launch(cbns_ctx* c, const double* q, bool check_done, bool every_step = false, unsigned widen = 0,
                  bool hold = false) {
  const SensorSet ss = sensor_set(c, q, check_done, every_step, widen, hold);
  int n = 0;
  {
    Prof p(c, PK_SENSOR);
    if (!hold) {
      CK(launch_sensor_mask(ss.m, c->stream));
      n += 2;
    }
    // widening (held: the count only)
    for (int dim = hold ? 2 : 0; dim < 3; ++dim) {
      CK(launch_sensor_dilate(ss.w[dim], c->stream));
      n += 1;
    }
  }
  {
    Prof p(c, PK_AUDIT);
    CK(launch_sensor_audit(ss.au, c->stream));
  }
  n += 1;
  if (!hold) {
    Prof p(c, PK_WENO);
    CK(launch_weno_list(c->d, c->mask, c->nfaces, c->st, c->wlist, check_done, ss.m.every, c->stream));
    n += 1;
  }
  c->launches += n;  // sensor sweeps, widening passes, the audit, the WENO5-face list
  return CBNS_OK;
}

bool hybrid(const cbns_ctx* c) { return c->ph.precision == CBNS_PREC_HYBRID; }
bool ogrid(const cbns_ctx* c) { return c->prm.bc_mode == CBNS_BC_OGRID; }

// One SSP-RK3 step on the fixed buffer roles P0 = Q, P1 = spare, P2 = Q_p.
int enqueue_step(cbns_ctx* c) {
  const bool visc = c->ph.viscous != 0;
  double* P0 = c->qb[c->lq];
  double* P1 = c->qb[c->ls];
  double* P2 = c->qb[c->lp];
  {
    Prof p(c, PK_STEP);
    CK(launch_step_prologue(c->st, c->ph.CFL, c->stream));
    c->launches += 1;
  }
  if (hybrid(c)) RET(sensor_launch(c, P0, true));
  struct S {
    const double *src, *q0, *qp;
    double* out;
  } s[3] = {{P0, P0, P0, P1}, {P1, P0, P1, P2}, {P2, P0, P2, P0}};
  for (int k = 0; k < 3; ++k) {
    const bool last = k == 2;
    // O-grid: the wrap copy rewrites nodes stage 3 updated, so the spectral
    // radius is swept after the boundary pass
    const bool fuse = last && !visc && !ogrid(c);
    RET(stage_launch(c, stage_args(c, s[k].src, s[k].q0, s[k].qp, s[k].out, fuse), k + 1));
    // no boundary pass in the step for a viscous far-field block: its
    // boundary and ghost nodes hold their Q, so their primitives (formed at
    // the start of the run) stand, the stage kernel recovering the interior
    // primitives and the viscous node kernel the spectral radii
    if (!(visc && c->prm.bc_mode == CBNS_BC_FARFIELD)) RET(bc_launch(c, bc_args(c, s[k].out, true, fuse), false));
    if (last && !visc && ogrid(c)) RET(sigma_launch(c));
    if (visc) RET(visc_launch(c, visc_args(c, true, last)));
  }
  return CBNS_OK;
}

// A stage kernel whose TMA wait ran out left the state invalid.
int stage_status(const StepState& h) {
  if (!h.stage_fail) return CBNS_OK;
  g_last = "a stage kernel's TMA wait timed out; the state is not valid";
  return CBNS_ERR_CUDA;
}

int check_ready(cbns_ctx* c) {
  if (!c) return CBNS_ERR_ARG;
  if (!c->have_metrics) {
    g_last = "metrics have not been computed (cbns_calc_metrics)";
    return CBNS_ERR_STATE;
  }
  return CBNS_OK;
}

// check_ready plus, for the flux evaluations of a hybrid context, the sensor.
int check_flux_ready(cbns_ctx* c) {
  RET(check_ready(c));
  if (hybrid(c) && !c->sensor_loaded) {
    g_last = "the hybrid flux needs the sensor network (cbns_sensor_load)";
    return CBNS_ERR_STATE;
  }
  return CBNS_OK;
}

// Start of a run: the step counter, finish and NaN flags reset, t_end set,
// and the spectral-radius maximum of the current state available.
int run_prepare(cbns_ctx* c, double t_end) {
  RET(check_flux_ready(c));
  StepState h;
  CK(cudaMemcpyAsync(&h, c->st, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
  RET(sync(c));
  h.t_end = t_end;
  h.done = 0;
  h.nan_dt = 0;
  h.steps = 0;
  CK(cudaMemcpyAsync(c->st, &h, sizeof(h), cudaMemcpyHostToDevice, c->stream));
  // viscous far field: the steps leave the boundary primitives as they are
  // (enqueue_step); form them here from the state the run starts from
  if (c->ph.viscous && c->prm.bc_mode == CBNS_BC_FARFIELD) RET(bc_launch(c, bc_args(c, c->qb[c->lq], false, false), false));
  RET(sync(c));
  if (!c->sigma_valid) {
    RET(sigma_launch(c));
    c->sigma_valid = true;
  }
  return CBNS_OK;
}

}  // namespace

// ---------------------------------------------------------------- batches
struct cbns_batch {
  std::vector<cbns_ctx*> blk;
  cudaStream_t stream = nullptr;           // the caller's, or owned by the batch
  bool own_stream = false;
  std::vector<cudaStream_t> saved;         // the blocks' streams before the batch
  // the blocks' own kernels (the sensor sweeps, widening, audit and WENO5-face
  // lists; boundary and viscous kernels unless every block is far field) are
  // captured on side streams, so the graph runs different blocks' small
  // kernels side by side between the batched launches
  std::vector<cudaStream_t> side;
  cudaEvent_t ev_fork = nullptr;
  std::vector<cudaEvent_t> ev_join;
  bool visc = false, fp32 = false, hyb = false;
  StageArgs* args = nullptr;  // device: 3 stages x nblocks
  std::vector<StageArgs> host_args;  // the same, on the host (hybrid: the WENO5-face passes)
  int* start = nullptr;       // device: nblocks + 1
  unsigned* counter = nullptr;
  int total = 0;
  // batched per-block kernels: the step prologues, and (every block in
  // CBNS_BC_FARFIELD) the far-field boundary and viscous node kernels of all
  // blocks in one launch per stage; device tables, block b owning CTAs
  // cta[b] .. cta[b+1]-1
  bool farfield = false;
  void* tables = nullptr;            // one allocation holding the tables below
  StepState** st_tab = nullptr;      // nblocks
  double* cfl_tab = nullptr;         // nblocks
  BCArgs* bc_tab = nullptr;          // 3 stages x nblocks
  ViscArgs* visc_tab = nullptr;      // 3 stages x nblocks
  int* bc_cta = nullptr;             // nblocks + 1
  int* visc_cta = nullptr;           // nblocks + 1
  int* div_cta = nullptr;            // nblocks + 1 (the divergence kernel's CTAs)
  int bc_total = 0, visc_total = 0, div_total = 0;
  // hybrid, every block with the same network: the sensor sweeps, widening
  // passes, audits and WENO5-face lists of all blocks in one launch each
  bool sensor_batched = false;
  void* stables = nullptr;           // one allocation holding the tables below
  MaskArgs* mask_tab = nullptr;      // nblocks
  DilateArgs* dil_tab = nullptr;     // 3 passes x nblocks
  AuditArgs* aud_tab = nullptr;      // nblocks
  ListArgs* list_tab = nullptr;      // nblocks
  int* dil_cta = nullptr;            // 3 passes x (nblocks + 1)
  int* aud_cta = nullptr;            // nblocks + 1
  int* list_cta = nullptr;           // nblocks + 1
  long* ipre = nullptr;              // 2 x (nblocks + 1): sweep work items of the two kinds
  int dil_total[3] = {0, 0, 0}, aud_total = 0, list_total = 0;
  long items_total[2] = {0, 0};
  std::vector<int> roles;     // (lq, lp, ls) per block at capture
  std::vector<unsigned long long> gens;  // the blocks' graph_gen at capture
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
};

namespace {

void batch_release_side(cbns_batch* b) {
  for (cudaStream_t s : b->side) cudaStreamDestroy(s);
  for (cudaEvent_t ev : b->ev_join) cudaEventDestroy(ev);
  if (b->ev_fork) cudaEventDestroy(b->ev_fork);
  b->side.clear();
  b->ev_join.clear();
  b->ev_fork = nullptr;
}

void batch_drop_graph(cbns_batch* b) {
  if (b->gexec) cudaGraphExecDestroy(b->gexec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->gexec = nullptr;
  b->graph = nullptr;
}

// Hybrid batches whose blocks all carry the same network: the tables of the
// batched sensor launches (for the fixed buffer roles, as batch_tables).
// Otherwise the blocks' sensor kernels stay per block, on the side streams.
int batch_sensor_tables(cbns_batch* b) {
  const int nb = (int)b->blk.size();
  b->sensor_batched = false;
  if (!b->hyb) return CBNS_OK;
  std::vector<float> p0(CBNS_SENSOR_NPARAM), pi(CBNS_SENSOR_NPARAM);
  CK(cudaDeviceSynchronize());  // the blocks' weight uploads, on whatever streams they were issued
  for (int i = 0; i < nb; ++i) {
    if (!b->blk[i]->sensor_params) return CBNS_OK;
    CK(cudaMemcpy(i ? pi.data() : p0.data(), b->blk[i]->sensor_params, CBNS_SENSOR_NPARAM * sizeof(float),
                  cudaMemcpyDeviceToHost));
    if (i && std::memcmp(p0.data(), pi.data(), CBNS_SENSOR_NPARAM * sizeof(float)) != 0) return CBNS_OK;
  }
  if (!b->stables) {
    auto up = [](size_t x) { return (x + 255) / 256 * 256; };
    const size_t o1 = up(nb * sizeof(MaskArgs)), o2 = o1 + up(3 * nb * sizeof(DilateArgs)),
                 o3 = o2 + up(nb * sizeof(AuditArgs)), o4 = o3 + up(nb * sizeof(ListArgs)),
                 o5 = o4 + up(3 * (nb + 1) * sizeof(int)), o6 = o5 + up((nb + 1) * sizeof(int)),
                 o7 = o6 + up((nb + 1) * sizeof(int)), o8 = o7 + up(2 * (nb + 1) * sizeof(long));
    CK(cudaMalloc(&b->stables, o8));
    char* t = static_cast<char*>(b->stables);
    b->mask_tab = reinterpret_cast<MaskArgs*>(t);
    b->dil_tab = reinterpret_cast<DilateArgs*>(t + o1);
    b->aud_tab = reinterpret_cast<AuditArgs*>(t + o2);
    b->list_tab = reinterpret_cast<ListArgs*>(t + o3);
    b->dil_cta = reinterpret_cast<int*>(t + o4);
    b->aud_cta = reinterpret_cast<int*>(t + o5);
    b->list_cta = reinterpret_cast<int*>(t + o6);
    b->ipre = reinterpret_cast<long*>(t + o7);
  }
  std::vector<MaskArgs> mt(nb);
  std::vector<DilateArgs> dt(3 * nb);
  std::vector<AuditArgs> at(nb);
  std::vector<ListArgs> lt(nb);
  std::vector<int> dc(3 * (nb + 1), 0), ac(nb + 1, 0), lc(nb + 1, 0);
  std::vector<long> ip(2 * (nb + 1), 0);
  for (int i = 0; i < nb; ++i) {
    cbns_ctx* c = b->blk[i];
    const SensorSet ss = sensor_set(c, c->qb[c->lq], true, false, 0, false);
    mt[i] = ss.m;
    for (int dim = 0; dim < 3; ++dim) dt[dim * nb + i] = ss.w[dim];
    at[i] = ss.au;
    lt[i] = ss.li;
    for (int dim = 0; dim < 3; ++dim)
      dc[dim * (nb + 1) + i + 1] = dc[dim * (nb + 1) + i] + sensor_dilate_ctas(c->d, dim);
    ac[i + 1] = ac[i] + sensor_audit_ctas(ss.au);
    lc[i + 1] = lc[i] + weno_list_ctas(c->d);
    long n0, n1;
    sensor_mask_items(c->d, &n0, &n1);
    ip[i + 1] = ip[i] + n0;
    ip[nb + 1 + i + 1] = ip[nb + 1 + i] + n1;
  }
  for (int dim = 0; dim < 3; ++dim) b->dil_total[dim] = dc[dim * (nb + 1) + nb];
  b->aud_total = ac[nb];
  b->list_total = lc[nb];
  b->items_total[0] = ip[nb];
  b->items_total[1] = ip[2 * nb + 1];
  CK(cudaMemcpyAsync(b->mask_tab, mt.data(), nb * sizeof(MaskArgs), cudaMemcpyHostToDevice, b->stream));
  CK(cudaMemcpyAsync(b->dil_tab, dt.data(), 3 * nb * sizeof(DilateArgs), cudaMemcpyHostToDevice, b->stream));
  CK(cudaMemcpyAsync(b->aud_tab, at.data(), nb * sizeof(AuditArgs), cudaMemcpyHostToDevice, b->stream));
  CK(cudaMemcpyAsync(b->list_tab, lt.data(), nb * sizeof(ListArgs), cudaMemcpyHostToDevice, b->stream));
  CK(cudaMemcpyAsync(b->dil_cta, dc.data(), 3 * (nb + 1) * sizeof(int), cudaMemcpyHostToDevice, b->stream));
  CK(cudaMemcpyAsync(b->aud_cta, ac.data(), (nb + 1) * sizeof(int), cudaMemcpyHostToDevice, b->stream));
  CK(cudaMemcpyAsync(b->list_cta, lc.data(), (nb + 1) * sizeof(int), cudaMemcpyHostToDevice, b->stream));
  CK(cudaMemcpyAsync(b->ipre, ip.data(), 2 * (nb + 1) * sizeof(long), cudaMemcpyHostToDevice, b->stream));
  b->sensor_batched = true;
  return CBNS_OK;
}

// The StageArgs of the three stages of every block for the fixed buffer roles
// P0 = Q, P1 = spare, P2 = Q_p (as enqueue_step), uploaded to the device.
// k planes per work item of a batch's stage launches: measured on the
// 64-block workload (16 planes: 11.31 ms per step, 32: 11.33, whole columns:
// 11.66, the blocks' own chunks of about 9 planes: 11.54)
constexpr int kBatchKChunk = 16;

int batch_tables(cbns_batch* b) {
  const int nb = (int)b->blk.size();
  std::vector<StageArgs> tab(3 * nb);
  std::vector<int> start(nb + 1, 0);
  b->roles.clear();
  for (int i = 0; i < nb; ++i) {
    cbns_ctx* c = b->blk[i];
    double* P0 = c->qb[c->lq];
    double* P1 = c->qb[c->ls];
    double* P2 = c->qb[c->lp];
    tab[0 * nb + i] = stage_args(c, P0, P0, P0, P1, false);
    tab[1 * nb + i] = stage_args(c, P1, P0, P1, P2, false);
    tab[2 * nb + i] = stage_args(c, P2, P0, P2, P0, !b->visc);
    // the batch's own chunking: its work queue balances the blocks' items, so
    // chunks of up to kBatchKChunk planes instead of each block's (sized for
    // the block alone on the whole GPU)
    const int kc = std::min(c->d.KM - 2, kBatchKChunk);
    for (int r = 0; r < 3; ++r) tab[r * nb + i].kchunk = kc;
    start[i + 1] = start[i] + c->ntile_i * c->ntile_j * ((c->d.KM - 2 + kc - 1) / kc);
    b->roles.insert(b->roles.end(), {c->lq, c->lp, c->ls});
  }
  b->total = start[nb];
  b->host_args = tab;
  CK(cudaMemcpyAsync(b->args, tab.data(), tab.size() * sizeof(StageArgs), cudaMemcpyHostToDevice, b->stream));
  CK(cudaMemcpyAsync(b->start, start.data(), start.size() * sizeof(int), cudaMemcpyHostToDevice, b->stream));
  // the batched per-block kernels' tables
  std::vector<StepState*> sts(nb);
  std::vector<double> cfl(nb);
  std::vector<BCArgs> bct(3 * nb);
  std::vector<ViscArgs> vt(3 * nb);
  std::vector<int> bcc(nb + 1, 0), vc(nb + 1, 0), dc(nb + 1, 0);
  for (int i = 0; i < nb; ++i) {
    cbns_ctx* c = b->blk[i];
    sts[i] = c->st;
    cfl[i] = c->ph.CFL;
    for (int k = 0; k < 3; ++k) {
      double* out = k == 0 ? c->qb[c->ls] : (k == 1 ? c->qb[c->lp] : c->qb[c->lq]);
      bct[k * nb + i] = bc_args(c, out, true, k == 2 && !b->visc);
      if (b->visc) vt[k * nb + i] = visc_args(c, true, k == 2);
    }
    bcc[i + 1] = bcc[i] + bc_farfield_ctas(c->d);
    vc[i + 1] = vc[i] + (b->visc ? visc_ctas(vt[i]) : 0);
    dc[i + 1] = dc[i] + (b->visc ? visc_div_ctas(c->d) : 0);
  }
  b->bc_total = bcc[nb];
  b->visc_total = vc[nb];
  b->div_total = dc[nb];
  CK(cudaMemcpyAsync(b->st_tab, sts.data(), nb * sizeof(StepState*), cudaMemcpyHostToDevice, b->stream));
  CK(cudaMemcpyAsync(b->cfl_tab, cfl.data(), nb * sizeof(double), cudaMemcpyHostToDevice, b->stream));
  CK(cudaMemcpyAsync(b->bc_tab, bct.data(), bct.size() * sizeof(BCArgs), cudaMemcpyHostToDevice, b->stream));
  if (b->visc)
    CK(cudaMemcpyAsync(b->visc_tab, vt.data(), vt.size() * sizeof(ViscArgs), cudaMemcpyHostToDevice, b->stream));
  CK(cudaMemcpyAsync(b->bc_cta, bcc.data(), bcc.size() * sizeof(int), cudaMemcpyHostToDevice, b->stream));
  CK(cudaMemcpyAsync(b->visc_cta, vc.data(), vc.size() * sizeof(int), cudaMemcpyHostToDevice, b->stream));
  CK(cudaMemcpyAsync(b->div_cta, dc.data(), dc.size() * sizeof(int), cudaMemcpyHostToDevice, b->stream));
  RET(batch_sensor_tables(b));
  CK(cudaStreamSynchronize(b->stream));
  return CBNS_OK;
}

// One SSP-RK3 step of every block: per-block prologue (own dt) and sensor,
// then per stage one persistent launch over all blocks' tiles followed by the
// blocks' boundary (and viscous) kernels.
// Side streams: fork them off the batch stream, or join them back into it.
int batch_fork(cbns_batch* b) {
  CK(cudaEventRecord(b->ev_fork, b->stream));
  for (cudaStream_t s : b->side) CK(cudaStreamWaitEvent(s, b->ev_fork, 0));
  return CBNS_OK;
}
int batch_join(cbns_batch* b) {
  for (size_t i = 0; i < b->side.size(); ++i) {
    CK(cudaEventRecord(b->ev_join[i], b->side[i]));
    CK(cudaStreamWaitEvent(b->stream, b->ev_join[i], 0));
  }
  return CBNS_OK;
}

// Block i's own kernels go on side stream i mod S while the step is captured.
struct SideStreams {
  cbns_batch* b;
  explicit SideStreams(cbns_batch* bb) : b(bb) {
    for (size_t i = 0; i < b->blk.size(); ++i) b->blk[i]->stream = b->side[i % b->side.size()];
  }
  ~SideStreams() {
    for (cbns_ctx* c : b->blk) c->stream = b->stream;
  }
};

int batch_enqueue_body(cbns_batch* b) {
  const int nb = (int)b->blk.size();
  // every block's prologue (own dt) in one launch
  CK(launch_step_prologue_batched(b->st_tab, b->cfl_tab, nb, b->stream));
  b->blk[0]->launches += 1;
  bool forked = false;
  if (b->hyb && b->sensor_batched) {
    // every block's decisions: sweeps, widening, audit, WENO5-face list
    CK(launch_sensor_mask_batched(b->mask_tab, b->ipre, b->ipre + nb + 1, b->items_total[0], b->items_total[1], nb,
                                  b->stream));
    for (int dim = 0; dim < 3; ++dim)
      CK(launch_sensor_dilate_batched(b->dil_tab + dim * nb, b->dil_cta + dim * (nb + 1), nb, b->dil_total[dim],
                                      b->stream));
    CK(launch_sensor_audit_batched(b->aud_tab, b->aud_cta, nb, b->aud_total, b->stream));
    CK(launch_weno_list_batched(b->list_tab, b->list_cta, nb, b->list_total, b->stream));
    b->blk[0]->launches += 8;
  } else if (b->hyb) {
    RET(batch_fork(b));
    forked = true;
    for (int i = 0; i < nb; ++i) {
      cbns_ctx* c = b->blk[i];
      RET(sensor_launch(c, c->qb[c->lq], true));
    }
  }
  for (int k = 0; k < 3; ++k) {
    const bool last = k == 2;
    if (forked) {
      RET(batch_join(b));
      forked = false;
    }
    if (b->hyb) {
      // the blocks' WENO5-face passes side by side on the side streams: one
      // launch over every block's list (tiles of one block per CTA, the
      // StageArgs staged in shared memory) measured 1.9% slower per step
      RET(batch_fork(b));
      for (int i = 0; i < nb; ++i) {
        CK(launch_weno_faces(b->host_args[k * nb + i], k + 1, b->blk[i]->nfaces, b->blk[i]->wlist,
                             b->blk[i]->stream));
        b->blk[i]->launches += 1;
      }
      RET(batch_join(b));
    }
    CK(cudaMemsetAsync(b->counter, 0, sizeof(unsigned), b->stream));
    BatchStage bs;
    bs.args = b->args + k * nb;
    bs.start = b->start;
    bs.nblocks = nb;
    bs.total = b->total;
    bs.counter = b->counter;
    CK(launch_stage_batched(bs, k + 1, b->visc, b->fp32, b->hyb, b->stream));
    b->blk[0]->launches += 1;
    if (b->farfield) {
      // inviscid: all blocks' boundary spectral radii in stage 3 (a viscous
      // far-field block's boundary primitives stand, see enqueue_step); then
      // all blocks' viscous node fluxes
      if (!b->visc && last) {
        CK(launch_bc_farfield_batched(b->bc_tab + k * nb, b->bc_cta, nb, b->bc_total, b->stream));
        b->blk[0]->launches += 1;
      }
      if (b->visc) {
        CK(launch_visc_batched(b->visc_tab + k * nb, b->visc_cta, nb, b->visc_total, b->div_cta, b->div_total,
                               b->fp32, b->stream));
        b->blk[0]->launches += 2;
      }
      continue;
    }
    RET(batch_fork(b));
    forked = true;
    for (cbns_ctx* c : b->blk) {
      double* out = k == 0 ? c->qb[c->ls] : (k == 1 ? c->qb[c->lp] : c->qb[c->lq]);
      RET(bc_launch(c, bc_args(c, out, true, last && !b->visc), false));
      if (b->visc) RET(visc_launch(c, visc_args(c, true, last)));
    }
  }
  if (forked) RET(batch_join(b));
  return CBNS_OK;
}

// One SSP-RK3 step of every block, captured: the blocks' own kernels on the
// side streams, the batched stage launches on the batch stream.
int batch_enqueue_step(cbns_batch* b) {
  SideStreams guard(b);
  return batch_enqueue_body(b);
}

int batch_run(cbns_batch* b, unsigned nsteps, double t_end, bool wait, unsigned* steps_min) {
  if (!b) return CBNS_ERR_ARG;
  for (cbns_ctx* c : b->blk) {
    c->percall_hold = 0;  // a run's decisions follow its own schedule
    c->percall_restart = true;
    c->sigma_pending = false;
  }
  for (cbns_ctx* c : b->blk) RET(run_prepare(c, t_end));
  bool stale = !b->gexec;
  for (size_t i = 0; i < b->blk.size() && !stale; ++i) {
    const cbns_ctx* c = b->blk[i];
    stale = b->roles[3 * i] != c->lq || b->roles[3 * i + 1] != c->lp || b->roles[3 * i + 2] != c->ls ||
            b->gens[i] != c->graph_gen;
  }
  if (stale) {
    batch_drop_graph(b);
    RET(batch_tables(b));
    b->gens.clear();
    for (const cbns_ctx* c : b->blk) b->gens.push_back(c->graph_gen);
    std::vector<unsigned long long> l0;
    for (cbns_ctx* c : b->blk) l0.push_back(c->launches);
    CK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    const int rc = batch_enqueue_step(b);
    cudaGraph_t g = nullptr;
    const cudaError_t ee = cudaStreamEndCapture(b->stream, &g);
    for (size_t i = 0; i < b->blk.size(); ++i) {
      b->blk[i]->launches_per_step = (int)(b->blk[i]->launches - l0[i]);
      b->blk[i]->launches = l0[i];
    }
    if (rc != CBNS_OK) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    CK(ee);
    b->graph = g;
    CK(cudaGraphInstantiate(&b->gexec, g, 0));
  }
  for (unsigned n = 0; n < nsteps; ++n) {
    CK(cudaGraphLaunch(b->gexec, b->stream));
    for (cbns_ctx* c : b->blk) c->launches += c->launches_per_step;
  }
  for (cbns_ctx* c : b->blk)
    if (c->ph.viscous) c->prims_of = c->lq;
  if (!wait) return CBNS_OK;
  CK(cudaStreamSynchronize(b->stream));
  unsigned mn = ~0u;
  bool nan = false;
  for (cbns_ctx* c : b->blk) {
    StepState h;
    CK(cudaMemcpy(&h, c->st, sizeof(h), cudaMemcpyDeviceToHost));
    RET(stage_status(h));
    mn = std::min(mn, h.steps);
    if (h.nan_dt) {
      nan = true;
      c->sigma_valid = false;
    }
  }
  if (steps_min) *steps_min = mn;
  return nan ? CBNS_ERR_NAN_DT : CBNS_OK;
}

}  // namespace

extern "C" {

const char* cbns_status_string(int status) {
  switch (status) {
    case CBNS_OK: return "ok";
    case CBNS_ERR_ARG: return "bad argument";
    case CBNS_ERR_CUDA: return g_last.empty() ? "CUDA error" : g_last.c_str();
    case CBNS_ERR_NAN_DT: return "An error occurred while calculating the time step.";
    case CBNS_ERR_STATE: return g_last.empty() ? "call out of order" : g_last.c_str();
    case CBNS_ERR_UNSUPPORTED: return "unsupported option";
    case CBNS_ERR_NOMEM: return "device allocation failed";
    case CBNS_ERR_TOO_LARGE: return "size beyond the entry point's fixed limit";
    default: return "unknown status";
  }
}

int cbns_create(const cbns_params* p, cbns_ctx** out) {
  if (!p || !out) return CBNS_ERR_ARG;
  *out = nullptr;
  if (p->IM < 4 || p->JM < 4 || p->KM < 4) return CBNS_ERR_ARG;
  if (p->viscous != 0 && p->viscous != 1) return CBNS_ERR_ARG;
  if (p->precision < CBNS_PREC_FP64 || p->precision > CBNS_PREC_HYBRID) return CBNS_ERR_ARG;
  if (p->vis_divergence != CBNS_VISDIV_REFERENCE && p->vis_divergence != CBNS_VISDIV_CENTERED) return CBNS_ERR_ARG;
  if (p->bc_mode < CBNS_BC_REFERENCE || p->bc_mode > CBNS_BC_OGRID) return CBNS_ERR_ARG;
  if (p->bc_mode == CBNS_BC_OGRID && p->IM - 2 * CBNS_OGRID_WRAP < 6) {
    g_last = "an O-grid block needs IM - 2*CBNS_OGRID_WRAP >= 6";
    return CBNS_ERR_ARG;
  }
  if (p->dt_viscous != CBNS_DTV_REFERENCE && p->dt_viscous != CBNS_DTV_FULL) return CBNS_ERR_ARG;
  for (int r : p->reserved)
    if (r != 0) return CBNS_ERR_ARG;
  const double ng = ((double)p->IM + 4) * ((double)p->JM + 4) * ((double)p->KM + 4);
  if (ng * 5 > 2.0e9) return CBNS_ERR_TOO_LARGE;

  cbns_ctx* c = new cbns_ctx();
  c->prm = *p;
  // derived parameters exactly as src/Block3d.cpp:99-113
  Phys& h = c->ph;
  h.gamma = p->gamma;
  h.Mach2 = p->Mach * p->Mach;
  h.Re_inv = 1.0 / p->Re;
  h.Pr_inv = 1.0 / p->Pr;
  h.gam1 = p->gamma - 1.0;
  h.gM2 = p->gamma * h.Mach2;
  h.gam1_inv = 1.0 / h.gam1;
  h.p_inf = 1.0 / h.gM2;
  h.C_T_inf = 110.5 / p->T_inf;
  h.C_dt_v = std::max(4.0 / 3.0, p->gamma * h.Pr_inv) * h.Re_inv;
  h.CFL = p->CFL;
  h.angle_attack = p->angle_attack;
  h.i_begin = p->i_begin;
  h.i_end = p->i_end;
  h.viscous = p->viscous;
  h.visdiv = p->vis_divergence;
  h.precision = p->precision;

  Dims& d = c->d;
  d.IM = (int)p->IM;
  d.JM = (int)p->JM;
  d.KM = (int)p->KM;
  d.IG = d.IM + 2 * NG;
  d.JG = d.JM + 2 * NG;
  d.KG = d.KM + 2 * NG;
  d.PX = round_up(LP + d.IG + 16, 16);  // +16: tiles may read a few nodes past IM+1
  d.PL = d.PX * d.JG;
  d.VOL = round_up(d.PL * (d.KG + 1), 32);  // one spare plane of padding at the end

  int rc = CBNS_OK;
  for (int b = 0; b < 3 && rc == CBNS_OK; ++b) rc = dalloc(c, &c->qb[b], (size_t)NEQ * d.VOL);
  for (int m = 0; m < 10 && rc == CBNS_OK; ++m) rc = dalloc(c, &c->f.met[m], d.VOL);
  {
    // one allocation, components VOL elements apart (one 4-D tensor map covers them)
    double* tmp = nullptr;
    rc = rc == CBNS_OK ? dalloc(c, &tmp, (size_t)10 * d.VOL) : rc;
    if (rc == CBNS_OK)
      for (int m = 0; m < 10; ++m) c->f.area[m] = tmp + (size_t)m * d.VOL;
  }
  for (int m = 0; m < 6; ++m) c->f.area32[m] = nullptr;
  if (p->precision != CBNS_PREC_FP64) {
    // one allocation, components VOL floats apart (one 4-D tensor map covers them)
    double* tmp = nullptr;
    rc = rc == CBNS_OK ? dalloc(c, &tmp, (size_t)3 * d.VOL) : rc;
    if (rc == CBNS_OK)
      for (int m = 0; m < 6; ++m) c->f.area32[m] = reinterpret_cast<float*>(tmp) + (size_t)m * d.VOL;
  }
  for (int m = 0; m < 7 && rc == CBNS_OK; ++m) rc = dalloc(c, &c->f.prim[m], d.VOL);
  for (int m = 0; m < 12; ++m) c->f.vflux[m] = nullptr;
  for (int m = 0; m < 4; ++m) c->f.dfv[m] = nullptr;
  if (p->viscous) {
    for (int m = 0; m < 12 && rc == CBNS_OK; ++m) rc = dalloc(c, &c->f.vflux[m], d.VOL);
    for (int m = 0; m < 4 && rc == CBNS_OK; ++m) rc = dalloc(c, &c->f.dfv[m], d.VOL);
  }
  const long NGt = (long)d.IG * d.JG * d.KG;
  c->staging_elems = (size_t)std::max(5 * NGt, 10L * d.IM * d.JM * d.KM);
  if (rc == CBNS_OK) rc = dalloc(c, &c->staging, c->staging_elems);
  c->nfaces = (long)(d.IM - 1) * (d.JM - 2) * (d.KM - 2) + (long)(d.IM - 2) * (d.JM - 1) * (d.KM - 2) +
              (long)(d.IM - 2) * (d.JM - 2) * (d.KM - 1);
  if (rc == CBNS_OK && p->precision == CBNS_PREC_HYBRID && (c->nfaces >= (1L << 31) || d.VOL >= (1L << 30))) {
    g_last = "the hybrid flux indexes faces with 32-bit integers: grid too large";
    rc = CBNS_ERR_TOO_LARGE;
  }
  if (rc == CBNS_OK && p->precision == CBNS_PREC_HYBRID) {
    double* tmp = nullptr;
    rc = dalloc(c, &tmp, (size_t)(c->nfaces + 7) / 8);
    c->mask = reinterpret_cast<unsigned char*>(tmp);
    if (rc == CBNS_OK) rc = dalloc(c, &tmp, (size_t)(c->nfaces + 7) / 8);
    c->mask_raw = reinterpret_cast<unsigned char*>(tmp);
    if (rc == CBNS_OK) rc = dalloc(c, &tmp, (size_t)c->nfaces * 4);
    c->wflux = reinterpret_cast<float*>(tmp);
    if (rc == CBNS_OK) rc = dalloc(c, &tmp, (size_t)c->nfaces);
    c->wlist = reinterpret_cast<int2*>(tmp);
    if (rc == CBNS_OK) {
      rc = dalloc(c, &tmp, (CBNS_SENSOR_NPARAM + 1) / 2);
      c->sensor_params = reinterpret_cast<float*>(tmp);
    }
  }
  if (rc == CBNS_OK) {
    void* s = nullptr;
    if (cudaMalloc(&s, sizeof(StepState)) != cudaSuccess) rc = CBNS_ERR_NOMEM;
    else {
      c->allocs.push_back(s);
      c->st = static_cast<StepState*>(s);
      cudaMemset(s, 0, sizeof(StepState));
    }
  }
  if (rc == CBNS_OK) {
    void* s = nullptr;
    if (cudaMalloc(&s, 256) != cudaSuccess) rc = CBNS_ERR_NOMEM;
    else {
      c->allocs.push_back(s);
      c->counter = static_cast<unsigned*>(s);
    }
  }
  if (rc == CBNS_OK && cudaStreamCreateWithFlags(&c->own, cudaStreamNonBlocking) != cudaSuccess) rc = CBNS_ERR_CUDA;
  if (rc != CBNS_OK) {
    cbns_destroy(c);
    return rc;
  }
  c->stream = c->own;
  {
    // the stage kernels' TMA boxes (stage.cu), per state buffer
    bool ok = true;
    const bool fp32 = p->precision != CBNS_PREC_FP64;
    for (int b = 0; b < 3; ++b) {
      StageMaps& m = c->tm[b];
      if (fp32) {  // halo boxes of the state, FP32 area vectors
        ok = ok && encode_node_map(&m.q_a, c->qb[b], 8, d.PX, d.JG, d.KG, d.VOL, NEQ, 4, 15, NEQ);
        ok = ok && encode_node_map(&m.q_b, c->qb[b], 8, d.PX, d.JG, d.KG, d.VOL, NEQ, 16, 3, NEQ);
        ok = ok && encode_node_map(&m.xi, c->f.area32[0], 4, d.PX, d.JG, d.KG, d.VOL, 6, 24, 15, 3);
        ok = ok && encode_node_map(&m.eta, c->f.area32[0], 4, d.PX, d.JG, d.KG, d.VOL, 6, 16, 17, 3);
      } else {  // ring column and plane boxes of the state, FP64 area vectors
        ok = ok && encode_node_map(&m.q_a, c->qb[b], 8, d.PX, d.JG, d.KG, d.VOL, NEQ, 16, 15, NEQ);
        ok = ok && encode_node_map(&m.q_b, c->qb[b], 8, d.PX, d.JG, d.KG, d.VOL, NEQ, 24, 21, NEQ);
        ok = ok && encode_node_map(&m.xi, c->f.area[0], 8, d.PX, d.JG, d.KG, d.VOL, 10, 24, 15, 3);
        ok = ok && encode_node_map(&m.eta, c->f.area[0], 8, d.PX, d.JG, d.KG, d.VOL, 10, 16, 17, 3);
      }
    }
    if (!ok) {
      g_last = "cuTensorMapEncodeTiled refused the stage kernel's tensor maps";
      cbns_destroy(c);
      return CBNS_ERR_CUDA;
    }
  }
  // zero everything once so padding never holds NaN garbage
  for (void* a : c->allocs) (void)a;
  for (int b = 0; b < 3; ++b) cudaMemsetAsync(c->qb[b], 0, (size_t)NEQ * d.VOL * sizeof(double), c->stream);
  for (int m = 0; m < 10; ++m) cudaMemsetAsync(c->f.met[m], 0, d.VOL * sizeof(double), c->stream);
  for (int m = 0; m < 10; ++m) cudaMemsetAsync(c->f.area[m], 0, d.VOL * sizeof(double), c->stream);
  for (int m = 0; m < 6; ++m)
    if (c->f.area32[m]) cudaMemsetAsync(c->f.area32[m], 0, d.VOL * sizeof(float), c->stream);
  for (int m = 0; m < 7; ++m) cudaMemsetAsync(c->f.prim[m], 0, d.VOL * sizeof(double), c->stream);
  if (p->viscous) {
    for (int m = 0; m < 12; ++m) cudaMemsetAsync(c->f.vflux[m], 0, d.VOL * sizeof(double), c->stream);
    for (int m = 0; m < 4; ++m) cudaMemsetAsync(c->f.dfv[m], 0, d.VOL * sizeof(double), c->stream);
  }

  stage_tiles(d, &c->ntile_i, &c->ntile_j);
  const int ntiles = c->ntile_i * c->ntile_j;
  const int nint = d.KM - 2;
  {
    int dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaGetLastError();
  }
  // until cbns_autotune says otherwise, the variants and chunks it picks on
  // B200 for grids of a few million nodes: FP64 stages by TMA (about 10%
  // faster than the synchronous variant) and the split precision runs 2 CTAs
  // per SM, both with about 9 waves of CTAs; the hybrid runs 3 per SM (8%
  // faster than 2) with chunks sized by the wave count and warm-up -- where
  // that gives at least two full waves of CTAs; a smaller hybrid grid keeps 2
  // per SM (its CTAs do not fill the GPU, and the 2-per-SM kernel holds more
  // in registers)
  c->stage_variant = p->precision == CBNS_PREC_SPLIT ? 0 : 1;
  c->kchunk = kchunk_for_waves(ntiles, nint, c->nsm * 2, 9.0);
  if (p->precision == CBNS_PREC_HYBRID) {
    const int kc3 = kchunk_by_waves(ntiles, nint, c->nsm * 3, 0.5);
    if ((long)ntiles * ((nint + kc3 - 1) / kc3) >= 2L * 3 * c->nsm) {
      c->kchunk = kc3;
    } else {
      c->stage_variant = 0;
      c->kchunk = kchunk_default(ntiles, nint, c->nsm);
    }
  }
  stage_prepare();
  if (p->precision == CBNS_PREC_HYBRID) (void)weno_prepare();
  if (cudaStreamSynchronize(c->stream) != cudaSuccess || cudaGetLastError() != cudaSuccess) {
    g_last = "context initialisation failed";
    cbns_destroy(c);
    return CBNS_ERR_CUDA;
  }
  *out = c;
  return CBNS_OK;
}

int cbns_destroy(cbns_ctx* c) {
  if (!c) return CBNS_ERR_ARG;
  if (c->stream) cudaStreamSynchronize(c->stream);
  drop_graph(c);
  for (auto& v : c->ev)
    for (auto& pr : v) {
      cudaEventDestroy(pr.first);
      cudaEventDestroy(pr.second);
    }
  for (auto e : c->ev_pool) cudaEventDestroy(e);
  for (void* a : c->allocs) cudaFree(a);
  if (c->own) cudaStreamDestroy(c->own);
  delete c;
  return CBNS_OK;
}

int cbns_set_stream(cbns_ctx* c, void* s) {
  if (!c) return CBNS_ERR_ARG;
  RET(sync(c));
  c->stream = s ? static_cast<cudaStream_t>(s) : c->own;
  drop_graph(c);
  return CBNS_OK;
}

int cbns_calc_metrics(cbns_ctx* c, const double* x, const double* y, const double* z) {
  if (!c || !x || !y || !z) return CBNS_ERR_ARG;
  const size_t N = (size_t)c->d.IM * c->d.JM * c->d.KM;
  double* sx = c->staging;
  CK(cudaMemcpyAsync(sx, x, N * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(sx + N, y, N * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(sx + 2 * N, z, N * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  const int wrap = ogrid(c) ? CBNS_OGRID_WRAP : 0;
  CK(launch_metrics(c->d, sx, sx + N, sx + 2 * N, c->f.met, c->f.area,
                    c->f.area32[0] ? c->f.area32 : nullptr, wrap, c->stream));
  c->launches += wrap ? 4 : 3;
  RET(sync(c));
  c->have_metrics = true;
  c->sigma_valid = false;
  c->sigma_pending = false;
  c->percall_hold = 0;  // a new state: the next per-call step evaluates the network
  c->percall_restart = true;
  return CBNS_OK;
}

int cbns_get_metrics(cbns_ctx* c, double* xi_x, double* xi_y, double* xi_z, double* eta_x, double* eta_y,
                     double* eta_z, double* zeta_x, double* zeta_y, double* zeta_z, double* Jac) {
  RET(check_ready(c));
  double* outs[10] = {xi_x, xi_y, xi_z, eta_x, eta_y, eta_z, zeta_x, zeta_y, zeta_z, Jac};
  const size_t N = (size_t)c->d.IM * c->d.JM * c->d.KM;
  for (int m = 0; m < 10; ++m) {
    if (!outs[m]) return CBNS_ERR_ARG;
    CK(launch_gather_nodes(c->d, c->f.met[m], c->staging, c->stream));
    c->launches += 1;
    CK(cudaMemcpyAsync(outs[m], c->staging, N * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    RET(sync(c));
  }
  return CBNS_OK;
}

int cbns_initial_condition(cbns_ctx* c) {
  if (!c) return CBNS_ERR_ARG;
  CK(launch_ic(c->d, c->f.prim, c->ph.angle_attack, c->ph.p_inf, c->ph.viscous, c->stream));
  c->launches += 1;
  c->prims_of = -1;
  return CBNS_OK;  // stream-ordered: the host-reading calls wait
}

int cbns_calc_conservative(cbns_ctx* c, int which) {
  if (!c || (which != CBNS_Q && which != CBNS_QP)) return CBNS_ERR_ARG;
  CK(launch_conservative(c->d, c->f.prim, buf(c, which), c->ph.gam1, c->stream));
  c->launches += 1;
  RET(replicate_q(c));
  c->sigma_valid = false;
  c->sigma_pending = false;
  c->percall_hold = 0;  // a new state: the next per-call step evaluates the network
  c->percall_restart = true;
  c->prims_of = -1;
  return CBNS_OK;  // stream-ordered: the host-reading calls wait
}

int cbns_set_conservative(cbns_ctx* c, const double* Q) {
  if (!c || !Q) return CBNS_ERR_ARG;
  const size_t n = (size_t)NEQ * c->d.IG * c->d.JG * c->d.KG;
  CK(cudaMemcpyAsync(c->staging, Q, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(launch_aos_to_soa(c->d, c->staging, c->qb[c->lq], c->stream));
  c->launches += 1;
  RET(replicate_q(c));
  c->sigma_valid = false;
  c->sigma_pending = false;
  c->percall_hold = 0;  // a new state: the next per-call step evaluates the network
  c->percall_restart = true;
  c->prims_of = -1;
  return sync(c);
}

int cbns_init_case(cbns_ctx* c, int kind, const double* x, const double* y, const double* z, const double* prm,
                   unsigned nprm) {
  if (!c || !x || !y || !z || (nprm > 0 && !prm) || nprm > 8) return CBNS_ERR_ARG;
  if (kind != CBNS_CASE_VORTEX && kind != CBNS_CASE_BLAST && kind != CBNS_CASE_SHOCK_VORTEX) return CBNS_ERR_ARG;
  const size_t N = (size_t)c->d.IM * c->d.JM * c->d.KM;
  double* sx = c->staging;
  CK(cudaMemcpyAsync(sx, x, N * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(sx + N, y, N * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(sx + 2 * N, z, N * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(launch_case_ic(c->d, sx, sx + N, sx + 2 * N, kind, prm, (int)nprm, c->ph.gamma, c->qb[c->lq], c->stream));
  c->launches += 1;
  RET(replicate_q(c));
  c->sigma_valid = false;
  c->sigma_pending = false;
  c->percall_hold = 0;  // a new state: the next per-call step evaluates the network
  c->percall_restart = true;
  c->prims_of = -1;
  return sync(c);
}

int cbns_get_conservative(cbns_ctx* c, int which, double* Q) {
  if (!c || !Q || (which != CBNS_Q && which != CBNS_QP)) return CBNS_ERR_ARG;
  const size_t n = (size_t)NEQ * c->d.IG * c->d.JG * c->d.KG;
  CK(launch_soa_to_aos(c->d, buf(c, which), c->staging, c->stream));
  c->launches += 1;
  CK(cudaMemcpyAsync(Q, c->staging, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  return sync(c);
}

int cbns_get_primitive(cbns_ctx* c, double* rho, double* u, double* v, double* w, double* p, double* T) {
  if (!c || !rho || !u || !v || !w || !p) return CBNS_ERR_ARG;
  if (!c->ph.viscous) {
    // inviscid runs keep no primitive arrays: recover them from Q
    CK(launch_primitive(c->d, c->qb[c->lq], c->f.prim, c->ph.gam1, c->ph.gM2, c->stream));
    c->launches += 1;
  }
  double* outs[6] = {rho, u, v, w, p, T};
  const size_t n = (size_t)c->d.IG * c->d.JG * c->d.KG;
  for (int m = 0; m < 6; ++m) {
    if (!outs[m]) continue;
    CK(launch_gather_ghosted(c->d, c->f.prim[m], c->staging, c->stream));
    c->launches += 1;
    CK(cudaMemcpyAsync(outs[m], c->staging, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    RET(sync(c));
  }
  return CBNS_OK;
}

int cbns_calc_primitive(cbns_ctx* c, int which) {
  if (!c || (which != CBNS_Q && which != CBNS_QP)) return CBNS_ERR_ARG;
  CK(launch_primitive(c->d, buf(c, which), c->f.prim, c->ph.gam1, c->ph.gM2, c->stream));
  c->launches += 1;
  c->prims_of = phys(c, which);
  return CBNS_OK;  // stream-ordered: the host-reading calls wait
}

int cbns_set_bc_calc_primitive(cbns_ctx* c, int which) {
  RET(check_ready(c));
  if (which != CBNS_Q && which != CBNS_QP) return CBNS_ERR_ARG;
  const int pb = phys(c, which);
  const bool interior = c->ph.viscous && c->prims_of != pb;
  // after an inviscid stage 3: add the boundary nodes to its spectral radii
  const bool sigma = c->sigma_pending && which == CBNS_Q && !c->ph.viscous;
  RET(bc_launch(c, bc_args(c, c->qb[pb], false, sigma), interior));
  if (c->ph.viscous) c->prims_of = pb;
  c->sigma_valid = sigma;
  c->sigma_pending = false;
  return CBNS_OK;  // stream-ordered: the host-reading calls wait
}

int cbns_calc_numerical_flux(cbns_ctx* c, int which) {
  RET(check_flux_ready(c));
  if (which != CBNS_Q && which != CBNS_QP) return CBNS_ERR_ARG;
  // the fluxes are formed inside the stage kernel launched by cbns_update_rk3
  c->pending_src = which;
  return CBNS_OK;
}

int cbns_calc_viscous_flux_contribution(cbns_ctx* c) {
  RET(check_ready(c));
  // the node fluxes and their divergence were formed by cbns_calc_viscous_terms
  // (visc.cu); the stage kernel subtracts the divergence
  return CBNS_OK;
}

int cbns_calc_viscous_terms(cbns_ctx* c) {
  RET(check_ready(c));
  if (!c->ph.viscous) return CBNS_OK;  // the inviscid build compiles this to nothing
  RET(visc_launch(c, visc_args(c, false, false)));
  return CBNS_OK;  // stream-ordered: the host-reading calls wait
}

int cbns_update_rk3(cbns_ctx* c, double dt, unsigned stage) {
  RET(check_flux_ready(c));
  if (stage < 1 || stage > 3) return CBNS_ERR_ARG;
  const int src_l = c->pending_src >= 0 ? c->pending_src : (stage == 1 ? CBNS_Q : CBNS_QP);
  c->pending_src = -1;
  const int src = phys(c, src_l);
  int out = stage == 3 ? c->lq : c->lp;
  const bool swap = out == src;
  if (swap) out = c->ls;
  {
    Prof p(c, PK_STEP);
    CK(launch_set_dt(c->st, dt, stage == 1, stage == 1 && c->percall_restart, c->stream));
    if (stage == 1) c->percall_restart = false;
    c->launches += 1;
  }
  if (hybrid(c) && stage == 1) {
    // the network runs on every sensor_every-th call of a sequence of steps
    // (as in cbns_run), its decisions widened to hold until the next one
    CK(cudaMemsetAsync(&c->st->force_weno, 0, sizeof(int), c->stream));
    const bool hold = c->percall_hold > 0;
    RET(sensor_launch(c, c->qb[src], false, true, c->sensor_every, hold));
    c->percall_hold = hold ? c->percall_hold - 1 : c->sensor_every - 1;
  }
  // inviscid stage 3 accumulates the spectral radius of the interior nodes it
  // updates; set_bc_calc_primitive(Q) adds the boundary nodes, and the next
  // cbns_calc_dt reads the maximum instead of sweeping the grid again
  const bool sigma = stage == 3 && !c->ph.viscous && !ogrid(c);
  if (sigma) CK(cudaMemsetAsync(&c->st->sigma_bits, 0, sizeof(unsigned long long), c->stream));
  const StageArgs a = stage_args(c, c->qb[src], c->qb[c->lq], c->qb[c->lp], c->qb[out], sigma);
  RET(stage_launch(c, a, (int)stage));
  if (swap) {
    if (stage == 3) std::swap(c->lq, c->ls);
    else std::swap(c->lp, c->ls);
  }
  if (c->ph.viscous) c->prims_of = out;
  c->sigma_valid = false;
  c->sigma_pending = sigma;
  return CBNS_OK;  // stream-ordered: the host-reading calls wait
}

int cbns_calc_dt(cbns_ctx* c, double* dt) {
  RET(check_ready(c));
  if (!dt) return CBNS_ERR_ARG;
  if (!c->sigma_valid) RET(sigma_launch(c));
  StepState h;
  CK(cudaMemcpyAsync(&h, c->st, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
  RET(sync(c));
  RET(stage_status(h));
  double smax;
  std::memcpy(&smax, &h.sigma_bits, sizeof(smax));
  *dt = c->ph.CFL / smax;
  c->sigma_valid = true;
  if (std::isnan(*dt)) return CBNS_ERR_NAN_DT;
  return CBNS_OK;
}

int cbns_set_time(cbns_ctx* c, double t_cur) {
  if (!c) return CBNS_ERR_ARG;
  CK(cudaMemcpyAsync(&c->st->t_cur, &t_cur, sizeof(double), cudaMemcpyHostToDevice, c->stream));
  return sync(c);
}

int cbns_get_time(cbns_ctx* c, double* t_cur, double* dt_last) {
  if (!c) return CBNS_ERR_ARG;
  StepState h;
  CK(cudaMemcpyAsync(&h, c->st, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
  RET(sync(c));
  if (t_cur) *t_cur = h.t_cur;
  if (dt_last) *dt_last = h.dt;
  return CBNS_OK;
}

static int run_impl(cbns_ctx* c, unsigned nsteps, double t_end, bool wait, unsigned* steps_done) {
  RET(run_prepare(c, t_end));
  c->percall_hold = 0;  // a run's decisions follow its own schedule
  c->percall_restart = true;
  c->sigma_pending = false;
  if (c->prof) {
    for (unsigned n = 0; n < nsteps; ++n) RET(enqueue_step(c));
  } else {
    if (!c->gexec || c->g_q != c->lq || c->g_p != c->lp || c->g_s != c->ls) {
      drop_graph(c);
      const unsigned long long l0 = c->launches;
      CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
      const int rc = enqueue_step(c);
      cudaGraph_t g = nullptr;
      const cudaError_t ee = cudaStreamEndCapture(c->stream, &g);
      if (rc != CBNS_OK) {
        if (g) cudaGraphDestroy(g);
        return rc;
      }
      CK(ee);
      c->graph = g;
      CK(cudaGraphInstantiate(&c->gexec, g, 0));
      c->launches_per_step = (int)(c->launches - l0);
      c->launches = l0;
      c->g_q = c->lq;
      c->g_p = c->lp;
      c->g_s = c->ls;
    }
    for (unsigned n = 0; n < nsteps; ++n) {
      CK(cudaGraphLaunch(c->gexec, c->stream));
      c->launches += c->launches_per_step;
    }
  }
  if (c->ph.viscous) c->prims_of = c->lq;
  if (!wait) return CBNS_OK;
  StepState h;
  CK(cudaMemcpyAsync(&h, c->st, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
  RET(sync(c));
  if (steps_done) *steps_done = h.steps;
  RET(stage_status(h));
  if (h.nan_dt) {
    c->sigma_valid = false;
    return CBNS_ERR_NAN_DT;
  }
  return CBNS_OK;
}

int cbns_run(cbns_ctx* c, unsigned nsteps, double t_end, unsigned* steps_done) {
  return run_impl(c, nsteps, t_end, true, steps_done);
}

int cbns_run_async(cbns_ctx* c, unsigned nsteps, double t_end) { return run_impl(c, nsteps, t_end, false, nullptr); }

int cbns_eval_rhs(cbns_ctx* c, int which, double* rhs) {
  RET(check_flux_ready(c));
  if (!rhs || (which != CBNS_Q && which != CBNS_QP)) return CBNS_ERR_ARG;
  if (hybrid(c)) {
    CK(cudaMemsetAsync(&c->st->force_weno, 0, sizeof(int), c->stream));
    RET(sensor_launch(c, buf(c, which), false, true));
    c->percall_hold = 0;  // unwidened decisions: the next per-call step evaluates again
  }
  const StageArgs a = stage_args(c, buf(c, which), nullptr, nullptr, c->staging, false);
  RET(stage_launch(c, a, 0));
  const size_t n = (size_t)NEQ * (c->d.IM - 2) * (c->d.JM - 2) * (c->d.KM - 2);
  CK(cudaMemcpyAsync(rhs, c->staging, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  return sync(c);
}

int cbns_sensor_sample(cbns_ctx* c, int which, unsigned stride, unsigned offset, float* feat, unsigned char* label,
                       float* dev, unsigned* index, unsigned capacity, unsigned* count) {
  RET(check_ready(c));
  if ((which != CBNS_Q && which != CBNS_QP) || stride == 0 || offset >= stride || !feat || !label || !count)
    return CBNS_ERR_ARG;
  SampleArgs a;
  a.d = c->d;
  a.gamma = (float)c->ph.gamma;
  a.gam1 = (float)c->ph.gam1;
  a.q = buf(c, which);
  for (int m = 0; m < 10; ++m) a.area[m] = c->f.area[m];
  a.stride = stride;
  a.offset = offset;
  a.feat = feat;
  a.label = label;
  a.dev = dev;
  a.index = index;
  a.capacity = capacity;
  a.count = c->counter;
  CK(cudaMemsetAsync(c->counter, 0, sizeof(unsigned), c->stream));
  CK(launch_sample_faces(a, c->stream));
  c->launches += 1;
  CK(cudaMemcpyAsync(count, c->counter, sizeof(unsigned), cudaMemcpyDeviceToHost, c->stream));
  return sync(c);
}

int cbns_mlp_grad(const float* P, const float* X, const unsigned char* Y, unsigned n, float pos_w, float* G,
                  float* loss, void* stream) {
  if (!P || !G || !loss || (n && (!X || !Y))) return CBNS_ERR_ARG;
  CK(launch_mlp_grad(P, X, Y, n, pos_w, G, loss, static_cast<cudaStream_t>(stream)));
  return CBNS_OK;
}

int cbns_mlp_adam(float* P, const float* G, float* M, float* V, unsigned step, float lr, void* stream) {
  if (!P || !G || !M || !V || step == 0) return CBNS_ERR_ARG;
  CK(launch_adam(P, G, M, V, step, lr, static_cast<cudaStream_t>(stream)));
  return CBNS_OK;
}

int cbns_mlp_predict(const float* P, const float* X, unsigned n, float* out, int use_tc, int* status, void* stream) {
  if (!P || !out || (n && !X)) return CBNS_ERR_ARG;
  if (use_tc) {
    if (!status) return CBNS_ERR_ARG;
    CK(launch_mlp_predict_tc(P, X, n, out, status, static_cast<cudaStream_t>(stream)));
  } else {
    CK(launch_mlp_predict(P, X, n, out, static_cast<cudaStream_t>(stream)));
  }
  return CBNS_OK;
}

int cbns_sensor_load(cbns_ctx* c, const float* params, float tau) {
  if (!c || !params) return CBNS_ERR_ARG;
  if (!hybrid(c)) {
    g_last = "cbns_sensor_load needs a context of precision CBNS_PREC_HYBRID";
    return CBNS_ERR_STATE;
  }
  if (!(tau > 0.f && tau < 1.f)) return CBNS_ERR_ARG;
  for (int k = 0; k < CBNS_SENSOR_NPARAM; ++k)
    if (!std::isfinite(params[k])) return CBNS_ERR_ARG;
  CK(cudaMemcpyAsync(c->sensor_params, params, CBNS_SENSOR_NPARAM * sizeof(float), cudaMemcpyHostToDevice,
                     c->stream));
  c->sensor_tau = tau;
  c->sensor_loaded = true;
  c->percall_hold = 0;
  drop_graph(c);
  return sync(c);
}

int cbns_sensor_load_file(cbns_ctx* c, const char* path) {
  if (!c || !path) return CBNS_ERR_ARG;
  FILE* f = std::fopen(path, "rb");
  if (!f) {
    g_last = "cannot open the sensor weights file";
    return CBNS_ERR_ARG;
  }
  char magic[8];
  unsigned n = 0;
  float tau = 0.f;
  std::vector<float> p(CBNS_SENSOR_NPARAM);
  const bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, "CBNSSNS1", 8) == 0 &&
                  std::fread(&n, 4, 1, f) == 1 && n == CBNS_SENSOR_NPARAM && std::fread(&tau, 4, 1, f) == 1 &&
                  std::fread(p.data(), 4, CBNS_SENSOR_NPARAM, f) == CBNS_SENSOR_NPARAM;
  std::fclose(f);
  if (!ok) {
    g_last = "malformed sensor weights file";
    return CBNS_ERR_ARG;
  }
  return cbns_sensor_load(c, p.data(), tau);
}

int cbns_sensor_audit(cbns_ctx* c, unsigned stride, float bound) {
  if (!c || stride == 0 || !(bound > 0.f)) return CBNS_ERR_ARG;
  c->audit_stride = stride;
  c->audit_bound = bound;
  drop_graph(c);
  return CBNS_OK;
}

int cbns_sensor_interval(cbns_ctx* c, unsigned every) {
  if (!c || every < 1 || every > 8) return CBNS_ERR_ARG;
  c->sensor_every = every;
  c->percall_hold = 0;
  drop_graph(c);
  return CBNS_OK;
}

int cbns_sensor_stats_get(cbns_ctx* c, cbns_sensor_stats* out) {
  if (!c || !out) return CBNS_ERR_ARG;
  StepState h;
  CK(cudaMemcpyAsync(&h, c->st, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
  RET(sync(c));
  out->weno_faces = h.weno_faces;
  out->audit_faces = h.audit_faces;
  out->audit_fail_steps = h.audit_fail_steps;
  out->audit_max = h.audit_max;
  out->sensor_fail = h.sensor_fail;
  out->faces_per_step = (unsigned long long)c->nfaces;
  return CBNS_OK;
}

int cbns_sensor_mask_get(cbns_ctx* c, unsigned char* mask, unsigned long long n, int* forced) {
  if (!c || !mask) return CBNS_ERR_ARG;
  if (!hybrid(c)) return CBNS_ERR_STATE;
  if (n < (unsigned long long)c->nfaces) return CBNS_ERR_ARG;
  CK(cudaMemcpyAsync(mask, c->mask, (size_t)c->nfaces, cudaMemcpyDeviceToHost, c->stream));
  int f = 0;
  CK(cudaMemcpyAsync(&f, &c->st->force_weno, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  RET(sync(c));
  if (forced) *forced = f;
  return CBNS_OK;
}

int cbns_sensor_stats_reset(cbns_ctx* c) {
  if (!c) return CBNS_ERR_ARG;
  StepState h;
  CK(cudaMemcpyAsync(&h, c->st, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
  RET(sync(c));
  h.weno_faces = 0;
  h.audit_faces = 0;
  h.audit_fail_steps = 0;
  h.audit_max = 0.f;
  h.sensor_fail = 0;
  CK(cudaMemcpyAsync(c->st, &h, sizeof(h), cudaMemcpyHostToDevice, c->stream));
  return sync(c);
}

int cbns_autotune(cbns_ctx* c, int* chosen) {
  RET(check_flux_ready(c));
  const bool fp32 = c->ph.precision != CBNS_PREC_FP64;
  const int nv = stage_variants(fp32, hybrid(c));
  // time every variant on the current state (RHS-only mode: nothing is updated);
  // the hybrid kernel is timed on the sensor's decisions for this state
  if (hybrid(c)) {
    CK(cudaMemsetAsync(&c->st->force_weno, 0, sizeof(int), c->stream));
    RET(sensor_launch(c, c->qb[c->lq], false, true));
    c->percall_hold = 0;
  }
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    g_last = "cudaEventCreate failed";
    return CBNS_ERR_CUDA;
  }
  // the faster of two rounds of three RHS launches after one warm-up launch
  auto time_it = [&](int v, int kc, float* ms) -> int {
    c->stage_variant = v;
    c->kchunk = kc;
    const StageArgs a = stage_args(c, c->qb[c->lq], nullptr, nullptr, c->staging, false);
    RET(stage_launch(c, a, 0));
    *ms = 1e30f;
    for (int round = 0; round < 2; ++round) {
      CK(cudaEventRecord(e0, c->stream));
      for (int r = 0; r < 3; ++r) RET(stage_launch(c, a, 0));
      CK(cudaEventRecord(e1, c->stream));
      CK(cudaEventSynchronize(e1));
      float t = 0.f;
      CK(cudaEventElapsedTime(&t, e0, e1));
      *ms = std::min(*ms, t);
    }
    return CBNS_OK;
  };
  // the context's current pair stays unless another is more than 1% faster:
  // the candidates' RHS-only times differ by about that much where their full
  // steps rank the other way
  const int v0 = c->stage_variant, kc0 = c->kchunk;
  int best = v0, best_kc = kc0, rc = CBNS_OK;
  float best_ms = 0.f;
  rc = time_it(v0, kc0, &best_ms);
  for (int v = 0; v < nv && rc == CBNS_OK; ++v) {
    // FP32 variant v runs 2 + v CTAs per SM, the FP64 ones 2; each with its candidate k chunks
    for (int kc : kchunk_candidates(c, fp32 ? 2 + v : 2)) {
      if (v == v0 && kc == kc0) continue;
      float ms = 0.f;
      if ((rc = time_it(v, kc, &ms)) != CBNS_OK) break;
      if (ms < 0.99f * best_ms) {
        best_ms = ms;
        best = v;
        best_kc = kc;
      }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  c->stage_variant = best;
  c->kchunk = best_kc;
  drop_graph(c);
  if (rc != CBNS_OK) return rc;
  if (chosen) *chosen = best;
  return CBNS_OK;
}

int cbns_synchronize(cbns_ctx* c) {
  if (!c) return CBNS_ERR_ARG;
  return sync(c);
}

int cbns_stage_variant(cbns_ctx* c, int variant, int* count) {
  if (!c) return CBNS_ERR_ARG;
  const int nv = stage_variants(c->ph.precision != CBNS_PREC_FP64, hybrid(c));
  if (count) *count = nv;
  if (variant == -1) return CBNS_OK;
  if (variant < 0 || variant >= nv) return CBNS_ERR_ARG;
  if (variant != c->stage_variant) {
    c->stage_variant = variant;
    drop_graph(c);
  }
  return CBNS_OK;
}

int cbns_stage_kchunk(cbns_ctx* c, int kchunk, int* current) {
  if (!c) return CBNS_ERR_ARG;
  if (kchunk != -1) {
    if (kchunk < 1 || kchunk > c->d.KM - 2) return CBNS_ERR_ARG;
    if (kchunk != c->kchunk) {
      c->kchunk = kchunk;
      drop_graph(c);
    }
  }
  if (current) *current = c->kchunk;
  return CBNS_OK;
}

int cbns_calc_gradient(unsigned IM, unsigned JM, unsigned KM, const double* f, double* fx, double* fy, double* fz) {
  if (!f || !fx || !fy || !fz || IM < 2 || JM < 2 || KM < 2) return CBNS_ERR_ARG;
  const size_t N = (size_t)IM * JM * KM;
  double* dbuf = nullptr;
  CK(cudaMalloc(&dbuf, 4 * N * sizeof(double)));
  int rc = CBNS_OK;
  if (cudaMemcpy(dbuf, f, N * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess ||
      launch_gradient_dense((int)IM, (int)JM, (int)KM, dbuf, dbuf + N, dbuf + 2 * N, dbuf + 3 * N, 0) !=
          cudaSuccess ||
      cudaMemcpy(fx, dbuf + N, N * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(fy, dbuf + 2 * N, N * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(fz, dbuf + 3 * N, N * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess) {
    g_last = cudaGetErrorString(cudaGetLastError());
    rc = CBNS_ERR_CUDA;
  }
  cudaFree(dbuf);
  return rc;
}

int cbns_prof_enable(cbns_ctx* c, int on) {
  if (!c) return CBNS_ERR_ARG;
  c->prof = on != 0;
  return CBNS_OK;
}

int cbns_prof_read(cbns_ctx* c, int id, double* total_ms, unsigned* launches) {
  if (!c || id < 0 || id >= PK_N) return CBNS_ERR_ARG;
  RET(sync(c));
  double tot = 0.0;
  for (auto& pr : c->ev[id]) {
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, pr.first, pr.second));
    tot += ms;
  }
  if (total_ms) *total_ms = tot;
  if (launches) *launches = (unsigned)c->ev[id].size();
  return CBNS_OK;
}

int cbns_prof_reset(cbns_ctx* c) {
  if (!c) return CBNS_ERR_ARG;
  RET(sync(c));
  for (auto& v : c->ev) {
    for (auto& pr : v) {
      c->ev_pool.push_back(pr.first);
      c->ev_pool.push_back(pr.second);
    }
    v.clear();
  }
  return CBNS_OK;
}

int cbns_launch_count(cbns_ctx* c, unsigned long long* n) {
  if (!c || !n) return CBNS_ERR_ARG;
  *n = c->launches;
  return CBNS_OK;
}

int cbns_batch_create(cbns_ctx* const* blocks, unsigned nblocks, void* stream, cbns_batch** out) {
  if (!blocks || !out || nblocks == 0) return CBNS_ERR_ARG;
  for (unsigned i = 0; i < nblocks; ++i) {
    if (!blocks[i]) return CBNS_ERR_ARG;
    for (unsigned j = 0; j < i; ++j)
      if (blocks[j] == blocks[i]) return CBNS_ERR_ARG;
    RET(check_flux_ready(blocks[i]));
    if (blocks[i]->ph.viscous != blocks[0]->ph.viscous || blocks[i]->ph.precision != blocks[0]->ph.precision) {
      g_last = "the blocks of a batch share the precision and the viscous flag";
      return CBNS_ERR_ARG;
    }
    if (ogrid(blocks[i])) {
      g_last = "O-grid blocks (CBNS_BC_OGRID) cannot join a batch";
      return CBNS_ERR_ARG;
    }
  }
  cbns_batch* b = new cbns_batch;
  b->blk.assign(blocks, blocks + nblocks);
  b->visc = blocks[0]->ph.viscous != 0;
  b->fp32 = blocks[0]->ph.precision != CBNS_PREC_FP64;
  b->hyb = blocks[0]->ph.precision == CBNS_PREC_HYBRID;
  cudaError_t e = cudaSuccess;
  if (stream) {
    b->stream = static_cast<cudaStream_t>(stream);
  } else {
    e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
      cudaGetLastError();
      delete b;
      g_last = "stream creation failed";
      return CBNS_ERR_CUDA;
    }
    b->own_stream = true;
  }
  // every block works on the batch's stream while the batch exists
  for (cbns_ctx* c : b->blk) {
    b->saved.push_back(c->stream == c->own ? nullptr : c->stream);
    const int rc = cbns_set_stream(c, b->stream);
    if (rc != CBNS_OK) {
      for (size_t i = 0; i + 1 < b->saved.size(); ++i) cbns_set_stream(b->blk[i], b->saved[i]);
      if (b->own_stream) cudaStreamDestroy(b->stream);
      delete b;
      return rc;
    }
  }
  b->farfield = true;
  for (cbns_ctx* c : b->blk) b->farfield = b->farfield && c->prm.bc_mode == CBNS_BC_FARFIELD;
  e = cudaMalloc(&b->args, 3 * nblocks * sizeof(StageArgs));
  if (e == cudaSuccess) e = cudaMalloc(&b->start, (nblocks + 1) * sizeof(int));
  if (e == cudaSuccess) {
    // tables of the batched per-block kernels, each on a 256-byte boundary
    auto up = [](size_t x) { return (x + 255) / 256 * 256; };
    const size_t o1 = up(nblocks * sizeof(StepState*)), o2 = o1 + up(nblocks * sizeof(double)),
                 o3 = o2 + up(3 * nblocks * sizeof(BCArgs)), o4 = o3 + up(3 * nblocks * sizeof(ViscArgs)),
                 o5 = o4 + up((nblocks + 1) * sizeof(int)), o6 = o5 + up((nblocks + 1) * sizeof(int)),
                 o7 = o6 + up((nblocks + 1) * sizeof(int));
    e = cudaMalloc(&b->tables, o7);
    if (e == cudaSuccess) {
      char* t = static_cast<char*>(b->tables);
      b->st_tab = reinterpret_cast<StepState**>(t);
      b->cfl_tab = reinterpret_cast<double*>(t + o1);
      b->bc_tab = reinterpret_cast<BCArgs*>(t + o2);
      b->visc_tab = reinterpret_cast<ViscArgs*>(t + o3);
      b->bc_cta = reinterpret_cast<int*>(t + o4);
      b->visc_cta = reinterpret_cast<int*>(t + o5);
      b->div_cta = reinterpret_cast<int*>(t + o6);
    }
  }
  if (e == cudaSuccess) e = cudaMalloc(&b->counter, sizeof(unsigned));
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming);
  for (unsigned i = 0; i < std::min(nblocks, 16u) && e == cudaSuccess; ++i) {
    cudaStream_t s = nullptr;
    cudaEvent_t ev = nullptr;
    e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (e == cudaSuccess) b->side.push_back(s);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    if (e == cudaSuccess) b->ev_join.push_back(ev);
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    cudaFree(b->args);
    cudaFree(b->start);
    cudaFree(b->counter);
    cudaFree(b->tables);
    batch_release_side(b);
    for (size_t i = 0; i < b->blk.size(); ++i) cbns_set_stream(b->blk[i], b->saved[i]);
    if (b->own_stream) cudaStreamDestroy(b->stream);
    delete b;
    g_last = "device allocation failed";
    return CBNS_ERR_NOMEM;
  }
  *out = b;
  return CBNS_OK;
}

int cbns_batch_destroy(cbns_batch* b) {
  if (!b) return CBNS_ERR_ARG;
  cudaStreamSynchronize(b->stream);
  batch_drop_graph(b);
  // the blocks go back to the streams they had
  for (size_t i = 0; i < b->blk.size(); ++i) cbns_set_stream(b->blk[i], b->saved[i]);
  cudaFree(b->args);
  cudaFree(b->start);
  cudaFree(b->counter);
  cudaFree(b->tables);
  cudaFree(b->stables);
  batch_release_side(b);
  if (b->own_stream) cudaStreamDestroy(b->stream);
  delete b;
  return CBNS_OK;
}

int cbns_batch_run(cbns_batch* b, unsigned nsteps, double t_end, unsigned* steps_min) {
  return batch_run(b, nsteps, t_end, true, steps_min);
}

int cbns_batch_run_async(cbns_batch* b, unsigned nsteps, double t_end) {
  return batch_run(b, nsteps, t_end, false, nullptr);
}

}  // extern "C"
