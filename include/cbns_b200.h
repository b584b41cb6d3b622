/*
 * cbns_b200.h - C ABI of the B200 (sm_100a) implementation of the cbns3d_cuda
 * RK3 right-hand-side path.
 *
 * Every entry point takes plain pointers and sizes and returns an int status
 * (CBNS_OK on success); nothing here calls exit() or throws.  The library owns
 * its device memory (structure-of-arrays, FP64 state), launches on the stream
 * given by cbns_set_stream (default: the legacy default stream) and keeps the
 * reference's synchronous contract: each call below returns after its work is
 * complete on the device unless its comment says otherwise.
 *
 * Reference interface each entry point replaces (paths inside the reference
 * project chenbei102/cbns3d_cuda):
 *   cbns_create                   copy_block_info   include/copy_block_info.h:9
 *                                 + allocate_mem    include/allocate_mem.h:9
 *   cbns_destroy                  free_mem          include/free_mem.h:9
 *   cbns_calc_metrics             calc_metrics      include/calc_metrics.h:9
 *   cbns_get_metrics              get_metrics       include/get_metrics.h:9
 *   cbns_initial_condition        initial_condition include/initial_condition.h:9
 *   cbns_calc_conservative        calc_conservative include/calc_conservative.h:9
 *   cbns_set_conservative         set_conservative  include/set_conservative.h:9
 *   cbns_get_conservative         get_conservative  include/get_conservative.h:9
 *   cbns_get_primitive            get_primitive     include/get_primitive.h:9
 *   cbns_calc_primitive           calc_primitive    include/calc_primitive.h:9-10
 *   cbns_set_bc_calc_primitive    set_bc_calc_primitive include/set_bc_calc_primitive.h:9
 *   cbns_calc_numerical_flux      calc_numerical_flux   include/calc_numerical_flux.h:9
 *   cbns_calc_viscous_terms       calc_viscous_terms    include/calc_viscous_terms.h:9
 *   cbns_calc_viscous_flux_contribution
 *                                 calc_viscous_flux_contribution
 *                                                   include/calc_viscous_flux_contribution.h:9
 *   cbns_update_rk3               update_rk3        include/time_integration.h:9-10
 *   cbns_calc_dt                  calc_dt           include/calc_dt.h:9
 *   cbns_calc_gradient            calc_gradient     include/calc_gradient.h:9
 *   cbns_run                      the time loop of Block3d::solve, src/Block3d.cpp:237-293
 * The remaining entry points (stream, time, timing, RHS evaluation) have no
 * single reference counterpart; their comments say what they are for.
 */
#ifndef CBNS_B200_H_
#define CBNS_B200_H_

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. */
#define CBNS_OK               0
#define CBNS_ERR_ARG          1  /* bad argument (null pointer, bad size, bad enum)    */
#define CBNS_ERR_CUDA         2  /* a CUDA runtime call or kernel launch failed        */
#define CBNS_ERR_NAN_DT       3  /* the CFL time step is NaN (calc_dt.cu:56-58 throws) */
#define CBNS_ERR_STATE        4  /* call out of order (e.g. stepping before metrics)   */
#define CBNS_ERR_UNSUPPORTED  5  /* option not available in this build                 */
#define CBNS_ERR_NOMEM        6  /* device allocation failed                           */
#define CBNS_ERR_TOO_LARGE    7  /* size beyond a fixed limit of the entry point       */

/* Which state buffer a call acts on: the reference passes block_data->Q or
 * block_data->Q_p explicitly (src/Block3d.cpp:249-284). */
#define CBNS_Q   0
#define CBNS_QP  1

/* Arithmetic of the inviscid face flux. */
#define CBNS_PREC_FP64    0  /* plain path, FP64 throughout (parity with the reference) */
#define CBNS_PREC_SPLIT   1  /* FP32 reconstruction + flux, FP64 state/metrics/reductions */
#define CBNS_PREC_HYBRID  2  /* SPLIT + learned shock sensor choosing WENO5 or upwind-5 */

/* Where the viscous flux divergence is evaluated. */
#define CBNS_VISDIV_REFERENCE 0 /* as src/viscous_contribution_kernel.cu:269-288: each
                                   directional derivative taken at the node shifted by -1
                                   in both transverse directions                        */
#define CBNS_VISDIV_CENTERED  1 /* every derivative taken at the node itself           */

/* cbns_params.bc_mode.  REFERENCE: the reference's boundary conditions
 * (src/primitive_bc_kernel.cu:13-494), the parity contract.  FARFIELD (no
 * counterpart in the reference): every boundary and ghost node holds the state
 * it was given by cbns_set_conservative / cbns_calc_conservative — the
 * free-stream far field on all faces that the vortex and batched-block
 * configurations ask for; only their primitives (viscous runs) and spectral
 * radii are recomputed. */
#define CBNS_BC_REFERENCE 0
#define CBNS_BC_FARFIELD  1
/* CHARACTERISTIC (no counterpart in the reference): a characteristic far field
 * on all six faces against the free stream (rho 1, velocity (cos a, sin a, 0)
 * at the angle of attack a, p_inf): per boundary node, Riemann invariants
 * along the outward unit normal from the node one step inward and from the
 * free stream; entropy and tangential velocity from the interior at outflow,
 * from the free stream at inflow; supersonic inflow takes the free stream,
 * supersonic outflow the inward node.  i faces (j, k interior), then j faces
 * (all i, k interior), then k faces (all i, j), each node's two ghosts set to
 * its state; the state depends on the buffer's interior only. */
#define CBNS_BC_CHARACTERISTIC 2
/* OGRID (no counterpart in the reference; the NACA 0012 O-grid configuration):
 * i wraps around, j = 0 is the wall (adiabatic no-slip in viscous runs, slip
 * in inviscid ones, on every i: the reference's wall branch with i_begin = 1,
 * i_end = IM whatever the parameters say), j = JM-1 the characteristic far
 * field above, the k faces the reference's zero-gradient copy.  The block
 * stores the periodic line of P = IM - 2*CBNS_OGRID_WRAP points at
 * i = CBNS_OGRID_WRAP .. IM-CBNS_OGRID_WRAP-1, with CBNS_OGRID_WRAP copies of
 * the points across the seam on either side (i < W holds point i + P,
 * i >= IM - W point i - P; the grid passed to cbns_calc_metrics must hold
 * them).  After every boundary pass those nodes and the i ghosts are copies of
 * the nodes P away (Q and primitives), and their metrics are copies too, so
 * every stencil of a stored point sees the periodic line.  Needs P >= 6.
 * Inviscid runs sweep the spectral radius after the boundary pass instead of
 * fusing it into stage 3; blocks in this mode cannot join a batch. */
#define CBNS_BC_OGRID 3
#define CBNS_OGRID_WRAP 4

/* cbns_params.dt_viscous: the viscous part of the spectral radius behind the
 * CFL time step.  REFERENCE: |grad xi|^2 * 2 mu C_dt_v |u| / (c rho) per
 * direction, as src/time_step_kernel.cu:54 (the local Mach number |u|/c scales
 * it, so it vanishes where the flow is at rest, e.g. at a no-slip wall).
 * FULL (no counterpart in the reference): |grad xi|^2 * 2 mu C_dt_v / rho, the
 * explicit diffusion limit without that factor, which the boundary layer of a
 * wall-resolved grid needs (first cells of 1e-5 chords). */
#define CBNS_DTV_REFERENCE 0
#define CBNS_DTV_FULL      1

/* cbns_init_case kinds (no counterpart in the reference) and their parameters:
 *   VORTEX        Mach, strength beta, centre x, centre y, radius R, stream
 *                 direction (dx, dy): isentropic vortex in a free stream
 *   BLAST         r2_in, p_in, p_out: pressure p_in where x^2+y^2+z^2 < r2_in,
 *                 p_out elsewhere, unit density, at rest
 *   SHOCK_VORTEX  shock Mach Ms, vortex strength eps, radius rc, centre x,
 *                 centre y, shock position x_s: stationary normal shock with a
 *                 vortex in the upstream flow */
#define CBNS_CASE_VORTEX       0
#define CBNS_CASE_BLAST        1
#define CBNS_CASE_SHOCK_VORTEX 2

/* Run parameters: the fields of Block3dInfo that Block3d::read_input fills
 * (src/Block3d.cpp:33-138, include/Block3d_cuda.h:32-78) plus build-time
 * switches of the reference that are run-time options here.  The derived
 * quantities (Mach^2, gamma*M^2, p_inf = 1/(gamma M^2), Sutherland constant
 * 110.5/T_inf, C_dt_v, ...) are computed inside cbns_create exactly as
 * src/Block3d.cpp:99-113 computes them. */
typedef struct cbns_params {
  unsigned IM, JM, KM;      /* grid points per direction (each >= 4)              */
  double   CFL;
  double   angle_attack;    /* degrees                                             */
  unsigned i_begin, i_end;  /* j=0 face: wake cut for i < i_begin-1, wall for
                               i < i_end (unsigned arithmetic, as the reference)   */
  double   Mach, Re, gamma, Pr, Pr_t, T_inf;
  int      viscous;         /* 0: INVIS_MODE=ON build; 1: viscous build            */
  int      precision;       /* CBNS_PREC_*                                         */
  int      vis_divergence;  /* CBNS_VISDIV_*                                       */
  int      bc_mode;         /* CBNS_BC_*                                           */
  int      dt_viscous;      /* CBNS_DTV_*                                          */
  int      reserved[3];     /* must be zero                                        */
} cbns_params;

typedef struct cbns_ctx cbns_ctx;

/* Lifecycle. */
int cbns_create(const cbns_params* params, cbns_ctx** out);
int cbns_destroy(cbns_ctx* ctx);
/* Launch stream for every later call (a cudaStream_t passed as void*). */
int cbns_set_stream(cbns_ctx* ctx, void* stream);
const char* cbns_status_string(int status);

/* Setup and I/O.  Host arrays: x,y,z are IM*JM*KM, i fastest (Plot3D order);
 * Q is the reference's AoS ghosted layout n + 5*(i + IM_G*(j + JM_G*k)) with
 * IM_G = IM+4 etc. (include/Block3d_cuda.h:100-108), i.e. the checkpoint body. */
int cbns_calc_metrics(cbns_ctx* ctx, const double* x, const double* y, const double* z);
int cbns_get_metrics(cbns_ctx* ctx, double* xi_x, double* xi_y, double* xi_z,
                     double* eta_x, double* eta_y, double* eta_z,
                     double* zeta_x, double* zeta_y, double* zeta_z, double* Jac);
int cbns_initial_condition(cbns_ctx* ctx);
int cbns_calc_conservative(cbns_ctx* ctx, int which);
int cbns_set_conservative(cbns_ctx* ctx, const double* Q_host);
/* Initial state of a configuration case (CBNS_CASE_*, nprm <= 8 parameters
 * as listed above) formed on the device from the grid coordinates (host,
 * IM*JM*KM each, as cbns_calc_metrics), the coordinates extended into the
 * ghost layers by odd reflection (k, then j, then i); the state of Q (and
 * Q_p) on the whole ghosted box in the reference's units.  The same as
 * forming it on the host and calling cbns_set_conservative, without the
 * host work or the 5-field upload. */
int cbns_init_case(cbns_ctx* ctx, int kind, const double* x, const double* y, const double* z, const double* prm,
                   unsigned nprm);
int cbns_get_conservative(cbns_ctx* ctx, int which, double* Q_host);
/* Ghosted primitive arrays (IM_G*JM_G*KM_G each); T may be null. */
int cbns_get_primitive(cbns_ctx* ctx, double* rho, double* u, double* v, double* w,
                       double* p, double* T);

/* The RK3 right-hand-side path, one reference entry point each.
 * Calls are stream-ordered on the context's stream: the entry points that only
 * launch device work (cbns_initial_condition, cbns_calc_conservative,
 * cbns_calc_primitive, cbns_set_bc_calc_primitive, cbns_calc_numerical_flux,
 * cbns_calc_viscous_terms, cbns_calc_viscous_flux_contribution,
 * cbns_update_rk3) return once their kernels are enqueued; every call that
 * reads into or from host memory (cbns_calc_dt, cbns_get_*, cbns_set_*,
 * cbns_calc_metrics, ...) waits for the stream first, so a caller sees the
 * results of all earlier calls.  Errors of enqueued kernels surface at the
 * next waiting call.  The block3d_cuda:: shims wait after every call, as the
 * reference does (each of its calls ends with cudaDeviceSynchronize). */
/* Wait for every call enqueued on the context's stream (no counterpart in the
 * reference; the shims' per-call cudaDeviceSynchronize). */
int cbns_synchronize(cbns_ctx* ctx);
int cbns_set_bc_calc_primitive(cbns_ctx* ctx, int which);
int cbns_calc_primitive(cbns_ctx* ctx, int which);
int cbns_calc_numerical_flux(cbns_ctx* ctx, int which);
int cbns_calc_viscous_terms(cbns_ctx* ctx);
int cbns_calc_viscous_flux_contribution(cbns_ctx* ctx);
int cbns_update_rk3(cbns_ctx* ctx, double dt, unsigned stage);
/* dt = CFL / max spectral radius of Q.  After an inviscid stage 3 followed by
 * cbns_set_bc_calc_primitive(CBNS_Q) (the reference's step order) the maximum
 * was accumulated by those two calls and is only read back; otherwise the
 * grid is swept (src/time_step_kernel.cu:13-96). */
int cbns_calc_dt(cbns_ctx* ctx, double* dt);

/* Whole SSP-RK3 steps with the time step kept on the device: per step the CFL
 * dt is formed from the previous step's spectral-radius maximum, clamped to
 * t_end - t_cur, and the loop stops once t_cur + 1e-8 > t_end, as the time
 * loop of src/Block3d.cpp:237-293 does.  Steps are replayed from a CUDA graph.
 * *steps_done (may be null) receives the steps actually taken. */
int cbns_run(cbns_ctx* ctx, unsigned nsteps, double t_end, unsigned* steps_done);
/* Same as cbns_run but returns without synchronising (steps_done unavailable). */
int cbns_run_async(cbns_ctx* ctx, unsigned nsteps, double t_end);
int cbns_set_time(cbns_ctx* ctx, double t_cur);
int cbns_get_time(cbns_ctx* ctx, double* t_cur, double* dt_last);

/* One right-hand-side evaluation for testing: rhs[n + 5*(i + (IM-2)*(j + (JM-2)*k))]
 * = ((E_{i+1/2}-E_{i-1/2}) + (F..) + (G..) - dfv)/J at interior node (i+1,j+1,k+1),
 * the quantity rk3_kernel forms (src/runge_kutta_kernel.cu:45-66).  The buffer's
 * boundary conditions (and viscous terms) must be current.  rhs is a host array. */
int cbns_eval_rhs(cbns_ctx* ctx, int which, double* rhs_host);

/* The 4th-order gradient of a standalone IM*JM*KM field (test helper of the
 * reference, src/calc_gradient.cu:17-51).  All arrays are host arrays. */
int cbns_calc_gradient(unsigned IM, unsigned JM, unsigned KM, const double* f,
                       double* fx, double* fy, double* fz);

/* The same gradient for callers that cannot allocate device memory: hosts
 * whose device memory belongs to their own pool allocator or a fixed budget,
 * and paths that cannot take the device-wide synchronisation of
 * cudaMalloc/cudaFree.  Synchronous, like cbns_calc_gradient.  It calls no
 * allocator; its device working copies live in one fixed array of
 * 4 x CBNS_NOALLOC_MAX_POINTS doubles (8 MiB) that every GPU loading this
 * library holds until the process exits.  IM*JM*KM above
 * CBNS_NOALLOC_MAX_POINTS returns CBNS_ERR_TOO_LARGE.  All calls on a device
 * share that array (it keeps the last call's contents; every element a call
 * reads it first writes), so calls overlapping on the GPU race and must be
 * serialised by the caller.  The first call on each device looks up the
 * array's device address (with that device current).  A CUDA failure returns
 * CBNS_ERR_CUDA with its text in cbns_status_string.  No counterpart in the
 * reference. */
#define CBNS_NOALLOC_MAX_POINTS 262144u
int cbns_calc_gradient_noalloc(unsigned IM, unsigned JM, unsigned KM, const double* f,
                               double* fx, double* fy, double* fz);

/* Self-test of the bounded waits' time-out path (no counterpart in the
 * reference): one GPU thread waits on an mbarrier that no MMA completes (the
 * sensor's tensor-core wait, both of its windows) and on a TMA transaction
 * barrier that no copy completes (the stage kernel's plane wait).
 * *mma_timed_out and *tma_timed_out receive 1 when the wait reported its
 * time-out, as it must; *mma_seconds and *tma_seconds (may be null) how long
 * each took on the GPU's clock.  Nothing faults or stays in flight: the
 * kernel returns and the device stays usable.  Synchronous. */
int cbns_selftest_waits(int* mma_timed_out, int* tma_timed_out, double* mma_seconds, double* tma_seconds);

/* Learned shock sensor (no counterpart in the reference).  A network of
 * CBNS_SENSOR_NIN inputs, two hidden layers of CBNS_SENSOR_NHID ReLU units and
 * one sigmoid output estimates, per grid face, the probability that the face
 * needs the full characteristic WENO5 flux.  Parameters are a float vector of
 * CBNS_SENSOR_NPARAM values: W1[32][15] b1[32] W2[32][32] b2[32] w3[32] b3.
 * Features of a face: the jumps of density, pressure and normal velocity
 * across its 5-point stencil, divided by the face's mean density, pressure and
 * sound speed, each compressed as sign(f) log2(1 + |f| / 0.01).  Faces whose
 * compressed features sum to less than 0.0045 in absolute value (flat
 * stencils) take the linear flux without evaluating the network.  Label: 1 when the WENO5 nonlinear weights of the face's
 * characteristic reconstruction depart from the linear weights by more than
 * 0.05.  Pointers marked _dev are device pointers; stream is a cudaStream_t. */
#define CBNS_SENSOR_NIN    15
#define CBNS_SENSOR_NHID   32
#define CBNS_SENSOR_NPARAM 1601
/* Features, labels (and, where the pointers are not null, the weight
 * deviation and the global face index) of the faces whose global index i
 * satisfies i % stride == offset, from the given state buffer.  Global face
 * index: i-faces, then j-faces, then k-faces, each in the order of the
 * reference's Ep/Fp/Gp arrays (include/Block3d_cuda.h:110-123).  Samples are
 * written in no particular order; at most capacity faces are written and
 * *count gets the number sampled (which may exceed capacity). */
int cbns_sensor_sample(cbns_ctx* ctx, int which, unsigned stride, unsigned offset, float* feat_dev,
                       unsigned char* label_dev, float* dev_dev, unsigned* index_dev, unsigned capacity,
                       unsigned* count);
/* Mean weighted binary cross-entropy over n samples (positive class weight
 * pos_weight) and its gradient with respect to every parameter. */
int cbns_mlp_grad(const float* params_dev, const float* x_dev, const unsigned char* y_dev, unsigned n,
                  float pos_weight, float* grad_dev, float* loss_dev, void* stream);
/* One Adam step (beta1 0.9, beta2 0.999, eps 1e-8) at step number step >= 1. */
int cbns_mlp_adam(float* params_dev, const float* grad_dev, float* m_dev, float* v_dev, unsigned step,
                  float lr, void* stream);
/* Probabilities for n feature vectors: FP32 on the CUDA cores, or BF16 on the
 * tcgen05 tensor cores (use_tensor_cores != 0; *status_dev is set non-zero if
 * a tensor-core wait timed out). */
int cbns_mlp_predict(const float* params_dev, const float* x_dev, unsigned n, float* out_dev,
                     int use_tensor_cores, int* status_dev, void* stream);

/* The hybrid flux (CBNS_PREC_HYBRID).  On every n-th time step
 * (cbns_sensor_interval, default 3) the network is evaluated on every face of
 * the step's starting state on the tensor cores; faces with probability >= tau
 * take the characteristic WENO5 flux -- the faces the network is confident
 * need it and those it is unsure about -- and only the faces it is confident
 * are smooth (p < tau) take the linear upwind-5 flux (same Lax-Friedrichs
 * splitting, component-wise).  The trained weights' tau is the lower edge of
 * that uncertainty band: at most 0.5, with a held-out recall floor of the
 * WENO5-labelled faces (cbns3d_cuda_b200/train_sensor.py).
 * The WENO5 decisions are then widened, per face direction, by 2 faces along
 * the face's own grid line and 1 face in the two other index directions (a
 * discontinuity moves less than a cell per step), and hold for the three
 * stages of the step (see cbns_sensor_interval for runs that evaluate the
 * network every n-th step).  An audit recomputes,
 * on the linear faces whose run of 128 consecutive global face indices r =
 * index / 128 has r % audit_stride equal to step % audit_stride, both
 * fluxes; a relative difference above audit_bound
 * on any of them makes the whole step take WENO5 everywhere.  The audit runs on
 * the step's starting state before its first stage, so a step that would
 * break the bound is taken with WENO5 from the start instead of being taken
 * and reverted (the same state, without the discarded stage work).  A context of
 * precision HYBRID refuses to step (CBNS_ERR_STATE) until cbns_sensor_load.
 * params_host: CBNS_SENSOR_NPARAM floats in host memory. */
int cbns_sensor_load(cbns_ctx* ctx, const float* params_host, float tau);
/* The same from a weights file: 8 bytes "CBNSSNS1", uint32 CBNS_SENSOR_NPARAM,
 * float32 tau, CBNS_SENSOR_NPARAM float32 parameters (little endian), as
 * written by cbns3d_cuda_b200/train_sensor.py.  CBNS_ERR_ARG if the file is
 * missing or malformed. */
int cbns_sensor_load_file(cbns_ctx* ctx, const char* path);
/* Evaluate the network on every n-th step of cbns_run / cbns_run_async (1 <=
 * n <= 8, default 3; the first step of each run always evaluates); in between,
 * the decisions of the last evaluation hold, widened by 1 + n faces along and
 * n faces across (a discontinuity moves less than a cell per step).  The
 * audit runs every step.  The per-call path follows the same schedule over
 * its cbns_update_rk3 stage-1 calls: the first call after a new state
 * (cbns_set_conservative, cbns_calc_conservative, cbns_calc_metrics), a run,
 * cbns_eval_rhs, cbns_autotune, cbns_sensor_load or cbns_sensor_interval
 * evaluates, the next n - 1 hold.  cbns_eval_rhs evaluates on every call,
 * with n = 1 widths. */
int cbns_sensor_interval(cbns_ctx* ctx, unsigned every);
/* audit_stride >= 1 (1 audits every linear face every step); audit_bound > 0
 * (relative to the face's largest flux component).  Defaults 97 and 1e-2. */
int cbns_sensor_audit(cbns_ctx* ctx, unsigned audit_stride, float audit_bound);
/* Counters since the last cbns_sensor_stats_reset: faces that took WENO5
 * (network decisions after widening, summed over steps), faces audited, steps whose decisions the audit
 * rejected, the largest relative difference the audit saw, and a non-zero
 * sensor_fail when a tensor-core wait timed out (the step then took WENO5). */
typedef struct cbns_sensor_stats {
  unsigned long long weno_faces;
  unsigned long long audit_faces;
  unsigned audit_fail_steps;
  float audit_max;
  int sensor_fail;
  unsigned long long faces_per_step;
} cbns_sensor_stats;
int cbns_sensor_stats_get(cbns_ctx* ctx, cbns_sensor_stats* stats);
/* The decisions of the latest sensor evaluation (one byte per face in global
 * face index order, 1 = WENO5) copied to mask_host, which holds n >=
 * faces_per_step bytes; *forced (may be null) = 1 when the audit (or a
 * tensor-core timeout) made that step take WENO5 everywhere. */
int cbns_sensor_mask_get(cbns_ctx* ctx, unsigned char* mask_host, unsigned long long n, int* forced);
int cbns_sensor_stats_reset(cbns_ctx* ctx);

/* Batches (no counterpart in the reference, which holds one block per
 * process): independent blocks, each a context created and initialised as
 * usual (its own grid, parameters, state and, for the hybrid, sensor),
 * advanced together.  Per RK stage one persistent launch of the stage kernel
 * works through a queue of the tiles of every block; each block keeps its own
 * time step (per-block dt) and boundary conditions; a whole step of the
 * batch is one CUDA graph.  The blocks share the precision and the viscous
 * flag; while the batch exists they work on the batch's stream — the
 * caller's `stream` (a cudaStream_t) or, when null, one the batch creates —
 * and go back to their previous streams at cbns_batch_destroy; the batch does
 * not own them (destroy the batch first).  cbns_batch_run advances every block by
 * nsteps steps (or to t_end), *steps_min receiving the fewest steps any block
 * took; CBNS_ERR_NAN_DT if any block's dt became NaN. */
typedef struct cbns_batch cbns_batch;
int cbns_batch_create(cbns_ctx* const* blocks, unsigned nblocks, void* stream, cbns_batch** batch);
int cbns_batch_destroy(cbns_batch* batch);
int cbns_batch_run(cbns_batch* batch, unsigned nsteps, double t_end, unsigned* steps_min);
int cbns_batch_run_async(cbns_batch* batch, unsigned nsteps, double t_end);

/* Pick, by timing on the current state, the fastest compiled variant of the
 * stage kernel for this context's precision and its k chunk (the state is not
 * modified; the current pair stays unless another is more than 1% faster);
 * *chosen (may be null) receives the variant index.  Later steps use it. */
int cbns_autotune(cbns_ctx* ctx, int* chosen);
/* Use compiled variant `variant` of the stage kernel (0 .. count-1; count from
 * *count when not null, variant -1 only queries it).  FP64: 0 stages each
 * plane synchronously, 1 by TMA (the same arithmetic, to the rounding of a
 * separate compilation); FP32:
 * 2 + variant CTAs per SM.  A new context starts on variant 1 (FP64; hybrid
 * grids of at least two waves of 3-per-SM CTAs) or 0 (split, smaller hybrid
 * grids).  No counterpart in the reference. */
int cbns_stage_variant(cbns_ctx* ctx, int variant, int* count);
/* Use k chunks of `kchunk` planes in the stage kernel's work items (one CTA
 * per tile and chunk; 1 .. KM-2, -1 only queries); *current (may be null)
 * receives the chunk in use.  cbns_autotune sets it with the variant.  No
 * counterpart in the reference. */
int cbns_stage_kchunk(cbns_ctx* ctx, int kchunk, int* current);

/* Per-kernel-group device timing with CUDA events on the launch stream.  Group
 * ids: 0 stage (fused sweep + RK update), 1 boundary conditions, 2 viscous
 * (node fluxes and their divergence), 3 dt/step bookkeeping, 4 hybrid sensor
 * network, 5 hybrid audit, 6 hybrid WENO5 faces (the per-step list and the
 * per-stage evaluation).  total_ms is the summed event time; *launches counts
 * the timed groups (one group can be several kernel launches, e.g. the three
 * ordered boundary launches); cbns_launch_count counts kernels. */
int cbns_prof_enable(cbns_ctx* ctx, int on);
int cbns_prof_read(cbns_ctx* ctx, int kernel_id, double* total_ms, unsigned* launches);
int cbns_prof_reset(cbns_ctx* ctx);
/* Number of kernels this context launched since creation (or the last reset). */
int cbns_launch_count(cbns_ctx* ctx, unsigned long long* launches);

#ifdef __cplusplus
}
#endif

#endif /* CBNS_B200_H_ */
