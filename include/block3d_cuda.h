/*
 * block3d_cuda.h - the reference's host-to-device API (namespace block3d_cuda)
 * with its exact names and signatures, implemented over the C ABI of
 * cbns_b200.h.  Host code written against the reference (its Block3d.cpp)
 * compiles against this header and links libcbns_b200.so unchanged.
 *
 * Reference declarations replaced (paths inside chenbei102/cbns3d_cuda):
 *   Block3dInfo, Block3dData          include/Block3d_cuda.h:32-231
 *   copy_block_info                   include/copy_block_info.h:9
 *   allocate_mem / free_mem           include/allocate_mem.h:9, include/free_mem.h:9
 *   calc_metrics / get_metrics        include/calc_metrics.h:9, include/get_metrics.h:9
 *   initial_condition                 include/initial_condition.h:9
 *   calc_conservative                 include/calc_conservative.h:9
 *   set_conservative / get_conservative include/set_conservative.h:9, include/get_conservative.h:9
 *   get_primitive / calc_primitive    include/get_primitive.h:9, include/calc_primitive.h:9-10
 *   set_bc_calc_primitive             include/set_bc_calc_primitive.h:9
 *   calc_numerical_flux               include/calc_numerical_flux.h:9
 *   calc_viscous_terms                include/calc_viscous_terms.h:9
 *   calc_viscous_flux_contribution    include/calc_viscous_flux_contribution.h:9
 *   update_rk3                        include/time_integration.h:9-10
 *   calc_dt                           include/calc_dt.h:9
 *   calc_gradient                     include/calc_gradient.h:9
 *
 * Behaviour kept: every call is synchronous; a failing CUDA call prints
 * "Error: file:line, code:N, reason: ..." and exits with EXIT_FAILURE like the
 * reference's ERROR_CHECK (include/Block3d_cuda.h:19-27); calc_dt throws
 * std::runtime_error on a NaN time step (src/calc_dt.cu:56-58).
 *
 * Differences a caller can see:
 *   - Block3dData's device arrays are owned by an opaque context; Q and Q_p are
 *     handles that identify the two state arrays when passed back to these
 *     functions and must not be dereferenced or copied by the caller (the
 *     reference's Block3d.cpp only passes them back).
 *   - The viscous/inviscid switch is a run-time field of Block3dInfo
 *     (is_viscous), defaulting from the IS_INVISCID macro as the reference's
 *     compile-time switch does; precision and the viscous-divergence placement
 *     are run-time fields too.
 *   - Only one block per process, as in the reference (its parameters live in
 *     one __constant__ singleton, src/copy_block_info.cu:8).
 */
#ifndef CBNS_BLOCK3D_CUDA_H_
#define CBNS_BLOCK3D_CUDA_H_

#include "cbns_b200.h"

typedef double value_type;
typedef unsigned int size_type;
typedef int index_type;

namespace constant {
const size_type NEQ = 5;
const size_type NG = 2;
const value_type PI = 3.14159265358979323846;
}  // namespace constant

#ifdef IS_INVISCID
#define CBNS_SHIM_VISCOUS_DEFAULT 0
#else
#define CBNS_SHIM_VISCOUS_DEFAULT 1
#endif

namespace block3d_cuda {

struct Block3dInfo {
  static const size_type NEQ{constant::NEQ};
  static const size_type NG{constant::NG};
  size_type IM, JM, KM;
  size_type IM_G, JM_G, KM_G;
  value_type CFL;
  value_type angle_attack;
  size_type i_begin;
  size_type i_end;
  value_type Mach;
  value_type Re;
  value_type Mach2;
  value_type gM2;
  value_type Re_inv;
  value_type p_inf;
  value_type gamma;
  value_type Pr;
  value_type Pr_t;
  value_type gam1;
  value_type gam1_inv;
  value_type Pr_inv;
  value_type Pr_t_inv;
  value_type gPr;
  value_type C_T_inf;
  value_type C_dt_v;
  /* run-time switches of this implementation */
  int is_viscous = CBNS_SHIM_VISCOUS_DEFAULT;
  int precision = CBNS_PREC_FP64;
  int vis_divergence = CBNS_VISDIV_REFERENCE;
  int bc_mode = CBNS_BC_REFERENCE;  /* CBNS_BC_*: the reference's boundaries by default */
  /* weights file of the learned sensor (cbns_sensor_load_file), required when
   * precision is CBNS_PREC_HYBRID */
  const char* sensor_weights = nullptr;
};

struct Block3dData {
  value_type* Q = nullptr;    /* handle of the reference's Q   */
  value_type* Q_p = nullptr;  /* handle of the reference's Q_p */
  cbns_ctx* ctx = nullptr;
};

void copy_block_info(const Block3dInfo* block_info);
void allocate_mem(const Block3dInfo* block_info, Block3dData* block_data);
void free_mem(Block3dData* block_data);
void calc_metrics(const Block3dInfo* block_info, Block3dData* block_data, const value_type* x, const value_type* y,
                  const value_type* z);
void get_metrics(const Block3dInfo* block_info, const Block3dData* block_data, value_type* xi_x, value_type* xi_y,
                 value_type* xi_z, value_type* eta_x, value_type* eta_y, value_type* eta_z, value_type* zeta_x,
                 value_type* zeta_y, value_type* zeta_z, value_type* Jac);
void initial_condition(const Block3dInfo* block_info, Block3dData* block_data);
void calc_conservative(const Block3dInfo* block_info, Block3dData* block_data, value_type* Q);
void set_conservative(const Block3dInfo* block_info, Block3dData* block_data, const value_type* Q);
void get_conservative(const Block3dInfo* block_info, const Block3dData* block_data, value_type* Q);
void get_primitive(const Block3dInfo* block_info, const Block3dData* block_data, value_type* rho, value_type* u,
                   value_type* v, value_type* w, value_type* p);
void calc_primitive(const Block3dInfo* block_info, Block3dData* block_data, const value_type* Q);
void set_bc_calc_primitive(const Block3dInfo* block_info, Block3dData* block_data, value_type* Q);
void calc_numerical_flux(const Block3dInfo* block_info, Block3dData* block_data, const value_type* Q);
void calc_viscous_terms(const Block3dInfo* block_info, Block3dData* block_data);
void calc_viscous_flux_contribution(const Block3dInfo* block_info, Block3dData* block_data);
void update_rk3(const Block3dInfo* block_info, Block3dData* block_data, const value_type dt, const size_type stage);
value_type calc_dt(const Block3dInfo* block_info, Block3dData* block_data);
void calc_gradient(const Block3dInfo* block_info, const value_type* f, value_type* fx, value_type* fy,
                   value_type* fz);

}  // namespace block3d_cuda

#endif /* CBNS_BLOCK3D_CUDA_H_ */
