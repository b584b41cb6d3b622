// block3d_shim.cpp - the reference's block3d_cuda:: host API over the C ABI.
// See include/block3d_cuda.h for the list of replaced declarations and the
// behaviour kept (synchronous calls, exit-on-error, throw on NaN dt).
#include "../../include/block3d_cuda.h"

#include <cstdio>
#include <cstdlib>
#include <stdexcept>

namespace block3d_cuda {

namespace {

Block3dInfo g_info;  // the reference keeps one copy in __constant__ memory
bool g_have_info = false;
char g_tag_q, g_tag_qp;  // addresses used as the Q / Q_p handles

void check(int rc, const char* file, int line) {
  if (rc != CBNS_OK) {
    std::printf("Error: %s:%d, ", file, line);
    std::printf("code:%d, reason: %s\n", rc, cbns_status_string(rc));
    std::exit(EXIT_FAILURE);
  }
}
#define SHIM_CHECK(call) check((call), __FILE__, __LINE__)

int which_of(const Block3dData* d, const value_type* Q) {
  if (Q == d->Q) return CBNS_Q;
  if (Q == d->Q_p) return CBNS_QP;
  std::printf("Error: %s:%d, code:%d, reason: pointer is neither block_data->Q nor block_data->Q_p\n", __FILE__,
              __LINE__, CBNS_ERR_ARG);
  std::exit(EXIT_FAILURE);
}

cbns_params params_of(const Block3dInfo* b) {
  cbns_params p{};
  p.IM = b->IM;
  p.JM = b->JM;
  p.KM = b->KM;
  p.CFL = b->CFL;
  p.angle_attack = b->angle_attack;
  p.i_begin = b->i_begin;
  p.i_end = b->i_end;
  p.Mach = b->Mach;
  p.Re = b->Re;
  p.gamma = b->gamma;
  p.Pr = b->Pr;
  p.Pr_t = b->Pr_t;
  p.T_inf = 110.5 / b->C_T_inf;  // Block3dInfo carries C_T_inf = 110.5 / T_inf
  p.viscous = b->is_viscous;
  p.precision = b->precision;
  p.vis_divergence = b->vis_divergence;
  p.bc_mode = b->bc_mode;
  return p;
}

}  // namespace

void copy_block_info(const Block3dInfo* block_info) {
  g_info = *block_info;
  g_have_info = true;
}

void allocate_mem(const Block3dInfo* block_info, Block3dData* block_data) {
  const cbns_params p = params_of(block_info);
  SHIM_CHECK(cbns_create(&p, &block_data->ctx));
  if (p.precision == CBNS_PREC_HYBRID) SHIM_CHECK(cbns_sensor_load_file(block_data->ctx, block_info->sensor_weights));
  block_data->Q = reinterpret_cast<value_type*>(&g_tag_q);
  block_data->Q_p = reinterpret_cast<value_type*>(&g_tag_qp);
}

void free_mem(Block3dData* block_data) {
  if (block_data->ctx) SHIM_CHECK(cbns_destroy(block_data->ctx));
  block_data->ctx = nullptr;
  block_data->Q = block_data->Q_p = nullptr;
}

void calc_metrics(const Block3dInfo*, Block3dData* d, const value_type* x, const value_type* y, const value_type* z) {
  SHIM_CHECK(cbns_calc_metrics(d->ctx, x, y, z));
}

void get_metrics(const Block3dInfo*, const Block3dData* d, value_type* xi_x, value_type* xi_y, value_type* xi_z,
                 value_type* eta_x, value_type* eta_y, value_type* eta_z, value_type* zeta_x, value_type* zeta_y,
                 value_type* zeta_z, value_type* Jac) {
  SHIM_CHECK(cbns_get_metrics(d->ctx, xi_x, xi_y, xi_z, eta_x, eta_y, eta_z, zeta_x, zeta_y, zeta_z, Jac));
}

void initial_condition(const Block3dInfo*, Block3dData* d) {
  SHIM_CHECK(cbns_initial_condition(d->ctx));
  SHIM_CHECK(cbns_synchronize(d->ctx));
}

void calc_conservative(const Block3dInfo*, Block3dData* d, value_type* Q) {
  SHIM_CHECK(cbns_calc_conservative(d->ctx, which_of(d, Q)));
  SHIM_CHECK(cbns_synchronize(d->ctx));
}

void set_conservative(const Block3dInfo*, Block3dData* d, const value_type* Q) {
  SHIM_CHECK(cbns_set_conservative(d->ctx, Q));
}

void get_conservative(const Block3dInfo*, const Block3dData* d, value_type* Q) {
  SHIM_CHECK(cbns_get_conservative(d->ctx, CBNS_Q, Q));
}

void get_primitive(const Block3dInfo*, const Block3dData* d, value_type* rho, value_type* u, value_type* v,
                   value_type* w, value_type* p) {
  SHIM_CHECK(cbns_get_primitive(d->ctx, rho, u, v, w, p, nullptr));
}

void calc_primitive(const Block3dInfo*, Block3dData* d, const value_type* Q) {
  SHIM_CHECK(cbns_calc_primitive(d->ctx, which_of(d, Q)));
  SHIM_CHECK(cbns_synchronize(d->ctx));
}

void set_bc_calc_primitive(const Block3dInfo*, Block3dData* d, value_type* Q) {
  SHIM_CHECK(cbns_set_bc_calc_primitive(d->ctx, which_of(d, Q)));
  SHIM_CHECK(cbns_synchronize(d->ctx));
}

void calc_numerical_flux(const Block3dInfo*, Block3dData* d, const value_type* Q) {
  SHIM_CHECK(cbns_calc_numerical_flux(d->ctx, which_of(d, Q)));
}

void calc_viscous_terms(const Block3dInfo*, Block3dData* d) {
  SHIM_CHECK(cbns_calc_viscous_terms(d->ctx));
  SHIM_CHECK(cbns_synchronize(d->ctx));
}

void calc_viscous_flux_contribution(const Block3dInfo*, Block3dData* d) {
  SHIM_CHECK(cbns_calc_viscous_flux_contribution(d->ctx));
}

void update_rk3(const Block3dInfo*, Block3dData* d, const value_type dt, const size_type stage) {
  SHIM_CHECK(cbns_update_rk3(d->ctx, dt, stage));
  SHIM_CHECK(cbns_synchronize(d->ctx));
}

value_type calc_dt(const Block3dInfo*, Block3dData* d) {
  value_type dt = 0.0;
  const int rc = cbns_calc_dt(d->ctx, &dt);
  if (rc == CBNS_ERR_NAN_DT) throw std::runtime_error("An error occurred while calculating the time step.\n");
  SHIM_CHECK(rc);
  return dt;
}

void calc_gradient(const Block3dInfo* b, const value_type* f, value_type* fx, value_type* fy, value_type* fz) {
  SHIM_CHECK(cbns_calc_gradient(b->IM, b->JM, b->KM, f, fx, fy, fz));
}

}  // namespace block3d_cuda
