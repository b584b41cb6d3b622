// Block3d.cpp - host driver (see Block3d.h).
#include "Block3d.h"

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <stdexcept>

namespace {
constexpr size_type NEQ = constant::NEQ;
constexpr size_type NG = constant::NG;

[[noreturn]] void die(const std::string& what) {
  std::cout << what << std::endl;
  std::exit(EXIT_FAILURE);
}
}  // namespace

// input.txt: the values of the .ini in section order [string] [real] [integer]
// [bool] (python/parser_ini.py:17-33), read positionally as src/Block3d.cpp:33-93.
void Block3d::read_input() {
  std::ifstream fh(opt_.input);
  if (!fh) die("Exception opening/reading file");
  value_type Pr = 0, Pr_t = 0, gamma = 0, Mach = 0, Re = 0, T_inf = 0, aoa = 0;
  size_type i_begin = 0, i_end = 0;
  fh >> grid_fname_ >> checkpoint_fname_ >> CFL_ >> t_cur_ >> t_end_ >> Pr >> Pr_t >> gamma >> Mach >> Re >> T_inf >>
      aoa >> nstep_max_ >> checkpoint_freq_ >> i_begin >> i_end >> is_restart_;
  if (!fh) die("Exception opening/reading file");
  std::cout << "grid_fname : " << grid_fname_ << "\ncheckpoint_fname : " << checkpoint_fname_ << "\nCFL : " << CFL_
            << "\nt_cur : " << t_cur_ << "\nt_end : " << t_end_ << "\nPr : " << Pr << "\nPr_t : " << Pr_t
            << "\ngamma : " << gamma << "\nMach : " << Mach << "\nRe : " << Re << "\nT_inf : " << T_inf
            << "\nangle_attack : " << aoa << "\nnstep_max : " << nstep_max_ << "\ncheckpoint_freq : "
            << checkpoint_freq_ << "\ni_begin : " << i_begin << "\ni_end : " << i_end
            << "\nis_restart : " << is_restart_ << std::endl;
  // derived quantities (src/Block3d.cpp:99-113)
  info_.CFL = CFL_;
  info_.angle_attack = aoa;
  info_.i_begin = i_begin;
  info_.i_end = i_end;
  info_.gamma = gamma;
  info_.Mach = Mach;
  info_.Re = Re;
  info_.Pr = Pr;
  info_.Pr_t = Pr_t;
  info_.Mach2 = Mach * Mach;
  info_.gM2 = gamma * info_.Mach2;
  info_.Re_inv = 1.0 / Re;
  info_.p_inf = 1.0 / info_.gM2;
  info_.gam1 = gamma - 1.0;
  info_.gam1_inv = 1.0 / info_.gam1;
  info_.Pr_inv = 1.0 / Pr;
  info_.Pr_t_inv = 1.0 / Pr_t;
  info_.gPr = gamma / Pr;
  info_.C_T_inf = 110.5 / T_inf;
  info_.C_dt_v = std::max(4.0 / 3.0, gamma * info_.Pr_inv) * info_.Re_inv;
  info_.is_viscous = opt_.viscous;
  info_.precision = opt_.precision;
  info_.vis_divergence = opt_.vis_divergence;
  info_.bc_mode = opt_.bc_mode;
  info_.sensor_weights = opt_.sensor.empty() ? nullptr : opt_.sensor.c_str();
}

// ASCII Plot3D single block: IM JM KM, then x, y, z with i fastest (src/Block3d.cpp:151-202).
void Block3d::read_mesh() {
  std::ifstream fh(grid_fname_);
  if (!fh) die("Exception opening/reading file");
  fh >> IM_ >> JM_ >> KM_;
  if (!fh) die("Exception opening/reading file");
  std::cout << IM_ << ", " << JM_ << ", " << KM_ << "\n";
  IM_G_ = IM_ + 2 * NG;
  JM_G_ = JM_ + 2 * NG;
  KM_G_ = KM_ + 2 * NG;
  const size_t n = (size_t)IM_ * JM_ * KM_;
  x_.resize(n);
  y_.resize(n);
  z_.resize(n);
  for (auto* a : {&x_, &y_, &z_})
    for (size_t i = 0; i < n; ++i) fh >> (*a)[i];
  if (!fh) die("Exception opening/reading file");
  const size_t ng = (size_t)IM_G_ * JM_G_ * KM_G_;
  for (auto* a : {&rho_, &u_, &v_, &w_, &p_}) a->resize(ng);
  Q_.resize(NEQ * ng);
  info_.IM = IM_;
  info_.JM = JM_;
  info_.KM = KM_;
  info_.IM_G = IM_G_;
  info_.JM_G = JM_G_;
  info_.KM_G = KM_G_;
}

// Legacy VTK, ASCII STRUCTURED_GRID with rho,u,v,w,p (src/Block3d.cpp:357-409).
void Block3d::output_vtk() const {
  FILE* f = std::fopen("output.vtk", "w");
  if (!f) return;
  const size_t n = (size_t)IM_ * JM_ * KM_;
  std::fprintf(f, "# vtk DataFile Version 3.0\nvtk output\nASCII\nDATASET STRUCTURED_GRID\n");
  std::fprintf(f, "DIMENSIONS %d %d %d\n", (int)IM_, (int)JM_, (int)KM_);
  std::fprintf(f, "POINTS %d double\n", (int)n);
  for (size_t i = 0; i < n; ++i) std::fprintf(f, "%E %E %E\n", x_[i], y_[i], z_[i]);
  std::fprintf(f, "POINT_DATA %d\n", (int)n);
  std::fprintf(f, "FIELD FieldData 5\n");
  const char* names[5] = {"rho", "u", "v", "w", "p"};
  const std::vector<value_type>* arrs[5] = {&rho_, &u_, &v_, &w_, &p_};
  for (int a = 0; a < 5; ++a) {
    std::fprintf(f, "%s 1 %d double\n", names[a], (int)n);
    for (size_type k = 0; k < KM_; ++k)
      for (size_type j = 0; j < JM_; ++j)
        for (size_type i = 0; i < IM_; ++i)
          std::fprintf(f, "%E\n", (*arrs[a])[(NG + i) + IM_G_ * ((NG + j) + JM_G_ * (NG + k))]);
  }
  std::cout << "The output is successful!\n";
  std::fclose(f);
}

namespace {

// legacy VTK binary data are big-endian
void put_be(std::vector<unsigned char>& buf, double v) {
  unsigned char b[8];
  std::memcpy(b, &v, 8);
  for (int i = 7; i >= 0; --i) buf.push_back(b[i]);
}

}  // namespace

// The same data set as output_vtk in legacy VTK BINARY: the header lines as
// text, each array as big-endian doubles followed by a newline.  One write per
// array instead of one formatted line per value.
void Block3d::output_vtk_binary() const {
  std::ofstream f("output.vtk", std::ios::out | std::ios::binary);
  if (!f) return;
  const size_t n = (size_t)IM_ * JM_ * KM_;
  std::ostringstream h;
  h << "# vtk DataFile Version 3.0\nvtk output\nBINARY\nDATASET STRUCTURED_GRID\n";
  h << "DIMENSIONS " << IM_ << " " << JM_ << " " << KM_ << "\n";
  h << "POINTS " << n << " double\n";
  f << h.str();
  std::vector<unsigned char> buf;
  buf.reserve(3 * n * 8 + 1);
  for (size_t i = 0; i < n; ++i) {
    put_be(buf, x_[i]);
    put_be(buf, y_[i]);
    put_be(buf, z_[i]);
  }
  buf.push_back('\n');
  f.write(reinterpret_cast<const char*>(buf.data()), (std::streamsize)buf.size());
  f << "POINT_DATA " << n << "\nFIELD FieldData 5\n";
  const char* names[5] = {"rho", "u", "v", "w", "p"};
  const std::vector<value_type>* arrs[5] = {&rho_, &u_, &v_, &w_, &p_};
  for (int a = 0; a < 5; ++a) {
    f << names[a] << " 1 " << n << " double\n";
    buf.clear();
    for (size_type k = 0; k < KM_; ++k)
      for (size_type j = 0; j < JM_; ++j)
        for (size_type i = 0; i < IM_; ++i) put_be(buf, (*arrs[a])[(NG + i) + IM_G_ * ((NG + j) + JM_G_ * (NG + k))]);
    buf.push_back('\n');
    f.write(reinterpret_cast<const char*>(buf.data()), (std::streamsize)buf.size());
  }
  std::cout << "The output is successful!\n";
}

// Binary Plot3D (whole 3D, single block, no record markers, native byte
// order): output.xyz = int32 IM JM KM, then x, y, z (float64, i fastest);
// output.q = int32 IM JM KM, float64 Mach, angle of attack, Re, time, then
// rho, rho u, rho v, rho w, rho E at the grid nodes (float64, i fastest).
void Block3d::output_plot3d() const {
  const int dims[3] = {(int)IM_, (int)JM_, (int)KM_};
  const size_t n = (size_t)IM_ * JM_ * KM_;
  {
    std::ofstream f("output.xyz", std::ios::out | std::ios::binary);
    if (!f) return;
    f.write(reinterpret_cast<const char*>(dims), sizeof(dims));
    for (const auto* a : {&x_, &y_, &z_}) f.write(reinterpret_cast<const char*>(a->data()), n * sizeof(value_type));
  }
  std::ofstream f("output.q", std::ios::out | std::ios::binary);
  if (!f) return;
  f.write(reinterpret_cast<const char*>(dims), sizeof(dims));
  const double head[4] = {info_.Mach, info_.angle_attack, info_.Re, t_cur_};
  f.write(reinterpret_cast<const char*>(head), sizeof(head));
  std::vector<double> q(n);
  for (int m = 0; m < NEQ; ++m) {
    size_t e = 0;
    for (size_type k = 0; k < KM_; ++k)
      for (size_type j = 0; j < JM_; ++j)
        for (size_type i = 0; i < IM_; ++i)
          q[e++] = Q_[m + NEQ * ((NG + i) + IM_G_ * ((NG + j) + JM_G_ * (NG + k)))];
    f.write(reinterpret_cast<const char*>(q.data()), n * sizeof(double));
  }
}

// Checkpoint: double t_cur; uint32 IM_G, JM_G, KM_G; double Q[5*IM_G*JM_G*KM_G]
// with the variable index fastest (src/Block3d.cpp:411-434).
void Block3d::output_bin(const std::string& fname) const {
  std::ofstream fh(fname, std::ios::out | std::ios::binary);
  if (!fh) {
    std::cout << "Cannot open file!" << std::endl;
    return;
  }
  fh.write(reinterpret_cast<const char*>(&t_cur_), sizeof(value_type));
  fh.write(reinterpret_cast<const char*>(&IM_G_), sizeof(size_type));
  fh.write(reinterpret_cast<const char*>(&JM_G_), sizeof(size_type));
  fh.write(reinterpret_cast<const char*>(&KM_G_), sizeof(size_type));
  fh.write(reinterpret_cast<const char*>(Q_.data()), Q_.size() * sizeof(value_type));
}

void Block3d::read_bin(const std::string& fname) {
  std::ifstream fh(fname, std::ios::in | std::ios::binary);
  if (!fh) die("Exception opening/reading file");
  fh.read(reinterpret_cast<char*>(&t_cur_), sizeof(value_type));
  size_type dims[3] = {0, 0, 0};
  fh.read(reinterpret_cast<char*>(dims), sizeof(dims));
  if (dims[0] != IM_G_ || dims[1] != JM_G_ || dims[2] != KM_G_) die("The dimensions do not match.\n");
  fh.read(reinterpret_cast<char*>(Q_.data()), Q_.size() * sizeof(value_type));
  if (!fh) die("Exception opening/reading file");
}

bool Block3d::is_finished() const {
  if (t_cur_ + 1.0e-8 > t_end_) {
    std::cout << "Finished!\n";
    return true;
  }
  return false;
}

// The solve sequence of src/Block3d.cpp:204-313.
int Block3d::solve() {
  using namespace block3d_cuda;
  read_input();
  read_mesh();
  copy_block_info(&info_);
  Block3dData data;
  allocate_mem(&info_, &data);
  calc_metrics(&info_, &data, x_.data(), y_.data(), z_.data());
  const bool visc = info_.is_viscous != 0;
  // note the reference's inverted flag: a non-zero is_restart starts from the
  // free stream, zero reads the checkpoint (src/Block3d.cpp:219-228)
  if (is_restart_) {
    initial_condition(&info_, &data);
    calc_conservative(&info_, &data, data.Q);
  } else {
    read_bin(checkpoint_fname_);
    set_conservative(&info_, &data, Q_.data());
    if (visc) calc_primitive(&info_, &data, data.Q);
  }
  set_bc_calc_primitive(&info_, &data, data.Q);
  if (visc) calc_viscous_terms(&info_, &data);

  const auto start = std::chrono::high_resolution_clock::now();
  if (opt_.graph) {
    // whole steps on the device, checkpoints between chunks
    size_type done_total = 0;
    if (cbns_set_time(data.ctx, t_cur_) != CBNS_OK) die("cbns_set_time failed");
    while (done_total < nstep_max_ && !is_finished()) {
      size_type chunk = nstep_max_ - done_total;
      if (checkpoint_freq_ > 0) chunk = std::min<size_type>(chunk, checkpoint_freq_ - done_total % checkpoint_freq_);
      unsigned got = 0;
      const int rc = cbns_run(data.ctx, chunk, t_end_, &got);
      double dt_last = 0.0;
      cbns_get_time(data.ctx, &t_cur_, &dt_last);
      if (rc == CBNS_ERR_NAN_DT) throw std::runtime_error("An error occurred while calculating the time step.\n");
      if (rc != CBNS_OK) die(std::string("cbns_run failed: ") + cbns_status_string(rc));
      done_total += got;
      if (!opt_.quiet) std::cout << done_total - 1 << ", " << dt_last << ", " << t_cur_ << std::endl;
      if (checkpoint_freq_ > 0 && done_total % checkpoint_freq_ == 0 && got == chunk) {
        get_conservative(&info_, &data, Q_.data());
        output_bin(checkpoint_fname_);
      }
      if (got < chunk) break;
    }
  } else {
    for (size_type n_t = 0; n_t < nstep_max_; ++n_t) {
      if (is_finished()) break;
      value_type dt = calc_dt(&info_, &data);
      if (t_end_ - t_cur_ < dt) dt = t_end_ - t_cur_;
      t_cur_ += dt;
      if (!opt_.quiet) std::cout << n_t << ", " << dt << ", " << t_cur_ << std::endl;
      for (size_type s = 1; s <= 3; ++s) {
        calc_numerical_flux(&info_, &data, s == 1 ? data.Q : data.Q_p);
        if (visc) calc_viscous_flux_contribution(&info_, &data);
        update_rk3(&info_, &data, dt, s);
        set_bc_calc_primitive(&info_, &data, s == 3 ? data.Q : data.Q_p);
        if (visc) calc_viscous_terms(&info_, &data);
      }
      // the reference takes this modulo even for checkpoint_freq = 0 (a division
      // by zero); zero here means "no periodic checkpoints"
      if (checkpoint_freq_ > 0 && (n_t + 1) % checkpoint_freq_ == 0) {
        get_conservative(&info_, &data, Q_.data());
        output_bin(checkpoint_fname_);
      }
    }
  }
  const auto end = std::chrono::high_resolution_clock::now();
  std::cout << "Elapsed Time = " << std::chrono::duration<double>(end - start).count() << "\n";
  if (0 < nstep_max_) {
    get_conservative(&info_, &data, Q_.data());
    output_bin(checkpoint_fname_);
  }
  get_primitive(&info_, &data, rho_.data(), u_.data(), v_.data(), w_.data(), p_.data());
  if (opt_.vtk_binary) output_vtk_binary();
  else output_vtk();
  if (opt_.plot3d) {
    get_conservative(&info_, &data, Q_.data());
    output_plot3d();
  }
  free_mem(&data);
  return 0;
}
