// Block3d.h - host driver of one curvilinear block: reads the parsed .ini
// (input.txt), the ASCII Plot3D mesh and an optional checkpoint, runs the SSP-RK3
// time loop through the block3d_cuda API and writes the checkpoint and the
// legacy VTK file.  The formats, the input order and the call sequence are
// those of the reference driver (include/Block3d.h:15-116, src/Block3d.cpp).
#pragma once

#include <string>
#include <vector>

#include "../../include/block3d_cuda.h"

class Block3d {
 public:
  struct Options {
    bool quiet = false;      // suppress the per-step "n, dt, t" line
    bool graph = false;      // whole steps from a CUDA graph (dt stays on the device)
    int precision = CBNS_PREC_FP64;
    int vis_divergence = CBNS_VISDIV_REFERENCE;
    int bc_mode = CBNS_BC_REFERENCE;
    int viscous = CBNS_SHIM_VISCOUS_DEFAULT;
    std::string input = "input.txt";
    std::string sensor = "";  // learned-sensor weights (precision hybrid)
    bool vtk_binary = false;  // output.vtk as legacy VTK BINARY (big-endian) instead of ASCII
    bool plot3d = false;      // also write output.xyz / output.q (binary Plot3D grid and solution)
  };

  explicit Block3d(const Options& o) : opt_(o) {}
  int solve();

 private:
  void read_input();
  void read_mesh();
  void output_vtk() const;
  void output_vtk_binary() const;
  void output_plot3d() const;
  void output_bin(const std::string& fname) const;
  void read_bin(const std::string& fname);
  bool is_finished() const;

  Options opt_;
  block3d_cuda::Block3dInfo info_{};
  std::string grid_fname_, checkpoint_fname_;
  size_type IM_ = 0, JM_ = 0, KM_ = 0, IM_G_ = 0, JM_G_ = 0, KM_G_ = 0;
  value_type CFL_ = 0, t_cur_ = 0, t_end_ = 0;
  bool is_restart_ = false;
  size_type nstep_max_ = 0, checkpoint_freq_ = 0;
  std::vector<value_type> x_, y_, z_, rho_, u_, v_, w_, p_, Q_;
};
