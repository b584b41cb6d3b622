// cbns3d.cpp - command-line entry of the B200 solver (the reference's
// src/cbns3d.cpp:17-25 with options).  Reads input.txt in the working
// directory like the reference.
//   --quiet          no per-step output line
//   --graph          whole steps replayed from a CUDA graph, dt on the device
//   --precision P    fp64 (default) | split | hybrid
//   --sensor FILE    learned-sensor weights for the hybrid (default: the
//                    trained weights shipped beside this executable,
//                    ../data/sensor_weights.bin)
//   --visdiv D       reference (default) | centered
//   --bc B           reference (default) | farfield | characteristic | ogrid
//                    (ogrid: the grid file stores the wrap copies of CBNS_BC_OGRID)
//   --inviscid / --viscous   override the build-time default
//   --input FILE     parameter file (default input.txt)
//   --vtk-binary     output.vtk in legacy VTK BINARY (same data set as the
//                    reference's ASCII file, written in one pass per array)
//   --plot3d         also write output.xyz / output.q (binary Plot3D)
#include <unistd.h>

#include <cstring>
#include <iostream>
#include <string>

#include "Block3d.h"

int main(int argc, char** argv) {
  Block3d::Options o;
  for (int a = 1; a < argc; ++a) {
    const std::string s = argv[a];
    auto next = [&]() -> std::string {
      if (a + 1 >= argc) {
        std::cerr << "missing value after " << s << "\n";
        std::exit(2);
      }
      return argv[++a];
    };
    if (s == "--quiet") o.quiet = true;
    else if (s == "--graph") o.graph = true;
    else if (s == "--inviscid") o.viscous = 0;
    else if (s == "--viscous") o.viscous = 1;
    else if (s == "--input") o.input = next();
    else if (s == "--vtk-binary") o.vtk_binary = true;
    else if (s == "--plot3d") o.plot3d = true;
    else if (s == "--precision") {
      const std::string v = next();
      o.precision = v == "split" ? CBNS_PREC_SPLIT : (v == "hybrid" ? CBNS_PREC_HYBRID : CBNS_PREC_FP64);
    } else if (s == "--sensor") {
      o.sensor = next();
    } else if (s == "--bc") {
      const std::string v = next();
      if (v == "reference") o.bc_mode = CBNS_BC_REFERENCE;
      else if (v == "farfield") o.bc_mode = CBNS_BC_FARFIELD;
      else if (v == "characteristic") o.bc_mode = CBNS_BC_CHARACTERISTIC;
      else if (v == "ogrid") o.bc_mode = CBNS_BC_OGRID;
      else {
        std::cerr << "unknown boundary mode " << v << "\n";
        return 2;
      }
    } else if (s == "--visdiv") {
      o.vis_divergence = next() == "centered" ? CBNS_VISDIV_CENTERED : CBNS_VISDIV_REFERENCE;
    } else {
      std::cerr << "unknown option " << s << "\n";
      return 2;
    }
  }
  if (o.precision == CBNS_PREC_HYBRID && o.sensor.empty()) {
    // the weights shipped with the library: <package>/data, the executable in <package>/bin
    char exe[4096];
    const ssize_t n = readlink("/proc/self/exe", exe, sizeof(exe) - 1);
    std::string dir = ".";
    if (n > 0) {
      exe[n] = 0;
      dir = std::string(exe);
      dir = dir.substr(0, dir.find_last_of('/'));
    }
    o.sensor = dir + "/../data/sensor_weights.bin";
  }
  Block3d block(o);
  return block.solve();
}
