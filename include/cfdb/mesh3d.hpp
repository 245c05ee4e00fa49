// Drop-in C++ facade over libcfdb's C ABI: the reference's Mesh3D API
// (include/mesh3d.hpp:118-237 of int0vrt/cfdARCOV2) without Eigen, OCCA or
// RMM.  Host vectors are std::vector<float>; device state lives in library
// buffers.  One process-wide context is created by CFDArcoGlobalInit.
#pragma once

#include <cstddef>
#include <stdexcept>
#include <string>
#include <vector>

#include "cfdb.h"

namespace cfdb {

// Throws std::runtime_error with the library's message on a non-zero status
// (the reference exits the process instead, include/cuda_operators.hpp:29-36).
void check(int status, const char* what);

// CFDArcoGlobalInit (include/cfdarcho_main_3d.hpp:33-79): binds a device and
// owns the library context.
class CFDArcoGlobalInit {
 public:
  // store_dir becomes store_path/run_<timestamp>, as the reference's
  // initialize sets it (src/cfdarcho_main_3d.cpp:276-299)
  static void initialize(int argc, char** argv, bool skip_history = true, const std::string& store_path = "./dumps");
  static void enable_cuda(int device = 0);
  static void finalize();
  static cfdb_ctx* ctx();
  static bool skip_history;
  static bool cuda_enabled;
  static bool store_stepping;
  static std::string store_dir;
  // use_jit equations on an exact lattice (cfdb_mesh_lattice_geometry) take
  // the geometry as constants instead of reading the face arrays; same bits
  static bool jit_lattice;
  // equations with use_jit = false run as generated kernels as well (the
  // generated kernels give the operator path's bits); false keeps them on
  // the operator-by-operator path as the reference runs them
  static bool jit_all;
  // print each generated kernel's entry, registers and local bytes to stderr
  // when it is built (a diagnostic, off by default)
  static bool jit_report;
};

class Mesh3D {
 public:
  Mesh3D(size_t x, size_t y, size_t z, float dx, float dy, float dz);
  ~Mesh3D();
  Mesh3D(const Mesh3D&) = delete;
  Mesh3D& operator=(const Mesh3D&) = delete;

  // The reference builds object graphs and computes every face's geometry
  // here (src/mesh3d.cpp:151-385).  init_basic_internals() does nothing;
  // compute() creates the library mesh and settles, on the GPU, whether it
  // is an exact lattice (cfdb_mesh_lattice_geometry), so that geometry work
  // happens before Equation::evaluate as in the reference.  Face arrays are
  // built on the device when an operator first needs them.
  void init_basic_internals();
  void compute();

  // Cell centre of cell id (z fastest, src/mesh3d.cpp:387-389).
  float x(size_t id) const;
  float y(size_t id) const;
  float z(size_t id) const;
  size_t square_node_coord_to_idx(size_t x, size_t y, size_t z) const { return _z * _y * x + _z * y + z; }
  bool is_boundary(size_t id) const;

  cfdb_mesh* handle();

  size_t _num_nodes, _x, _y, _z;
  float _lx, _ly, _lz, _dx, _dy, _dz;

 private:
  cfdb_mesh* mesh_ = nullptr;
};

using CudaMesh3D = Mesh3D;

}  // namespace cfdb
