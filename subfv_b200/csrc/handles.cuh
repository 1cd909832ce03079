// Opaque handle types of the C-ABI, shared by the translation units that implement it.
#pragma once
#include "../../include/subfv.h"
#include "common.cuh"
#include "mesh_dev.cuh"

// A device mesh plus the scratch buffers the stateless reference-shaped calls need.
struct subfv_mesh {
  subfv::DevMesh d;
  double* stage = nullptr;  // host-layout staging, max(5*ne, 3*nv) doubles
  double* sol6 = nullptr;   // [ne][kRec] cell records
  double* rhs6 = nullptr;   // [ne][kRhs]
  double* mass = nullptr;   // [ne]
  subfv::LagScalars* sc = nullptr;
  // the backward-Euler Jacobian's host pattern, built on first use and kept with the mesh
  void* imp_pattern = nullptr;
  void (*imp_pattern_free)(void*) = nullptr;
};

namespace subfv {
int handle_check_status(DevMesh& d);
int handle_clear_status(DevMesh& d);
int handle_ensure_scratch(subfv_mesh* m);
// full geometry when Lagrangian steps left only the step's subset current
int handle_ensure_full_geometry(DevMesh& d);
// the Lagrangian step's per-mesh arrays (allocated on the mesh's stream)
int handle_ensure_lag_arrays(DevMesh& d);
}  // namespace subfv
