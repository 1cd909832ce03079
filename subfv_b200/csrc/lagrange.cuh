// Launchers of the Lagrangian step kernels (lagrange.cu).
#pragma once
#include "common.cuh"
#include "mesh_dev.cuh"

namespace subfv {

// the face records (k_lag_face) then the nodal solve (k_lag_node); the mesh's frec must
// be allocated (devmesh_ensure_lag)
void launch_lag_node(const DevMesh& m, const double* sol6, const LagScalars* sc, int precision);
void launch_lag_face_only(const DevMesh& m, const double* sol6, const LagScalars* sc, int precision);
void launch_lag_node_only(const DevMesh& m, const LagScalars* sc, int precision);
// mode bit 1: rhs into rhs6; bit 2: CFL terms min-reduced into *dt_slot
void launch_lag_cell(const DevMesh& m, const double* sol6, double* rhs6, LagScalars* sc, double* dt_slot,
                     int precision, int mode);
void launch_lag_finalize(const DevMesh& m, LagScalars* sc);
void launch_lag_move(const DevMesh& m, const LagScalars* sc, double dt_host);
void launch_pack6(const DevMesh& m, int n, const double* s5, const double* mass, double* s6);
// record (stride doubles per cell) -> (5, n) host layout
void launch_unpack6(const DevMesh& m, int n, int stride, const double* s6, double* s5);
void launch_vp_out(const DevMesh& m, double* out);
void launch_vp_in(const DevMesh& m, const double* in);
void launch_set_scalar(const DevMesh& m, double* p, double v);
// fills m.centry (allocated by the caller, ncsf records) from the cell CSR
void launch_build_cell_entries(const DevMesh& m);
// scheme 0 "classic", 1 "sidil" (method_length `method`, FP64)
// the step up to lagrange_finalize (nodal solve, fluxes, dt); the rest is move_mesh and
// the geometry, with the update fused in (enqueue_lag_step) or launched on its own
void enqueue_lag_step_head(const DevMesh& m, double* sol6, double* rhs6, LagScalars* sc, int precision,
                           int scheme = 0, int method = 0);
void enqueue_lag_step(const DevMesh& m, double* sol6, double* rhs6, LagScalars* sc, int precision, int scheme = 0,
                      int method = 0);
// scheme "sidil": vertex volumes of the current mesh, then vp = (velocity, nodal pressure)
void launch_lag_sidil_node(const DevMesh& m, const double* sol6, const LagScalars* sc, int method);

// One problem of a batch: its mesh (moved by the steps), cell records, residual records
// and scalars.
struct LagItem {
  DevMesh m;
  double *sol6, *rhs6;
  LagScalars* sc;
};
// Table of in-flight problems: items, work-block prefixes over faces (wf, kLagFaceBlock
// faces per block), vertices (wv, kLagVertBlock) and cells (wc, kLagCellBlock), and
// hdr[0] = the number of problems; persistent grids of `grid` blocks.
constexpr int kLagFaceBlock = 128, kLagVertBlock = 128, kLagCellBlock = 64;
struct LagTable {
  LagItem* items = nullptr;
  int *wf = nullptr, *wv = nullptr, *wc = nullptr, *hdr = nullptr;
  int cap = 0, grid = 1;
};
// One step of lagrange_main.F90:89-127 for every problem of the table, in shared launches.
void launch_lag_batch_step(const LagTable& t, int precision, cudaStream_t s);

}  // namespace subfv
