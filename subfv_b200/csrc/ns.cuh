// Explicit Euler (subfvns) on the GPU: launchers and device-side parameter blocks.
#pragma once
#include "../../include/subfv.h"
#include "common.cuh"
#include "mesh_dev.cuh"

namespace subfv {

constexpr int kNsMaxSf = 32;  // subfaces around a vertex (a 3-D hex vertex has 12)
constexpr int kNsFs = 6;      // per-subcell record: five corner flux sums and the wave-speed sum
constexpr int kCellLanes = 8;  // lanes per cell of the grouped cell gradient (cells of up to 8 vertices)

struct NsParams {
  int scheme, second_order, method, bc_style, b2d, excl, lts, n_bc;
  int bc_type[16];
  double bc_val[16][5];
  double cfl, tmax;
  int precision;
  int node_group;  // 0: one thread per vertex; else a group of lanes per vertex, at least node_group
                  // (and, on meshes whose cells have at most kCellLanes vertices, a group of
                  // kCellLanes lanes per cell in the solo cell gradient)
  int diff, diff_kd;  // diffusion terms to apply in the time discretisation, doubles per corner record
};

struct NsScalars {
  double dtred;    // running min of V / sum_lambda of the current stage (starts at 1e10)
  double omega;    // running min of the positivity limiter (starts at 1; reset by the finalize)
  double omega_step;  // the limiter of the last finalized stage, which the update applies
  unsigned arrive;    // blocks of the current stage's time discretisation that finished
  double dt;       // time step of the last stage (after the omega correction)
  double t, final_res;
  double res, resv[5];
  unsigned long long steps;
  int done, skip;
  double tmax;     // end time of this problem (tmax of the namelist)
};

// One problem of a batch: its mesh and state buffers. Batched launches walk a table of
// these; work blocks never straddle two problems, so every per-problem reduction is the
// same as in a solo run.
struct NsItem {
  DevMesh m;
  double *U0, *U1, *fs, *rhs1, *rhs2, *ngrad, *grad, *delta, *partial;
  NsScalars* sc;
};

// Per-vertex array bound of the node kernel for a mesh: the smallest of 8, 16, 32 that
// holds every vertex's subfaces and subcells (0: a vertex has more than 32).
int ns_node_lanes(const DevMesh& m);
// Fills (or refills after the geometry changed) the mesh's per-vertex pseudo-inverses of
// the nodal-gradient matrices (DevMesh::npinv), on the mesh stream; nothing for a moving
// mesh. The solo gradient launches read them while they match the current geometry.
int ensure_nodal_pinv(DevMesh* m);
// Table of in-flight problems on the device: items, work-block prefixes over their
// vertices (wv, block_v vertices per work block) and cells (wc, 128 cells per work
// block), and hdr[0] = the number of problems. Up to cap problems; the grids are
// persistent (grid_v, grid_c blocks whatever the table holds). block_v: threads (one
// per vertex) per block of the vertex kernels (64, 128 or 256); group: the node
// kernel's per-vertex array bound (8, 16, 32), the largest the table needs.
struct NsTable {
  NsItem* items = nullptr;
  int* wv = nullptr;
  int* wc = nullptr;
  int* hdr = nullptr;
  int cap = 0;
  int block_v = 128, group = 8, grid_v = 1, grid_c = 1;
};
constexpr int kNsCellBlock = 128;
// One step of the time loop for every problem of the table, in shared launches.
void launch_ns_batch_step(const NsTable& t, const NsParams& P, cudaStream_t s);

NsParams ns_params_from(const subfv_ns_cfg& c);

// One residual evaluation at state U (records of kRec doubles): rhs1/sl (first order),
// and for second order ngrad, grad, rhs2. rhs records: kRhs doubles (5 + sum_lambda).
void launch_ns_rhs(const DevMesh& m, const NsParams& P, const double* U, double* fs, double* rhs1, double* rhs2,
                   double* ngrad, double* grad, NsScalars* sc);
// flux limiting + add_timedisc_and_solve + update (stage coefficients a1, a2)
// (dterm: the diffusion corner records when P.diff, else null)
void launch_ns_timedisc(const DevMesh& m, const NsParams& P, const double* U_rhs, const double* rhs1,
                        const double* rhs2, const double* U_td, double* U_out, double* delta, double* partial,
                        NsScalars* sc, double a1, double a2, int last_stage, const double* dterm = nullptr);
void launch_ns_pack(const DevMesh& m, const double* s5, double* U);
void launch_ns_flux_limiting(const DevMesh& m, const NsParams& P, const double* U, double* rhs1, const double* rhs2,
                             const NsScalars* sc);
// Backward-Euler Jacobian of the first-order two-wave residual (frozen wave speeds)
void launch_be_assemble(const DevMesh& m, const NsParams& P, const double* U, const int* jq_off, const int* jq,
                        const int* jblk, const int* row_off, const int* dblk, double* v, double dt,
                        const NsScalars* sc);
void launch_be_pack_rhs(const DevMesh& m, const double* rhs, double* b);
void launch_be_update(const DevMesh& m, double* U, const double* x);
// the diffusion blocks diag25 (column-major 5 x 5 per cell) onto the diagonal blocks
// (dblk) of the Jacobian values v, and b -= diag25 U
void launch_be_add_diffusion(const DevMesh& m, const int* dblk, const double* diag25, const double* U, double* v,
                             double* b);
int ns_partial_blocks(const DevMesh& m);

// The reference's module procedures one at a time (host-buffer entries of ns_procs.cu):
// compute_euler_flux, compute_cell_grad_from_nodal_grad, and the kernels of
// flux_limiting and add_timedisc_and_solve on arrays in the reference's layouts.
void launch_ns_euler_flux(const DevMesh& m, const NsParams& P, const double* U, const double* grad, double* fs,
                          double* rhs, int second_order, NsScalars* sc);
void launch_ns_cell_grads(const DevMesh& m, const NsParams& P, const double* U, double* ngrad, double* grad,
                          NsScalars* sc);
void launch_proc_dtmin(const DevMesh& m, const double* sl, double* slot);
void launch_proc_flux_limiting(const DevMesh& m, const double* sol5, double* rhs5, const double* rhso2_5,
                               const double* sl, double dt);
void launch_proc_timedisc(const DevMesh& m, const double* sol5, double* rhs5, double* diag25, double* delta5,
                          double* rn, double* rsq, double a1, double a2, double dt, double* omega_slot,
                          double* sums6);
void launch_proc_apply(const DevMesh& m, double* sol5, const double* delta5, double aw);

}  // namespace subfv
