// Navier-Stokes diffusion on the GPU (activate_diffusion): the momentum system of
// ns_vectorial_diffusion_module.F90 (with the viscous work) and the heat system of
// ns_diffusion_module.F90, assembled point-implicitly into the cells' 5x5 blocks.
//
// A warp per vertex builds and solves the vertex's sub-cell systems in shared memory and
// writes, per corner (sub-cell), the terms the reference adds into its cell's mat_diag
// and rhs, in the reference's order. The cell side (inside the time discretisation, or
// for the residual entry point) walks the cell's corners in ascending vertex order, the
// order of the reference's vertex loop, and applies them: first every corner's momentum
// terms, then every corner's heat terms, as the reference runs the momentum routine over
// all vertices before the heat routine.
//
// Per-corner record (kd doubles):
//   [0, 9)    momentum rhs(2:4): per component i, SNS_Ve, SNS_ll Ve, SB at 3 i + 0..2
//   [9, 27)   momentum diag(2:4,2:4): per (i, j) SNS_ll(i,j) / rho, blc_3(i,j) at 9 + 2 (i + 3 j)
//   [27, 31)  viscous work into rhs(5): one term per subface of the sub-cell
//   [31, 36)  heat diag(5, k): (blc_1 - SNS_ll) P(k)
//   [36, 40)  heat rhs(5): SNS_ll P.U, (blc_1 - SNS_ll) P.U, blc_1 theta, SB
//   [40, 40 + nsen)  heat rhs(5): SNS(l, p) theta(p), p over the vertex's sub-cells
#pragma once
#include "../../include/subfv.h"
#include "mesh_dev.cuh"

namespace subfv {

constexpr int kDiffHead = 40;

struct DiffParams {
  int sutherland;
  double mu_p, mu0, T0, Cv_p;
  int bcV[16], bcT[16];  // 0 or 1 neumann, 2 dirichlet
  double valV[16][3], valT[16];
  double prandtl;
  int kd;  // doubles per corner record
};

DiffParams diff_params_from(const subfv_ns_cfg& c, const DevMesh& m);
// shared memory one vertex's systems need (bytes), from the mesh's largest vertex
size_t diffusion_smem_bytes(const DevMesh& m);
// lets the vertex kernel use smem bytes of dynamic shared memory
int diffusion_prepare(size_t smem);
// mu0corr (into *mu0c) and the corner records of state U; from the mesh's cache when it
// holds the arrays for D's constants
void launch_ns_diffusion(const DevMesh& m, const DiffParams& D, const double* U, double* dterm, double* mu0c);
// With a constant viscosity, computes each vertex's state-independent diffusion arrays
// once into the mesh's cache (also writing the corner records of U into dterm), unless
// the mesh has a cache already (for any constants) or it would take more than half the
// free device memory; at state creation, outside any stream capture.
int diffusion_cache_build(DevMesh* m, const DiffParams& D, const double* U, double* dterm, double* mu0c);
// rhs1 (kRhs records) += the diffusion terms; diag (25 per cell, column-major) = the
// diffusion blocks (the residual entry point; the time loop applies them in place)
void launch_ns_diffusion_apply(const DevMesh& m, const double* dterm, int kd, double* rhs1, double* diag);

// The cell's diffusion terms onto its residual r (after flux limiting) and its block D
// (column-major, zero on entry).
// M: DevMesh or any view with its ev_off, cse_sorted, se_sf, se_vert and dse_off arrays
template <class M>
__device__ inline void apply_diffusion_terms(const M& m, int c, const double* __restrict__ dterm, int kd,
                                             double* r, double* D) {
  const int e0 = m.ev_off[c], e1 = m.ev_off[c + 1];
  for (int q = e0; q < e1; ++q) {
    const int se = m.cse_sorted[q];
    const double* t = dterm + (size_t)kd * se;
    for (int j = 0; j < 3; ++j)
      for (int i = 0; i < 3; ++i) {
        double& d = D[(1 + i) + 5 * (1 + j)];
        d = (d - t[9 + 2 * (i + 3 * j)]) + t[10 + 2 * (i + 3 * j)];
      }
    for (int i = 0; i < 3; ++i) r[1 + i] = ((r[1 + i] + t[3 * i]) - t[3 * i + 1]) + t[3 * i + 2];
    const int4 s4 = m.se_sf[se];
    const int nsf = (s4.x >= 0) + (s4.y >= 0) + (s4.z >= 0) + (s4.w >= 0);
    for (int k = 0; k < nsf; ++k) r[4] = r[4] + t[27 + k];
  }
  for (int q = e0; q < e1; ++q) {
    const int se = m.cse_sorted[q];
    const double* t = dterm + (size_t)kd * se;
    const int v = m.se_vert[se];
    const int nsen = m.dse_off[v + 1] - m.dse_off[v];  // the length of the writing vertex's stencil
    for (int p = 0; p < nsen; ++p) r[4] = r[4] + t[kDiffHead + p];
    for (int k = 0; k < 5; ++k) D[4 + 5 * k] = D[4 + 5 * k] + t[31 + k];
    r[4] = (((r[4] - t[36]) + t[37]) - t[38]) + t[39];
  }
}

// dgetrf + dgetrs (lu_solve_inplace_lapack) of the 5x5 column-major A, in the netlib
// operation order (right-looking elimination, first largest pivot, column scaled by the
// pivot's reciprocal); b is overwritten by the solution
__device__ inline void lu_solve5(double* A, double* b) {
  int ipiv[5];
  for (int j = 0; j < 5; ++j) {
    int p = j;
    double big = fabs(A[j + 5 * j]);
    for (int i = j + 1; i < 5; ++i)
      if (fabs(A[i + 5 * j]) > big) {
        big = fabs(A[i + 5 * j]);
        p = i;
      }
    ipiv[j] = p;
    if (A[p + 5 * j] != 0.0) {
      if (p != j)
        for (int k = 0; k < 5; ++k) {
          const double t = A[j + 5 * k];
          A[j + 5 * k] = A[p + 5 * k];
          A[p + 5 * k] = t;
        }
      if (fabs(A[j + 5 * j]) >= 2.2250738585072014e-308) {
        const double rr = 1.0 / A[j + 5 * j];
        for (int i = j + 1; i < 5; ++i) A[i + 5 * j] = rr * A[i + 5 * j];
      } else {
        for (int i = j + 1; i < 5; ++i) A[i + 5 * j] = A[i + 5 * j] / A[j + 5 * j];
      }
    }
    for (int k = j + 1; k < 5; ++k)
      for (int i = j + 1; i < 5; ++i) A[i + 5 * k] = A[i + 5 * k] - A[i + 5 * j] * A[j + 5 * k];
  }
  for (int j = 0; j < 5; ++j)
    if (ipiv[j] != j) {
      const double t = b[j];
      b[j] = b[ipiv[j]];
      b[ipiv[j]] = t;
    }
  for (int k = 0; k < 5; ++k)
    if (b[k] != 0.0)
      for (int i = k + 1; i < 5; ++i) b[i] = b[i] - b[k] * A[i + 5 * k];
  for (int k = 4; k >= 0; --k)
    if (b[k] != 0.0) {
      b[k] = b[k] / A[k + 5 * k];
      for (int i = 0; i < k; ++i) b[i] = b[i] - b[k] * A[i + 5 * k];
    }
}

}  // namespace subfv
