// Block-CSR matrices and the restarted, block-Jacobi right-preconditioned GMRES of
// src/linear_algebra/sparse_bcsr_linear_module.F90 on the GPU.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "common.cuh"

namespace subfv {

constexpr int kBcsrMaxBs = 8;

struct DevBcsr {
  int m = 0, bs = 0, nnz = 0;
  int* row = nullptr;      // (m+1) 0-based offsets
  int* col = nullptr;      // (nnz) 0-based block columns
  double* v = nullptr;     // (bs, bs, nnz) column-major blocks
  float* v32 = nullptr;    // FP32 copy for the iterative-refinement inner solves
  int* diag = nullptr;     // (m) index of the diagonal block, -1 if absent
  double* lu = nullptr;    // (bs*bs, m) no-pivot LU, element-major: multipliers below the diagonal, U on and above
  // colouring for the parallel LU-SGS preconditioner (bcsr_parallel_lusgs): colour per
  // block row (1..ncs), the rows grouped by colour, and the groups' offsets (host)
  int ncs = 0;
  int* color = nullptr;
  int* set_rows = nullptr;
  std::vector<int> set_off;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  size_t bytes = 0;
};

struct GmresStats {
  int restarts = 0;
  int conv = 0;
  double rho = 0.0;
  int inner_total = 0;
  int outer = 0;
};

// Workspace for GMRES(m) on n = bs*m unknowns.
struct GmresWork {
  int krylov = 0;
  long n = 0;
  double *V = nullptr, *r = nullptr, *w = nullptr, *zp = nullptr, *z = nullptr;
  double *partial = nullptr, *H = nullptr, *scal = nullptr;
  double *d = nullptr, *rr = nullptr;  // refinement correction and residual
  double* ty = nullptr;                 // the LU-SGS forward sweep
  size_t bytes = 0;
  cudaGraphExec_t cycle = nullptr;  // the captured Arnoldi cycle and what it was captured for
  uintptr_t cycle_key[10] = {};
};

int bcsr_upload(DevBcsr* A, int m, int bs, const int* row1, const int* col1, const double* v, cudaStream_t s);
int bcsr_set_values(DevBcsr* A, const double* v_dev_or_host, bool on_device);
void bcsr_free(DevBcsr* A);
int gmres_work_alloc(GmresWork* W, long n, int krylov);
void gmres_work_free(GmresWork* W);

void launch_bcsr_spmv(const DevBcsr& A, const double* x, double* y, bool fp32_matrix);
void launch_bcsr_factor_diag(const DevBcsr& A);
void launch_bcsr_bjacobi(const DevBcsr& A, const double* b, double* x);
// bcsr_parallel_lusgs (:1438-1502): x = (U+D)^-1 D (L+D)^-1 b by colour sets; ty is an
// n-vector of scratch (the forward sweep)
void launch_bcsr_lusgs(const DevBcsr& A, const double* b, double* x, double* ty);
// colours (1..ncs) per block row, host array; rejects colours out of range
int bcsr_set_colors(DevBcsr* A, int ncs, const int* color);

// preconditioners of gmres_device
enum GmresPrecond { kPrecondNone = 0, kPrecondDiag = 1, kPrecondLusgs = 2 };

// bcsr_gmres_diag (precond 1), bcsr_gmres_parallel_lusgs (2) or bcsr_gmres (0); x, b
// device vectors; tol absolute.
int gmres_device(const DevBcsr& A, GmresWork& W, double* x, const double* b, double tol, int precond,
                 bool fp32_matrix, int maxit, GmresStats* st, double* H_first_host);
// FP64 iterative refinement around FP32-matrix GMRES: stops at |b - A x| < rel_tol * |b|.
int gmres_refine_device(const DevBcsr& A, GmresWork& W, double* x, const double* b, double rel_tol,
                        double inner_rel_tol, int max_outer, GmresStats* st, int precond = kPrecondDiag);
double device_norm2(const DevBcsr& A, GmresWork& W, const double* x, long n);

struct PcgStats {
  int iters = 0;
  int status = 0;  // 0 converged, 1 not converged, 2 singular diagonal block
  double res = 0.0;
};
// bcsr_pcgm (:1110-1169) from the initial guess in x (device vectors)
int pcg_device(const DevBcsr& A, GmresWork& W, double* x, const double* b, double tol, PcgStats* st);

}  // namespace subfv
