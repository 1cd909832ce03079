// C-ABI of the BCSR linear algebra (include/subfv.h, subfv_bcsr_*).
#include <cstring>
#include <vector>

#include "../../include/subfv.h"
#include "bcsr.cuh"

using namespace subfv;

struct subfv_bcsr {
  DevBcsr A;
  GmresWork W;
  double *x = nullptr, *b = nullptr, *y = nullptr;
};

namespace {
int ensure_vecs(subfv_bcsr* h) {
  if (h->x) return 0;
  const size_t n = (size_t)h->A.m * h->A.bs;
  SUBFV_CUDA(cudaMalloc(&h->x, n * sizeof(double)));
  SUBFV_CUDA(cudaMalloc(&h->b, n * sizeof(double)));
  SUBFV_CUDA(cudaMalloc(&h->y, n * sizeof(double)));
  return 0;
}
int ensure_work(subfv_bcsr* h, int krylov) {
  if (h->W.V && h->W.krylov == krylov) return 0;
  gmres_work_free(&h->W);
  return gmres_work_alloc(&h->W, (long)h->A.m * h->A.bs, krylov);
}
}  // namespace

extern "C" {

int subfv_bcsr_create(int m, int bs, const int32_t* row, const int32_t* col, const double* v, subfv_bcsr** out) {
  if (!row || !col || !out) {
    set_error("subfv_bcsr_create: null argument");
    return -2;
  }
  auto* h = new subfv_bcsr();
  int rc = bcsr_upload(&h->A, m, bs, row, col, v, nullptr);
  if (rc) {
    bcsr_free(&h->A);
    delete h;
    return rc;
  }
  *out = h;
  return 0;
}

int subfv_bcsr_destroy(subfv_bcsr* h) {
  if (!h) return 0;
  cudaFree(h->x);
  cudaFree(h->b);
  cudaFree(h->y);
  gmres_work_free(&h->W);
  bcsr_free(&h->A);
  delete h;
  return 0;
}

int subfv_bcsr_set_values(subfv_bcsr* h, const double* v) { return bcsr_set_values(&h->A, v, false); }

int subfv_bcsr_matmul(subfv_bcsr* h, const double* x, double* y) {
  if (ensure_vecs(h)) return -1;
  const size_t n = (size_t)h->A.m * h->A.bs;
  SUBFV_CUDA(cudaMemcpyAsync(h->x, x, n * sizeof(double), cudaMemcpyHostToDevice, h->A.stream));
  launch_bcsr_spmv(h->A, h->x, h->y, false);
  SUBFV_CUDA(cudaMemcpyAsync(y, h->y, n * sizeof(double), cudaMemcpyDeviceToHost, h->A.stream));
  SUBFV_CUDA(cudaStreamSynchronize(h->A.stream));
  SUBFV_CUDA(cudaGetLastError());
  return 0;
}

int subfv_bcsr_diag(subfv_bcsr* h, double* x, const double* b) {
  if (ensure_vecs(h)) return -1;
  const size_t n = (size_t)h->A.m * h->A.bs;
  SUBFV_CUDA(cudaMemcpyAsync(h->b, b, n * sizeof(double), cudaMemcpyHostToDevice, h->A.stream));
  launch_bcsr_bjacobi(h->A, h->b, h->x);
  SUBFV_CUDA(cudaMemcpyAsync(x, h->x, n * sizeof(double), cudaMemcpyDeviceToHost, h->A.stream));
  SUBFV_CUDA(cudaStreamSynchronize(h->A.stream));
  SUBFV_CUDA(cudaGetLastError());
  return 0;
}

int subfv_bcsr_gmres_ex(subfv_bcsr* h, double* x, const double* b, double tol, int m, int precond, int* conv,
                        int* restarts, double* rho, double* H_first) {
  if (m < 1 || m > 200) {
    set_error("subfv_bcsr_gmres: Krylov dimension must be in [1, 200]");
    return -2;
  }
  if (precond < 0 || precond > 2 || (precond == kPrecondLusgs && h->A.ncs < 1)) {
    set_error("subfv_bcsr_gmres: precond 0, 1 or 2 (2 needs subfv_bcsr_set_colors first)");
    return -2;
  }
  if (ensure_vecs(h) || ensure_work(h, m)) return -1;
  const size_t n = (size_t)h->A.m * h->A.bs;
  SUBFV_CUDA(cudaMemcpyAsync(h->b, b, n * sizeof(double), cudaMemcpyHostToDevice, h->A.stream));
  GmresStats st;
  // maxit: 40 restarts for bcsr_gmres_diag (:1603), 20 for bcsr_gmres and the LU-SGS variant (:205, :898)
  if (gmres_device(h->A, h->W, h->x, h->b, tol, precond, false, precond == kPrecondDiag ? 40 : 20, &st, H_first))
    return -1;
  SUBFV_CUDA(cudaMemcpyAsync(x, h->x, n * sizeof(double), cudaMemcpyDeviceToHost, h->A.stream));
  SUBFV_CUDA(cudaStreamSynchronize(h->A.stream));
  if (conv) *conv = st.conv;
  if (restarts) *restarts = st.restarts;
  if (rho) *rho = st.rho;
  return st.conv ? 0 : SUBFV_ERR_GMRES;
}

int subfv_bcsr_set_colors(subfv_bcsr* h, int n_color_sets, const int32_t* color) {
  if (!h || !color) {
    set_error("subfv_bcsr_set_colors: null argument");
    return -2;
  }
  return bcsr_set_colors(&h->A, n_color_sets, color);
}

int subfv_bcsr_parallel_lusgs(subfv_bcsr* h, double* x, const double* b) {
  if (h->A.ncs < 1) {
    set_error("subfv_bcsr_parallel_lusgs: no colouring (subfv_bcsr_set_colors)");
    return -2;
  }
  if (ensure_vecs(h) || ensure_work(h, h->W.krylov > 0 ? h->W.krylov : 1)) return -1;
  const size_t n = (size_t)h->A.m * h->A.bs;
  SUBFV_CUDA(cudaMemcpyAsync(h->b, b, n * sizeof(double), cudaMemcpyHostToDevice, h->A.stream));
  launch_bcsr_lusgs(h->A, h->b, h->x, h->W.ty);
  SUBFV_CUDA(cudaMemcpyAsync(x, h->x, n * sizeof(double), cudaMemcpyDeviceToHost, h->A.stream));
  SUBFV_CUDA(cudaStreamSynchronize(h->A.stream));
  SUBFV_CUDA(cudaGetLastError());
  return 0;
}

int subfv_bcsr_gmres_parallel_lusgs(subfv_bcsr* h, double* x, const double* b, double tol, int m, int* conv,
                                    int* restarts, double* rho) {
  return subfv_bcsr_gmres_ex(h, x, b, tol, m, kPrecondLusgs, conv, restarts, rho, nullptr);
}

int subfv_bcsr_pcgm(subfv_bcsr* h, double* x, const double* b, double tol, int* iters, double* res) {
  if (!h || !x || !b) {
    set_error("subfv_bcsr_pcgm: null argument");
    return -2;
  }
  if (ensure_vecs(h) || ensure_work(h, h->W.krylov > 0 ? h->W.krylov : 1)) return -1;
  const size_t n = (size_t)h->A.m * h->A.bs;
  SUBFV_CUDA(cudaMemcpyAsync(h->b, b, n * sizeof(double), cudaMemcpyHostToDevice, h->A.stream));
  SUBFV_CUDA(cudaMemcpyAsync(h->x, x, n * sizeof(double), cudaMemcpyHostToDevice, h->A.stream));
  PcgStats st;
  if (pcg_device(h->A, h->W, h->x, h->b, tol, &st)) return -1;
  SUBFV_CUDA(cudaMemcpyAsync(x, h->x, n * sizeof(double), cudaMemcpyDeviceToHost, h->A.stream));
  SUBFV_CUDA(cudaStreamSynchronize(h->A.stream));
  if (iters) *iters = st.iters;
  if (res) *res = st.res;
  if (st.status == 2) return SUBFV_ERR_NONFINITE;
  return st.status ? SUBFV_ERR_GMRES : 0;
}

int subfv_bcsr_gmres_diag(subfv_bcsr* h, double* x, const double* b, double tol, int m, int* conv, int* restarts,
                          double* rho) {
  return subfv_bcsr_gmres_ex(h, x, b, tol, m, 1, conv, restarts, rho, nullptr);
}
int subfv_bcsr_gmres(subfv_bcsr* h, double* x, const double* b, double tol, int m, int* conv, int* restarts,
                     double* rho) {
  return subfv_bcsr_gmres_ex(h, x, b, tol, m, 0, conv, restarts, rho, nullptr);
}

int subfv_bcsr_gmres_refine(subfv_bcsr* h, double* x, const double* b, double rel_tol, int m, int* conv,
                            int* outer, double* rho) {
  if (ensure_vecs(h) || ensure_work(h, m)) return -1;
  const size_t n = (size_t)h->A.m * h->A.bs;
  SUBFV_CUDA(cudaMemcpyAsync(h->b, b, n * sizeof(double), cudaMemcpyHostToDevice, h->A.stream));
  GmresStats st;
  if (gmres_refine_device(h->A, h->W, h->x, h->b, rel_tol, 1e-4, 30, &st)) return -1;
  SUBFV_CUDA(cudaMemcpyAsync(x, h->x, n * sizeof(double), cudaMemcpyDeviceToHost, h->A.stream));
  SUBFV_CUDA(cudaStreamSynchronize(h->A.stream));
  if (conv) *conv = st.conv;
  if (outer) *outer = st.outer;
  if (rho) *rho = st.rho;
  return st.conv ? 0 : SUBFV_ERR_GMRES;
}

int subfv_bcsr_profile_spmv(subfv_bcsr* h, int n_iter, int fp32, double* ms_per_spmv) {
  if (ensure_vecs(h)) return -1;
  const size_t n = (size_t)h->A.m * h->A.bs;
  SUBFV_CUDA(cudaMemsetAsync(h->x, 0, n * sizeof(double), h->A.stream));
  cudaEvent_t e0, e1;
  SUBFV_CUDA(cudaEventCreate(&e0));
  SUBFV_CUDA(cudaEventCreate(&e1));
  launch_bcsr_spmv(h->A, h->x, h->y, fp32 != 0);
  SUBFV_CUDA(cudaEventRecord(e0, h->A.stream));
  for (int i = 0; i < n_iter; ++i) launch_bcsr_spmv(h->A, h->x, h->y, fp32 != 0);
  SUBFV_CUDA(cudaEventRecord(e1, h->A.stream));
  SUBFV_CUDA(cudaEventSynchronize(e1));
  float ms = 0.f;
  SUBFV_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *ms_per_spmv = ms / n_iter;
  SUBFV_CUDA(cudaGetLastError());
  return 0;
}

}  // extern "C"
