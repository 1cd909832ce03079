// BCSR SpMV, block-Jacobi application and restarted GMRES on the GPU.
// Reference: src/linear_algebra/sparse_bcsr_linear_module.F90 bcsr_matmul (:13-29),
// bcsr_diag (:1414-1436) with lu_solve_noswp (linear_solver_module.F90:413-445),
// modifiedArnoldi(_diag) and bcsr_gmres(_diag) (:194-340, :1568-1691).
//
// * SpMV: a group of bs lanes per block row, lane r owns row component r and walks the
//   row's blocks in order; each block's product is summed over its columns first, then
//   added, exactly as y(blk) = y(blk) + matmul(v(:,:,j), x(blk(col(j)))). Bit-identical.
// * block Jacobi: the no-pivot LU of each diagonal block is factored once per matrix
//   (multipliers and upper factor kept), then applied with the same operations and order
//   as lu_solve_noswp. Bit-identical.
// * dot products and norms: a fixed grid of 592 blocks x 256 threads (4 per SM); each
//   thread sums a fixed strided slice, each block a fixed warp-shuffle tree, and the
//   consumer of the block partials (every block of the next kernel, or one finishing
//   block) sums them with the same fixed tree. Deterministic run to run; not the
//   reference's left-to-right order.
// * Gram-Schmidt (modified, as the reference's): the axpy of step i is fused with the dot
//   product of step i+1, so one Arnoldi column of step j costs j passes over the vectors.
// * One restart cycle's Arnoldi process (m columns) has no host decision in it: it is
//   captured once per matrix and workspace as a CUDA graph and replayed.
// * Givens rotations and the back substitution run on the host in the reference's order.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "bcsr.cuh"

namespace subfv {

namespace {

constexpr int kRedBlocks = 592;  // 4 x 148 SMs
constexpr int kRedThreads = 256;

// Four blocks of the row are in flight at once (their column indices, values and x
// entries are loaded before any product); the arithmetic order is unchanged.
template <int BS, class MT>
__global__ void __launch_bounds__(128) k_spmv(int m, const int* __restrict__ row, const int* __restrict__ col,
                                              const MT* __restrict__ v, const double* __restrict__ x,
                                              double* __restrict__ y) {
  constexpr int GPW = 32 / BS;
  constexpr int U = 4;
  const int lane = threadIdx.x & 31;
  if (lane >= GPW * BS) return;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int i = warp * GPW + lane / BS;
  const int r = lane % BS;
  if (i >= m) return;
  double acc = 0.0;
  const int je = row[i + 1];
  for (int j = row[i]; j < je; j += U) {
    int cc[U];
    MT bv[U][BS];
    double xv[U][BS];
#pragma unroll
    for (int u = 0; u < U; ++u) cc[u] = j + u < je ? col[j + u] : -1;
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const MT* blk = v + (size_t)BS * BS * (j + u);
#pragma unroll
      for (int c = 0; c < BS; ++c) bv[u][c] = cc[u] >= 0 ? blk[r + BS * c] : MT(0);
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const double* xc = x + (size_t)BS * (cc[u] >= 0 ? cc[u] : 0);
#pragma unroll
      for (int c = 0; c < BS; ++c) xv[u][c] = cc[u] >= 0 ? xc[c] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (cc[u] < 0) break;
      double t = 0.0;
#pragma unroll
      for (int c = 0; c < BS; ++c) t = t + (double)bv[u][c] * xv[u][c];
      acc = acc + t;
    }
  }
  y[(size_t)BS * i + r] = acc;
}

// The no-pivot LU of each diagonal block, packed in one block (multipliers below the
// diagonal, the upper factor on and above it) and stored element-major: entry q of
// block row i at lu[q * m + i], so that a thread per block row reads coalesced.
template <int BS>
__global__ void k_factor_diag(int m, const int* __restrict__ diag, const double* __restrict__ v,
                              double* __restrict__ lu) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  double C[BS * BS];
  const int dj = diag[i];
  for (int q = 0; q < BS * BS; ++q)
    C[q] = dj >= 0 ? v[(size_t)BS * BS * dj + q] : (q % (BS + 1) == 0 ? 1.0 : 0.0);
  for (int k = 0; k < BS; ++k) {
    const double invdiag = 1.0 / C[k + BS * k];
    for (int ii = k + 1; ii < BS; ++ii) {
      const double lik = C[ii + BS * k] * invdiag;
      for (int jj = k + 1; jj < BS; ++jj) C[ii + BS * jj] = C[ii + BS * jj] - lik * C[k + BS * jj];
      C[ii + BS * k] = lik;
    }
  }
  for (int q = 0; q < BS * BS; ++q) lu[(size_t)q * m + i] = C[q];
}

// xv = D_i^-1 xv with the packed no-pivot LU of block row i (lu_solve_noswp's operations)
template <int BS>
__device__ inline void lu_apply(const double* __restrict__ lu, int m, int i, double* xv) {
  double C[BS * BS];
#pragma unroll
  for (int q = 0; q < BS * BS; ++q) C[q] = lu[(size_t)q * m + i];
#pragma unroll
  for (int k = 0; k < BS; ++k)
#pragma unroll
    for (int ii = k + 1; ii < BS; ++ii) xv[ii] = xv[ii] - C[ii + BS * k] * xv[k];
  xv[BS - 1] = xv[BS - 1] / C[(BS - 1) + BS * (BS - 1)];
#pragma unroll
  for (int k = BS - 2; k >= 0; --k) {
#pragma unroll
    for (int j = k + 1; j < BS; ++j) xv[k] = xv[k] - C[k + BS * j] * xv[j];
    xv[k] = xv[k] / C[k + BS * k];
  }
}

template <int BS>
__global__ void k_bjacobi(int m, const double* __restrict__ lu, const double* __restrict__ b,
                          double* __restrict__ x) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  double xv[BS];
#pragma unroll
  for (int k = 0; k < BS; ++k) xv[k] = b[(size_t)BS * i + k];
  lu_apply<BS>(lu, m, i, xv);
#pragma unroll
  for (int k = 0; k < BS; ++k) x[(size_t)BS * i + k] = xv[k];
}

// lu_solve (linear_solver_module.F90:447-484) on block row i's diagonal block: partial
// pivoting on the first largest |C(k:n, k)|, whole rows swapped; a pivot below 1e-12 at
// the last step (where the reference stops) sets bit 2 of *flag and skips the back
// substitution
template <int BS>
__global__ void k_pivot_diag(int m, const int* __restrict__ diag, const double* __restrict__ v,
                             const double* __restrict__ r, double* __restrict__ mr, unsigned* flag) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const int dj = diag[i];
  double C[BS * BS], x[BS];
  for (int q = 0; q < BS * BS; ++q) C[q] = dj >= 0 ? v[(size_t)BS * BS * dj + q] : (q % (BS + 1) == 0 ? 1.0 : 0.0);
  for (int k = 0; k < BS; ++k) x[k] = r[(size_t)BS * i + k];
  for (int k = 0; k < BS; ++k) {
    int p = k;
    for (int ii = k + 1; ii < BS; ++ii)
      if (fabs(C[ii + BS * k]) > fabs(C[p + BS * k])) p = ii;
    for (int j = 0; j < BS; ++j) {
      const double t = C[k + BS * j];
      C[k + BS * j] = C[p + BS * j];
      C[p + BS * j] = t;
    }
    const double tx = x[k];
    x[k] = x[p];
    x[p] = tx;
    const double invdiag = 1.0 / C[k + BS * k];
    for (int ii = k + 1; ii < BS; ++ii) {
      const double lik = C[ii + BS * k] * invdiag;
      for (int j = k; j < BS; ++j) C[ii + BS * j] = C[ii + BS * j] - lik * C[k + BS * j];
      x[ii] = x[ii] - lik * x[k];
    }
  }
  if (fabs(C[BS * BS - 1]) < 1e-12) {
    atomicOr(flag, 2u);
  } else {
    x[BS - 1] = x[BS - 1] / C[BS * BS - 1];
    for (int k = BS - 2; k >= 0; --k) {
      for (int j = k + 1; j < BS; ++j) x[k] = x[k] - C[k + BS * j] * x[j];
      x[k] = x[k] / C[k + BS * k];
    }
  }
  for (int k = 0; k < BS; ++k) mr[(size_t)BS * i + k] = x[k];
}

// x += a p; r -= a q; p = z + b p (conjugate gradients, bcsr_pcgm's vector updates)
__global__ void k_cg_update(double* __restrict__ x, double* __restrict__ r, const double* __restrict__ p,
                            const double* __restrict__ q, double a, long n) {
  const long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  x[k] = x[k] + a * p[k];
  r[k] = r[k] - a * q[k];
}
__global__ void k_cg_dir(double* __restrict__ p, const double* __restrict__ z, double beta, long n) {
  const long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) p[k] = z[k] + beta * p[k];
}

// The sweeps use BS lanes per block row, as the SpMV does (lane r owns component r, and
// the row's blocks are walked in order, each product summed over its columns first);
// the backward sweep then gathers the row's components by shuffles and every lane of
// the group applies the diagonal LU to the whole block, keeping its own component.
template <int BS, bool FWD>
__device__ inline double lusgs_lane(const int* __restrict__ row, const int* __restrict__ col,
                                    const double* __restrict__ v, const int* __restrict__ color, int cs, int i, int r,
                                    const double* u, double acc) {
  for (int j = row[i]; j < row[i + 1]; ++j) {
    const int c = col[j];
    const int cc = color[c];
    if (FWD ? !(cc < cs) : !(cc > cs)) continue;
    const double* blk = v + (size_t)BS * BS * j;
    const double* uc = u + (size_t)BS * c;
    double t = 0.0;
#pragma unroll
    for (int k = 0; k < BS; ++k) t = t + blk[r + BS * k] * uc[k];
    acc = acc - t;
  }
  return acc;
}

// forward sweep of colour set cs: y_i = b_i - sum over lower colours of A_ij y_j
template <int BS>
__global__ void __launch_bounds__(128) k_lusgs_fwd(int nrows, const int* __restrict__ rows,
                                                   const int* __restrict__ row, const int* __restrict__ col,
                                                   const double* __restrict__ v, const int* __restrict__ color,
                                                   int cs, const double* __restrict__ b, double* y) {
  constexpr int GPW = 32 / BS;
  const int lane = threadIdx.x & 31;
  if (lane >= GPW * BS) return;
  const int t = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * GPW + lane / BS;
  if (t >= nrows) return;
  const int i = rows[t], r = lane % BS;
  y[(size_t)BS * i + r] = lusgs_lane<BS, true>(row, col, v, color, cs, i, r, y, b[(size_t)BS * i + r]);
}
// backward sweep of colour set cs: x_i = D_i^-1 (y_i - sum over higher colours of A_ij x_j)
template <int BS>
__global__ void __launch_bounds__(128) k_lusgs_bwd(int nrows, const int* __restrict__ rows,
                                                   const int* __restrict__ row, const int* __restrict__ col,
                                                   const double* __restrict__ v, const int* __restrict__ color,
                                                   int cs, const double* __restrict__ lu, int m,
                                                   const double* __restrict__ y, double* x) {
  constexpr int GPW = 32 / BS;
  const int lane = threadIdx.x & 31;
  const int g = lane / BS, r = lane % BS;
  const int t = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * GPW + g;
  const bool live = lane < GPW * BS && t < nrows;  // every lane joins the shuffles
  const int i = live ? rows[t] : 0;
  double xr = 0.0;
  if (live) xr = lusgs_lane<BS, false>(row, col, v, color, cs, i, r, x, y[(size_t)BS * i + r]);
  double xv[BS];
#pragma unroll
  for (int k = 0; k < BS; ++k) xv[k] = __shfl_sync(0xffffffffu, xr, (lane < GPW * BS ? g * BS : 0) + k);
  if (!live) return;
  lu_apply<BS>(lu, m, i, xv);
  x[(size_t)BS * i + r] = xv[r];
}

__device__ inline double warp_tree(double v) {
  for (int o = 16; o > 0; o >>= 1) v = v + __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

__device__ inline double block_sum(double v) {
  __shared__ double sh[kRedThreads / 32];
  v = warp_tree(v);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < kRedThreads / 32; ++w) s = s + sh[w];
  return s;  // valid in thread 0
}

// sum of the nb block partials by a fixed tree (thread slices, warp shuffles, warps in
// order); every block that calls it gets the same value. Returned to all threads.
__device__ inline double sum_partials(const double* __restrict__ p, int nb) {
  __shared__ double sh[kRedThreads / 32];
  __shared__ double tot;
  double v = 0.0;
  for (int q = threadIdx.x; q < nb; q += kRedThreads) v = v + p[q];
  v = warp_tree(v);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < kRedThreads / 32; ++w) s = s + sh[w];
    tot = s;
  }
  __syncthreads();
  return tot;
}

constexpr int kUnroll = 4;

// partial[b] = sum over the block's fixed slice of a*b
__global__ void __launch_bounds__(kRedThreads) k_dot(const double* __restrict__ a, const double* __restrict__ b,
                                                     long n, double* __restrict__ partial) {
  const long T = (long)gridDim.x * blockDim.x;
  long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
  double s = 0.0;
  for (; k + (kUnroll - 1) * T < n; k += kUnroll * T) {
    double av[kUnroll], bv[kUnroll];
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      av[u] = a[k + u * T];
      bv[u] = b[k + u * T];
    }
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) s = s + av[u] * bv[u];
  }
  for (; k < n; k += T) s = s + a[k] * b[k];
  s = block_sum(s);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

// *out = the fixed-tree sum of the partials (one block)
__global__ void __launch_bounds__(kRedThreads) k_finish(const double* __restrict__ pin, int nb, double* out) {
  const double s = sum_partials(pin, nb);
  if (threadIdx.x == 0) *out = s;
}

// h = sum(pin); y -= h*x; then pout = partial dot(y_new, nx), or of y_new with itself
// when nx is null (the squared norm that closes a Gram-Schmidt column). Block 0 stores h.
__global__ void __launch_bounds__(kRedThreads) k_axpy_dot(double* __restrict__ y, const double* __restrict__ x,
                                                          const double* __restrict__ pin, int nb, double* hout,
                                                          const double* __restrict__ nx, double* __restrict__ pout,
                                                          long n) {
  const double h = sum_partials(pin, nb);
  if (blockIdx.x == 0 && threadIdx.x == 0 && hout) *hout = h;
  const long T = (long)gridDim.x * blockDim.x;
  long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
  double s = 0.0;
  if (nx) {
    for (; k + (kUnroll - 1) * T < n; k += kUnroll * T) {
      double yv[kUnroll], xv[kUnroll], nv[kUnroll];
#pragma unroll
      for (int u = 0; u < kUnroll; ++u) {
        yv[u] = y[k + u * T];
        xv[u] = x[k + u * T];
        nv[u] = nx[k + u * T];
      }
#pragma unroll
      for (int u = 0; u < kUnroll; ++u) {
        const double yk = yv[u] - h * xv[u];
        y[k + u * T] = yk;
        s = s + yk * nv[u];
      }
    }
    for (; k < n; k += T) {
      const double yk = y[k] - h * x[k];
      y[k] = yk;
      s = s + yk * nx[k];
    }
  } else {
    for (; k + (kUnroll - 1) * T < n; k += kUnroll * T) {
      double yv[kUnroll], xv[kUnroll];
#pragma unroll
      for (int u = 0; u < kUnroll; ++u) {
        yv[u] = y[k + u * T];
        xv[u] = x[k + u * T];
      }
#pragma unroll
      for (int u = 0; u < kUnroll; ++u) {
        const double yk = yv[u] - h * xv[u];
        y[k + u * T] = yk;
        s = s + yk * yk;
      }
    }
    for (; k < n; k += T) {
      const double yk = y[k] - h * x[k];
      y[k] = yk;
      s = s + yk * yk;
    }
  }
  s = block_sum(s);
  if (threadIdx.x == 0) pout[blockIdx.x] = s;
}

// nrm = sqrt(sum(pin)); y = src / nrm (src may be y); block 0 stores nrm at *hout
__global__ void __launch_bounds__(kRedThreads) k_normalize(const double* src, double* y, const double* __restrict__ pin,
                                                           int nb, double* hout, long n) {
  const double h = sqrt(sum_partials(pin, nb));
  if (blockIdx.x == 0 && threadIdx.x == 0) *hout = h;
  const long T = (long)gridDim.x * blockDim.x;
  for (long k = (long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += T) y[k] = src[k] / h;
}

__global__ void k_sub(const double* __restrict__ b, const double* __restrict__ w, double* __restrict__ r, long n) {
  const long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) r[k] = b[k] - w[k];
}
__global__ void k_add(double* __restrict__ x, const double* __restrict__ d, long n) {
  const long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) x[k] = x[k] + d[k];
}
// out = base + sum_i z_i V_i, summed left to right from base (base may alias out)
__global__ void k_lincomb(const double* __restrict__ V, long n, const double* __restrict__ z, int nr,
                          const double* base, double* out) {
  const long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  double acc = base ? base[k] : 0.0;
  for (int i = 0; i < nr; ++i) acc = acc + z[i] * V[(size_t)i * n + k];
  out[k] = acc;
}
__global__ void k_d2f(const double* __restrict__ a, float* __restrict__ b, size_t n) {
  const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) b[k] = (float)a[k];
}

int egrid(long n) { return (int)((n + 255) / 256); }

}  // namespace

int bcsr_upload(DevBcsr* A, int m, int bs, const int* row1, const int* col1, const double* v, cudaStream_t s) {
  if (m <= 0 || bs < 1 || bs > kBcsrMaxBs || (bs != 5 && bs != 4 && bs != 1 && bs != 3)) {
    set_error("subfv_bcsr: supported block sizes are 1, 3, 4 and 5");
    return -2;
  }
  const int nnz = row1[m] - 1;
  std::vector<int> row(m + 1), col(nnz), diag(m, -1);
  for (int i = 0; i <= m; ++i) row[i] = row1[i] - 1;
  for (int j = 0; j < nnz; ++j) {
    col[j] = col1[j] - 1;
    if (col[j] < 0 || col[j] >= m) {
      set_error("subfv_bcsr: column index out of range");
      return -2;
    }
  }
  for (int i = 0; i < m; ++i)
    for (int j = row[i]; j < row[i + 1]; ++j)
      if (col[j] == i) {
        diag[i] = j;
        break;
      }
  A->m = m;
  A->bs = bs;
  A->nnz = nnz;
  if (s) {
    A->stream = s;
  } else {
    SUBFV_CUDA(cudaStreamCreateWithFlags(&A->stream, cudaStreamNonBlocking));
    A->own_stream = true;
  }
  const size_t vb = (size_t)bs * bs * std::max(nnz, 1);
  SUBFV_CUDA(cudaMalloc(&A->row, (m + 1) * sizeof(int)));
  SUBFV_CUDA(cudaMalloc(&A->col, std::max(nnz, 1) * sizeof(int)));
  SUBFV_CUDA(cudaMalloc(&A->diag, m * sizeof(int)));
  SUBFV_CUDA(cudaMalloc(&A->v, vb * sizeof(double)));
  SUBFV_CUDA(cudaMalloc(&A->v32, vb * sizeof(float)));
  SUBFV_CUDA(cudaMalloc(&A->lu, (size_t)bs * bs * m * sizeof(double)));
  A->bytes = (m + 1 + nnz + m) * sizeof(int) + vb * 12 + (size_t)bs * bs * m * 8;
  SUBFV_CUDA(cudaMemcpyAsync(A->row, row.data(), (m + 1) * sizeof(int), cudaMemcpyHostToDevice, A->stream));
  SUBFV_CUDA(cudaMemcpyAsync(A->col, col.data(), nnz * sizeof(int), cudaMemcpyHostToDevice, A->stream));
  SUBFV_CUDA(cudaMemcpyAsync(A->diag, diag.data(), m * sizeof(int), cudaMemcpyHostToDevice, A->stream));
  SUBFV_CUDA(cudaStreamSynchronize(A->stream));
  if (v) return bcsr_set_values(A, v, false);
  return 0;
}

int bcsr_set_values(DevBcsr* A, const double* v, bool on_device) {
  const size_t vb = (size_t)A->bs * A->bs * A->nnz;
  if (v != A->v)
    SUBFV_CUDA(cudaMemcpyAsync(A->v, v, vb * sizeof(double), on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                               A->stream));
  k_d2f<<<(int)((vb + 255) / 256), 256, 0, A->stream>>>(A->v, A->v32, vb);
  launch_bcsr_factor_diag(*A);
  SUBFV_CUDA(cudaGetLastError());
  SUBFV_CUDA(cudaStreamSynchronize(A->stream));
  return 0;
}

void bcsr_free(DevBcsr* A) {
  void* p[] = {A->row, A->col, A->v, A->v32, A->diag, A->lu, A->color, A->set_rows};
  for (void* q : p)
    if (q) cudaFree(q);
  if (A->own_stream && A->stream) cudaStreamDestroy(A->stream);
  *A = DevBcsr();
}

int gmres_work_alloc(GmresWork* W, long n, int krylov) {
  W->n = n;
  W->krylov = krylov;
  SUBFV_CUDA(cudaMalloc(&W->V, (size_t)n * (krylov + 1) * sizeof(double)));
  SUBFV_CUDA(cudaMalloc(&W->r, n * sizeof(double)));
  SUBFV_CUDA(cudaMalloc(&W->w, n * sizeof(double)));
  SUBFV_CUDA(cudaMalloc(&W->zp, n * sizeof(double)));
  SUBFV_CUDA(cudaMalloc(&W->d, n * sizeof(double)));
  SUBFV_CUDA(cudaMalloc(&W->rr, n * sizeof(double)));
  SUBFV_CUDA(cudaMalloc(&W->ty, n * sizeof(double)));
  SUBFV_CUDA(cudaMalloc(&W->z, (krylov + 2) * sizeof(double)));
  SUBFV_CUDA(cudaMalloc(&W->partial, 2 * kRedBlocks * sizeof(double)));
  SUBFV_CUDA(cudaMalloc(&W->H, (size_t)(krylov + 1) * krylov * sizeof(double)));
  SUBFV_CUDA(cudaMalloc(&W->scal, 8 * sizeof(double)));
  W->bytes = (size_t)n * (krylov + 7) * 8;
  return 0;
}

void gmres_work_free(GmresWork* W) {
  if (W->cycle) cudaGraphExecDestroy(W->cycle);
  void* p[] = {W->V, W->r, W->w, W->zp, W->z, W->partial, W->H, W->scal, W->d, W->rr, W->ty};
  for (void* q : p)
    if (q) cudaFree(q);
  *W = GmresWork();
}

void launch_bcsr_spmv(const DevBcsr& A, const double* x, double* y, bool fp32) {
  const int gpw = 32 / A.bs;
  const long warps = (A.m + gpw - 1) / gpw;
  const int grid = (int)((warps * 32 + 127) / 128);
  switch (A.bs) {
    case 5:
      if (fp32) k_spmv<5, float><<<grid, 128, 0, A.stream>>>(A.m, A.row, A.col, A.v32, x, y);
      else k_spmv<5, double><<<grid, 128, 0, A.stream>>>(A.m, A.row, A.col, A.v, x, y);
      break;
    case 4:
      if (fp32) k_spmv<4, float><<<grid, 128, 0, A.stream>>>(A.m, A.row, A.col, A.v32, x, y);
      else k_spmv<4, double><<<grid, 128, 0, A.stream>>>(A.m, A.row, A.col, A.v, x, y);
      break;
    case 3:
      if (fp32) k_spmv<3, float><<<grid, 128, 0, A.stream>>>(A.m, A.row, A.col, A.v32, x, y);
      else k_spmv<3, double><<<grid, 128, 0, A.stream>>>(A.m, A.row, A.col, A.v, x, y);
      break;
    default:
      if (fp32) k_spmv<1, float><<<grid, 128, 0, A.stream>>>(A.m, A.row, A.col, A.v32, x, y);
      else k_spmv<1, double><<<grid, 128, 0, A.stream>>>(A.m, A.row, A.col, A.v, x, y);
  }
}

void launch_bcsr_factor_diag(const DevBcsr& A) {
  const int g = (A.m + 127) / 128;
  switch (A.bs) {
    case 5: k_factor_diag<5><<<g, 128, 0, A.stream>>>(A.m, A.diag, A.v, A.lu); break;
    case 4: k_factor_diag<4><<<g, 128, 0, A.stream>>>(A.m, A.diag, A.v, A.lu); break;
    case 3: k_factor_diag<3><<<g, 128, 0, A.stream>>>(A.m, A.diag, A.v, A.lu); break;
    default: k_factor_diag<1><<<g, 128, 0, A.stream>>>(A.m, A.diag, A.v, A.lu);
  }
}

void launch_bcsr_bjacobi(const DevBcsr& A, const double* b, double* x) {
  const int g = (A.m + 127) / 128;
  switch (A.bs) {
    case 5: k_bjacobi<5><<<g, 128, 0, A.stream>>>(A.m, A.lu, b, x); break;
    case 4: k_bjacobi<4><<<g, 128, 0, A.stream>>>(A.m, A.lu, b, x); break;
    case 3: k_bjacobi<3><<<g, 128, 0, A.stream>>>(A.m, A.lu, b, x); break;
    default: k_bjacobi<1><<<g, 128, 0, A.stream>>>(A.m, A.lu, b, x);
  }
}

double device_norm2(const DevBcsr& A, GmresWork& W, const double* x, long n) {
  k_dot<<<kRedBlocks, kRedThreads, 0, A.stream>>>(x, x, n, W.partial);
  k_finish<<<1, kRedThreads, 0, A.stream>>>(W.partial, kRedBlocks, W.scal + 1);
  double s = 0.0;
  if (cudaMemcpyAsync(&s, W.scal + 1, sizeof(double), cudaMemcpyDeviceToHost, A.stream) != cudaSuccess ||
      cudaStreamSynchronize(A.stream) != cudaSuccess) {
    set_error("device_norm2: CUDA error");
    return -1.0;
  }
  return std::sqrt(s);
}

namespace {
// blocks of 128 threads (4 warps of 32 / bs row groups) covering n rows
int lusgs_grid(int bs, int n) {
  const int gpw = 32 / bs;
  const long warps = (n + gpw - 1) / gpw;
  return (int)((warps * 32 + 127) / 128);
}
}  // namespace

void launch_bcsr_lusgs(const DevBcsr& A, const double* b, double* x, double* ty) {
  for (int cs = 1; cs <= A.ncs; ++cs) {
    const int o = A.set_off[cs - 1], n = A.set_off[cs] - o;
    if (n == 0) continue;
    const int g = lusgs_grid(A.bs, n);
    switch (A.bs) {
      case 5: k_lusgs_fwd<5><<<g, 128, 0, A.stream>>>(n, A.set_rows + o, A.row, A.col, A.v, A.color, cs, b, ty); break;
      case 4: k_lusgs_fwd<4><<<g, 128, 0, A.stream>>>(n, A.set_rows + o, A.row, A.col, A.v, A.color, cs, b, ty); break;
      case 3: k_lusgs_fwd<3><<<g, 128, 0, A.stream>>>(n, A.set_rows + o, A.row, A.col, A.v, A.color, cs, b, ty); break;
      default: k_lusgs_fwd<1><<<g, 128, 0, A.stream>>>(n, A.set_rows + o, A.row, A.col, A.v, A.color, cs, b, ty);
    }
  }
  for (int cs = A.ncs; cs >= 1; --cs) {
    const int o = A.set_off[cs - 1], n = A.set_off[cs] - o;
    if (n == 0) continue;
    const int g = lusgs_grid(A.bs, n);
    switch (A.bs) {
      case 5:
        k_lusgs_bwd<5><<<g, 128, 0, A.stream>>>(n, A.set_rows + o, A.row, A.col, A.v, A.color, cs, A.lu, A.m, ty, x);
        break;
      case 4:
        k_lusgs_bwd<4><<<g, 128, 0, A.stream>>>(n, A.set_rows + o, A.row, A.col, A.v, A.color, cs, A.lu, A.m, ty, x);
        break;
      case 3:
        k_lusgs_bwd<3><<<g, 128, 0, A.stream>>>(n, A.set_rows + o, A.row, A.col, A.v, A.color, cs, A.lu, A.m, ty, x);
        break;
      default:
        k_lusgs_bwd<1><<<g, 128, 0, A.stream>>>(n, A.set_rows + o, A.row, A.col, A.v, A.color, cs, A.lu, A.m, ty, x);
    }
  }
}

int bcsr_set_colors(DevBcsr* A, int ncs, const int* color) {
  if (ncs < 1 || ncs > A->m) {
    set_error("subfv_bcsr_set_colors: the number of colour sets must be in [1, m]");
    return -2;
  }
  std::vector<int> cnt(ncs + 1, 0);
  for (int i = 0; i < A->m; ++i) {
    if (color[i] < 1 || color[i] > ncs) {
      set_error("subfv_bcsr_set_colors: colour out of [1, n_color_sets]");
      return -2;
    }
    cnt[color[i]]++;
  }
  std::vector<int> off(ncs + 1, 0), rows(A->m);
  for (int c = 1; c <= ncs; ++c) off[c] = off[c - 1] + cnt[c];
  std::vector<int> fill(off.begin(), off.end() - 1);
  for (int i = 0; i < A->m; ++i) rows[fill[color[i] - 1]++] = i;  // ascending rows within a set
  if (A->color) cudaFree(A->color);
  if (A->set_rows) cudaFree(A->set_rows);
  A->color = A->set_rows = nullptr;
  SUBFV_CUDA(cudaMalloc(&A->color, A->m * sizeof(int)));
  SUBFV_CUDA(cudaMalloc(&A->set_rows, A->m * sizeof(int)));
  SUBFV_CUDA(cudaMemcpyAsync(A->color, color, A->m * sizeof(int), cudaMemcpyHostToDevice, A->stream));
  SUBFV_CUDA(cudaMemcpyAsync(A->set_rows, rows.data(), A->m * sizeof(int), cudaMemcpyHostToDevice, A->stream));
  SUBFV_CUDA(cudaStreamSynchronize(A->stream));
  A->ncs = ncs;
  A->set_off = off;
  return 0;
}

namespace {
// One restart cycle's Arnoldi process: V_1 = r/|r| (|r|^2 from the partials that the
// preceding device_norm2 left in W.partial), then columns 2..m+1 with modified
// Gram-Schmidt, H on the device. Launch-only (no host decision), so it can be captured.
void arnoldi_cycle(const DevBcsr& A, GmresWork& W, int precond, bool fp32) {
  const int m = W.krylov;
  const long n = W.n;
  cudaStream_t s = A.stream;
  double* pa = W.partial;
  double* pb = W.partial + kRedBlocks;
  auto Vc = [&](int j) { return W.V + (size_t)(j - 1) * n; };  // 1-based
  auto Hd = [&](int i, int j) { return W.H + (i - 1) + (size_t)(m + 1) * (j - 1); };
  cudaMemsetAsync(W.H, 0, (size_t)(m + 1) * m * sizeof(double), s);
  k_normalize<<<kRedBlocks, kRedThreads, 0, s>>>(W.r, Vc(1), pa, kRedBlocks, W.scal, n);
  for (int jj = 2; jj <= m + 1; ++jj) {
    if (precond) {
      if (precond == kPrecondLusgs) launch_bcsr_lusgs(A, Vc(jj - 1), W.zp, W.ty);
      else launch_bcsr_bjacobi(A, Vc(jj - 1), W.zp);
      launch_bcsr_spmv(A, W.zp, Vc(jj), fp32);
    } else {
      launch_bcsr_spmv(A, Vc(jj - 1), Vc(jj), fp32);
    }
    k_dot<<<kRedBlocks, kRedThreads, 0, s>>>(Vc(1), Vc(jj), n, pa);
    for (int i = 1; i <= jj - 1; ++i) {
      const double* nx = i < jj - 1 ? Vc(i + 1) : nullptr;  // the last one is |V_jj|^2
      k_axpy_dot<<<kRedBlocks, kRedThreads, 0, s>>>(Vc(jj), Vc(i), pa, kRedBlocks, Hd(i, jj - 1), nx, pb, n);
      std::swap(pa, pb);
    }
    k_normalize<<<kRedBlocks, kRedThreads, 0, s>>>(Vc(jj), Vc(jj), pa, kRedBlocks, Hd(jj, jj - 1), n);
  }
}

// Replays the cycle from a graph captured for this matrix, workspace and mode.
int run_arnoldi_cycle(const DevBcsr& A, GmresWork& W, int precond, bool fp32) {
  const uintptr_t key[] = {(uintptr_t)A.row, (uintptr_t)A.col, (uintptr_t)A.v, (uintptr_t)A.v32, (uintptr_t)A.lu,
                           (uintptr_t)A.nnz, (uintptr_t)A.m, (uintptr_t)A.set_rows, (uintptr_t)A.stream,
                           (uintptr_t)precond | (fp32 ? 4 : 0) | ((uintptr_t)A.bs << 3) | ((uintptr_t)A.ncs << 8)};
  static_assert(sizeof(key) == sizeof(W.cycle_key), "cycle key size");
  if (W.cycle && std::memcmp(key, W.cycle_key, sizeof(key)) != 0) {
    cudaGraphExecDestroy(W.cycle);
    W.cycle = nullptr;
  }
  if (!W.cycle) {
    cudaGraph_t g = nullptr;
    SUBFV_CUDA(cudaStreamBeginCapture(A.stream, cudaStreamCaptureModeThreadLocal));
    arnoldi_cycle(A, W, precond, fp32);
    const cudaError_t le = cudaGetLastError();
    const cudaError_t ce = cudaStreamEndCapture(A.stream, &g);
    SUBFV_CUDA(le);
    SUBFV_CUDA(ce);
    const cudaError_t ie = cudaGraphInstantiate(&W.cycle, g, 0);
    cudaGraphDestroy(g);
    SUBFV_CUDA(ie);
    std::memcpy(W.cycle_key, key, sizeof(key));
  }
  SUBFV_CUDA(cudaGraphLaunch(W.cycle, A.stream));
  return 0;
}
}  // namespace

int gmres_device(const DevBcsr& A, GmresWork& W, double* x, const double* b, double tol, int precond, bool fp32,
                 int maxit, GmresStats* st, double* H_first_host) {
  const int m = W.krylov;
  const long n = W.n;
  cudaStream_t s = A.stream;
  std::vector<double> H((size_t)(m + 1) * m), y(m + 1), c(m + 1), sn(m + 1), z(m + 1);
  auto h = [&](int i, int j) -> double& { return H[(i - 1) + (size_t)(m + 1) * (j - 1)]; };
  st->conv = 0;
  SUBFV_CUDA(cudaMemsetAsync(x, 0, n * sizeof(double), s));
  launch_bcsr_spmv(A, x, W.w, fp32);
  k_sub<<<egrid(n), 256, 0, s>>>(b, W.w, W.r, n);
  double rho = device_norm2(A, W, W.r, n);
  if (rho < 0.0) return -1;
  int it = 0;
  // A zero residual is solved by x = 0 whatever tol is; the reference, given tol = 0 (a
  // relative tolerance on b = 0), would divide the residual by its zero norm
  if (rho < tol || rho == 0.0) {
    st->conv = 1;
    st->rho = rho;
    st->restarts = 0;
    return 0;
  }
  for (int j = 1; j <= maxit; ++j) {
    it = j;
    std::fill(y.begin(), y.end(), 0.0);
    y[0] = rho;
    if (run_arnoldi_cycle(A, W, precond, fp32)) return -1;
    SUBFV_CUDA(cudaMemcpyAsync(H.data(), W.H, H.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
    SUBFV_CUDA(cudaStreamSynchronize(s));
    SUBFV_CUDA(cudaGetLastError());
    if (j == 1 && H_first_host) std::memcpy(H_first_host, H.data(), H.size() * sizeof(double));
    int nr = m, i;
    for (i = 1; i <= m; ++i) {  // Givens rotations (:1634-1658)
      for (int k = 2; k <= i; ++k) {
        double tmp = h(k - 1, i);
        h(k - 1, i) = c[k - 2] * h(k - 1, i) + sn[k - 2] * h(k, i);
        h(k, i) = -sn[k - 2] * tmp + c[k - 2] * h(k, i);
      }
      double delta = std::sqrt(h(i, i) * h(i, i) + h(i + 1, i) * h(i + 1, i));
      c[i - 1] = h(i, i) / delta;
      sn[i - 1] = h(i + 1, i) / delta;
      h(i, i) = c[i - 1] * h(i, i) + sn[i - 1] * h(i + 1, i);
      for (int k = i + 1; k <= m + 1; ++k) h(k, i) = 0.0;
      y[i] = -sn[i - 1] * y[i - 1];
      y[i - 1] = c[i - 1] * y[i - 1];
      rho = std::fabs(y[i]);
      if (rho < tol) {
        nr = i + 1;
        break;
      }
    }
    std::fill(z.begin(), z.end(), 0.0);  // back substitution (:1660-1673)
    if (i >= m) {
      nr = m;
      z[nr - 1] = y[nr - 1] / h(nr, nr);
    }
    for (int k = nr - 1; k >= 1; --k) {
      z[k - 1] = y[k - 1];
      for (int l = k + 1; l <= nr; ++l) z[k - 1] = z[k - 1] - h(k, l) * z[l - 1];
      z[k - 1] = z[k - 1] / h(k, k);
    }
    SUBFV_CUDA(cudaMemcpyAsync(W.z, z.data(), nr * sizeof(double), cudaMemcpyHostToDevice, s));
    if (precond) {
      k_lincomb<<<egrid(n), 256, 0, s>>>(W.V, n, W.z, nr, nullptr, W.r);
      if (precond == kPrecondLusgs) launch_bcsr_lusgs(A, W.r, W.zp, W.ty);
      else launch_bcsr_bjacobi(A, W.r, W.zp);
      k_add<<<egrid(n), 256, 0, s>>>(x, W.zp, n);
    } else {
      k_lincomb<<<egrid(n), 256, 0, s>>>(W.V, n, W.z, nr, x, x);
    }
    launch_bcsr_spmv(A, x, W.w, fp32);
    k_sub<<<egrid(n), 256, 0, s>>>(b, W.w, W.r, n);
    rho = device_norm2(A, W, W.r, n);
    if (rho < 0.0) return -1;
    if (rho < tol) {
      if (precond == kPrecondDiag) st->conv = 1;
      break;
    }
  }
  if (precond != kPrecondDiag) {  // bcsr_gmres (:284-289) and bcsr_gmres_parallel_lusgs (:987-992)
    launch_bcsr_spmv(A, x, W.w, fp32);
    k_sub<<<egrid(n), 256, 0, s>>>(b, W.w, W.r, n);
    const double r2 = device_norm2(A, W, W.r, n);
    if (r2 < 0.0) return -1;
    st->conv = !(r2 > tol);
  }
  st->rho = rho;
  st->restarts = it;
  SUBFV_CUDA(cudaGetLastError());
  return 0;
}

int gmres_refine_device(const DevBcsr& A, GmresWork& W, double* x, const double* b, double rel_tol,
                        double inner_rel_tol, int max_outer, GmresStats* st, int precond) {
  const long n = W.n;
  cudaStream_t s = A.stream;
  const double bnorm = device_norm2(A, W, b, n);
  if (bnorm < 0.0) return -1;
  SUBFV_CUDA(cudaMemsetAsync(x, 0, n * sizeof(double), s));
  SUBFV_CUDA(cudaMemcpyAsync(W.rr, b, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
  st->conv = 0;
  st->inner_total = 0;
  double rn = bnorm;
  int outer = 0;
  for (outer = 1; outer <= max_outer; ++outer) {
    if (rn < rel_tol * bnorm || rn == 0.0) {
      st->conv = 1;
      break;
    }
    GmresStats in;
    if (gmres_device(A, W, W.d, W.rr, inner_rel_tol * rn, precond, true, 40, &in, nullptr)) return -1;
    st->inner_total += in.restarts;
    k_add<<<egrid(n), 256, 0, s>>>(x, W.d, n);
    launch_bcsr_spmv(A, x, W.w, false);  // FP64 residual
    k_sub<<<egrid(n), 256, 0, s>>>(b, W.w, W.rr, n);
    rn = device_norm2(A, W, W.rr, n);
    if (rn < 0.0) return -1;
  }
  if (!st->conv && (rn < rel_tol * bnorm || rn == 0.0)) st->conv = 1;
  st->outer = outer - (st->conv ? 1 : 0);
  st->rho = rn;
  SUBFV_CUDA(cudaGetLastError());
  return 0;
}

namespace {
double device_dot(const DevBcsr& A, GmresWork& W, const double* a, const double* b, long n) {
  k_dot<<<kRedBlocks, kRedThreads, 0, A.stream>>>(a, b, n, W.partial);
  k_finish<<<1, kRedThreads, 0, A.stream>>>(W.partial, kRedBlocks, W.scal + 1);
  double s = 0.0;
  if (cudaMemcpyAsync(&s, W.scal + 1, sizeof(double), cudaMemcpyDeviceToHost, A.stream) != cudaSuccess ||
      cudaStreamSynchronize(A.stream) != cudaSuccess)
    return std::nan("");
  return s;
}
void launch_pivot_diag(const DevBcsr& A, const double* r, double* mr, unsigned* flag) {
  const int g = (A.m + 127) / 128;
  switch (A.bs) {
    case 5: k_pivot_diag<5><<<g, 128, 0, A.stream>>>(A.m, A.diag, A.v, r, mr, flag); break;
    case 4: k_pivot_diag<4><<<g, 128, 0, A.stream>>>(A.m, A.diag, A.v, r, mr, flag); break;
    case 3: k_pivot_diag<3><<<g, 128, 0, A.stream>>>(A.m, A.diag, A.v, r, mr, flag); break;
    default: k_pivot_diag<1><<<g, 128, 0, A.stream>>>(A.m, A.diag, A.v, r, mr, flag);
  }
}
}  // namespace

// bcsr_pcgm (:1110-1169): CG from the caller's x (device), preconditioned by lu_solve on
// each diagonal block. Dot products by the fixed tree (not left to right). status 0, 1
// not converged (the reference stops), 2 a singular diagonal block.
int pcg_device(const DevBcsr& A, GmresWork& W, double* x, const double* b, double tol, PcgStats* st) {
  const long n = (long)A.m * A.bs;
  cudaStream_t s = A.stream;
  double *r = W.r, *p = W.zp, *Ap = W.w, *mr = W.ty;
  unsigned* flag = reinterpret_cast<unsigned*>(W.scal + 4);
  SUBFV_CUDA(cudaMemsetAsync(flag, 0, sizeof(unsigned), s));
  st->status = 0;
  st->iters = 0;
  double rpdrp = 0.0;
  launch_bcsr_spmv(A, x, Ap, false);
  k_sub<<<egrid(n), 256, 0, s>>>(b, Ap, r, n);
  launch_pivot_diag(A, r, mr, flag);
  double rdr = device_dot(A, W, mr, r, n);
  st->res = std::sqrt(rdr);
  // a zero residual is already solved (the recurrence would divide 0 by 0 with tol = 0)
  const bool done0 = std::sqrt(rdr) < tol || (rdr == 0.0 && device_norm2(A, W, r, n) == 0.0);
  if (!done0) SUBFV_CUDA(cudaMemcpyAsync(p, mr, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
  for (long k = 1; k <= n && !done0; ++k) {
    st->iters = (int)k;
    launch_bcsr_spmv(A, p, Ap, false);
    const double alpha = rdr / device_dot(A, W, p, Ap, n);
    k_cg_update<<<egrid(n), 256, 0, s>>>(x, r, p, Ap, alpha, n);
    launch_pivot_diag(A, r, mr, flag);
    rpdrp = device_dot(A, W, mr, r, n);
    if (!(rpdrp == rpdrp)) return -1;  // a CUDA error inside device_dot
    if (std::sqrt(rpdrp) <= tol && device_norm2(A, W, r, n) <= tol) break;
    k_cg_dir<<<egrid(n), 256, 0, s>>>(p, mr, rpdrp / rdr, n);
    rdr = rpdrp;
  }
  if (!done0) st->res = std::sqrt(rpdrp);
  unsigned f = 0;
  SUBFV_CUDA(cudaMemcpyAsync(&f, flag, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
  SUBFV_CUDA(cudaStreamSynchronize(s));
  SUBFV_CUDA(cudaGetLastError());
  st->status = (f & 2u) ? 2 : (!done0 && std::sqrt(rpdrp) > tol ? 1 : 0);
  return 0;
}

}  // namespace subfv
