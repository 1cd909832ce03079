// Navier-Stokes diffusion kernels: the per-vertex momentum and heat systems of
// src/ns/ns_vectorial_diffusion_module.F90:7-318 and src/ns/ns_diffusion_module.F90:7-184,
// a warp per vertex with the vertex's matrices in shared memory. Every output element of
// a matrix product, solve or inverse is produced by one lane in the order the reference
// (netlib LAPACK / BLAS) accumulates it, so the results are those of the serial code.
#include <algorithm>
#include <cstring>
#include <vector>

#include "ns.cuh"
#include "ns_diffusion.cuh"

namespace subfv {

namespace {

constexpr double kGamma = 1.4, kC0 = 110.4;  // ns_global_data_module.F90:9,20

__device__ inline double temp_u(const double* u, double cv) {  // ns_euler_primitives_module.F90:52-63
  const double tau = 1.0 / u[0];
  const double uu = u[1] * u[1] + u[2] * u[2] + u[3] * u[3];
  return (u[4] * tau - 0.5 * uu * (tau * tau)) / cv;
}
__device__ inline double mu_of(const DiffParams& D, const double* u) {  // compute_mu / mu_sutherland
  if (!D.sutherland) return D.mu_p;
  const double T = temp_u(u, D.Cv_p);
  return D.mu0 * pow(T / D.T0, 1.5) * (D.T0 + kC0) / (T + kC0);
}
__device__ inline void load_u(const double* U, int c, double* u) {
  const double* p = U + kRec * (size_t)c;
  for (int k = 0; k < 5; ++k) u[k] = p[k];
}
__device__ inline double scaled_norm3(double a0, double a1, double a2) {  // gfortran NORM2
  const double a[3] = {a0, a1, a2};
  double scale = 1.0, res = 0.0;
  for (int i = 0; i < 3; ++i)
    if (a[i] != 0.0) {
      const double ax = fabs(a[i]);
      if (ax > scale) {
        const double q = scale / ax;
        res = 1.0 + res * q * q;
        scale = ax;
      } else {
        const double q = ax / scale;
        res += q * q;
      }
    }
  return scale * sqrt(res);
}

// the subface's normal oriented out of sub-cell se, and its area
__device__ inline double oriented(const DevMesh& m, int sf, int se, double* n) {
  const double4 s = m.sfn[sf];
  const double sg = m.sf_se[sf].x == se ? 1.0 : -1.0;
  n[0] = sg == 1.0 ? s.x : -s.x;
  n[1] = sg == 1.0 ? s.y : -s.y;
  n[2] = sg == 1.0 ? s.z : -s.z;
  return s.w;
}
__device__ inline int n_sub_faces(const int4 q) { return (q.x >= 0) + (q.y >= 0) + (q.z >= 0) + (q.w >= 0); }
__device__ inline int sf_of(const int4 q, int p) { return p == 0 ? q.x : p == 1 ? q.y : p == 2 ? q.z : q.w; }

// Warp-parallel dgetrf + dgetri of the n x n column-major matrix a (inv_lapack,
// linear_solver_module.F90:629-641), n <= 96. Each row-parallel phase gives lane r the
// rows r, r + 32, r + 64 (only the groups that still hold live rows), keeps their
// running values in registers and issues each group of four loads before using them,
// so no phase divides indices or waits on a shuffle chain; every element still
// receives the same operations in the same order as in the serial algorithm.

// dgetf2's rank-1 update of the trailing block after column j (dger with alpha = -1:
// a(i,k) - l(i) u(k)), rows j + 1 + lane + 32 g
template <int G, int NC>
__device__ __forceinline__ void lu_update(double* a, int n_rt, int j, int lane) {
  const int n = NC > 0 ? NC : n_rt;
  double l[G];
  double* row[G];
  bool ok[G];
#pragma unroll
  for (int g = 0; g < G; ++g) {
    const int i = j + 1 + lane + 32 * g;
    ok[g] = i < n;
    const int ic = ok[g] ? i : j + 1;  // a dead lane reads a live row and stores nothing
    l[g] = a[ic + n * j];
    row[g] = a + ic;
  }
  const double* pr = a + j;  // the pivot row, a broadcast
  int k = j + 1;
  for (; k + 3 < n; k += 4) {
    double u[4];
#pragma unroll
    for (int t = 0; t < 4; ++t) u[t] = pr[n * (k + t)];
#pragma unroll
    for (int g = 0; g < G; ++g) {
      double x[4];
#pragma unroll
      for (int t = 0; t < 4; ++t) x[t] = row[g][n * (k + t)];
      if (ok[g]) {
#pragma unroll
        for (int t = 0; t < 4; ++t) row[g][n * (k + t)] = x[t] - l[g] * u[t];
      }
    }
  }
  for (; k < n; ++k) {
    const double u = pr[n * k];
#pragma unroll
    for (int g = 0; g < G; ++g)
      if (ok[g]) row[g][n * k] = row[g][n * k] - l[g] * u;
  }
}

// Column j > 0 of dtrti2 ('Upper', 'Non-unit'): x := T x with T the already inverted
// leading block (dtrmv, upper, no transpose), then x := -x / U(j,j) (dscal). In dtrmv,
// step jj reads x(jj) before any step has changed it (later steps only add to rows
// above them), and when it is non-zero scales x(jj) by T(jj,jj) and adds x(jj) T(i,jj)
// to each row i < jj. So a row's result is its own value scaled by the diagonal, then
// the original x(jj) T(i,jj) added in increasing jj, each skipped when x(jj) is zero:
// every lane reads the original column and accumulates its rows i < j (G groups).
template <int G, int NC>
__device__ __forceinline__ void trti_col(double* a, int n_rt, int j, int lane) {
  const int n = NC > 0 ? NC : n_rt;
  const double ajj = -a[j + n * j];
  double* x = a + n * j;
  double acc[G];
  int ii[G];
#pragma unroll
  for (int g = 0; g < G; ++g) {
    const int i = lane + 32 * g;
    ii[g] = i < j ? i : j;  // a dead lane never adds (ii >= every jj) and is never stored
    const int ic = i < j ? i : 0;
    const double x0 = x[ic], d = a[ic + n * ic];
    acc[g] = x0 != 0.0 ? x0 * d : x0;  // dtrmv's step jj = i
  }
  int jj = 1;
  for (; jj + 3 < j; jj += 4) {
    double t[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) t[u] = x[jj + u];
#pragma unroll
    for (int g = 0; g < G; ++g) {
      const int ic = ii[g] < j ? ii[g] : 0;
      double av[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) av[u] = a[ic + n * (jj + u)];
#pragma unroll
      for (int u = 0; u < 4; ++u)
        if (t[u] != 0.0 && ii[g] < jj + u) acc[g] = acc[g] + t[u] * av[u];
    }
  }
  for (; jj < j; ++jj) {
    const double t = x[jj];
#pragma unroll
    for (int g = 0; g < G; ++g) {
      const int ic = ii[g] < j ? ii[g] : 0;
      const double av = a[ic + n * jj];
      if (t != 0.0 && ii[g] < jj) acc[g] = acc[g] + t * av;
    }
  }
  __syncwarp();  // every lane has read the column before it is overwritten
#pragma unroll
  for (int g = 0; g < G; ++g)
    if (ii[g] < j) x[ii[g]] = ajj * acc[g];
  __syncwarp();
}

// dgetri's unblocked sweep, inv(A) L = inv(U) column by column from the last: column j
// becomes (its upper part, zero below the diagonal) - sum over jj > j, in increasing jj,
// of L(jj,j) times column jj; then the column interchanges of ipiv from the last. Rows
// are independent: lane r keeps rows r + 32 g, and each column's L entries are copied
// to work (2 n doubles, alternate halves per column) before any row overwrites them.
template <int NQ, int NC>
__device__ __forceinline__ void getri_sweep(double* a, int n_rt, const int* ipiv, double* work, int lane) {
  const int n = NC > 0 ? NC : n_rt;
  int ic[NQ];
#pragma unroll
  for (int g = 0; g < NQ; ++g) ic[g] = lane + 32 * g < n ? lane + 32 * g : 0;
  for (int j = n - 1; j >= 0; --j) {
    double* w = work + (j & 1) * n;
    for (int i = j + 1 + lane; i < n; i += 32) w[i] = a[i + n * j];
    __syncwarp();
    double acc[NQ];
#pragma unroll
    for (int g = 0; g < NQ; ++g) acc[g] = lane + 32 * g <= j ? a[ic[g] + n * j] : 0.0;
    int jj = j + 1;
    for (; jj + 3 < n; jj += 4) {
      double wv[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) wv[u] = -w[jj + u];
#pragma unroll
      for (int g = 0; g < NQ; ++g) {
        double av[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) av[u] = a[ic[g] + n * (jj + u)];
#pragma unroll
        for (int u = 0; u < 4; ++u) acc[g] = acc[g] + wv[u] * av[u];
      }
    }
    for (; jj < n; ++jj) {
      const double wv = -w[jj];
#pragma unroll
      for (int g = 0; g < NQ; ++g) acc[g] = acc[g] + wv * a[ic[g] + n * jj];
    }
#pragma unroll
    for (int g = 0; g < NQ; ++g)
      if (lane + 32 * g < n) a[lane + 32 * g + n * j] = acc[g];
  }
#pragma unroll
  for (int g = 0; g < NQ; ++g) {
    const int i = lane + 32 * g;
    if (i < n)
      for (int j = n - 2; j >= 0; --j) {
        const int p = ipiv[j];
        if (p != j) {
          const double t = a[i + n * j];
          a[i + n * j] = a[i + n * p];
          a[i + n * p] = t;
        }
      }
  }
  __syncwarp();
}

// work: 2 n doubles. NC > 0 fixes n at compile time (every index product a constant).
template <int NC>
__device__ void warp_inverse_n(double* a, int n_rt, int* ipiv, double* work, int lane) {
  const int n = NC > 0 ? NC : n_rt;
  for (int j = 0; j < n; ++j) {  // dgetf2
    double big = -1.0;
    int bi = n;
    for (int i = j + lane; i < n; i += 32) {
      const double x = fabs(a[i + n * j]);
      if (x > big) {
        big = x;
        bi = i;
      }
    }
    for (int o = 16; o > 0; o >>= 1) {  // largest |x|, the first index among equals
      const double ob = __shfl_xor_sync(0xffffffffu, big, o);
      const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
      if (ob > big || (ob == big && oi < bi)) {
        big = ob;
        bi = oi;
      }
    }
    const int p = bi < n ? bi : j;
    if (lane == 0) ipiv[j] = p;
    const bool nz = a[p + n * j] != 0.0;
    __syncwarp();
    if (nz) {
      if (p != j) {
        for (int k = lane; k < n; k += 32) {
          const double t = a[j + n * k];
          a[j + n * k] = a[p + n * k];
          a[p + n * k] = t;
        }
        __syncwarp();
      }
      const double piv = a[j + n * j];
      if (fabs(piv) >= 2.2250738585072014e-308) {
        const double r = 1.0 / piv;
        for (int i = j + 1 + lane; i < n; i += 32) a[i + n * j] = r * a[i + n * j];
      } else {
        for (int i = j + 1 + lane; i < n; i += 32) a[i + n * j] = a[i + n * j] / piv;
      }
    }
    __syncwarp();
    const int w = n - j - 1;
    if (w > 64) lu_update<3, NC>(a, n, j, lane);
    else if (w > 32) lu_update<2, NC>(a, n, j, lane);
    else if (w > 0) lu_update<1, NC>(a, n, j, lane);
    __syncwarp();
  }
  for (int j = 0; j < n; ++j) {  // dtrti2
    if (lane == 0) a[j + n * j] = 1.0 / a[j + n * j];
    __syncwarp();
    if (j > 64) trti_col<3, NC>(a, n, j, lane);
    else if (j > 32) trti_col<2, NC>(a, n, j, lane);
    else if (j > 0) trti_col<1, NC>(a, n, j, lane);
  }
  if (n > 64) getri_sweep<3, NC>(a, n, ipiv, work, lane);
  else if (n > 32) getri_sweep<2, NC>(a, n, ipiv, work, lane);
  else getri_sweep<1, NC>(a, n, ipiv, work, lane);
}

// The sizes of hexahedral meshes (momentum 36, heat 12 per vertex) and of one-layer slabs
// of hexahedra (24, 8) with their index arithmetic fixed; others at run time.
__device__ inline void warp_inverse(double* a, int n, int* ipiv, double* work, int lane) {
  switch (n) {
    case 36: warp_inverse_n<36>(a, n, ipiv, work, lane); break;
    case 24: warp_inverse_n<24>(a, n, ipiv, work, lane); break;
    case 12: warp_inverse_n<12>(a, n, ipiv, work, lane); break;
    case 8: warp_inverse_n<8>(a, n, ipiv, work, lane); break;
    default: warp_inverse_n<0>(a, n, ipiv, work, lane);
  }
}

// C(m x p) = A(m x k) B(k x p), netlib dgemm order: C(i,j) = sum over l, in order, of
// B(l,j) A(i,l). C is written over B's storage with leading dimension m <= k: column j of
// C needs only column j of B, so each block of columns is summed into registers and
// stored once the whole warp has read that block of B (the stored block ends at
// m (j0 + JB) <= k (j0 + JB), below the columns still to be read). A lane owns rows
// lane + 32 g, so one load of A(i,l) serves JB sums and B(l,j) is a broadcast.
template <int NQ, int JB, int MC, int KC>
__device__ __forceinline__ void gemm_block(int m_rt, int k_rt, const double* A, double* BC, int j0, int lane) {
  const int m = MC > 0 ? MC : m_rt, k = KC > 0 ? KC : k_rt;
  double s[NQ][JB];
#pragma unroll
  for (int g = 0; g < NQ; ++g)
#pragma unroll
    for (int jj = 0; jj < JB; ++jj) s[g][jj] = 0.0;
  const double* b = BC + (size_t)k * j0;
  int ic[NQ];
#pragma unroll
  for (int g = 0; g < NQ; ++g) ic[g] = lane + 32 * g < m ? lane + 32 * g : 0;
  int l = 0;
  for (; l + 1 < k; l += 2) {
    double bv[2][JB];
#pragma unroll
    for (int u = 0; u < 2; ++u)
#pragma unroll
      for (int jj = 0; jj < JB; ++jj) bv[u][jj] = b[l + u + k * jj];
#pragma unroll
    for (int g = 0; g < NQ; ++g) {
      const double a0 = A[ic[g] + m * l], a1 = A[ic[g] + m * (l + 1)];
#pragma unroll
      for (int jj = 0; jj < JB; ++jj) s[g][jj] = s[g][jj] + bv[0][jj] * a0;
#pragma unroll
      for (int jj = 0; jj < JB; ++jj) s[g][jj] = s[g][jj] + bv[1][jj] * a1;
    }
  }
  if (l < k) {
#pragma unroll
    for (int g = 0; g < NQ; ++g) {
      const double a0 = A[ic[g] + m * l];
#pragma unroll
      for (int jj = 0; jj < JB; ++jj) s[g][jj] = s[g][jj] + b[l + k * jj] * a0;
    }
  }
  __syncwarp();
#pragma unroll
  for (int g = 0; g < NQ; ++g)
    if (lane + 32 * g < m)
#pragma unroll
      for (int jj = 0; jj < JB; ++jj) BC[lane + 32 * g + m * (j0 + jj)] = s[g][jj];
}
template <int NQ, int MC = 0, int KC = 0>
__device__ void gemm_over_b_rows(int m, int p, int k, const double* A, double* BC, int lane) {
  int j0 = 0;
  for (; j0 + 4 <= p; j0 += 4) gemm_block<NQ, 4, MC, KC>(m, k, A, BC, j0, lane);
  for (; j0 < p; ++j0) gemm_block<NQ, 1, MC, KC>(m, k, A, BC, j0, lane);
  __syncwarp();
}
// (m, k) of the hexahedral and one-layer-slab vertices fixed at compile time, as above
__device__ inline void warp_gemm_over_b(int m, int p, int k, const double* A, double* BC, int lane) {
  if (m == 24 && k == 36) gemm_over_b_rows<1, 24, 36>(m, p, k, A, BC, lane);
  else if (m == 8 && k == 12) gemm_over_b_rows<1, 8, 12>(m, p, k, A, BC, lane);
  else if (m == 12 && k == 24) gemm_over_b_rows<1, 12, 24>(m, p, k, A, BC, lane);
  else if (m == 4 && k == 8) gemm_over_b_rows<1, 4, 8>(m, p, k, A, BC, lane);
  else if (m <= 32) gemm_over_b_rows<1>(m, p, k, A, BC, lane);
  else if (m <= 64) gemm_over_b_rows<2>(m, p, k, A, BC, lane);
  else gemm_over_b_rows<3>(m, p, k, A, BC, lane);
}
// y(m) = A(m x n) x, netlib dgemv order
__device__ inline void warp_gemv(int m, int n, const double* A, const double* x, double* y, int lane) {
  for (int i = lane; i < m; i += 32) {
    double s = 0.0;
    for (int j = 0; j < n; ++j) s = s + x[j] * A[i + m * j];
    y[i] = s;
  }
  __syncwarp();
}
// y1 = A x1 and y2 = A x2 in one pass over A, each in netlib dgemv order
__device__ inline void warp_gemv2(int m, int n, const double* A, const double* x1, const double* x2, double* y1,
                                  double* y2, int lane) {
  for (int i = lane; i < m; i += 32) {
    double s1 = 0.0, s2 = 0.0;
    for (int j = 0; j < n; ++j) {
      const double av = A[i + m * j];
      s1 = s1 + x1[j] * av;
      s2 = s2 + x2[j] * av;
    }
    y1[i] = s1;
    y2[i] = s2;
  }
  __syncwarp();
}

// Offsets (doubles) of one vertex's work arrays, for the mesh's largest vertex. N holds
// the nodal matrix, then its inverse, then St N^-1; S holds S, then SNS = St N^-1 S. The
// heat system reuses the same arrays at its smaller sizes, with its per-subcell theta,
// P and b1 placed in St past the heat St's ne x nf entries.
struct DiffSmem {
  int N, S, St, B, Vf, tmp, work, Ve, SB, SNSVe, blc3, ipiv, total;
};
__host__ __device__ inline DiffSmem diff_layout(int max_vsf, int max_vse) {
  const int F = 3 * max_vsf, E = 3 * max_vse;
  DiffSmem L{};
  int o = 0;
  L.N = o, o += F * F;
  L.S = o, o += F * E;
  L.St = o, o += E * F;
  L.B = o, o += F;
  L.Vf = o, o += F;
  L.tmp = o, o += F;
  L.work = o, o += F;  // tmp and work together are the inverse's 2 F scratch
  L.Ve = o, o += E;
  L.SB = o, o += E;
  L.SNSVe = o, o += E;
  L.blc3 = o, o += 3 * E;
  L.ipiv = o, o += F;  // ints stored in double slots
  L.total = o;
  return L;
}

__global__ void k_diff_mu0c(DevMesh m, DiffParams D, const double* __restrict__ U, double* mu0c, int init) {
  if (init) {
    if (blockIdx.x == 0 && threadIdx.x == 0) *mu0c = D.sutherland ? 1e12 : D.mu_p;
    return;
  }
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= m.ne || !D.sutherland) return;
  double u[5];
  load_u(U, c, u);
  atomic_min_pos(mu0c, mu_of(D, u));
}

// The momentum blc_3 (ns_vectorial_diffusion_module.F90:85-91) and the Neumann face's
// N / S block (:149-152), row-major b[i][j]
__device__ inline void mom_block(double al, double ap, double vol, double mu, double mu0c, const double* nl,
                                 const double* np, double b[3][3]) {
  const double s = al * ap * (1.0 / vol);
  const double d = nl[0] * np[0] + nl[1] * np[1] + nl[2] * np[2];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      const double e = i == j ? 1.0 : 0.0;
      const double tp = np[i] * nl[j], tpt = np[j] * nl[i];
      b[i][j] = s * ((mu * d * e + (mu - mu0c) * tp) + (mu0c - (2.0 / 3.0) * mu) * tpt);
    }
}
__device__ inline void neumann_block(double al, double ap, double vol, const double* nl, const double* np,
                                     double b[3][3]) {
  const double s = al * ap * (1.0 / vol);
  const double d = nl[0] * np[0] + nl[1] * np[1] + nl[2] * np[2];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      const double e = i == j ? 1.0 : 0.0;
      b[i][j] = s * (d * e + (np[j] * nl[i]) / 3.0);
    }
}

// Where a vertex's invariant diffusion arrays sit in the cache (constant viscosity): S
// (F x E), B (F), N^-1 (F x F), SNS (E x E), SB (E), the per-subcell sums of St (9 per
// subcell, blc3's numerators), then the heat system's SNS (ne x ne), SB (ne) and b1 (ne).
struct DiffCacheView {
  double *S, *B, *Ninv, *SNS, *SB, *Spc, *SNSh, *SBh, *b1;
};
__host__ __device__ inline long long diff_cache_doubles(int nf, int ne) {
  const long long F = 3 * nf, E = 3 * ne;
  return F * E + F + F * F + E * E + E + 3 * E + (long long)ne * ne + 2LL * ne;
}
__device__ inline DiffCacheView diff_cache_view(double* c, int nf, int ne) {
  const int F = 3 * nf, E = 3 * ne;
  DiffCacheView w;
  w.S = c;
  w.B = w.S + (size_t)F * E;
  w.Ninv = w.B + F;
  w.SNS = w.Ninv + (size_t)F * F;
  w.SB = w.SNS + (size_t)E * E;
  w.Spc = w.SB + E;
  w.SNSh = w.Spc + 3 * E;
  w.SBh = w.SNSh + (size_t)ne * ne;
  w.b1 = w.SBh + ne;
  return w;
}

// FILL: the same computation, which also stores the state-independent arrays of each
// vertex in the cache (only with a constant viscosity, where they do not depend on U)
template <bool FILL>
__global__ void __launch_bounds__(32) k_ns_diffusion(DevMesh m, DiffParams D, const double* __restrict__ U,
                                                     double* __restrict__ dterm, const double* __restrict__ mu0c_p,
                                                     double* __restrict__ cache, const long long* __restrict__ coff) {
  extern __shared__ double sm[];
  const DiffSmem L = diff_layout(m.max_dsf, m.max_dse);
  const int lane = threadIdx.x;
  double *N = sm + L.N, *S = sm + L.S, *St = sm + L.St, *B = sm + L.B;
  double *Vf = sm + L.Vf, *tmp = sm + L.tmp, *work = sm + L.work, *Ve = sm + L.Ve, *SB = sm + L.SB;
  double *SNSVe = sm + L.SNSVe, *blc3 = sm + L.blc3;
  int* ipiv = reinterpret_cast<int*>(sm + L.ipiv);
  const double mu0c = *mu0c_p;
  for (int v = blockIdx.x; v < m.nv; v += gridDim.x) {
    const int f0 = m.dsf_off[v], nf = m.dsf_off[v + 1] - f0;
    const int s0 = m.dse_off[v], ne = m.dse_off[v + 1] - s0;
    const int F = 3 * nf, E = 3 * ne;
    DiffCacheView cw{};
    if (FILL) cw = diff_cache_view(cache + coff[v], nf, ne);
    // ---- momentum: build_momentum_diff_nodal_system (:7-193)
    for (int e = lane; e < F * F; e += 32) N[e] = 0.0;
    for (int e = lane; e < F * E; e += 32) S[e] = St[e] = 0.0;
    for (int e = lane; e < F; e += 32) B[e] = 0.0;
    __syncwarp();
    for (int l = lane; l < nf; l += 32) {  // lane l owns row block l of N and S, column block l of St
      const int sf = m.dsf[f0 + l];
      const int ifl0 = 3 * l;
      const int2 lr = m.flr[m.sf_face[sf]];
      const int2 se2 = m.dsf_se[f0 + l], sep = m.dsf_seloc[f0 + l];
      const double4 sn = m.sfn[sf];
      const double al = sn.w;
      int kind = 0;  // 0 interior, 1 neumann (the default wall, and a tag's "" or "neumann"), 2 dirichlet
      int tag = 0;
      if (lr.y == -1) {
        kind = 1;
      } else if (lr.y < -1) {
        tag = -(lr.y + 1) - 1;
        kind = D.bcV[tag] == 2 ? 2 : 1;
      }
      auto side = [&](int se, int elem, const double* nl, int mode, int sp) {
        double u[5];
        load_u(U, elem, u);
        const double mue = mu_of(D, u);
        const int ise0 = 3 * sp;
        const int4 q4 = m.se_sf[se], ql = m.dse_sfloc[s0 + sp];
        const double vol = m.vol_se[se];
        const int nsf = n_sub_faces(q4);
        for (int p = 0; p < nsf; ++p) {
          const int sfp = sf_of(q4, p);
          const int ifp0 = 3 * sf_of(ql, p);
          double np[3];
          const double ap = oriented(m, sfp, se, np);
          double blc[3][3], bn[3][3];
          mom_block(al, ap, vol, mue, mu0c, nl, np, blc);
          if (mode == 1) neumann_block(al, ap, vol, nl, np, bn);
          for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
              St[(ise0 + i) + E * (ifl0 + j)] += blc[j][i];
              if (mode != 2) {
                const double x = mode == 1 ? bn[i][j] : blc[i][j];
                N[(ifl0 + i) + F * (ifp0 + j)] += x;
                S[(ifl0 + i) + F * (ise0 + j)] += x;
              }
            }
        }
      };
      const double nl[3] = {sn.x, sn.y, sn.z}, nr[3] = {-sn.x, -sn.y, -sn.z};
      if (kind == 0) {
        side(se2.x, lr.x, nl, 0, sep.x);
        side(se2.y, lr.y, nr, 0, sep.y);
      } else if (kind == 1) {
        side(se2.x, lr.x, nl, 1, sep.x);
      } else {
        side(se2.x, lr.x, nl, 2, sep.x);
        for (int k = 0; k < 3; ++k) B[ifl0 + k] = al * D.valV[tag][k];
        for (int i = 0; i < 3; ++i) {
          for (int c = 0; c < E; ++c) S[(ifl0 + i) + F * c] = 0.0;
          for (int c = 0; c < F; ++c) N[(ifl0 + i) + F * c] = 0.0;
          for (int j = 0; j < 3; ++j) N[(ifl0 + i) + F * (ifl0 + j)] = al * (i == j ? 1.0 : 0.0);
        }
      }
    }
    __syncwarp();
    // ---- build_momentum_diff_mat_into_global_mat_diag (:233-318)
    for (int l = lane; l < ne; l += 32) {
      double u[5];
      load_u(U, m.se_elem[m.dse[s0 + l]], u);
      for (int k = 0; k < 3; ++k) Ve[3 * l + k] = u[1 + k] / u[0];
      double Spc[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
      for (int c = 0; c < nf; ++c)
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j) Spc[i][j] = Spc[i][j] + St[(3 * l + i) + E * (3 * c + j)];
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) blc3[9 * l + i + 3 * j] = Spc[j][i] / u[0];
      if (FILL)
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j) cw.Spc[9 * l + i + 3 * j] = Spc[j][i];
    }
    if (FILL) {
      for (int e = lane; e < F * E; e += 32) cw.S[e] = S[e];
      for (int e = lane; e < F; e += 32) cw.B[e] = B[e];
    }
    __syncwarp();
    warp_gemv(F, E, S, Ve, Vf, lane);
    for (int i = lane; i < F; i += 32) Vf[i] = Vf[i] + B[i];
    __syncwarp();
    warp_inverse(N, F, ipiv, tmp, lane);  // tmp and work (adjacent, 2 F) as its scratch
    if (FILL)
      for (int e = lane; e < F * F; e += 32) cw.Ninv[e] = N[e];
    // the products of the reference, the two with N^-1 as a vector first, then
    // T1 = St N^-1 over N and SNS = T1 S over S (each product's own arithmetic unchanged)
    warp_gemv2(F, F, N, B, Vf, tmp, work, lane);  // N^-1 B, and N^-1 (S Ve + B): the face velocities
    warp_gemm_over_b(E, F, F, St, N, lane);
    const double* T1 = N;
    warp_gemm_over_b(E, E, F, T1, S, lane);
    const double* SNSm = S;
    warp_gemv(E, F, St, tmp, SB, lane);
    warp_gemv(E, E, SNSm, Ve, SNSVe, lane);
    if (FILL) {
      for (int e = lane; e < E * E; e += 32) cw.SNS[e] = SNSm[e];
      for (int e = lane; e < E; e += 32) cw.SB[e] = SB[e];
    }
    for (int l = lane; l < ne; l += 32) {
      const int se = m.dse[s0 + l];
      if (m.se_vert[se] != v) continue;  // a periodic image's subcell: its own vertex writes it
      double u[5];
      load_u(U, m.se_elem[se], u);
      double* t = dterm + (size_t)D.kd * se;
      const int4 ql = m.dse_sfloc[s0 + l];
      for (int i = 0; i < 3; ++i) {
        double mv = 0.0;
        for (int k = 0; k < 3; ++k) mv = mv + SNSm[(3 * l + i) + E * (3 * l + k)] * Ve[3 * l + k];
        t[3 * i] = SNSVe[3 * l + i];
        t[3 * i + 1] = mv;
        t[3 * i + 2] = SB[3 * l + i];
      }
      for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i) {
          t[9 + 2 * (i + 3 * j)] = SNSm[(3 * l + i) + E * (3 * l + j)] / u[0];
          t[10 + 2 * (i + 3 * j)] = blc3[9 * l + i + 3 * j];
        }
      // viscous work (:285-313)
      const int4 q4 = m.se_sf[se];
      const int nsf = n_sub_faces(q4);
      double Spc[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
      for (int k = 0; k < nsf; ++k) {
        const int sf = sf_of(q4, k);
        double nl[3];
        const double a = oriented(m, sf, se, nl);
        const int q = 3 * sf_of(ql, k);
        double vm[3];
        for (int d = 0; d < 3; ++d) vm[d] = work[q + d] - Ve[3 * l + d];
        const double dd = vm[0] * nl[0] + vm[1] * nl[1] + vm[2] * nl[2];
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j) {
            const double e = i == j ? 1.0 : 0.0;
            Spc[i][j] = Spc[i][j] + a * ((vm[i] * nl[j] + vm[j] * nl[i]) - (2.0 / 3.0) * dd * e);
          }
      }
      const double mue = mu_of(D, u), vse = m.vol_se[se];
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) Spc[i][j] = Spc[i][j] * mue / vse;
      for (int k = 0; k < 4; ++k) t[27 + k] = 0.0;
      for (int k = 0; k < nsf; ++k) {
        const int sf = sf_of(q4, k);
        double nl[3];
        const double a = oriented(m, sf, se, nl);
        const int q = 3 * sf_of(ql, k);
        double sv[3];
        for (int i = 0; i < 3; ++i) {
          double s = 0.0;
          for (int c = 0; c < 3; ++c) s = s + Spc[i][c] * work[q + c];
          sv[i] = s;
        }
        t[27 + k] = a * (sv[0] * nl[0] + sv[1] * nl[1] + sv[2] * nl[2]);
      }
    }
    __syncwarp();
    // ---- heat: build_diff_nodal_system (ns_diffusion_module.F90:7-110)
    for (int e = lane; e < nf * nf; e += 32) N[e] = 0.0;
    for (int e = lane; e < nf * ne; e += 32) S[e] = St[e] = 0.0;
    for (int e = lane; e < nf; e += 32) B[e] = 0.0;
    __syncwarp();
    for (int l = lane; l < nf; l += 32) {
      const int sf = m.dsf[f0 + l];
      const int il = l;
      const int2 lr = m.flr[m.sf_face[sf]];
      const int2 se2 = m.dsf_se[f0 + l], sep = m.dsf_seloc[f0 + l];
      const double4 sn = m.sfn[sf];
      const double al = sn.w;
      auto side = [&](int se, int elem, const double* nl, int sp) {
        double u[5];
        load_u(U, elem, u);
        const double kap = mu_of(D, u) * D.Cv_p * kGamma / D.prandtl;
        const int ie = sp;
        const int4 q4 = m.se_sf[se], ql = m.dse_sfloc[s0 + sp];
        const double vol = m.vol_se[se];
        const int nsf = n_sub_faces(q4);
        for (int p = 0; p < nsf; ++p) {
          const int sfp = sf_of(q4, p);
          const int ip = sf_of(ql, p);
          double np[3];
          const double ap = oriented(m, sfp, se, np);
          const double b = kap * al * ap * (1.0 / vol) * (np[0] * nl[0] + np[1] * nl[1] + np[2] * nl[2]);
          N[il + nf * ip] += b;
          S[il + nf * ie] += b;
          St[ie + ne * il] += b;
        }
      };
      const double nl[3] = {sn.x, sn.y, sn.z}, nr[3] = {-sn.x, -sn.y, -sn.z};
      side(se2.x, lr.x, nl, sep.x);
      if (se2.y >= 0) {
        side(se2.y, lr.y, nr, sep.y);
      } else if (lr.y < -1 && D.bcT[-(lr.y + 1) - 1] == 2) {
        B[il] = al * D.valT[-(lr.y + 1) - 1];
        for (int c = 0; c < ne; ++c) S[il + nf * c] = 0.0;
        for (int c = 0; c < nf; ++c) N[il + nf * c] = 0.0;
        N[il + nf * il] = al;
      }
    }
    __syncwarp();
    warp_inverse(N, nf, ipiv, tmp, lane);
    warp_gemv(nf, nf, N, B, tmp, lane);
    warp_gemm_over_b(ne, nf, nf, St, N, lane);
    warp_gemm_over_b(ne, ne, nf, T1, S, lane);
    warp_gemv(ne, nf, St, tmp, SB, lane);
    double* theta = St + ne * nf;  // past the heat St, which the loops below still read
    double* P = theta + ne;
    double* b1 = P + 5 * ne;
    for (int l = lane; l < ne; l += 32) {
      double u[5];
      load_u(U, m.se_elem[m.dse[s0 + l]], u);
      theta[l] = temp_u(u, D.Cv_p);
      const double nn = scaled_norm3(u[1] / u[0], u[2] / u[0], u[3] / u[0]);
      P[5 * l] = (nn * nn - u[4] / u[0]) / (u[0] * D.Cv_p);
      for (int k = 1; k < 4; ++k) P[5 * l + k] = -u[k] / ((u[0] * u[0]) * D.Cv_p);
      P[5 * l + 4] = 1.0 / (u[0] * D.Cv_p);
      double s = 0.0;
      for (int c = 0; c < nf; ++c) s = s + St[l + ne * c];
      b1[l] = s;
    }
    __syncwarp();
    if (FILL) {
      for (int e = lane; e < ne * ne; e += 32) cw.SNSh[e] = SNSm[e];
      for (int e = lane; e < ne; e += 32) {
        cw.SBh[e] = SB[e];
        cw.b1[e] = b1[e];
      }
    }
    for (int l = lane; l < ne; l += 32) {
      const int se = m.dse[s0 + l];
      if (m.se_vert[se] != v) continue;
      double u[5];
      load_u(U, m.se_elem[se], u);
      double* t = dterm + (size_t)D.kd * se;
      for (int p = 0; p < ne; ++p) t[kDiffHead + p] = SNSm[l + ne * p] * theta[p];
      const double snl = SNSm[l + ne * l], cc = b1[l] - snl;
      for (int k = 0; k < 5; ++k) t[31 + k] = cc * P[5 * l + k];
      double pu = 0.0;
      for (int k = 0; k < 5; ++k) pu = pu + P[5 * l + k] * u[k];
      t[36] = snl * pu;
      t[37] = cc * pu;
      t[38] = b1[l] * theta[l];
      t[39] = SB[l];
    }
    __syncwarp();
  }
}

// The corner records from the cache (constant viscosity): the state-dependent part of
// k_ns_diffusion only, with the same operations in the same order on the same stored
// values, so the records are bit-identical to the full kernel's. A warp per vertex,
// kDiffWarps per block; the matrices are read from the cache with the rows on the lanes.
constexpr int kDiffWarps = 4;
__global__ void __launch_bounds__(32 * kDiffWarps) k_ns_diffusion_cached(DevMesh m, DiffParams D,
                                                                         const double* __restrict__ U,
                                                                         double* __restrict__ dterm,
                                                                         const double* __restrict__ cache,
                                                                         const long long* __restrict__ coff) {
  extern __shared__ double smc[];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int MF = 3 * m.max_dsf, ME = 3 * m.max_dse;
  double* base = smc + (size_t)wid * (2 * MF + 7 * ME);
  double *Vf = base, *work = Vf + MF, *Ve = work + MF, *SNSVe = Ve + ME, *blc3 = SNSVe + ME;
  double *theta = blc3 + 3 * ME, *P = theta + ME / 3;
  for (int v = blockIdx.x * kDiffWarps + wid; v < m.nv; v += gridDim.x * kDiffWarps) {
    const int f0 = m.dsf_off[v], nf = m.dsf_off[v + 1] - f0;
    const int s0 = m.dse_off[v], ne = m.dse_off[v + 1] - s0;
    const int F = 3 * nf, E = 3 * ne;
    const DiffCacheView c = diff_cache_view(const_cast<double*>(cache) + coff[v], nf, ne);
    (void)f0;
    for (int l = lane; l < ne; l += 32) {
      double u[5];
      load_u(U, m.se_elem[m.dse[s0 + l]], u);
      for (int k = 0; k < 3; ++k) Ve[3 * l + k] = u[1 + k] / u[0];
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) blc3[9 * l + i + 3 * j] = c.Spc[9 * l + i + 3 * j] / u[0];
    }
    __syncwarp();
    for (int i = lane; i < F; i += 32) {  // S Ve + B
      double s = 0.0;
      for (int j = 0; j < E; ++j) s = s + Ve[j] * c.S[i + F * j];
      Vf[i] = s;
    }
    __syncwarp();
    for (int i = lane; i < F; i += 32) Vf[i] = Vf[i] + c.B[i];
    __syncwarp();
    for (int i = lane; i < F; i += 32) {  // N^-1 (S Ve + B): the face velocities
      double s = 0.0;
      for (int j = 0; j < F; ++j) s = s + Vf[j] * c.Ninv[i + F * j];
      work[i] = s;
    }
    for (int i = lane; i < E; i += 32) {  // SNS Ve
      double s = 0.0;
      for (int j = 0; j < E; ++j) s = s + Ve[j] * c.SNS[i + E * j];
      SNSVe[i] = s;
    }
    __syncwarp();
    const double* SNSm = c.SNS;
    const double* SB = c.SB;
    for (int l = lane; l < ne; l += 32) {
      const int se = m.dse[s0 + l];
      if (m.se_vert[se] != v) continue;  // a periodic image's subcell: its own vertex writes it
      double u[5];
      load_u(U, m.se_elem[se], u);
      double* t = dterm + (size_t)D.kd * se;
      const int4 ql = m.dse_sfloc[s0 + l];
      for (int i = 0; i < 3; ++i) {
        double mv = 0.0;
        for (int k = 0; k < 3; ++k) mv = mv + SNSm[(3 * l + i) + E * (3 * l + k)] * Ve[3 * l + k];
        t[3 * i] = SNSVe[3 * l + i];
        t[3 * i + 1] = mv;
        t[3 * i + 2] = SB[3 * l + i];
      }
      for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i) {
          t[9 + 2 * (i + 3 * j)] = SNSm[(3 * l + i) + E * (3 * l + j)] / u[0];
          t[10 + 2 * (i + 3 * j)] = blc3[9 * l + i + 3 * j];
        }
      // viscous work (:285-313)
      const int4 q4 = m.se_sf[se];
      const int nsf = n_sub_faces(q4);
      double Spc[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
      for (int k = 0; k < nsf; ++k) {
        const int sf = sf_of(q4, k);
        double nl[3];
        const double a = oriented(m, sf, se, nl);
        const int q = 3 * sf_of(ql, k);
        double vm[3];
        for (int d = 0; d < 3; ++d) vm[d] = work[q + d] - Ve[3 * l + d];
        const double dd = vm[0] * nl[0] + vm[1] * nl[1] + vm[2] * nl[2];
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j) {
            const double e = i == j ? 1.0 : 0.0;
            Spc[i][j] = Spc[i][j] + a * ((vm[i] * nl[j] + vm[j] * nl[i]) - (2.0 / 3.0) * dd * e);
          }
      }
      const double mue = mu_of(D, u), vse = m.vol_se[se];
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) Spc[i][j] = Spc[i][j] * mue / vse;
      for (int k = 0; k < 4; ++k) t[27 + k] = 0.0;
      for (int k = 0; k < nsf; ++k) {
        const int sf = sf_of(q4, k);
        double nl[3];
        const double a = oriented(m, sf, se, nl);
        const int q = 3 * sf_of(ql, k);
        double sv[3];
        for (int i = 0; i < 3; ++i) {
          double s = 0.0;
          for (int cc = 0; cc < 3; ++cc) s = s + Spc[i][cc] * work[q + cc];
          sv[i] = s;
        }
        t[27 + k] = a * (sv[0] * nl[0] + sv[1] * nl[1] + sv[2] * nl[2]);
      }
    }
    __syncwarp();
    // ---- heat
    for (int l = lane; l < ne; l += 32) {
      double u[5];
      load_u(U, m.se_elem[m.dse[s0 + l]], u);
      theta[l] = temp_u(u, D.Cv_p);
      const double nn = scaled_norm3(u[1] / u[0], u[2] / u[0], u[3] / u[0]);
      P[5 * l] = (nn * nn - u[4] / u[0]) / (u[0] * D.Cv_p);
      for (int k = 1; k < 4; ++k) P[5 * l + k] = -u[k] / ((u[0] * u[0]) * D.Cv_p);
      P[5 * l + 4] = 1.0 / (u[0] * D.Cv_p);
    }
    __syncwarp();
    for (int l = lane; l < ne; l += 32) {
      const int se = m.dse[s0 + l];
      if (m.se_vert[se] != v) continue;
      double u[5];
      load_u(U, m.se_elem[se], u);
      double* t = dterm + (size_t)D.kd * se;
      for (int p = 0; p < ne; ++p) t[kDiffHead + p] = c.SNSh[l + ne * p] * theta[p];
      const double snl = c.SNSh[l + ne * l], cc = c.b1[l] - snl;
      for (int k = 0; k < 5; ++k) t[31 + k] = cc * P[5 * l + k];
      double pu = 0.0;
      for (int k = 0; k < 5; ++k) pu = pu + P[5 * l + k] * u[k];
      t[36] = snl * pu;
      t[37] = cc * pu;
      t[38] = c.b1[l] * theta[l];
      t[39] = c.SBh[l];
    }
    __syncwarp();
  }
}

__global__ void k_ns_diffusion_apply(DevMesh m, const double* __restrict__ dterm, int kd, double* __restrict__ rhs1,
                                     double* __restrict__ diag) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= m.ne) return;
  double* r1 = rhs1 + kRhs * (size_t)c;
  double r[5], Dm[25];
  for (int k = 0; k < 5; ++k) r[k] = r1[k];
  for (int k = 0; k < 25; ++k) Dm[k] = 0.0;
  apply_diffusion_terms(m, c, dterm, kd, r, Dm);
  for (int k = 0; k < 5; ++k) r1[k] = r[k];
  if (diag)
    for (int k = 0; k < 25; ++k) diag[25 * (size_t)c + k] = Dm[k];
}

}  // namespace

DiffParams diff_params_from(const subfv_ns_cfg& c, const DevMesh& m) {
  DiffParams D{};
  D.sutherland = c.use_sutherland;
  D.mu_p = c.mu_p;
  D.mu0 = c.mu0;
  D.T0 = c.T0;
  D.Cv_p = c.Cv_p;
  D.prandtl = c.prandtl > 0.0 ? c.prandtl : 0.71;  // ns_global_data_module.F90:10
  for (int i = 0; i < 16; ++i) {
    D.bcV[i] = c.bc_type_V[i];
    D.bcT[i] = c.bc_type_T[i];
    D.valT[i] = c.bc_val_T[i];
    for (int k = 0; k < 3; ++k) D.valV[i][k] = c.bc_val_V[i][k];
  }
  D.kd = kDiffHead + std::max(1, m.max_dse);
  return D;
}

size_t diffusion_smem_bytes(const DevMesh& m) {
  return sizeof(double) * (size_t)diff_layout(m.max_dsf, m.max_dse).total;
}

int diffusion_prepare(size_t smem) {
  // the attribute is per kernel: only ever raised, so every live state's launch fits
  static size_t granted = 0;
  if (smem > granted) {
    SUBFV_CUDA(cudaFuncSetAttribute(k_ns_diffusion<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    SUBFV_CUDA(cudaFuncSetAttribute(k_ns_diffusion<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    granted = smem;
  }
  return 0;
}

namespace {
// The constants the cached arrays depend on (besides the mesh): zero-filled, so that
// whole objects compare bytewise.
struct DiffCacheKey {
  int sutherland;
  int bcV[16], bcT[16];
  double mu_p, Cv_p, prandtl;
  double valV[16][3], valT[16];
};
DiffCacheKey cache_key_of(const DiffParams& D) {
  DiffCacheKey k;
  std::memset(&k, 0, sizeof k);
  k.sutherland = D.sutherland;
  for (int i = 0; i < 16; ++i) {
    k.bcV[i] = D.bcV[i];
    k.bcT[i] = D.bcT[i];
    k.valT[i] = D.valT[i];
    for (int c = 0; c < 3; ++c) k.valV[i][c] = D.valV[i][c];
  }
  k.mu_p = D.mu_p;
  k.Cv_p = D.Cv_p;
  k.prandtl = D.prandtl;
  return k;
}
// the constants and the geometry epoch the cache was filled for
struct DiffCacheMeta {
  DiffCacheKey key;
  unsigned long long epoch;
};
bool cache_matches(const DevMesh& m, const DiffParams& D) {
  if (!m.dcache || !m.dcache_key || D.sutherland || m.moving) return false;
  const auto* meta = static_cast<const DiffCacheMeta*>(m.dcache_key);
  const DiffCacheKey k = cache_key_of(D);
  return meta->epoch == m.geom_epoch && std::memcmp(&k, &meta->key, sizeof k) == 0;
}
int grid_full(const DevMesh& m) { return std::max(1, std::min(m.nv, 148 * 32)); }
}  // namespace

void diffusion_cache_forget(DevMesh* m) {
  delete static_cast<DiffCacheMeta*>(m->dcache_key);
  m->dcache_key = nullptr;
}

// Built once per mesh geometry and never rewritten for other constants: a state whose
// step graph reads the cache keeps its constants, and a later state with other constants
// takes the full kernel. After the geometry changed (a new epoch) the arrays are refilled
// in place for the next state; a mesh that a Lagrangian state or batch moves has none.
int diffusion_cache_build(DevMesh* m, const DiffParams& D, const double* U, double* dterm, double* mu0c) {
  if (D.sutherland || m->moving) return 0;
  if (m->dcache && m->dcache_key && static_cast<const DiffCacheMeta*>(m->dcache_key)->epoch == m->geom_epoch)
    return 0;
  cudaStream_t s = m->stream;
  if (!m->dcache) {
    std::vector<int> fo(m->nv + 1), so(m->nv + 1);
    SUBFV_CUDA(cudaMemcpyAsync(fo.data(), m->dsf_off, fo.size() * sizeof(int), cudaMemcpyDeviceToHost, s));
    SUBFV_CUDA(cudaMemcpyAsync(so.data(), m->dse_off, so.size() * sizeof(int), cudaMemcpyDeviceToHost, s));
    SUBFV_CUDA(cudaStreamSynchronize(s));
    std::vector<long long> off(m->nv + 1, 0);
    for (int v = 0; v < m->nv; ++v) off[v + 1] = off[v] + diff_cache_doubles(fo[v + 1] - fo[v], so[v + 1] - so[v]);
    const size_t bytes = sizeof(double) * (size_t)off[m->nv] + sizeof(long long) * off.size();
    size_t free_b = 0, total_b = 0;
    SUBFV_CUDA(cudaMemGetInfo(&free_b, &total_b));
    if (bytes > free_b / 2) return 0;  // no room to spare: every step recomputes them
    SUBFV_CUDA(cudaMallocAsync((void**)&m->dcache, sizeof(double) * (size_t)off[m->nv], s));
    SUBFV_CUDA(cudaMallocAsync((void**)&m->dcache_off, sizeof(long long) * off.size(), s));
    SUBFV_CUDA(cudaMemcpyAsync(m->dcache_off, off.data(), sizeof(long long) * off.size(), cudaMemcpyHostToDevice, s));
    SUBFV_CUDA(cudaStreamSynchronize(s));  // off goes out of scope
    m->bytes += bytes;
  }
  diffusion_cache_forget(m);  // invalid until refilled
  k_diff_mu0c<<<1, 1, 0, s>>>(*m, D, U, mu0c, 1);
  k_ns_diffusion<true><<<grid_full(*m), 32, diffusion_smem_bytes(*m), s>>>(*m, D, U, dterm, mu0c, m->dcache,
                                                                            m->dcache_off);
  SUBFV_CUDA(cudaGetLastError());
  SUBFV_CUDA(cudaStreamSynchronize(s));
  m->dcache_key = new DiffCacheMeta{cache_key_of(D), m->geom_epoch};
  return 0;
}

void launch_ns_diffusion(const DevMesh& m, const DiffParams& D, const double* U, double* dterm, double* mu0c) {
  k_diff_mu0c<<<1, 1, 0, m.stream>>>(m, D, U, mu0c, 1);
  if (D.sutherland) k_diff_mu0c<<<grid_for(m.ne, 256), 256, 0, m.stream>>>(m, D, U, mu0c, 0);
  if (cache_matches(m, D)) {
    const size_t smem = sizeof(double) * kDiffWarps * (size_t)(2 * 3 * m.max_dsf + 7 * 3 * m.max_dse);
    const int grid = std::max(1, std::min((m.nv + kDiffWarps - 1) / kDiffWarps, 148 * 16));
    k_ns_diffusion_cached<<<grid, 32 * kDiffWarps, smem, m.stream>>>(m, D, U, dterm, m.dcache, m.dcache_off);
    return;
  }
  // a warp per vertex: as many warps as shared memory lets reside (up to 32 per SM)
  k_ns_diffusion<false><<<grid_full(m), 32, diffusion_smem_bytes(m), m.stream>>>(m, D, U, dterm, mu0c, nullptr,
                                                                                 nullptr);
}

void launch_ns_diffusion_apply(const DevMesh& m, const double* dterm, int kd, double* rhs1, double* diag) {
  k_ns_diffusion_apply<<<grid_for(m.ne, 128), 128, 0, m.stream>>>(m, dterm, kd, rhs1, diag);
}

}  // namespace subfv
