// Test infrastructure only (oracle). Restatement of the BCSR linear algebra of
// src/linear_algebra/sparse_bcsr_linear_module.F90: bcsr_matmul (:13-29), bcsr_diag
// (:1414-1436) with lu_solve_noswp (linear_solver_module.F90:413-445),
// modifiedArnoldi_diag + bcsr_gmres_diag (:1568-1691), the unpreconditioned
// bcsr_gmres (:194-290), and bcsr_parallel_lusgs with bcsr_gmres_parallel_lusgs and
// modifiedArnoldi_parallel_lusgs (:1438-1502, :885-993, :583-611), and bcsr_pcgm
// (:1110-1169) with lu_solve (linear_solver_module.F90:447-484). norm2 is gfortran's scaled sum of squares and dot_product a
// left-to-right sum, as the serial reference evaluates them.
// PARITY UNPINNED (no Fortran compiler here).
#include "oracle.h"
#include <cmath>
#include <vector>

namespace oracle {

struct Bcsr {
  int m, n, bs;
  const int* row;    // (m+1), 1-based
  const int* col;    // (nnz), 1-based
  const double* v;   // (bs, bs, nnz) column-major blocks
};

// :13-29
static void bcsr_matmul(const Bcsr& A, const double* x, double* y) {
  const int bs = A.bs;
  for (int i = 0; i < bs * A.m; ++i) y[i] = 0.0;
  std::vector<double> t(bs);
  for (int i = 1; i <= A.m; ++i)
    for (int j = A.row[i - 1]; j <= A.row[i] - 1; ++j) {
      const double* blk = A.v + (size_t)bs * bs * (j - 1);
      const double* xc = x + (size_t)bs * (A.col[j - 1] - 1);
      for (int r = 0; r < bs; ++r) {
        double s = 0.0;
        for (int c = 0; c < bs; ++c) s = s + blk[r + bs * c] * xc[c];
        t[r] = s;
      }
      for (int r = 0; r < bs; ++r) y[bs * (i - 1) + r] = y[bs * (i - 1) + r] + t[r];
    }
}

// linear_solver_module.F90:413-445 (no pivoting)
static void lu_solve_noswp(int n, const double* A, double* x, const double* b) {
  std::vector<double> C(A, A + n * n);
  for (int i = 0; i < n; ++i) x[i] = b[i];
  auto c = [&](int i, int j) -> double& { return C[i + n * j]; };
  for (int k = 0; k < n; ++k) {
    double invdiag = 1.0 / c(k, k);
    for (int i = k + 1; i < n; ++i) {
      double lik = c(i, k) * invdiag;
      for (int j = k; j < n; ++j) c(i, j) = c(i, j) - lik * c(k, j);
      x[i] = x[i] - lik * x[k];
    }
  }
  x[n - 1] = x[n - 1] / c(n - 1, n - 1);
  for (int k = n - 2; k >= 0; --k) {
    for (int j = k + 1; j < n; ++j) x[k] = x[k] - c(k, j) * x[j];
    x[k] = x[k] / c(k, k);
  }
}

// :1414-1436
static void bcsr_diag(const Bcsr& A, double* x, const double* b) {
  const int bs = A.bs;
  for (int i = 1; i <= A.m; ++i)
    for (int j = A.row[i - 1]; j <= A.row[i] - 1; ++j)
      if (A.col[j - 1] == i) {
        lu_solve_noswp(bs, A.v + (size_t)bs * bs * (j - 1), x + bs * (i - 1), b + bs * (i - 1));
        break;
      }
}

// bcsr_parallel_lusgs (:1438-1502): colour sets ascending for (L+D) y = b (only blocks of
// lower colours), descending for (U+D) x = D y (higher colours, then the diagonal LU);
// color (m) 1..ncs, the rows of a set in ascending order
static void bcsr_parallel_lusgs(const Bcsr& A, double* x, const double* b, int ncs, const int* color) {
  const int bs = A.bs;
  std::vector<double> y((size_t)bs * A.m), t(bs), tmp(bs);
  std::vector<int> d(A.m);
  for (int i = 1; i <= A.m; ++i)
    for (int j = A.row[i - 1]; j <= A.row[i] - 1; ++j)
      if (A.col[j - 1] == i) {
        d[i - 1] = j;
        break;
      }
  auto sub_blocks = [&](int i, int cs, bool lower, double* v, const double* u) {
    for (int j = A.row[i - 1]; j <= A.row[i] - 1; ++j) {
      const int c = A.col[j - 1];
      if (lower ? !(color[c - 1] < cs) : !(color[c - 1] > cs)) continue;
      const double* blk = A.v + (size_t)bs * bs * (j - 1);
      const double* uc = u + (size_t)bs * (c - 1);
      for (int r = 0; r < bs; ++r) {
        double s = 0.0;
        for (int k = 0; k < bs; ++k) s = s + blk[r + bs * k] * uc[k];
        t[r] = s;
      }
      for (int r = 0; r < bs; ++r) v[r] = v[r] - t[r];
    }
  };
  for (int cs = 1; cs <= ncs; ++cs)
    for (int i = 1; i <= A.m; ++i) {
      if (color[i - 1] != cs) continue;
      double* yi = y.data() + (size_t)bs * (i - 1);
      for (int r = 0; r < bs; ++r) yi[r] = b[(size_t)bs * (i - 1) + r];
      sub_blocks(i, cs, true, yi, y.data());
    }
  for (int cs = ncs; cs >= 1; --cs)
    for (int i = 1; i <= A.m; ++i) {
      if (color[i - 1] != cs) continue;
      double* xi = x + (size_t)bs * (i - 1);
      double* yi = y.data() + (size_t)bs * (i - 1);
      for (int r = 0; r < bs; ++r) xi[r] = yi[r];
      sub_blocks(i, cs, false, xi, x);
      for (int r = 0; r < bs; ++r) yi[r] = xi[r];
      lu_solve_noswp(bs, A.v + (size_t)bs * bs * (d[i - 1] - 1), xi, yi);
    }
}

static double dotp(const double* a, const double* b, long n) {
  double s = 0.0;
  for (long i = 0; i < n; ++i) s = s + a[i] * b[i];
  return s;
}

// linear_solver_module.F90:447-484 (lu_solve): partial pivoting on the first largest
// |C(k:n, k)|, whole rows swapped; returns false where the reference stops on
// |C(n,n)| < 1e-12
static bool lu_solve_pivot(int n, const double* A, double* x, const double* b) {
  std::vector<double> C(A, A + n * n);
  auto c = [&](int i, int j) -> double& { return C[i + n * j]; };
  for (int i = 0; i < n; ++i) x[i] = b[i];
  for (int k = 0; k < n; ++k) {
    int p = k;
    for (int i = k + 1; i < n; ++i)
      if (std::fabs(c(i, k)) > std::fabs(c(p, k))) p = i;
    for (int j = 0; j < n; ++j) std::swap(c(k, j), c(p, j));
    std::swap(x[k], x[p]);
    const double invdiag = 1.0 / c(k, k);
    for (int i = k + 1; i < n; ++i) {
      const double lik = c(i, k) * invdiag;
      for (int j = k; j < n; ++j) c(i, j) = c(i, j) - lik * c(k, j);
      x[i] = x[i] - lik * x[k];
    }
  }
  if (std::fabs(c(n - 1, n - 1)) < 1e-12) return false;
  x[n - 1] = x[n - 1] / c(n - 1, n - 1);
  for (int k = n - 2; k >= 0; --k) {
    for (int j = k + 1; j < n; ++j) x[k] = x[k] - c(k, j) * x[j];
    x[k] = x[k] / c(k, k);
  }
  return true;
}

// bcsr_pcgm (:1110-1169): conjugate gradients from the caller's x, preconditioned by
// lu_solve on each diagonal block (the reference passes n = 3: blocks of size 3).
// Returns the iterations; *status 0, 1 not converged (the reference stops), 2 a
// singular diagonal block.
static int bcsr_pcgm(const Bcsr& A, double* x, const double* b, double tol, int* status, double* res) {
  const long n = (long)A.bs * A.m;
  const int bs = A.bs;
  std::vector<double> r(n), p(n), Ap(n), mr(n), w(n);
  std::vector<int> d(A.m);
  for (int i = 1; i <= A.m; ++i)
    for (int j = A.row[i - 1]; j <= A.row[i] - 1; ++j)
      if (A.col[j - 1] == i) {
        d[i - 1] = j;
        break;
      }
  *status = 0;
  auto precond = [&]() {
    for (int i = 0; i < A.m; ++i)
      if (!lu_solve_pivot(bs, A.v + (size_t)bs * bs * (d[i] - 1), mr.data() + (size_t)bs * i,
                          r.data() + (size_t)bs * i))
        *status = 2;
  };
  double rpdrp = 0.0;
  bcsr_matmul(A, x, w.data());
  for (long k = 0; k < n; ++k) r[k] = b[k] - w[k];
  precond();
  double rdr = dotp(mr.data(), r.data(), n);
  *res = std::sqrt(rdr);
  if (std::sqrt(rdr) < tol) return 0;
  p = mr;
  long it = 0;
  for (long k = 1; k <= n; ++k) {
    it = k;
    bcsr_matmul(A, p.data(), Ap.data());
    const double alpha = rdr / dotp(p.data(), Ap.data(), n);
    for (long q = 0; q < n; ++q) x[q] = x[q] + alpha * p[q];
    for (long q = 0; q < n; ++q) r[q] = r[q] - alpha * Ap[q];
    precond();
    rpdrp = dotp(mr.data(), r.data(), n);
    if (std::sqrt(rpdrp) <= tol)
      if (fnorm2(r.data(), (int)n) <= tol) break;
    for (long q = 0; q < n; ++q) p[q] = mr[q] + (rpdrp / rdr) * p[q];
    rdr = rpdrp;
  }
  *res = std::sqrt(rpdrp);
  if (std::sqrt(rpdrp) > tol && *status == 0) *status = 1;
  return (int)it;
}

// GMRES(m) with restarts; precond 1 = bcsr_gmres_diag (maxit 40), 2 =
// bcsr_gmres_parallel_lusgs (:885-993, maxit 20, colours ncs/color), 0 = bcsr_gmres
// (maxit 20). H is (m+1, m) column-major; returns restarts used; *conv as the reference
// sets it.
static int gmres(const Bcsr& A, double* x, const double* b, double tol, int m, int precond, bool* conv,
                 double* rho_out, double* H_first, int ncs = 0, const int* color = nullptr) {
  const long n = (long)A.bs * A.m;
  const int maxit = precond == 1 ? 40 : 20;
  auto apply_precond = [&](double* out, const double* in) {
    if (precond == 2) bcsr_parallel_lusgs(A, out, in, ncs, color);
    else bcsr_diag(A, out, in);
  };
  std::vector<double> H((m + 1) * m, 0.0), V(n * (m + 1)), r(n), y(m + 1), c(m + 1), s(m + 1), z(m + 1), zp(n), w(n);
  auto h = [&](int i, int j) -> double& { return H[(i - 1) + (m + 1) * (j - 1)]; };  // 1-based
  auto Vc = [&](int j) { return V.data() + n * (j - 1); };
  *conv = false;
  for (long i = 0; i < n; ++i) x[i] = 0.0;
  bcsr_matmul(A, x, w.data());
  for (long i = 0; i < n; ++i) r[i] = b[i] - w[i];
  double rho = fnorm2(r.data(), (int)n);
  int it = 0;
  if (rho < tol) {
    *conv = true;
    *rho_out = rho;
    return 0;
  }
  for (int j = 1; j <= maxit; ++j) {
    it = j;
    for (int i = 0; i <= m; ++i) y[i] = 0.0;
    y[0] = rho;
    for (long i = 0; i < n; ++i) r[i] = r[i] / y[0];
    // modifiedArnoldi(_diag) (:1568-1590)
    for (long i = 0; i < n; ++i) Vc(1)[i] = r[i];
    for (int jj = 2; jj <= m + 1; ++jj) {
      if (precond) {
        apply_precond(Vc(jj), Vc(jj - 1));
        bcsr_matmul(A, Vc(jj), w.data());
      } else {
        bcsr_matmul(A, Vc(jj - 1), w.data());
      }
      for (long i = 0; i < n; ++i) Vc(jj)[i] = w[i];
      for (int i = 1; i <= jj - 1; ++i) {
        h(i, jj - 1) = dotp(Vc(i), Vc(jj), n);
        for (long k = 0; k < n; ++k) Vc(jj)[k] = Vc(jj)[k] - h(i, jj - 1) * Vc(i)[k];
      }
      h(jj, jj - 1) = fnorm2(Vc(jj), (int)n);
      for (long k = 0; k < n; ++k) Vc(jj)[k] = Vc(jj)[k] / h(jj, jj - 1);
    }
    if (j == 1 && H_first)
      for (int q = 0; q < (m + 1) * m; ++q) H_first[q] = H[q];
    // Givens rotations (:1634-1658)
    int nr = m, i;
    for (i = 1; i <= m; ++i) {
      for (int k = 2; k <= i; ++k) {
        double tmp = h(k - 1, i);
        h(k - 1, i) = c[k - 2] * h(k - 1, i) + s[k - 2] * h(k, i);
        h(k, i) = -s[k - 2] * tmp + c[k - 2] * h(k, i);
      }
      double delta = std::sqrt(h(i, i) * h(i, i) + h(i + 1, i) * h(i + 1, i));
      c[i - 1] = h(i, i) / delta;
      s[i - 1] = h(i + 1, i) / delta;
      h(i, i) = c[i - 1] * h(i, i) + s[i - 1] * h(i + 1, i);
      for (int k = i + 1; k <= m + 1; ++k) h(k, i) = 0.0;
      y[i] = -s[i - 1] * y[i - 1];
      y[i - 1] = c[i - 1] * y[i - 1];
      rho = std::fabs(y[i]);
      if (rho < tol) {
        nr = i + 1;
        break;
      }
    }
    // back substitution (:1660-1673); i is m+1 when the loop ran to the end
    for (int k = 0; k <= m; ++k) z[k] = 0.0;
    if (i >= m) {
      nr = m;
      z[nr - 1] = y[nr - 1] / h(nr, nr);
    }
    for (int k = nr - 1; k >= 1; --k) {
      z[k - 1] = y[k - 1];
      for (int l = k + 1; l <= nr; ++l) z[k - 1] = z[k - 1] - h(k, l) * z[l - 1];
      z[k - 1] = z[k - 1] / h(k, k);
    }
    if (precond) {
      for (long k = 0; k < n; ++k) r[k] = 0.0;
      for (int q = 1; q <= nr; ++q)
        for (long k = 0; k < n; ++k) r[k] = r[k] + z[q - 1] * Vc(q)[k];
      apply_precond(zp.data(), r.data());
      for (long k = 0; k < n; ++k) x[k] = x[k] + zp[k];
    } else {
      for (int q = 1; q <= nr; ++q)
        for (long k = 0; k < n; ++k) x[k] = x[k] + z[q - 1] * Vc(q)[k];
    }
    bcsr_matmul(A, x, w.data());
    for (long k = 0; k < n; ++k) r[k] = b[k] - w[k];
    rho = fnorm2(r.data(), (int)n);
    if (rho < tol) {
      if (precond == 1) *conv = true;
      break;
    }
  }
  if (precond != 1) {  // :284-289 and :987-992
    bcsr_matmul(A, x, w.data());
    for (long k = 0; k < n; ++k) r[k] = b[k] - w[k];
    *conv = !(fnorm2(r.data(), (int)n) > tol);
  }
  *rho_out = rho;
  return it;
}

}  // namespace oracle

using namespace oracle;

extern "C" {

void or_bcsr_matmul(int m, int n, int bs, const int* row, const int* col, const double* v, const double* x, double* y) {
  Bcsr A{m, n, bs, row, col, v};
  bcsr_matmul(A, x, y);
}
void or_bcsr_diag(int m, int bs, const int* row, const int* col, const double* v, double* x, const double* b) {
  Bcsr A{m, m, bs, row, col, v};
  bcsr_diag(A, x, b);
}
int or_bcsr_gmres(int m, int bs, const int* row, const int* col, const double* v, double* x, const double* b,
                  double tol, int krylov, int precond, int* conv, double* rho, double* H_first) {
  Bcsr A{m, m, bs, row, col, v};
  bool cv = false;
  int it = gmres(A, x, b, tol, krylov, precond != 0 ? 1 : 0, &cv, rho, H_first);
  *conv = cv ? 1 : 0;
  return it;
}
int or_bcsr_pcgm(int m, int bs, const int* row, const int* col, const double* v, double* x, const double* b,
                 double tol, int* status, double* res) {
  Bcsr A{m, m, bs, row, col, v};
  return bcsr_pcgm(A, x, b, tol, status, res);
}
void or_bcsr_parallel_lusgs(int m, int bs, const int* row, const int* col, const double* v, int ncs,
                            const int* color, double* x, const double* b) {
  Bcsr A{m, m, bs, row, col, v};
  bcsr_parallel_lusgs(A, x, b, ncs, color);
}
int or_bcsr_gmres_lusgs(int m, int bs, const int* row, const int* col, const double* v, int ncs, const int* color,
                        double* x, const double* b, double tol, int krylov, int* conv, double* rho) {
  Bcsr A{m, m, bs, row, col, v};
  bool cv = false;
  int it = gmres(A, x, b, tol, krylov, 2, &cv, rho, nullptr, ncs, color);
  *conv = cv ? 1 : 0;
  return it;
}

}  // extern "C"
