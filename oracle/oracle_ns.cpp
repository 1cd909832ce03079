// Test infrastructure only (oracle). Restatement of the subfv explicit Euler path
// (subfvns): src/ns/ns_euler_primitives_module.F90, src/ns/ns_euler_recon_module.F90,
// src/ns/ns_euler_rs_module.F90 (two_wave, multi_point, the multi-point nodal velocity
// solver), src/ns/ns_euler_module.F90 (compute_euler_flux, compute_rhs_around_vert,
// add_timedisc_and_solve), the contained compute_rhs_ns and the time loop of
// src/ns/ns_main.F90:83-130, and the Gresho initial state of
// src/ns/ns_euler_exact_sol_module.F90:7-44.
//
// LAPACK stand-ins (the reference links an unpinned system LAPACK):
//  * dgesvd-based pseudo_inverse_inplace_lapack (linear_solver_module.F90:683-715):
//    one-sided Jacobi SVD, six sweeps, same singular-value cut n*1e-12*max(sigma);
//  * lu_solve_inplace_lapack (:643-657): LU with partial pivoting in LAPACK's
//    dgetrf2 / dgetrs operation order, reference-BLAS triangular solves.
// PARITY UNPINNED (no Fortran compiler or LAPACK build of the reference here).
#include "oracle.h"
#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <map>
#include <vector>

namespace oracle {

static const double G = 1.4;  // ns_global_data_module.F90:9

struct NsCfg {
  int scheme;  // 1 multi_point, 2 _iso, 3 three_wave, 4 two_wave, 5 modified_three_wave, 6/8 multi_point_pressure(_ph)
  int second_order;    // 0/1
  int method;          // 0/1 (no gradient), 2-6 (compute_cell_grad_method_2..6)
  int bc_style;        // 0, 1, 2
  int b2d;
  int exclude_bound_vert;
  double cfl, tmax;
  int local_time_step;
  int n_bc;
  const int* bc_type;     // per tag: 1 wall, 3 freestream, 4 outflow supersonic
  const double* bc_val;   // per tag: 5 primitive values
};

// ---------------------------------------------------------------- primitives (:7-111)
static void p2c(const double* w, double* u) {
  u[0] = w[0];
  for (int k = 1; k < 4; ++k) u[k] = w[k] * w[0];
  u[4] = w[4] / (G - 1) + 0.5 * w[0] * (w[1] * w[1] + w[2] * w[2] + w[3] * w[3]);
}
static void c2p(const double* u, double* w) {
  w[0] = u[0];
  for (int k = 1; k < 4; ++k) w[k] = u[k] / u[0];
  w[4] = (G - 1) * (u[4] - 0.5 * w[0] * (w[1] * w[1] + w[2] * w[2] + w[3] * w[3]));
}
static double sound_speed_w(const double* w) { return std::sqrt(G * w[4] / w[0]); }
static double fmax2(double a, double b) { return b > a ? b : a; }
static double fmin2(double a, double b) { return b < a ? b : a; }
static double dot3(const double* a, const double* b) {
  double s = 0.0;
  for (int k = 0; k < 3; ++k) s = s + a[k] * b[k];
  return s;
}

double max_omega_for_positivity(const double* U, const double* dU) {
  double omega = 1.0, US[5], WS[5];
  for (int k = 0; k < 5; ++k) US[k] = U[k] + omega * dU[k];
  c2p(US, WS);
  bool pos = WS[0] > 1e-17 && WS[4] > 1e-17;
  while (!pos && omega > 1e-6) {
    omega = omega * 0.9;
    for (int k = 0; k < 5; ++k) US[k] = U[k] + omega * dU[k];
    c2p(US, WS);
    pos = WS[0] > 1e-17 && WS[4] > 1e-17;
  }
  return omega;
}

// ---------------------------------------------------------------- LAPACK stand-ins
// When every singular value passes the cut, the pseudo-inverse is the inverse. The cut
// (3e-12 * sigma_max) is certainly passed when |det A| > 3e-12 ||A||_F^3, because
// sigma_min >= |det A| / sigma_max^2 and sigma_max <= ||A||_F. Then A^-1 = adj(A) / det,
// refined by one Newton step X <- X + X (I - A X); otherwise the Jacobi SVD below runs.
static bool inv3_if_regular(double A[3][3]) {
  double f2 = 0.0;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) f2 = f2 + A[i][j] * A[i][j];
  double C[3][3];  // cofactors
  C[0][0] = A[1][1] * A[2][2] - A[1][2] * A[2][1];
  C[0][1] = A[1][2] * A[2][0] - A[1][0] * A[2][2];
  C[0][2] = A[1][0] * A[2][1] - A[1][1] * A[2][0];
  C[1][0] = A[0][2] * A[2][1] - A[0][1] * A[2][2];
  C[1][1] = A[0][0] * A[2][2] - A[0][2] * A[2][0];
  C[1][2] = A[0][1] * A[2][0] - A[0][0] * A[2][1];
  C[2][0] = A[0][1] * A[1][2] - A[0][2] * A[1][1];
  C[2][1] = A[0][2] * A[1][0] - A[0][0] * A[1][2];
  C[2][2] = A[0][0] * A[1][1] - A[0][1] * A[1][0];
  const double det = A[0][0] * C[0][0] + A[0][1] * C[0][1] + A[0][2] * C[0][2];
  if (!(det * det > 9e-24 * (f2 * f2 * f2))) return false;
  const double r = 1.0 / det;
  double X[3][3], R[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) X[i][j] = C[j][i] * r;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double s = i == j ? 1.0 : 0.0;
      for (int k = 0; k < 3; ++k) s = s - A[i][k] * X[k][j];
      R[i][j] = s;
    }
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double s = 0.0;
      for (int k = 0; k < 3; ++k) s = s + X[i][k] * R[k][j];
      A[i][j] = X[i][j] + s;
    }
  return true;
}

// Optional real LAPACK (Fortran calling convention, no hidden string lengths): when set
// by or_set_lapack, pinv3 and lu_solve3 call it exactly as pseudo_inverse_inplace_lapack
// and lu_solve_inplace_lapack do (linear_solver_module.F90:643-657, 683-715), in place
// of the restated algorithms above and below. Test infrastructure only: it measures how
// far the restatement's results drift from the reference's LAPACK calls.
typedef void (*dgesvd_fn)(char*, char*, int*, int*, double*, int*, double*, double*, int*, double*, int*, double*,
                          int*, int*);
typedef void (*dgetrf_fn)(int*, int*, double*, int*, int*, int*);
typedef void (*dgetrs_fn)(char*, int*, int*, double*, int*, int*, double*, int*, int*);
static dgesvd_fn g_dgesvd = nullptr;
static dgetrf_fn g_dgetrf = nullptr;
static dgetrs_fn g_dgetrs = nullptr;

// pseudo_inverse_inplace_lapack(3, mat), linear_solver_module.F90:683-715: dgesvd('A', 'O')
// with LWORK = 5 n (the reference passes 5*n, not the queried size), VT written over A,
// cut n 1e-12 max(Sigma), then A = matmul(transpose(A), matmul(Sigma_plus, transpose(U)))
// with gfortran's matmul summing k ascending.
static void pinv3_lapack(double A[3][3]) {
  double a[9], U[9], S[3], work[15];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) a[c * 3 + r] = A[r][c];
  int n = 3, lda = 3, ldu = 3, ldvt = 3, lwork = 15, info = 0;
  char ju = 'A', jvt = 'O';
  g_dgesvd(&ju, &jvt, &n, &n, a, &lda, S, U, &ldu, a, &ldvt, work, &lwork, &info);
  double smax = S[0];
  for (int i = 1; i < 3; ++i) smax = std::fmax(smax, S[i]);
  const double tol = 3 * 1e-12 * smax;
  double Sp[3][3] = {};
  for (int i = 0; i < 3; ++i) Sp[i][i] = S[i] > tol ? 1.0 / S[i] : 0.0;
  double T[3][3];  // matmul(Sigma_plus, transpose(U)): T(i,j) = sum_k Sp(i,k) U(j,k)
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double s = 0.0;
      for (int k = 0; k < 3; ++k) s = s + Sp[i][k] * U[k * 3 + j];
      T[i][j] = s;
    }
  for (int i = 0; i < 3; ++i)  // matmul(transpose(VT), T): sum_k VT(k,i) T(k,j)
    for (int j = 0; j < 3; ++j) {
      double s = 0.0;
      for (int k = 0; k < 3; ++k) s = s + a[i * 3 + k] * T[k][j];
      A[i][j] = s;
    }
}

// A[r][c] = mat(r+1, c+1). The inverse when the cut cannot bite, else one-sided Jacobi
// on the columns: A V = U S.
void pinv3(double A[3][3]) {
  if (g_dgesvd) {
    pinv3_lapack(A);
    return;
  }
  if (inv3_if_regular(A)) return;
  double U[3][3], V[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  std::memcpy(U, A, sizeof(U));
  const int pr[3][2] = {{0, 1}, {0, 2}, {1, 2}};
  for (int sweep = 0; sweep < 6; ++sweep)
    for (const auto& pq : pr) {
      int p = pq[0], q = pq[1];
      double al = 0.0, be = 0.0, ga = 0.0;
      for (int i = 0; i < 3; ++i) {
        al = al + U[i][p] * U[i][p];
        be = be + U[i][q] * U[i][q];
        ga = ga + U[i][p] * U[i][q];
      }
      if (!(std::fabs(ga) > 1e-15 * std::sqrt(al * be))) continue;
      double zeta = (be - al) / (2.0 * ga);
      double t = 1.0 / (std::fabs(zeta) + std::sqrt(1.0 + zeta * zeta));
      if (zeta < 0.0) t = -t;
      double c = 1.0 / std::sqrt(1.0 + t * t), s = c * t;
      for (int i = 0; i < 3; ++i) {
        double up = U[i][p], uq = U[i][q];
        U[i][p] = c * up - s * uq;
        U[i][q] = s * up + c * uq;
        double vp = V[i][p], vq = V[i][q];
        V[i][p] = c * vp - s * vq;
        V[i][q] = s * vp + c * vq;
      }
    }
  double sig[3], smax = 0.0;
  for (int k = 0; k < 3; ++k) {
    double s = 0.0;
    for (int i = 0; i < 3; ++i) s = s + U[i][k] * U[i][k];
    sig[k] = std::sqrt(s);
    smax = fmax2(smax, sig[k]);
  }
  double tol = 3 * 1e-12 * smax;
  double SUt[3][3];  // Sigma_plus * U^T, U^T row k = u_k = U[:,k] / sig_k
  for (int k = 0; k < 3; ++k)
    for (int j = 0; j < 3; ++j) SUt[k][j] = sig[k] > tol ? (1.0 / sig[k]) * (U[j][k] / sig[k]) : 0.0;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double s = 0.0;
      for (int k = 0; k < 3; ++k) s = s + V[i][k] * SUt[k][j];
      A[i][j] = s;
    }
}

// dgetrf2 + dgetrs ('N') on a 3x3 system; A is overwritten.
void lu_solve3(double A[3][3], double* x, const double* b) {
  if (g_dgetrf && g_dgetrs) {  // lu_solve_inplace_lapack, linear_solver_module.F90:643-657
    double a[9], bc[3] = {b[0], b[1], b[2]};
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) a[c * 3 + r] = A[r][c];
    int n = 3, one = 1, ipiv[3], info = 0;
    char tr = 'N';
    g_dgetrf(&n, &n, a, &n, ipiv, &info);
    g_dgetrs(&tr, &n, &one, a, &n, ipiv, bc, &n, &info);
    for (int k = 0; k < 3; ++k) x[k] = bc[k];
    return;
  }
  const double sfmin = 2.2250738585072014e-308;
  int ipiv[3];
  for (int j = 0; j < 3; ++j) {
    int p = j;
    double amax = std::fabs(A[j][j]);
    for (int i = j + 1; i < 3; ++i)
      if (std::fabs(A[i][j]) > amax) {
        amax = std::fabs(A[i][j]);
        p = i;
      }
    ipiv[j] = p;
    if (A[p][j] != 0.0) {
      if (p != j)
        for (int k = 0; k < 3; ++k) std::swap(A[j][k], A[p][k]);
      if (std::fabs(A[j][j]) >= sfmin) {
        double r = 1.0 / A[j][j];
        for (int i = j + 1; i < 3; ++i) A[i][j] = r * A[i][j];
      } else {
        for (int i = j + 1; i < 3; ++i) A[i][j] = A[i][j] / A[j][j];
      }
    }
    for (int i = j + 1; i < 3; ++i)
      for (int k = j + 1; k < 3; ++k) A[i][k] = A[i][k] - A[j][k] * A[i][j];
  }
  double y[3] = {b[0], b[1], b[2]};
  for (int j = 0; j < 3; ++j)
    if (ipiv[j] != j) std::swap(y[j], y[ipiv[j]]);
  for (int k = 0; k < 3; ++k)
    if (y[k] != 0.0)
      for (int i = k + 1; i < 3; ++i) y[i] = y[i] - y[k] * A[i][k];
  for (int k = 2; k >= 0; --k)
    if (y[k] != 0.0) {
      y[k] = y[k] / A[k][k];
      for (int i = 0; i < k; ++i) y[i] = y[i] - y[k] * A[i][k];
    }
  for (int k = 0; k < 3; ++k) x[k] = y[k];
}

// ---------------------------------------------------------------- fluxes (ns_euler_rs_module.F90)
// :154-198
static void two_wave(const double* wl, const double* wr, const double* n, double lr[2][5], double* sl, double* sr) {
  double rhol = wl[0], vnl = dot3(wl + 1, n), pl = wl[4], al = sound_speed_w(wl), ul[5];
  p2c(wl, ul);
  double rhor = wr[0], vnr = dot3(wr + 1, n), pr = wr[4], ar = sound_speed_w(wr), ur[5];
  p2c(wr, ur);
  double fl[5], fr[5];
  fl[0] = vnl * ul[0];
  for (int k = 1; k < 4; ++k) fl[k] = vnl * ul[k] + pl * n[k - 1];
  fl[4] = (ul[4] + pl) * vnl;
  fr[0] = vnr * ur[0];
  for (int k = 1; k < 4; ++k) fr[k] = vnr * ur[k] + pr * n[k - 1];
  fr[4] = (ur[4] + pr) * vnr;
  double lam_l = fmax2(fmax2(al * rhol, std::sqrt(rhol * fmax2(0.0, pr - pl))), -rhol * (vnr - vnl));
  double lam_r = fmax2(fmax2(ar * rhor, std::sqrt(rhor * fmax2(0.0, pl - pr))), -rhor * (vnr - vnl));
  *sl = vnl - lam_l / rhol;
  *sr = vnr + lam_r / rhor;
  for (int k = 0; k < 5; ++k) {
    double et = (*sr * ur[k] - *sl * ul[k] - (fr[k] - fl[k])) / (*sr - *sl);
    lr[0][k] = 0.5 * (fl[k] + fr[k]) - 0.5 * (std::fabs(*sl) * (et - ul[k]) + std::fabs(*sr) * (ur[k] - et));
    lr[1][k] = -lr[0][k];
  }
}

// three_wave (:9-75) and modified_three_wave (:77-152): the two-wave bounds, v* = v_bar,
// HLLC-type star states (the modified form also averages the tangential velocity and
// carries its jump energy), no nodal solve.
static void three_wave(const double* wl, const double* wr, const double* n, double lr[2][5], double* sl, double* sr,
                       bool modified) {
  double rhol = wl[0], vnl = dot3(wl + 1, n), pl = wl[4], ul[5];
  p2c(wl, ul);
  double el = ul[4] / rhol, al = sound_speed_w(wl);
  double rhor = wr[0], vnr = dot3(wr + 1, n), pr = wr[4], ur[5];
  p2c(wr, ur);
  double er = ur[4] / rhor, ar = sound_speed_w(wr);
  double fl[5], fr[5];
  fl[0] = vnl * ul[0];
  for (int k = 1; k < 4; ++k) fl[k] = vnl * ul[k] + pl * n[k - 1];
  fl[4] = (ul[4] + pl) * vnl;
  fr[0] = vnr * ur[0];
  for (int k = 1; k < 4; ++k) fr[k] = vnr * ur[k] + pr * n[k - 1];
  fr[4] = (ur[4] + pr) * vnr;
  double lam_l = fmax2(fmax2(al * rhol, std::sqrt(rhol * fmax2(0.0, pr - pl))), -rhol * (vnr - vnl));
  double lam_r = fmax2(fmax2(ar * rhor, std::sqrt(rhor * fmax2(0.0, pl - pr))), -rhor * (vnr - vnl));
  double v_et = (lam_l * vnl + lam_r * vnr - (pr - pl)) / (lam_r + lam_l);
  double vt_et[3] = {0.0, 0.0, 0.0}, tang_energy = 0.0;
  if (modified) {
    double vt_l[3], vt_r[3], dvt[3];
    for (int d = 0; d < 3; ++d) {
      vt_l[d] = wl[1 + d] - vnl * n[d];
      vt_r[d] = wr[1 + d] - vnr * n[d];
    }
    for (int d = 0; d < 3; ++d) vt_et[d] = (lam_l * vt_l[d] + lam_r * vt_r[d]) / (lam_l + lam_r);
    for (int d = 0; d < 3; ++d) dvt[d] = vt_r[d] - vt_l[d];
    double tang_coeff = -(lam_l * lam_r / (lam_l + lam_r));
    tang_energy = tang_coeff * dot3(dvt, vt_et);
  }
  double rhol_et = 1.0 / (1.0 / rhol + (v_et - vnl) / lam_l);
  double pl_bar = pl - lam_l * (v_et - vnl);
  double rhor_et = 1.0 / (1.0 / rhor + (vnr - v_et) / lam_r);
  double pr_bar = pr + lam_r * (v_et - vnr);
  double sle[5], sre[5];
  sle[0] = rhol_et;
  sre[0] = rhor_et;
  if (modified) {
    for (int k = 1; k < 4; ++k) sle[k] = rhol_et * (v_et * n[k - 1] + vt_et[k - 1]);
    sle[4] = rhol_et * (el + (pl * vnl - pl_bar * v_et - tang_energy) / lam_l);
    for (int k = 1; k < 4; ++k) sre[k] = rhor_et * (v_et * n[k - 1] + vt_et[k - 1]);
    sre[4] = rhor_et * (er + (pr_bar * v_et - pr * vnr + tang_energy) / lam_r);
  } else {
    for (int k = 1; k < 4; ++k) sle[k] = rhol_et * (wl[k] + (v_et - vnl) * n[k - 1]);
    sle[4] = rhol_et * (el + (pl * vnl - pl_bar * v_et) / lam_l);
    for (int k = 1; k < 4; ++k) sre[k] = rhor_et * (wr[k] + (v_et - vnr) * n[k - 1]);
    sre[4] = rhor_et * (er + (pr_bar * v_et - pr * vnr) / lam_r);
  }
  *sl = vnl - lam_l / rhol;
  *sr = vnr + lam_r / rhor;
  for (int k = 0; k < 5; ++k) {
    lr[0][k] = 0.5 * (fl[k] + fr[k]) - 0.5 * (std::fabs(*sl) * (sle[k] - ul[k]) + std::fabs(v_et) * (sre[k] - sle[k]) +
                                              std::fabs(*sr) * (ur[k] - sre[k]));
    lr[1][k] = -lr[0][k];
  }
}

// multi_point_pressure (:555-616) and multi_point_pressure_ph (:618-679): star states from
// the nodal pressure p_nodal and the bounds of the nodal pressure solver
static void multi_point_pressure(const double* wl, const double* wr, const double* n, double lr[2][5],
                                 double p_nodal, double lam_l, double lam_r, double* sl, double* sr, bool ph) {
  double rhol = wl[0], vnl = dot3(wl + 1, n), pl = wl[4], ul[5], vt_l[3];
  for (int d = 0; d < 3; ++d) vt_l[d] = wl[1 + d] - vnl * n[d];
  p2c(wl, ul);
  double el = ul[4] / rhol;
  double rhor = wr[0], vnr = dot3(wr + 1, n), pr = wr[4], ur[5], vt_r[3];
  for (int d = 0; d < 3; ++d) vt_r[d] = wr[1 + d] - vnr * n[d];
  p2c(wr, ur);
  double er = ur[4] / rhor;
  double fl[5], fr[5];
  fl[0] = vnl * ul[0];
  for (int k = 1; k < 4; ++k) fl[k] = vnl * ul[k] + pl * n[k - 1];
  fl[4] = (ul[4] + pl) * vnl;
  fr[0] = vnr * ur[0];
  for (int k = 1; k < 4; ++k) fr[k] = vnr * ur[k] + pr * n[k - 1];
  fr[4] = (ur[4] + pr) * vnr;
  double vn_bar = (lam_l * vnl + lam_r * vnr - (pr - pl)) / (lam_r + lam_l);
  double vn_l_et = vnl - (p_nodal - pl) / lam_l;
  double rhol_et = 1.0 / (1.0 / rhol + (vn_bar - vnl) / lam_l);
  double sle[5], sre[5];
  sle[0] = rhol_et;
  for (int k = 1; k < 4; ++k) sle[k] = rhol_et * (vt_l[k - 1] + vn_l_et * n[k - 1]);
  sle[4] = rhol_et * (el + (pl * vnl - p_nodal * (ph ? vn_l_et : vn_bar)) / lam_l);
  double vn_r_et = vnr + (p_nodal - pr) / lam_r;
  double rhor_et = 1.0 / (1.0 / rhor + (vnr - vn_bar) / lam_r);
  sre[0] = rhor_et;
  for (int k = 1; k < 4; ++k) sre[k] = rhor_et * (vt_r[k - 1] + vn_r_et * n[k - 1]);
  sre[4] = rhor_et * (er + (p_nodal * (ph ? vn_r_et : vn_bar) - pr * vnr) / lam_r);
  *sl = vnl - lam_l / rhol;
  *sr = vnr + lam_r / rhor;
  for (int k = 0; k < 5; ++k) {
    lr[0][k] = 0.5 * (fl[k] + fr[k]) - 0.5 * (std::fabs(*sl) * (sle[k] - ul[k]) + std::fabs(vn_bar) * (sre[k] - sle[k]) +
                                              std::fabs(*sr) * (ur[k] - sre[k]));
    lr[1][k] = -lr[0][k];
  }
}

// :200-286; returns false on a negative star density (the reference error-stops)
static bool multi_point(const double* wl, const double* wr, const double* n, double lr[2][5], double vn_nodal,
                        double lam_l, double lam_r, double* sl, double* sr) {
  double rhol = wl[0], vnl = dot3(wl + 1, n), pl = wl[4], ul[5];
  p2c(wl, ul);
  double el = ul[4] / rhol;
  double rhor = wr[0], vnr = dot3(wr + 1, n), pr = wr[4], ur[5];
  p2c(wr, ur);
  double er = ur[4] / rhor;
  double fl[5], fr[5];
  fl[0] = vnl * ul[0];
  for (int k = 1; k < 4; ++k) fl[k] = vnl * ul[k] + pl * n[k - 1];
  fl[4] = (ul[4] + pl) * vnl;
  fr[0] = vnr * ur[0];
  for (int k = 1; k < 4; ++k) fr[k] = vnr * ur[k] + pr * n[k - 1];
  fr[4] = (ur[4] + pr) * vnr;
  double v_et = vn_nodal;
  double rhol_et = 1.0 / (1.0 / rhol + (v_et - vnl) / lam_l);
  double pl_bar = pl - lam_l * (v_et - vnl);
  double sle[5], sre[5];
  sle[0] = rhol_et;
  for (int k = 1; k < 4; ++k) sle[k] = rhol_et * (wl[k] + (v_et - vnl) * n[k - 1]);
  sle[4] = rhol_et * (el + (pl * vnl - pl_bar * v_et) / lam_l);
  double rhor_et = 1.0 / (1.0 / rhor + (vnr - v_et) / lam_r);
  double pr_bar = pr + lam_r * (v_et - vnr);
  sre[0] = rhor_et;
  for (int k = 1; k < 4; ++k) sre[k] = rhor_et * (wr[k] + (v_et - vnr) * n[k - 1]);
  sre[4] = rhor_et * (er + (pr_bar * v_et - pr * vnr) / lam_r);
  bool ok = !(rhol_et < 0.0 || rhor_et < 0.0);
  *sl = vnl - lam_l / rhol;
  *sr = vnr + lam_r / rhor;
  const double e[5] = {0.0, n[0], n[1], n[2], v_et};
  for (int k = 0; k < 5; ++k) {
    double base = 0.5 * (fl[k] + fr[k]) -
                  0.5 * (std::fabs(*sl) * (sle[k] - ul[k]) + std::fabs(v_et) * (sre[k] - sle[k]) +
                         std::fabs(*sr) * (ur[k] - sre[k]));
    double jump = 0.5 * (pr_bar - pl_bar) * e[k];
    lr[0][k] = base - jump;
    lr[1][k] = -(base + jump);
  }
  return ok;
}

// ---------------------------------------------------------------- reconstruction (ns_euler_recon_module.F90)
static bool is_wall(const NsCfg& cfg, int re) {
  if (re > 0) return false;
  if (re == 0) return true;
  return cfg.bc_type[-re - 1] == 1;
}

// :331-409 (wall, freestream, outflow supersonic); sol_l/sol_r conservative
// the time of the step being evaluated (ns_global_data_module's t, read by the
// time-dependent boundary states); set by the time loop
static double g_ns_time = 0.0;

// :413-419 (sol_potential_flow_2d / _3d, ns_euler_exact_sol_module.F90:105-170)
static void potential_flow(const double* x, bool three_d, double* w) {
  // the 2-D routine declares its Mach number with a default-kind (single precision)
  // literal, 1e-4, so its value is the float nearest 1e-4; the 3-D one uses 1e-4_DOUBLE
  const double r0 = 0.5, r1 = 5.5, rhoinf = 1.4, pinf = 1.0;
  const double mach = three_d ? 1e-4 : (double)1e-4f;
  const double vinf = mach * std::sqrt(G * pinf / rhoinf);
  double ux, uy, uz;
  if (!three_d) {
    const double r = std::sqrt(x[0] * x[0] + x[1] * x[1]);
    const double th = std::atan2(x[1], x[0]);
    const double c = r1 * r1 / (r1 * r1 - r0 * r0), q = (r0 / r) * (r0 / r);
    const double vr = c * (1.0 - q) * std::cos(th);
    const double vt = -c * (1.0 + q) * std::sin(th);
    ux = vinf * (std::cos(th) * vr - std::sin(th) * vt);
    uy = vinf * (std::sin(th) * vr + std::cos(th) * vt);
    uz = 0.0;
  } else {
    const double r = std::sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
    const double f = r0 * r0 * r0 / (2.0 * (r * r * r * r * r));
    ux = vinf * (1.0 + f * (r * r - 3.0 * (x[0] * x[0])));
    uy = -3.0 * vinf * f * x[0] * x[1];
    uz = -3.0 * vinf * f * x[0] * x[2];
  }
  const double vmag2 = ux * ux + uy * uy + uz * uz;
  w[0] = rhoinf;
  w[1] = ux;
  w[2] = uy;
  w[3] = uz;
  w[4] = pinf + 0.5 * rhoinf * (vinf * vinf - vmag2);
}

// :331-409: the ghost state by boundary kind (1 wall, 2 adherence wall, 3 freestream,
// 4 supersonic outflow, 5 pondered inflow, 6 and 7 the double-Mach inflow/outflow and
// bottom, 8 and 9 the potential flows), sol_l / sol_r conservative
static void compute_right_state(const Mesh& m, const NsCfg& cfg, int sf, int re, const double* sol_l, double* sol_r) {
  const double* n = &m.sub_face[sf].norm[1];
  const double* fx = &m.face[m.sub_face[sf].mesh_face].coord[1];
  int kind = re == 0 ? 1 : cfg.bc_type[-re - 1];
  const double* bv = re < 0 ? cfg.bc_val + 5 * (-re - 1) : nullptr;
  auto mirror = [&]() {
    for (int k = 0; k < 5; ++k) sol_r[k] = sol_l[k];
    double d = dot3(sol_r + 1, n);
    for (int k = 1; k < 4; ++k) sol_r[k] = sol_r[k] - 2.0 * d * n[k - 1];
  };
  const double post[5] = {8.0, 7.145, -4.125, 0.0, 116.5}, pre[5] = {1.4, 0.0, 0.0, 0.0, 1.0};
  if (kind == 1) {
    mirror();
  } else if (kind == 2) {
    for (int k = 0; k < 5; ++k) sol_r[k] = sol_l[k];
    for (int k = 1; k < 4; ++k) sol_r[k] = 2.0 * sol_l[0] * bv[k] - sol_l[k];
    double ul[3], ur[3];
    for (int d = 0; d < 3; ++d) {
      ul[d] = sol_l[1 + d] / sol_l[0];
      ur[d] = sol_r[1 + d] / sol_r[0];
    }
    const double nl = fnorm2(ul, 3), nr = fnorm2(ur, 3);
    sol_r[4] = sol_l[4] - 0.5 * sol_l[0] * (nl * nl) + 0.5 * sol_l[0] * (nr * nr);
  } else if (kind == 3) {
    p2c(bv, sol_r);
  } else if (kind == 5) {
    p2c(bv, sol_r);
    if (dot3(sol_r + 1, n) > 0.0)
      for (int k = 0; k < 5; ++k) sol_r[k] = sol_l[k];
  } else if (kind == 6) {
    p2c(fx[1] > 1.732 * (fx[0] - 0.1667 - 10.0 * g_ns_time) ? post : pre, sol_r);
  } else if (kind == 7) {
    if (fx[0] < 0.1667) p2c(post, sol_r);
    else mirror();
  } else if (kind == 8 || kind == 9) {
    double w[5];
    potential_flow(fx, kind == 9, w);
    p2c(w, sol_r);
  } else {
    for (int k = 0; k < 5; ++k) sol_r[k] = sol_l[k];
  }
}

// :427-451; grad[c*15 + d*5 + var] = grad(d+1, var+1, c+1)
static void reconstruct_lr_w(const Mesh& m, const NsCfg& cfg, const double* sol, const double* grad, int v, int sf,
                             int le, int re, bool so, double* wl, double* wr) {
  c2p(sol + 5 * (le - 1), wl);
  if (so) {
    double dx[3];
    for (int d = 0; d < 3; ++d) dx[d] = m.vert[v].coord[d + 1] - m.elem[le].coord[d + 1];
    const double* g = grad + 15 * (le - 1);
    for (int k = 0; k < 5; ++k) {
      double s = 0.0;
      for (int d = 0; d < 3; ++d) s = s + g[5 * d + k] * dx[d];
      wl[k] = wl[k] + s;
    }
  }
  if (re > 0) {
    c2p(sol + 5 * (re - 1), wr);
    if (so) {
      double dx[3];
      for (int d = 0; d < 3; ++d) dx[d] = m.vert[v].coord[d + 1] - m.elem[re].coord[d + 1];
      const double* g = grad + 15 * (re - 1);
      for (int k = 0; k < 5; ++k) {
        double s = 0.0;
        for (int d = 0; d < 3; ++d) s = s + g[5 * d + k] * dx[d];
        wr[k] = wr[k] + s;
      }
    }
  } else {
    double ul[5], ghost[5];
    p2c(wl, ul);
    compute_right_state(m, cfg, sf, re, ul, ghost);
    c2p(ghost, wr);
  }
}

// :453-490
static void compute_nodal_grad(const Mesh& m, int v, const double* sol, double* ng) {
  double g[3][5] = {{0}}, mat[3][3] = {{0}};
  const Vert& vv = m.vert[v];
  for (int i = 1; i <= vv.n_sub_faces_neigh; ++i) {
    int sf = vv.sub_face_neigh[i];
    const Face& f = m.face[m.sub_face[sf].mesh_face];
    int le = f.left_neigh, re = f.right_neigh;
    if (re > 0) {
      double wl[5], wr[5];
      c2p(sol + 5 * (le - 1), wl);
      c2p(sol + 5 * (re - 1), wr);
      const double* n = &m.sub_face[sf].norm[1];
      double a = m.sub_face[sf].area;
      for (int d = 0; d < 3; ++d)
        for (int k = 0; k < 5; ++k) g[d][k] = g[d][k] + a * (n[d] * (wr[k] - wl[k]));
      for (int d = 0; d < 3; ++d)
        for (int e = 0; e < 3; ++e)
          mat[d][e] = mat[d][e] + a * (n[d] * (m.elem[re].coord[e + 1] - m.elem[le].coord[e + 1]));
    }
  }
  pinv3(mat);
  for (int d = 0; d < 3; ++d)
    for (int k = 0; k < 5; ++k) {
      double s = 0.0;
      for (int e = 0; e < 3; ++e) s = s + mat[d][e] * g[e][k];
      ng[5 * d + k] = vv.is_bound ? 0.0 : s;
    }
}

static double OI(double a, double b, double c) {
  const double x[3] = {a, b, c};
  return fnorm2(x, 3);
}

// :8-59 (methods 2-6, :166-320) with physical_slope_limiter (:129-164) and
// relaxed_maximum_principle (:61-127)
static void compute_cell_grads(const Mesh& m, const NsCfg& cfg, const double* sol, double* grad, double* ngrad) {
  for (int v = 1; v <= m.n_vert; ++v) compute_nodal_grad(m, v, sol, ngrad + 15 * (v - 1));
  if (cfg.method == 0 || cfg.method == 1) {
    for (int i = 0; i < 15 * m.n_elems; ++i) grad[i] = 0.0;
    return;
  }
  const double eps = 1e-3, tol = 1e-8;
  for (int c = 1; c <= m.n_elems; ++c) {
    const Elem& e = m.elem[c];
    double* g = grad + 15 * (c - 1);
    double ws[5] = {0, 0, 0, 0, 0};
    for (int i = 0; i < 15; ++i) g[i] = 0.0;
    if (cfg.method == 2) {  // :166-187 dual-volume average
      double dvs = 0.0;
      for (int j = 1; j <= e.n_vert; ++j) {
        int v = e.vert[j];
        const double* ng = ngrad + 15 * (v - 1);
        for (int i = 0; i < 15; ++i) g[i] = g[i] + m.vert[v].volume * ng[i];
        dvs = dvs + m.vert[v].volume;
      }
      for (int i = 0; i < 15; ++i) g[i] = g[i] / dvs;
    } else if (cfg.method == 3) {  // :189-209 the vertex gradient of smallest norm, per variable
      const double* ng1 = ngrad + 15 * (e.vert[1] - 1);
      for (int i = 0; i < 15; ++i) g[i] = ng1[i];
      for (int j = 2; j <= e.n_vert; ++j) {
        const double* ng = ngrad + 15 * (e.vert[j] - 1);
        for (int k = 0; k < 5; ++k)
          if (OI(ng[k], ng[5 + k], ng[10 + k]) < OI(g[k], g[5 + k], g[10 + k]))
            for (int d = 0; d < 3; ++d) g[5 * d + k] = ng[5 * d + k];
      }
    } else {  // 4 (:211-241): weights V/(eps+|g|); 5, 6 (:243-320): V/(eps+|g|)^2
      double cg[15] = {0}, cws = 0.0;
      for (int j = 1; j <= e.n_vert; ++j) {
        int v = e.vert[j];
        const double* ng = ngrad + 15 * (v - 1);
        for (int k = 0; k < 5; ++k) {
          const double q = eps + OI(ng[k], ng[5 + k], ng[10 + k]);
          double w = cfg.method == 4 ? m.vert[v].volume / q : m.vert[v].volume / (q * q);
          for (int d = 0; d < 3; ++d) g[5 * d + k] = g[5 * d + k] + w * ng[5 * d + k];
          ws[k] = ws[k] + w;
        }
        if (cfg.method == 6) {
          for (int i = 0; i < 15; ++i) cg[i] = cg[i] + m.vert[v].volume * ng[i];
          cws = cws + m.vert[v].volume;
        }
      }
      if (cfg.method == 6) {
        // the central gradient's weight: OI of the whole (3, 5) array is, by sequence
        // association with OI's dimension(3) argument, the norm of its first column
        for (int i = 0; i < 15; ++i) cg[i] = cg[i] / cws;
        const double q = eps + OI(cg[0], cg[5], cg[10]);
        const double wc = cws / (q * q);
        for (int i = 0; i < 15; ++i) g[i] = g[i] + wc * cg[i];
        for (int k = 0; k < 5; ++k) ws[k] = ws[k] + wc;
      }
      for (int k = 0; k < 5; ++k)
        for (int d = 0; d < 3; ++d) g[5 * d + k] = g[5 * d + k] / ws[k];
    }
    // physical_slope_limiter
    double w0[5];
    c2p(sol + 5 * (c - 1), w0);
    double omega = 1.0;
    for (int j = 1; j <= e.n_vert; ++j) {
      int v = e.vert[j];
      double dx[3], dw[5];
      for (int d = 0; d < 3; ++d) dx[d] = m.vert[v].coord[d + 1] - e.coord[d + 1];
      for (int k = 0; k < 5; ++k) {
        double s = 0.0;
        for (int d = 0; d < 3; ++d) s = s + g[5 * d + k] * dx[d];
        dw[k] = s;
      }
      if (dw[0] < 0.0) omega = fmin2(omega, fmax2(0.0, w0[0] / (tol - dw[0])));
      if (dw[4] < 0.0) omega = fmin2(omega, fmax2(0.0, w0[4] / (tol - dw[4])));
    }
    for (int i = 0; i < 15; ++i) g[i] = omega * g[i];
    // relaxed_maximum_principle
    double rmin = 1e100, rmax = 0.0, pmin = 1e100, pmax = 0.0;
    for (int j = 1; j <= e.n_vert; ++j) {
      const Vert& vv = m.vert[e.vert[j]];
      for (int k = 1; k <= vv.n_elems_neigh; ++k) {
        double w[5];
        c2p(sol + 5 * (vv.elem_neigh[k] - 1), w);
        pmin = fmin2(pmin, w[4]);
        pmax = fmax2(pmax, w[4]);
        rmin = fmin2(rmin, w[0]);
        rmax = fmax2(rmax, w[0]);
      }
    }
    pmin = (1.0 - 1e-2) * pmin;
    rmin = (1.0 - 1e-2) * rmin;
    pmax = (1.0 + 1e-2) * pmax;
    rmax = (1.0 + 1e-2) * rmax;
    omega = 1.0;
    for (int j = 1; j <= e.n_vert; ++j) {
      int v = e.vert[j];
      double dx[3], dw[5];
      for (int d = 0; d < 3; ++d) dx[d] = m.vert[v].coord[d + 1] - e.coord[d + 1];
      for (int k = 0; k < 5; ++k) {
        double s = 0.0;
        for (int d = 0; d < 3; ++d) s = s + g[5 * d + k] * dx[d];
        dw[k] = s;
      }
      if (dw[0] < 0.0)
        omega = fmin2(omega, fmax2(0.0, (w0[0] - rmin) / (tol - dw[0])));
      else
        omega = fmin2(omega, fmax2(0.0, -(w0[0] - rmax) / (tol + dw[0])));
      if (dw[4] < 0.0)
        omega = fmin2(omega, fmax2(0.0, (w0[4] - pmin) / (tol - dw[4])));
      else
        omega = fmin2(omega, fmax2(0.0, -(w0[4] - pmax) / (tol + dw[4])));
    }
    for (int i = 0; i < 15; ++i) g[i] = omega * g[i];
  }
}

// ns_euler_primitives_module.F90:162-190
static void wall_normal(const Mesh& m, const NsCfg& cfg, int v, double* B) {
  B[0] = B[1] = B[2] = 0.0;
  const Vert& vv = m.vert[v];
  for (int j = 1; j <= vv.n_sub_faces_neigh; ++j) {
    int sf = vv.sub_face_neigh[j];
    int re = m.face[m.sub_face[sf].mesh_face].right_neigh;
    if (re <= 0) {
      const double* n = &m.sub_face[sf].norm[1];
      if (!(cfg.b2d && std::fabs(n[2]) > 1e-12))
        if (re == 0 || cfg.bc_type[-re - 1] == 1)
          for (int d = 0; d < 3; ++d) B[d] = B[d] + m.sub_face[sf].area * n[d];
    }
  }
}

// ns_euler_rs_module.F90:288-422
static void nodal_velocity(const Mesh& m, const NsCfg& cfg, int v, const std::vector<double>& wlr,
                           std::vector<double>& lam, std::vector<double>& vbar, double* vnode) {
  const Vert& vv = m.vert[v];
  int nsfn = vv.n_sub_faces_neigh;
  double Bp[3];
  wall_normal(m, cfg, v, Bp);
  vnode[0] = vnode[1] = vnode[2] = 0.0;
  for (int iter = 1; iter <= 4; ++iter) {
    double mat[3][3] = {{0}}, Rp[3] = {0, 0, 0};
    for (int j = 0; j < nsfn; ++j) {
      int sf = vv.sub_face_neigh[j + 1];
      int re = m.face[m.sub_face[sf].mesh_face].right_neigh;
      const double* n = &m.sub_face[sf].norm[1];
      double area = m.sub_face[sf].area;
      const double* wl = &wlr[10 * j];
      const double* wr = &wlr[10 * j + 5];
      double rhol = wl[0], vnl = dot3(wl + 1, n), pl = wl[4], al = sound_speed_w(wl);
      double rhor = wr[0], vnr = dot3(wr + 1, n), pr = wr[4], ar = sound_speed_w(wr);
      double lam_l = lam[2 * j], lam_r = lam[2 * j + 1];
      if (iter == 1) {
        lam_l = fmax2(fmax2(fmax2(lam_l, al * rhol), std::sqrt(rhol * fmax2(0.0, pr - pl))), -rhol * (vnr - vnl));
        lam_r = fmax2(fmax2(fmax2(lam_r, ar * rhor), std::sqrt(rhor * fmax2(0.0, pl - pr))), -rhor * (vnr - vnl));
        vbar[j] = (lam_l * vnl + lam_r * vnr - (pr - pl)) / (lam_r + lam_l);
        lam_l = fmax2(lam_l, al * rhol * (1.0 + 1.5 * fmax2(0.0, -(vbar[j] - vnl) / al)));
        lam_r = fmax2(lam_r, ar * rhor * (1.0 + 1.5 * fmax2(0.0, (vbar[j] - vnr) / ar)));
      } else if (is_wall(cfg, re) && cfg.bc_style == 1) {
        lam_l = fmax2(lam_l, al * rhol * (1.0 + 1.5 * fmax2(0.0, -(vbar[j] - vnl) / al)));
        lam_r = fmax2(lam_r, ar * rhor * (1.0 + 1.5 * fmax2(0.0, (vbar[j] - vnr) / ar)));
      } else {
        double v_et = dot3(vnode, n);
        lam_l = fmax2(lam_l, al * rhol * (1.0 + 1.5 * fmax2(0.0, -(v_et - vnl) / al)));
        lam_r = fmax2(lam_r, ar * rhor * (1.0 + 1.5 * fmax2(0.0, (v_et - vnr) / ar)));
      }
      lam[2 * j] = lam_l;
      lam[2 * j + 1] = lam_r;
      vbar[j] = (lam_l * vnl + lam_r * vnr - (pr - pl)) / (lam_r + lam_l);
      bool wall = is_wall(cfg, re);
      // multi_point_iso (compute_lambdas_and_solve_nodal_velocity_iso, :424-553) drops
      // the subface area from M and R
      const bool iso = cfg.scheme == 2;
      if (!wall || cfg.bc_style == 0 || cfg.bc_style == 2) {
        double w = iso ? (lam_r + lam_l) : (lam_r + lam_l) * area;
        for (int d = 0; d < 3; ++d)
          for (int e = 0; e < 3; ++e) mat[d][e] = mat[d][e] + w * (n[d] * n[e]);
      }
      if (!wall || cfg.bc_style == 0) {
        double q = iso ? (lam_r + lam_l) * vbar[j] : area * (lam_r + lam_l) * vbar[j];
        for (int d = 0; d < 3; ++d) Rp[d] = Rp[d] + q * n[d];
      } else if (cfg.bc_style == 2) {
        if (!cfg.b2d || std::fabs(n[2]) < 1e-8) {
          double q = iso ? pl : area * pl;
          for (int d = 0; d < 3; ++d) Rp[d] = Rp[d] + q * n[d];
        }
      }
    }
    auto mv = [&](const double* x, double* y) {
      for (int d = 0; d < 3; ++d) {
        double s = 0.0;
        for (int e = 0; e < 3; ++e) s = s + mat[d][e] * x[e];
        y[d] = s;
      }
    };
    if (cfg.bc_style == 2) {
      double bmax = fmax2(fmax2(std::fabs(Bp[0]), std::fabs(Bp[1])), std::fabs(Bp[2]));
      if (bmax > 1e-8) {
        pinv3(mat);
        double mr[3], mb[3], r2[3];
        mv(Rp, mr);
        mv(Bp, mb);
        double p_bound = dot3(mr, Bp) / dot3(mb, Bp);
        for (int d = 0; d < 3; ++d) r2[d] = Rp[d] - p_bound * Bp[d];
        mv(r2, vnode);
        double f = dot3(vnode, Bp) / dot3(Bp, Bp);
        for (int d = 0; d < 3; ++d) vnode[d] = vnode[d] - f * Bp[d];
      } else {
        lu_solve3(mat, vnode, Rp);
      }
    } else {
      pinv3(mat);
      double r[3] = {Rp[0], Rp[1], Rp[2]};
      mv(r, vnode);
    }
  }
}

// compute_lambdas_and_solve_nodal_pressure (ns_euler_rs_module.F90:681-758): ten
// fixed-point iterations of p_node = s1 / s2 over the vertex's subfaces
static double nodal_pressure(const Mesh& m, const NsCfg& cfg, int v, const std::vector<double>& wlr,
                             std::vector<double>& lam) {
  const Vert& vv = m.vert[v];
  int nsfn = vv.n_sub_faces_neigh;
  std::vector<double> pbar(nsfn, 0.0);
  double p_node = 0.0;
  for (int iter = 1; iter <= 10; ++iter) {
    double s1 = 0.0, s2 = 0.0;
    for (int j = 0; j < nsfn; ++j) {
      int sf = vv.sub_face_neigh[j + 1];
      int re = m.face[m.sub_face[sf].mesh_face].right_neigh;
      const double* n = &m.sub_face[sf].norm[1];
      double area = m.sub_face[sf].area;
      const double* wl = &wlr[10 * j];
      const double* wr = &wlr[10 * j + 5];
      double rhol = wl[0], vnl = dot3(wl + 1, n), pl = wl[4], al = sound_speed_w(wl);
      double rhor = wr[0], vnr = dot3(wr + 1, n), pr = wr[4], ar = sound_speed_w(wr);
      double lam_l = lam[2 * j], lam_r = lam[2 * j + 1];
      const bool wall1 = cfg.bc_style == 1 && is_wall(cfg, re);
      if (iter == 1) {
        lam_l = fmax2(fmax2(fmax2(lam_l, al * rhol), std::sqrt(rhol * fmax2(0.0, pr - pl))), -rhol * (vnr - vnl));
        lam_r = fmax2(fmax2(fmax2(lam_r, ar * rhor), std::sqrt(rhor * fmax2(0.0, pl - pr))), -rhor * (vnr - vnl));
        pbar[j] = (lam_r * pl + lam_l * pr - lam_r * lam_l * (vnr - vnl)) / (lam_r + lam_l);
        lam_l = fmax2(lam_l, al * rhol + 1.5 * std::sqrt(fmax2(0.0, (pbar[j] - pl) * rhol)));
        lam_r = fmax2(lam_r, ar * rhor + 1.5 * std::sqrt(fmax2(0.0, (pbar[j] - pr) * rhor)));
      } else {
        const double pq = wall1 ? pbar[j] : p_node;
        lam_l = fmax2(lam_l, al * rhol + 1.5 * std::sqrt(fmax2(0.0, (pq - pl) * rhol)));
        lam_r = fmax2(lam_r, ar * rhor + 1.5 * std::sqrt(fmax2(0.0, (pq - pr) * rhor)));
      }
      pbar[j] = (lam_r * pl + lam_l * pr - lam_r * lam_l * (vnr - vnl)) / (lam_r + lam_l);
      if (wall1) {
        s1 = s1 + (1.0 / lam_r + 1.0 / lam_l) * area * (lam_r * pl + lam_r * lam_l * vnl) / (lam_r + lam_l);
        s2 = s2 + (1.0 / lam_l) * area;
      } else {
        s1 = s1 + (1.0 / lam_r + 1.0 / lam_l) * area * pbar[j];
        s2 = s2 + (1.0 / lam_r + 1.0 / lam_l) * area;
      }
      lam[2 * j] = lam_l;
      lam[2 * j + 1] = lam_r;
    }
    p_node = s1 / s2;
  }
  return p_node;
}

// ns_euler_module.F90:151-339 (scheme_id multi_point, multi_point_iso, three_wave,
// two_wave, modified_three_wave, multi_point_pressure(_ph)) + :341-519
static int compute_euler_flux(const Mesh& m, const NsCfg& cfg, const double* sol, double* rhs, const double* grad,
                              double* sum_lambda, bool so, double* vp) {
  for (int i = 0; i < 5 * m.n_elems; ++i) rhs[i] = 0.0;
  for (int i = 0; i < m.n_elems; ++i) sum_lambda[i] = 1e-12;
  int status = 0;
  std::vector<double> wlr, lam, vbar, fsv, slv;
  for (int v = 1; v <= m.n_vert; ++v) {
    const Vert& vv = m.vert[v];
    int nsfn = vv.n_sub_faces_neigh, nsen = vv.n_sub_elems_neigh;
    wlr.assign(10 * nsfn, 0.0);
    lam.assign(2 * nsfn, 0.0);
    vbar.assign(nsfn, 0.0);
    fsv.assign(5 * nsen, 0.0);
    slv.assign(nsen, 0.0);
    double amin = 0.0;  // minval of the subface areas (warea, ns_euler_module.F90:386-397)
    for (int j = 0; j < nsfn; ++j) {
      int sf = vv.sub_face_neigh[j + 1];
      const Face& f = m.face[m.sub_face[sf].mesh_face];
      reconstruct_lr_w(m, cfg, sol, grad, v, sf, f.left_neigh, f.right_neigh, so, &wlr[10 * j], &wlr[10 * j + 5]);
      amin = j == 0 ? m.sub_face[sf].area : fmin2(amin, m.sub_face[sf].area);
    }
    double vv3[3] = {0, 0, 0};
    bool excl = vv.is_bound && cfg.exclude_bound_vert;
    double p_nodal = 0.0;
    const bool pres = cfg.scheme == 6 || cfg.scheme == 8;
    if (pres) p_nodal = nodal_pressure(m, cfg, v, wlr, lam);
    if (cfg.scheme == 1 || cfg.scheme == 2) {
      if (!excl) nodal_velocity(m, cfg, v, wlr, lam, vbar, vv3);
      for (int d = 0; d < 3; ++d) vp[3 * (v - 1) + d] = vv3[d];
    }
    int rse_loc = 0;
    for (int j = 0; j < nsfn; ++j) {
      int sf = vv.sub_face_neigh[j + 1];
      const SubFace& s = m.sub_face[sf];
      int re = m.face[s.mesh_face].right_neigh;
      int lse = s.left_sub_elem_neigh, rse = s.right_sub_elem_neigh;
      int lse_loc = m.sub_elem[lse].id_loc_around_node;
      if (rse > 0) rse_loc = m.sub_elem[rse].id_loc_around_node;
      double lr[2][5], sl, sr;
      const double* n = &s.norm[1];
      if ((cfg.scheme == 1 || cfg.scheme == 2) && !excl) {
        double vn = is_wall(cfg, re) ? 0.0 : dot3(vv3, n);
        if (!multi_point(&wlr[10 * j], &wlr[10 * j + 5], n, lr, vn, lam[2 * j], lam[2 * j + 1], &sl, &sr))
          status |= 4;
      } else if (cfg.scheme == 3 || cfg.scheme == 5) {
        three_wave(&wlr[10 * j], &wlr[10 * j + 5], n, lr, &sl, &sr, cfg.scheme == 5);
      } else if (pres) {
        multi_point_pressure(&wlr[10 * j], &wlr[10 * j + 5], n, lr, p_nodal, lam[2 * j], lam[2 * j + 1], &sl, &sr,
                             cfg.scheme == 8);
      } else {
        two_wave(&wlr[10 * j], &wlr[10 * j + 5], n, lr, &sl, &sr);
      }
      if (cfg.scheme == 2) {  // blend with three_wave by warea = min area / area; sl, sr from three_wave
        double lr3[2][5];
        three_wave(&wlr[10 * j], &wlr[10 * j + 5], n, lr3, &sl, &sr, false);
        const double wa = amin / s.area;
        for (int q = 0; q < 2; ++q)
          for (int k = 0; k < 5; ++k) lr[q][k] = wa * lr[q][k] + (1.0 - wa) * lr3[q][k];
      }
      if (m.sub_elem[lse].mesh_vert == v) {
        slv[lse_loc - 1] = slv[lse_loc - 1] + s.area * fmax2(0.0, -sl);
        for (int k = 0; k < 5; ++k) fsv[5 * (lse_loc - 1) + k] = fsv[5 * (lse_loc - 1) + k] + s.area * lr[0][k];
        if (rse > 0 && m.sub_elem[rse].mesh_vert == v) {
          slv[rse_loc - 1] = slv[rse_loc - 1] + s.area * fmax2(0.0, sr);
          for (int k = 0; k < 5; ++k) fsv[5 * (rse_loc - 1) + k] = fsv[5 * (rse_loc - 1) + k] + s.area * lr[1][k];
        }
      }
    }
    for (int j = 0; j < nsen; ++j) {
      int ide = m.sub_elem[vv.sub_elem_neigh[j + 1]].mesh_elem;
      for (int k = 0; k < 5; ++k) rhs[5 * (ide - 1) + k] = rhs[5 * (ide - 1) + k] - fsv[5 * j + k];
      sum_lambda[ide - 1] = sum_lambda[ide - 1] + slv[j];
    }
  }
  return status;
}

// ns_euler_recon_module.F90:560-601
static void flux_limiting(const Mesh& m, const double* sol, double* rhs, const double* rhs_o2,
                          const double* sum_lambda, double cfl) {
  double dt = 1e10;
  for (int i = 1; i <= m.n_elems; ++i) dt = fmin2(dt, m.elem[i].volume / sum_lambda[i - 1]);
  dt = cfl * dt;
  for (int i = 1; i <= m.n_elems; ++i) {
    double den = m.elem[i].volume / dt + sum_lambda[i - 1];
    double U[5], dU[5];
    for (int k = 0; k < 5; ++k) {
      U[k] = sol[5 * (i - 1) + k] + rhs[5 * (i - 1) + k] / den;
      dU[k] = (rhs_o2[5 * (i - 1) + k] - rhs[5 * (i - 1) + k]) / den;
    }
    double omega = max_omega_for_positivity(U, dU);
    double w = fmin2(1.0, omega);
    for (int k = 0; k < 5; ++k)
      rhs[5 * (i - 1) + k] = rhs[5 * (i - 1) + k] + w * (rhs_o2[5 * (i - 1) + k] - rhs[5 * (i - 1) + k]);
  }
}

struct NsWork {
  std::vector<double> rhs, rhs_o2, sl, sl_o2, grad, ngrad, vp, delta, diag;
};

// ------------------------------------------------------------------------------------
// Diffusion (activate_diffusion): ns_vectorial_diffusion_module.F90 (momentum) and
// ns_diffusion_module.F90 (heat), point-implicit blocks in mat_diag and terms in rhs.
// The LAPACK / BLAS calls are restated in the reference (netlib) implementations'
// operation order: dgetrf for n < 64 is dgetrf2, which for these sizes performs the
// right-looking elimination with partial pivoting (first largest |pivot|, the column
// scaled by the pivot's reciprocal); dgetri (the workspace of n the reference passes
// selects the unblocked code) is dtrti2 then the column sweep with dgemv; dgemm / dgemv
// accumulate each output from zero over the inner index in ascending order.

struct DiffCfg {
  int active = 0, use_sutherland = 0;
  double mu_p = 1.329e-5, mu0 = 1.716e-5, T0 = 273.15, Cv_p = 720.19471;
  double prandtl = 0.71;             // ns_global_data_module.F90:10 (a parameter there)
  int bcV[16] = {0}, bcT[16] = {0};  // 0 or 1 neumann, 2 dirichlet
  double valV[16][3] = {{0}}, valT[16] = {0};
};
static DiffCfg g_diff;
static const double kC0 = 110.4;  // ns_global_data_module.F90:20

// column-major n x n, A(i,j) = a[i + n*j]
static void lapack_getrf(int n, double* a, int* ipiv) {
  const double sfmin = 2.2250738585072014e-308;  // dlamch('S')
  for (int j = 0; j < n; ++j) {
    int p = j;
    double big = std::fabs(a[j + n * j]);
    for (int i = j + 1; i < n; ++i)
      if (std::fabs(a[i + n * j]) > big) {
        big = std::fabs(a[i + n * j]);
        p = i;
      }
    ipiv[j] = p;
    if (a[p + n * j] != 0.0) {
      if (p != j)
        for (int k = 0; k < n; ++k) std::swap(a[j + n * k], a[p + n * k]);
      if (std::fabs(a[j + n * j]) >= sfmin) {
        const double r = 1.0 / a[j + n * j];
        for (int i = j + 1; i < n; ++i) a[i + n * j] = r * a[i + n * j];
      } else {
        for (int i = j + 1; i < n; ++i) a[i + n * j] = a[i + n * j] / a[j + n * j];
      }
    }
    for (int k = j + 1; k < n; ++k)
      for (int i = j + 1; i < n; ++i) a[i + n * k] = a[i + n * k] - a[i + n * j] * a[j + n * k];
  }
}
// dgetrs('N') for one right-hand side
static void lapack_getrs(int n, const double* a, const int* ipiv, double* b) {
  for (int j = 0; j < n; ++j)
    if (ipiv[j] != j) std::swap(b[j], b[ipiv[j]]);
  for (int k = 0; k < n; ++k)
    if (b[k] != 0.0)
      for (int i = k + 1; i < n; ++i) b[i] = b[i] - b[k] * a[i + n * k];
  for (int k = n - 1; k >= 0; --k)
    if (b[k] != 0.0) {
      b[k] = b[k] / a[k + n * k];
      for (int i = 0; i < k; ++i) b[i] = b[i] - b[k] * a[i + n * k];
    }
}
// inv_lapack (linear_solver_module.F90:629-641): dgetrf + dgetri
static void lapack_inverse(int n, double* a) {
  std::vector<int> ipiv(n);
  std::vector<double> work(n);
  lapack_getrf(n, a, ipiv.data());
  for (int j = 0; j < n; ++j) {  // dtrti2 ('Upper', 'Non-unit')
    a[j + n * j] = 1.0 / a[j + n * j];
    const double ajj = -a[j + n * j];
    double* x = a + n * j;  // dtrmv on x(0:j-1) with the inverted leading block
    for (int jj = 0; jj < j; ++jj)
      if (x[jj] != 0.0) {
        const double temp = x[jj];
        for (int i = 0; i < jj; ++i) x[i] = x[i] + temp * a[i + n * jj];
        x[jj] = x[jj] * a[jj + n * jj];
      }
    for (int i = 0; i < j; ++i) x[i] = ajj * x[i];
  }
  for (int j = n - 1; j >= 0; --j) {
    for (int i = j + 1; i < n; ++i) {
      work[i] = a[i + n * j];
      a[i + n * j] = 0.0;
    }
    for (int jj = j + 1; jj < n; ++jj) {  // dgemv: A(:,j) += -work(jj) * A(:,jj)
      const double temp = -work[jj];
      for (int i = 0; i < n; ++i) a[i + n * j] = a[i + n * j] + temp * a[i + n * jj];
    }
  }
  for (int j = n - 2; j >= 0; --j)
    if (ipiv[j] != j)
      for (int i = 0; i < n; ++i) std::swap(a[i + n * j], a[i + n * ipiv[j]]);
}
// C(m x p) = A(m x k) * B(k x p), netlib dgemm order
static void blas_gemm(int m, int p, int k, const double* A, const double* B, double* C) {
  for (int j = 0; j < p; ++j)
    for (int i = 0; i < m; ++i) {
      double s = 0.0;
      for (int l = 0; l < k; ++l) s = s + B[l + k * j] * A[i + m * l];
      C[i + m * j] = s;
    }
}
// y(m) = A(m x n) x, netlib dgemv order
static void blas_gemv(int m, int n, const double* A, const double* x, double* y) {
  for (int i = 0; i < m; ++i) {
    double s = 0.0;
    for (int j = 0; j < n; ++j) s = s + x[j] * A[i + m * j];
    y[i] = s;
  }
}

// temp_u (ns_euler_primitives_module.F90:52-63)
static double temp_u(const double* u) {
  const double tau = 1.0 / u[0];
  const double uu = u[1] * u[1] + u[2] * u[2] + u[3] * u[3];
  return (u[4] * tau - 0.5 * uu * (tau * tau)) / g_diff.Cv_p;
}
// mu_sutherland / compute_mu (ns_vectorial_diffusion_module.F90:320-357)
static double mu_of(const double* u) {
  if (!g_diff.use_sutherland) return g_diff.mu_p;
  const double T = temp_u(u);
  return g_diff.mu0 * std::pow(T / g_diff.T0, 1.5) * (g_diff.T0 + kC0) / (T + kC0);
}

// the sub_elem / sub_face relations of one vertex in the reference's local numbering
static double se_sign_norm(const Mesh& m, int isfp, int se, double* np) {
  const SubFace& s = m.sub_face[isfp];
  for (int d = 0; d < 3; ++d) np[d] = s.left_sub_elem_neigh == se ? s.norm[1 + d] : -s.norm[1 + d];
  return s.area;
}

// the momentum blc_3 (:85-91): s * (mu (nl.np) I + (mu - mu0corr) np (x) nl + (mu0corr - 2/3 mu) nl (x) np)
static void mom_block(double al, double ap, double vol, double mu, double mu0c, const double* nl, const double* np,
                      double blc[3][3]) {
  const double s = al * ap * (1.0 / vol);
  const double d = nl[0] * np[0] + nl[1] * np[1] + nl[2] * np[2];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      const double e = i == j ? 1.0 : 0.0;
      const double tp = np[i] * nl[j], tpt = np[j] * nl[i];
      blc[i][j] = s * ((mu * d * e + (mu - mu0c) * tp) + (mu0c - (2.0 / 3.0) * mu) * tpt);
    }
}
// the Neumann face's N and S block (:149-152): s * ((nl.np) I + (np (x) nl)^T / 3)
static void neumann_block(double al, double ap, double vol, const double* nl, const double* np, double blc[3][3]) {
  const double s = al * ap * (1.0 / vol);
  const double d = nl[0] * np[0] + nl[1] * np[1] + nl[2] * np[2];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      const double e = i == j ? 1.0 : 0.0;
      blc[i][j] = s * (d * e + (np[j] * nl[i]) / 3.0);
    }
}

// The stencil of a vertex's diffusion systems. Not the reference's: at a periodic node
// its extended lists (build_periodic_stencil, mesh_connectivity_module.F90:1075-1328)
// index the images' subfaces and subcells by their own id_loc_around_node, which
// collide, and at periodic edges and corners they name subcells the list does not hold.
// Here every image of a periodic node (vertices joined through the subface lists) gets
// the union over the images, in ascending vertex order: each image's subfaces in list
// order, the second copy of a periodic face dropped (key: its two cells, unordered; a
// boundary face: its cell, boundary and face), then each image's own subcells (mesh_vert
// the image) in list order. Rows and columns are positions in these lists, and an image
// applies the terms of its own subcells only. Without periodic faces the stencil is the
// vertex's own lists, and the positions are its id_loc_around_node.
struct DiffStencil {
  std::vector<int> sf, se;              // 1-based ids
  std::vector<int> lse, rse, lpos, rpos;  // per stencil subface: its cells' subcells (0 none), positions (-1)
  std::vector<std::array<int, 4>> fpos;  // per stencil subcell: its subfaces' positions (-1 pad)
};

static std::vector<DiffStencil> diffusion_stencils(const Mesh& m) {
  const int nv = m.n_vert;
  std::vector<int> up(nv + 1);
  for (int v = 1; v <= nv; ++v) up[v] = v;
  auto root = [&](int x) {
    while (up[x] != x) x = up[x];
    return x;
  };
  for (int v = 1; v <= nv; ++v)
    for (int k = 1; k <= m.vert[v].n_sub_faces_neigh; ++k) {
      const int a = root(v), b = root(m.sub_face[m.vert[v].sub_face_neigh[k]].mesh_vert);
      if (a < b) up[b] = a;
      else if (b < a) up[a] = b;
    }
  std::map<int, std::vector<int>> images;
  for (int v = 1; v <= nv; ++v) images[root(v)].push_back(v);
  auto fkey = [&](int s) {
    const int f = m.sub_face[s].mesh_face, l = m.face[f].left_neigh, r = m.face[f].right_neigh;
    if (r > 0) return std::array<int, 3>{std::min(l, r), std::max(l, r), 0};
    return std::array<int, 3>{l, r, f};
  };
  std::vector<DiffStencil> out(nv + 1);
  for (auto& kv : images) {
    DiffStencil st;
    std::map<std::array<int, 3>, int> where;
    std::map<int, int> cellpos;
    for (int v : kv.second)
      for (int k = 1; k <= m.vert[v].n_sub_faces_neigh; ++k) {
        const int s = m.vert[v].sub_face_neigh[k];
        if (where.find(fkey(s)) == where.end()) {
          where[fkey(s)] = (int)st.sf.size();
          st.sf.push_back(s);
        }
      }
    for (int v : kv.second)
      for (int k = 1; k <= m.vert[v].n_sub_elems_neigh; ++k) {
        const int e = m.vert[v].sub_elem_neigh[k];
        if (m.sub_elem[e].mesh_vert != v) continue;
        cellpos[m.sub_elem[e].mesh_elem] = (int)st.se.size();
        st.se.push_back(e);
      }
    for (int s : st.sf) {
      const Face& f = m.face[m.sub_face[s].mesh_face];
      int lp = -1, rp = -1;
      if (cellpos.count(f.left_neigh)) lp = cellpos[f.left_neigh];
      if (f.right_neigh > 0 && cellpos.count(f.right_neigh)) rp = cellpos[f.right_neigh];
      st.lpos.push_back(lp);
      st.rpos.push_back(rp);
      st.lse.push_back(lp >= 0 ? st.se[lp] : 0);
      st.rse.push_back(rp >= 0 ? st.se[rp] : 0);
    }
    for (int e : st.se) {
      std::array<int, 4> q = {-1, -1, -1, -1};
      for (int p = 1; p <= m.sub_elem[e].n_sub_faces && p <= 4; ++p) {
        auto it = where.find(fkey(m.sub_elem[e].sub_face[p]));
        q[p - 1] = it == where.end() ? -1 : it->second;
      }
      st.fpos.push_back(q);
    }
    for (int v : kv.second) out[v] = st;
  }
  return out;
}

// build_momentum_diff_mat_into_global_mat_diag (:195-318), all vertices
static void momentum_diffusion(const Mesh& m, const double* sol, const double* mu, double mu0c, double* diag,
                               double* rhs) {
  const std::vector<DiffStencil> stencils = diffusion_stencils(m);
  for (int v = 1; v <= m.n_vert; ++v) {
    const DiffStencil& Z = stencils[v];
    const int nf = (int)Z.sf.size(), ne = (int)Z.se.size(), F = 3 * nf, E = 3 * ne;
    std::vector<double> N(F * F, 0.0), S(F * E, 0.0), St(E * F, 0.0), B(F, 0.0);
    // build_momentum_diff_nodal_system (:7-193)
    for (int l = 0; l < nf; ++l) {
      const int isfl = Z.sf[l];
      const SubFace& sl = m.sub_face[isfl];
      const int ifl0 = 3 * l;
      const int re = sl.right_elem_neigh;
      bool neu = false, dir = false;
      if (re < 0) {  // bc_V_id: "" and "neumann" are Neumann (ns_global_data_module.F90:229-236)
        dir = g_diff.bcV[-re - 1] == 2;
        neu = !dir;
      } else if (re == 0) {
        neu = true;
      }
      auto side = [&](int se, int elem, const double* nl, int mode, int sp) {
        // mode 0: N, S, St with the full block; 1: Neumann (N, S the plain block, St the
        // full one); 2: Dirichlet (St only)
        const SubElem& E0 = m.sub_elem[se];
        const int ise0 = 3 * sp;
        const double mue = mu[elem - 1];
        for (int p = 0; p < E0.n_sub_faces; ++p) {
          const int isfp = E0.sub_face[p + 1];
          const int ifp0 = 3 * Z.fpos[sp][p];
          double np[3];
          const double ap = se_sign_norm(m, isfp, se, np);
          double blc[3][3], bn[3][3];
          mom_block(sl.area, ap, E0.volume, mue, mu0c, nl, np, blc);
          if (mode == 1) neumann_block(sl.area, ap, E0.volume, nl, np, bn);
          const double (*bNS)[3] = mode == 1 ? bn : blc;
          for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
              St[(ise0 + i) + E * (ifl0 + j)] += blc[j][i];
              if (mode != 2) {
                N[(ifl0 + i) + F * (ifp0 + j)] += bNS[i][j];
                S[(ifl0 + i) + F * (ise0 + j)] += bNS[i][j];
              }
            }
        }
      };
      const double nl[3] = {sl.norm[1], sl.norm[2], sl.norm[3]};
      const double nr[3] = {-sl.norm[1], -sl.norm[2], -sl.norm[3]};
      const Face& fl = m.face[sl.mesh_face];
      if (!neu && !dir) {
        side(Z.lse[l], fl.left_neigh, nl, 0, Z.lpos[l]);
        side(Z.rse[l], fl.right_neigh, nr, 0, Z.rpos[l]);
      } else if (neu) {
        side(Z.lse[l], fl.left_neigh, nl, 1, Z.lpos[l]);
      } else {
        side(Z.lse[l], fl.left_neigh, nl, 2, Z.lpos[l]);
        for (int k = 0; k < 3; ++k) B[ifl0 + k] = sl.area * g_diff.valV[-re - 1][k];
        for (int i = 0; i < 3; ++i) {
          for (int c = 0; c < E; ++c) S[(ifl0 + i) + F * c] = 0.0;
          for (int c = 0; c < F; ++c) N[(ifl0 + i) + F * c] = 0.0;
          for (int j = 0; j < 3; ++j) N[(ifl0 + i) + F * (ifl0 + j)] = sl.area * (i == j ? 1.0 : 0.0);
        }
      }
    }
    std::vector<double> Ve(E), Vf(F), SB(E), SNS(E * E), T1(E * F), tmp(F), SNSVe(E), blc3(9 * ne);
    for (int l = 0; l < ne; ++l) {
      const double* u = sol + 5 * (m.sub_elem[Z.se[l]].mesh_elem - 1);
      for (int k = 0; k < 3; ++k) Ve[3 * l + k] = u[1 + k] / u[0];
    }
    for (int p = 0; p < ne; ++p) {
      const double* u = sol + 5 * (m.sub_elem[Z.se[p]].mesh_elem - 1);
      double Spc[3][3] = {{0}};
      for (int l = 0; l < nf; ++l)
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j) Spc[i][j] = Spc[i][j] + St[(3 * p + i) + E * (3 * l + j)];
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) blc3[9 * p + i + 3 * j] = Spc[j][i] / u[0];
    }
    blas_gemv(F, E, S.data(), Ve.data(), Vf.data());
    for (int i = 0; i < F; ++i) Vf[i] = Vf[i] + B[i];
    lapack_inverse(F, N.data());
    blas_gemm(E, F, F, St.data(), N.data(), T1.data());
    blas_gemm(E, E, F, T1.data(), S.data(), SNS.data());
    blas_gemv(F, F, N.data(), B.data(), tmp.data());
    blas_gemv(E, F, St.data(), tmp.data(), SB.data());
    blas_gemv(F, F, N.data(), Vf.data(), B.data());
    Vf = B;
    blas_gemv(E, E, SNS.data(), Ve.data(), SNSVe.data());
    for (int l = 0; l < ne; ++l) {
      if (m.sub_elem[Z.se[l]].mesh_vert != v) continue;  // a periodic image's subcell
      const int iel = m.sub_elem[Z.se[l]].mesh_elem;
      const double* u = sol + 5 * (iel - 1);
      double* D = diag + 25 * (iel - 1);
      double* r = rhs + 5 * (iel - 1);
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
          D[(1 + i) + 5 * (1 + j)] =
              (D[(1 + i) + 5 * (1 + j)] - SNS[(3 * l + i) + E * (3 * l + j)] / u[0]) + blc3[9 * l + i + 3 * j];
      for (int i = 0; i < 3; ++i) {
        double mv = 0.0;
        for (int k = 0; k < 3; ++k) mv = mv + SNS[(3 * l + i) + E * (3 * l + k)] * Ve[3 * l + k];
        r[1 + i] = ((r[1 + i] + SNSVe[3 * l + i]) - mv) + SB[3 * l + i];
      }
    }
    for (int p = 0; p < ne; ++p) {  // viscous work
      const int isep = Z.se[p];
      if (m.sub_elem[isep].mesh_vert != v) continue;
      const SubElem& Ep = m.sub_elem[isep];
      const int iep = Ep.mesh_elem;
      double Spc[3][3] = {{0}};
      for (int l = 0; l < Ep.n_sub_faces; ++l) {
        const int isfl = Ep.sub_face[l + 1];
        double nl[3];
        const double a = se_sign_norm(m, isfl, isep, nl);
        const int q = 3 * Z.fpos[p][l];
        double vm[3];
        for (int k = 0; k < 3; ++k) vm[k] = Vf[q + k] - Ve[3 * p + k];
        const double dd = vm[0] * nl[0] + vm[1] * nl[1] + vm[2] * nl[2];
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j) {
            const double e = i == j ? 1.0 : 0.0;
            Spc[i][j] = Spc[i][j] + a * ((vm[i] * nl[j] + vm[j] * nl[i]) - (2.0 / 3.0) * dd * e);
          }
      }
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) Spc[i][j] = Spc[i][j] * mu[iep - 1] / Ep.volume;
      for (int l = 0; l < Ep.n_sub_faces; ++l) {
        const int isfl = Ep.sub_face[l + 1];
        double nl[3];
        const double a = se_sign_norm(m, isfl, isep, nl);
        const int q = 3 * Z.fpos[p][l];
        double sv[3];
        for (int i = 0; i < 3; ++i) {
          double s = 0.0;
          for (int k = 0; k < 3; ++k) s = s + Spc[i][k] * Vf[q + k];
          sv[i] = s;
        }
        rhs[5 * (iep - 1) + 4] = rhs[5 * (iep - 1) + 4] + a * (sv[0] * nl[0] + sv[1] * nl[1] + sv[2] * nl[2]);
      }
    }
  }
}

// build_diff_mat_into_global_mat_diag (ns_diffusion_module.F90:112-184), all vertices
static void heat_diffusion(const Mesh& m, const double* sol, const double* mu, double* diag, double* rhs) {
  const std::vector<DiffStencil> stencils = diffusion_stencils(m);
  for (int v = 1; v <= m.n_vert; ++v) {
    const DiffStencil& Z = stencils[v];
    const int nf = (int)Z.sf.size(), ne = (int)Z.se.size();
    std::vector<double> N(nf * nf, 0.0), S(nf * ne, 0.0), St(ne * nf, 0.0), B(nf, 0.0);
    for (int l = 0; l < nf; ++l) {  // build_diff_nodal_system (:7-110)
      const int isfl = Z.sf[l];
      const SubFace& sl = m.sub_face[isfl];
      const int il = l;
      const Face& fl = m.face[sl.mesh_face];
      auto side = [&](int se, int elem, const double* nl, int sp) {
        const SubElem& E0 = m.sub_elem[se];
        const int ie = sp;
        const double kap = mu[elem - 1] * g_diff.Cv_p * G / g_diff.prandtl;
        for (int p = 0; p < E0.n_sub_faces; ++p) {
          const int isfp = E0.sub_face[p + 1];
          const int ip = Z.fpos[sp][p];
          double np[3];
          const double ap = se_sign_norm(m, isfp, se, np);
          const double b = kap * sl.area * ap * (1.0 / E0.volume) * (np[0] * nl[0] + np[1] * nl[1] + np[2] * nl[2]);
          N[il + nf * ip] += b;
          S[il + nf * ie] += b;
          St[ie + ne * il] += b;
        }
      };
      const double nl[3] = {sl.norm[1], sl.norm[2], sl.norm[3]};
      const double nr[3] = {-sl.norm[1], -sl.norm[2], -sl.norm[3]};
      side(Z.lse[l], fl.left_neigh, nl, Z.lpos[l]);
      if (Z.rse[l] > 0) {
        side(Z.rse[l], fl.right_neigh, nr, Z.rpos[l]);
      } else if (fl.right_neigh < 0 && g_diff.bcT[-fl.right_neigh - 1] == 2) {
        B[il] = sl.area * g_diff.valT[-fl.right_neigh - 1];
        for (int c = 0; c < ne; ++c) S[il + nf * c] = 0.0;
        for (int c = 0; c < nf; ++c) N[il + nf * c] = 0.0;
        N[il + nf * il] = sl.area;
      }
    }
    std::vector<double> SNS(ne * ne), T1(ne * nf), tmp(nf), SB(ne), theta(ne), P(5 * ne), b1(ne);
    lapack_inverse(nf, N.data());
    blas_gemm(ne, nf, nf, St.data(), N.data(), T1.data());
    blas_gemm(ne, ne, nf, T1.data(), S.data(), SNS.data());
    blas_gemv(nf, nf, N.data(), B.data(), tmp.data());
    blas_gemv(ne, nf, St.data(), tmp.data(), SB.data());
    for (int l = 0; l < ne; ++l) {
      const double* u = sol + 5 * (m.sub_elem[Z.se[l]].mesh_elem - 1);
      theta[l] = temp_u(u);
      const double uv[3] = {u[1] / u[0], u[2] / u[0], u[3] / u[0]};
      const double nn = fnorm2(uv, 3);
      P[5 * l] = (nn * nn - u[4] / u[0]) / (u[0] * g_diff.Cv_p);
      for (int k = 1; k < 4; ++k) P[5 * l + k] = -u[k] / ((u[0] * u[0]) * g_diff.Cv_p);
      P[5 * l + 4] = 1.0 / (u[0] * g_diff.Cv_p);
      double s = 0.0;
      for (int c = 0; c < nf; ++c) s = s + St[l + ne * c];
      b1[l] = s;
    }
    for (int l = 0; l < ne; ++l) {
      if (m.sub_elem[Z.se[l]].mesh_vert != v) continue;
      const int iel = m.sub_elem[Z.se[l]].mesh_elem;
      const double* u = sol + 5 * (iel - 1);
      double* D = diag + 25 * (iel - 1);
      double& r5 = rhs[5 * (iel - 1) + 4];
      for (int p = 0; p < ne; ++p) r5 = r5 + SNS[l + ne * p] * theta[p];
      const double snl = SNS[l + ne * l], cc = b1[l] - snl;
      for (int k = 0; k < 5; ++k) D[4 + 5 * k] = D[4 + 5 * k] + cc * P[5 * l + k];
      double pu = 0.0;
      for (int k = 0; k < 5; ++k) pu = pu + P[5 * l + k] * u[k];
      r5 = (((r5 - snl * pu) + cc * pu) - b1[l] * theta[l]) + SB[l];
    }
  }
}

// ns_main.F90:130-179
static int compute_rhs_ns(const Mesh& m, const NsCfg& cfg, const double* sol, NsWork& w) {
  w.grad.assign(15 * m.n_elems, 0.0);
  w.ngrad.assign(15 * m.n_vert, 0.0);
  w.diag.assign(25 * m.n_elems, 0.0);
  int st = compute_euler_flux(m, cfg, sol, w.rhs.data(), w.grad.data(), w.sl.data(), false, w.vp.data());
  if (cfg.second_order) {
    compute_cell_grads(m, cfg, sol, w.grad.data(), w.ngrad.data());
    st |= compute_euler_flux(m, cfg, sol, w.rhs_o2.data(), w.grad.data(), w.sl_o2.data(), true, w.vp.data());
    flux_limiting(m, sol, w.rhs.data(), w.rhs_o2.data(), w.sl.data(), cfg.cfl);
  }
  if (g_diff.active) {
    std::vector<double> mu(m.n_elems);
    double mu0c = g_diff.use_sutherland ? 1e12 : g_diff.mu_p;
    for (int i = 0; i < m.n_elems; ++i) {
      mu[i] = mu_of(sol + 5 * i);
      if (g_diff.use_sutherland) mu0c = fmin2(mu0c, mu[i]);
    }
    momentum_diffusion(m, sol, mu.data(), mu0c, w.diag.data(), w.rhs.data());
    heat_diffusion(m, sol, mu.data(), w.diag.data(), w.rhs.data());
  }
  return st;
}

// the caller's diag goes through the 5x5 LU even without diffusion (the standalone
// add_timedisc_and_solve entry, whose diag may hold any blocks)
static bool g_force_lu = false;

// ns_euler_module.F90:521-609 (no diffusion blocks: diag = a1*(V/dt + sum_lambda)*I)
static int add_timedisc_and_solve(const Mesh& m, const NsCfg& cfg, double* sol, double* rhs, double* sum_lambda,
                                  double* delta, double* res, double* res_vect, double a1, double a2, double t,
                                  double* dt_io, double* diag) {
  double dt = 1e10;
  for (int i = 1; i <= m.n_elems; ++i) dt = fmin2(dt, m.elem[i].volume / sum_lambda[i - 1]);
  dt = cfg.cfl * dt;
  if (!cfg.local_time_step) {
    dt = fmin2(cfg.tmax - t + 1e-12, dt);
    for (int i = 0; i < m.n_elems; ++i) sum_lambda[i] = 0.0;
  }
  *res = 0.0;
  for (int k = 0; k < 5; ++k) res_vect[k] = 0.0;
  double omega = 1.0;
  for (int i = 1; i <= m.n_elems; ++i) {
    double* r = rhs + 5 * (i - 1);
    double* u = sol + 5 * (i - 1);
    for (int k = 0; k < 5; ++k) res_vect[k] = res_vect[k] + r[k] * r[k];
    double s = a1 * (m.elem[i].volume / dt + sum_lambda[i - 1]);
    double nw[5], d5[5], ad[5];
    for (int k = 0; k < 5; ++k) r[k] = r[k] + s * u[k];
    if (g_diff.active || g_force_lu) {  // diag + s I, then lu_solve_inplace_lapack (dgetrf + dgetrs)
      double* D = diag + 25 * (i - 1);
      for (int a = 0; a < 5; ++a)
        for (int b = 0; b < 5; ++b) D[a + 5 * b] = D[a + 5 * b] + s * (a == b ? 1.0 : 0.0);
      int ipiv[5];
      lapack_getrf(5, D, ipiv);
      for (int k = 0; k < 5; ++k) nw[k] = r[k];
      lapack_getrs(5, D, ipiv, nw);
    } else {
      for (int k = 0; k < 5; ++k) nw[k] = r[k] / s;
    }
    for (int k = 0; k < 5; ++k) {
      d5[k] = nw[k] - u[k];
      delta[5 * (i - 1) + k] = d5[k];
      ad[k] = a2 * d5[k];
    }
    omega = fmin2(omega, max_omega_for_positivity(u, ad));
    *res = *res + fnorm2(d5, 5);
  }
  for (int k = 0; k < 5; ++k) res_vect[k] = std::sqrt(res_vect[k]);
  int st = 0;
  if (omega <= 1e-6) st |= 8;
  if (!cfg.local_time_step && omega < 1.0) dt = (1.0 - omega) * dt;
  for (int i = 0; i < 5 * m.n_elems; ++i) sol[i] = sol[i] + a2 * omega * delta[i];
  *dt_io = dt;
  return st;
}

// ns_main.F90:72-107: while (res > final_res .and. iter <= n_max_iter); second order is
// the two-stage scheme (stage 1 a1 = 2 on sol, stage 2 a1 = 1 on soln), each stage with
// its own dt. Returns status bits; *iters, *t and *res are updated.
int ns_run(const Mesh& m, const NsCfg& cfg, double* sol, int n_max_iter, double final_res, double* t_io,
           int* iters, double* res_out, double* res_vect, double* vp_out) {
  NsWork w;
  w.rhs.assign(5 * m.n_elems, 0.0);
  w.rhs_o2.assign(5 * m.n_elems, 0.0);
  w.sl.assign(m.n_elems, 0.0);
  w.sl_o2.assign(m.n_elems, 0.0);
  w.vp.assign(3 * m.n_vert, 0.0);
  w.delta.assign(5 * m.n_elems, 0.0);
  std::vector<double> soln(5 * m.n_elems);
  double t = *t_io, res = final_res + 1.0, dt = 0.0;
  int iter = 0, st = 0;
  while (res > final_res && iter <= n_max_iter) {
    g_ns_time = t;
    st |= compute_rhs_ns(m, cfg, sol, w);
    if (cfg.second_order) {
      std::memcpy(soln.data(), sol, soln.size() * sizeof(double));
      st |= add_timedisc_and_solve(m, cfg, sol, w.rhs.data(), w.sl.data(), w.delta.data(), &res, res_vect, 2.0,
                                   1.0, t, &dt, w.diag.data());
      st |= compute_rhs_ns(m, cfg, sol, w);
      st |= add_timedisc_and_solve(m, cfg, soln.data(), w.rhs.data(), w.sl.data(), w.delta.data(), &res,
                                   res_vect, 1.0, 1.0, t, &dt, w.diag.data());
      std::memcpy(sol, soln.data(), soln.size() * sizeof(double));
    } else {
      st |= add_timedisc_and_solve(m, cfg, sol, w.rhs.data(), w.sl.data(), w.delta.data(), &res, res_vect, 1.0,
                                   1.0, t, &dt, w.diag.data());
    }
    iter = iter + 1;
    t = t + dt;
    if (st) break;
    if (!cfg.local_time_step && t >= cfg.tmax) break;
  }
  *t_io = t;
  *iters = iter;
  *res_out = res;
  if (vp_out) std::memcpy(vp_out, w.vp.data(), w.vp.size() * sizeof(double));
  return st;
}

// One compute_rhs_ns evaluation (rhs after flux limiting, first-order sum_lambda).
int ns_rhs(const Mesh& m, const NsCfg& cfg, const double* sol, double* rhs, double* sum_lambda, double* vp,
           double* cell_grad, double* mat_diag = nullptr) {
  NsWork w;
  w.rhs.assign(5 * m.n_elems, 0.0);
  w.rhs_o2.assign(5 * m.n_elems, 0.0);
  w.sl.assign(m.n_elems, 0.0);
  w.sl_o2.assign(m.n_elems, 0.0);
  w.vp.assign(3 * m.n_vert, 0.0);
  g_ns_time = 0.0;
  int st = compute_rhs_ns(m, cfg, sol, w);
  std::memcpy(rhs, w.rhs.data(), w.rhs.size() * sizeof(double));
  std::memcpy(sum_lambda, w.sl.data(), w.sl.size() * sizeof(double));
  if (vp) std::memcpy(vp, w.vp.data(), w.vp.size() * sizeof(double));
  if (cell_grad) std::memcpy(cell_grad, w.grad.data(), w.grad.size() * sizeof(double));
  if (mat_diag) std::memcpy(mat_diag, w.diag.data(), w.diag.size() * sizeof(double));
  return st;
}

// ns_euler_exact_sol_module.F90:7-44 evaluated at the cell centroids, then
// primit_to_conserv (ns_euler_module.F90:49-53).
void init_gresho(const Mesh& m, double mach, double* sol) {
  for (int i = 1; i <= m.n_elems; ++i) {
    const double* x = &m.elem[i].coord[1];
    double w[5];
    double wg = 0.2, pg = 1.0 / (G * (mach * mach));
    double r = fnorm2(x, 2);
    if (r < wg) {
      w[0] = 1.0;
      w[1] = -5.0 * x[1];
      w[2] = 5.0 * x[0];
      w[3] = 0.0;
      w[4] = pg + 12.5 * (r * r);
    } else if (r > 1.0 * wg && r < 2.0 * wg) {
      w[0] = 1.0;
      w[1] = (5.0 - 2.0 / r) * x[1];
      w[2] = (-5.0 + 2.0 / r) * x[0];
      w[3] = 0.0;
      w[4] = pg + 12.5 * (r * r) + 4.0 - 20.0 * r + 4.0 * std::log(5.0 * r);
    } else {
      w[0] = 1.0;
      w[1] = w[2] = w[3] = 0.0;
      w[4] = pg - 2.0 + 4.0 * std::log(2.0);
    }
    p2c(w, sol + 5 * (i - 1));
  }
}

// ------------------------------------------------------------------------------------
// Backward-Euler Jacobian (no counterpart in the reference, whose NS path is only
// point-implicit): A = V/dt I - d rhs/dU for the first-order two-wave residual, the
// wave speeds sl, sr frozen at their current values. The oracle restates the same
// formulas the product uses; a CPU test also checks them against finite differences.

// dF.n/dU for the Euler flux, conservative variables
static void euler_jac(const double* U, const double* n, double A[5][5]) {
  const double rho = U[0];
  const double u[3] = {U[1] / rho, U[2] / rho, U[3] / rho};
  const double q2 = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
  const double p = (G - 1) * (U[4] - 0.5 * rho * q2);
  const double vn = dot3(u, n);
  const double H = (U[4] + p) / rho;
  const double phi = 0.5 * (G - 1) * q2;
  A[0][0] = 0.0;
  for (int m = 0; m < 3; ++m) A[0][m + 1] = n[m];
  A[0][4] = 0.0;
  for (int k = 0; k < 3; ++k) {
    A[k + 1][0] = phi * n[k] - u[k] * vn;
    for (int m = 0; m < 3; ++m) {
      double a = u[k] * n[m] - (G - 1) * u[m] * n[k];
      A[k + 1][m + 1] = k == m ? a + vn : a;
    }
    A[k + 1][4] = (G - 1) * n[k];
  }
  A[4][0] = vn * (phi - H);
  for (int m = 0; m < 3; ++m) A[4][m + 1] = H * n[m] - (G - 1) * u[m] * vn;
  A[4][4] = G * vn;
}

// d(two_wave flux)/dU_L and /dU_R at frozen sl, sr
static void two_wave_jac(const double* wl, const double* wr, const double* n, double JL[5][5], double JR[5][5]) {
  double rhol = wl[0], vnl = dot3(wl + 1, n), pl = wl[4], al = sound_speed_w(wl), ul[5];
  p2c(wl, ul);
  double rhor = wr[0], vnr = dot3(wr + 1, n), pr = wr[4], ar = sound_speed_w(wr), ur[5];
  p2c(wr, ur);
  double lam_l = fmax2(fmax2(al * rhol, std::sqrt(rhol * fmax2(0.0, pr - pl))), -rhol * (vnr - vnl));
  double lam_r = fmax2(fmax2(ar * rhor, std::sqrt(rhor * fmax2(0.0, pl - pr))), -rhor * (vnr - vnl));
  double sl = vnl - lam_l / rhol, sr = vnr + lam_r / rhor;
  double AL[5][5], AR[5][5];
  euler_jac(ul, n, AL);
  euler_jac(ur, n, AR);
  const double den = sr - sl, asl = std::fabs(sl), asr = std::fabs(sr), d = asl - asr;
  const double rden = 1.0 / den;  // one division per subface; both sides multiply by it
  for (int r = 0; r < 5; ++r)
    for (int c = 0; c < 5; ++c) {
      const bool I = r == c;
      const double dL = (AL[r][c] - (I ? sl : 0.0)) * rden;
      const double dR = ((I ? sr : 0.0) - AR[r][c]) * rden;
      JL[r][c] = 0.5 * AL[r][c] - 0.5 * (d * dL - (I ? asl : 0.0));
      JR[r][c] = 0.5 * AR[r][c] - 0.5 * (d * dR + (I ? asr : 0.0));
    }
}

// Pattern (rows sorted, self included) and values of A = V/dt I - d rhs/dU; blocks are
// (5, 5) column-major as bcsr_matrix_type stores them. Cells' subfaces in ascending id.
void be_jacobian(const Mesh& m, const NsCfg& cfg, const double* sol, double dt, std::vector<int>& row,
                 std::vector<int>& col, std::vector<double>& v) {
  row.assign(m.n_elems + 1, 1);
  col.clear();
  std::vector<std::vector<int>> cols(m.n_elems + 1);
  for (int i = 1; i <= m.n_elems; ++i) {
    std::vector<int> cs{i};
    for (int k = 1; k <= m.elem[i].n_sub_faces; ++k) {
      const Face& f = m.face[m.sub_face[m.elem[i].sub_face[k]].mesh_face];
      int o = f.left_neigh == i ? f.right_neigh : f.left_neigh;
      if (o > 0) cs.push_back(o);
    }
    std::sort(cs.begin(), cs.end());
    cs.erase(std::unique(cs.begin(), cs.end()), cs.end());
    cols[i] = cs;
    row[i] = row[i - 1] + (int)cs.size();
    col.insert(col.end(), cs.begin(), cs.end());
  }
  v.assign((size_t)25 * col.size(), 0.0);
  auto blk = [&](int i, int j) -> double* {
    const auto& cs = cols[i];
    int q = (int)(std::lower_bound(cs.begin(), cs.end(), j) - cs.begin());
    return &v[(size_t)25 * (row[i - 1] - 1 + q)];
  };
  for (int i = 1; i <= m.n_elems; ++i) {
    double* D = blk(i, i);
    const double vdt = m.elem[i].volume / dt;
    for (int r = 0; r < 5; ++r) D[r + 5 * r] = vdt;
    for (int k = 1; k <= m.elem[i].n_sub_faces; ++k) {
      const int sf = m.elem[i].sub_face[k];
      const SubFace& s = m.sub_face[sf];
      const Face& f = m.face[s.mesh_face];
      const double* n = &s.norm[1];
      const double area = s.area;
      const int L = f.left_neigh, R = f.right_neigh;
      double wl[5], wr[5];
      reconstruct_lr_w(m, cfg, sol, nullptr, s.mesh_vert, sf, L, R, false, wl, wr);
      double JL[5][5], JR[5][5];
      two_wave_jac(wl, wr, n, JL, JR);
      if (i == L) {
        if (R > 0) {
          for (int r = 0; r < 5; ++r)
            for (int c = 0; c < 5; ++c) D[r + 5 * c] = D[r + 5 * c] + area * JL[r][c];
          double* O = blk(i, R);
          for (int r = 0; r < 5; ++r)
            for (int c = 0; c < 5; ++c) O[r + 5 * c] = O[r + 5 * c] + area * JR[r][c];
        } else {  // ghost state U_R(U_L) through M = dU_R/dU_L: reflections, I or 0
          const int kind = R == 0 ? 1 : cfg.bc_type[-R - 1];
          const double* bv = R < 0 ? cfg.bc_val + 5 * (-R - 1) : nullptr;
          const double fx0 = m.face[s.mesh_face].coord[1];
          double M[5][5] = {{0}};
          if (kind == 1 || (kind == 7 && !(fx0 < 0.1667))) {
            M[0][0] = M[4][4] = 1.0;
            for (int a = 0; a < 3; ++a)
              for (int b = 0; b < 3; ++b) M[a + 1][b + 1] = (a == b ? 1.0 : 0.0) - 2.0 * n[a] * n[b];
          } else if (kind == 4) {
            for (int a = 0; a < 5; ++a) M[a][a] = 1.0;
          } else if (kind == 5) {
            double ub[5];
            p2c(bv, ub);
            if (dot3(ub + 1, n) > 0.0)
              for (int a = 0; a < 5; ++a) M[a][a] = 1.0;
          } else if (kind == 2) {  // rho_r = rho, m_r = 2 rho b - m, E_r = E - |m|^2/2rho + |m_r|^2/2rho
            double uu = 0.0, rb = 0.0, rr = 0.0;
            for (int a = 0; a < 3; ++a) {
              const double r = 2.0 * bv[a + 1] - wl[a + 1];
              uu = uu + wl[a + 1] * wl[a + 1];
              rb = rb + r * bv[a + 1];
              rr = rr + r * r;
            }
            M[0][0] = 1.0;
            for (int a = 0; a < 3; ++a) {
              M[a + 1][0] = 2.0 * bv[a + 1];
              M[a + 1][a + 1] = -1.0;
              M[4][a + 1] = -2.0 * bv[a + 1];
            }
            M[4][0] = 0.5 * uu + 2.0 * rb - 0.5 * rr;
            M[4][4] = 1.0;
          }
          for (int r = 0; r < 5; ++r)
            for (int c = 0; c < 5; ++c) {
              double t = 0.0;
              for (int q = 0; q < 5; ++q) t = t + JR[r][q] * M[q][c];
              D[r + 5 * c] = D[r + 5 * c] + area * (JL[r][c] + t);
            }
        }
      } else {
        for (int r = 0; r < 5; ++r)
          for (int c = 0; c < 5; ++c) D[r + 5 * c] = D[r + 5 * c] - area * JR[r][c];
        double* O = blk(i, L);
        for (int r = 0; r < 5; ++r)
          for (int c = 0; c < 5; ++c) O[r + 5 * c] = O[r + 5 * c] - area * JL[r][c];
      }
    }
  }
}

int oracle_pinv3(double* a9) {
  double A[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) A[i][j] = a9[3 * i + j];
  pinv3(A);
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) a9[3 * i + j] = A[i][j];
  return 0;
}
void oracle_lu3(double* a9, double* x, const double* b) {
  double A[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) A[i][j] = a9[3 * i + j];
  lu_solve3(A, x, b);
}

}  // namespace oracle

using namespace oracle;
struct OHandleNs;  // the mesh handle of oracle_capi.cpp
namespace oracle {
Mesh& handle_mesh(void* h);
}

extern "C" {

static NsCfg make_cfg(const int* ic, const double* dc, const int* bc_type, const double* bc_val) {
  NsCfg c;
  c.scheme = ic[0];
  c.second_order = ic[1];
  c.method = ic[2];
  c.bc_style = ic[3];
  c.b2d = ic[4];
  c.exclude_bound_vert = ic[5];
  c.local_time_step = ic[6];
  c.n_bc = ic[7];
  c.cfl = dc[0];
  c.tmax = dc[1];
  c.bc_type = bc_type;
  c.bc_val = bc_val;
  return c;
}

// ic = {scheme, second_order, method, bc_style, b2d, exclude_bound_vert, local_time_step, n_bc}
// dc = {cfl, tmax}
int or_ns_rhs(void* h, const int* ic, const double* dc, const int* bc_type, const double* bc_val,
              const double* sol, double* rhs, double* sum_lambda, double* vp, double* grad) {
  return ns_rhs(handle_mesh(h), make_cfg(ic, dc, bc_type, bc_val), sol, rhs, sum_lambda, vp, grad);
}
// compute_rhs_ns with mat_diag (5, 5, n) column-major per cell
int or_ns_rhs_diag(void* h, const int* ic, const double* dc, const int* bc_type, const double* bc_val,
                   const double* sol, double* rhs, double* sum_lambda, double* mat_diag) {
  return ns_rhs(handle_mesh(h), make_cfg(ic, dc, bc_type, bc_val), sol, rhs, sum_lambda, nullptr, nullptr, mat_diag);
}
int or_ns_run(void* h, const int* ic, const double* dc, const int* bc_type, const double* bc_val, double* sol,
              int n_max_iter, double final_res, double* t_io, int* iters, double* res, double* res_vect, double* vp) {
  return ns_run(handle_mesh(h), make_cfg(ic, dc, bc_type, bc_val), sol, n_max_iter, final_res, t_io, iters, res,
                res_vect, vp);
}
void or_ns_gresho(void* h, double mach, double* sol) { init_gresho(handle_mesh(h), mach, sol); }
// The procedures one at a time (grad and ngrad in the oracle's layout, 15 per entity,
// g[5 d + var]).
int or_euler_flux(void* h, const int* ic, const double* dc, const int* bc_type, const double* bc_val,
                  const double* sol, const double* grad, int second_order, double* rhs, double* sum_lambda,
                  double* vp) {
  const Mesh& m = handle_mesh(h);
  std::vector<double> vpw(3 * m.n_vert, 0.0);
  g_ns_time = 0.0;
  int st = compute_euler_flux(m, make_cfg(ic, dc, bc_type, bc_val), sol, rhs, grad, sum_lambda, second_order != 0,
                              vp ? vp : vpw.data());
  return st;
}
void or_cell_grads(void* h, const int* ic, const double* dc, const int* bc_type, const double* bc_val,
                   const double* sol, double* grad, double* ngrad) {
  const Mesh& m = handle_mesh(h);
  for (int i = 0; i < 15 * m.n_elems; ++i) grad[i] = 0.0;
  for (int i = 0; i < 15 * m.n_vert; ++i) ngrad[i] = 0.0;
  compute_cell_grads(m, make_cfg(ic, dc, bc_type, bc_val), sol, grad, ngrad);
}
void or_flux_limiting(void* h, const double* sol, double* rhs, const double* rhs_o2, const double* sum_lambda,
                      double cfl) {
  flux_limiting(handle_mesh(h), sol, rhs, rhs_o2, sum_lambda, cfl);
}
int or_add_timedisc(void* h, const int* ic, const double* dc, const int* bc_type, const double* bc_val, double* sol,
                    double* rhs, double* diag, double* sum_lambda, double* delta, double* res, double* res_vect,
                    double a1, double a2, double t, double* dt) {
  const Mesh& m = handle_mesh(h);
  std::vector<double> zero;
  if (!diag) zero.assign(25 * m.n_elems, 0.0);
  g_force_lu = diag != nullptr;
  int st = add_timedisc_and_solve(m, make_cfg(ic, dc, bc_type, bc_val), sol, rhs, sum_lambda, delta, res, res_vect,
                                  a1, a2, t, dt, diag ? diag : zero.data());
  g_force_lu = false;
  return st;
}
void or_pinv3(double* a9) { oracle_pinv3(a9); }
void or_set_lapack(void* dgesvd, void* dgetrf, void* dgetrs) {
  g_dgesvd = reinterpret_cast<dgesvd_fn>(dgesvd);
  g_dgetrf = reinterpret_cast<dgetrf_fn>(dgetrf);
  g_dgetrs = reinterpret_cast<dgetrs_fn>(dgetrs);
}
// one subface flux: scheme 3 three_wave, 5 modified_three_wave, else two_wave; lr (5, 2)
void or_ns_flux(int scheme, const double* wl, const double* wr, const double* n, double* lr10, double* slsr) {
  double lr[2][5];
  if (scheme == 3 || scheme == 5) three_wave(wl, wr, n, lr, &slsr[0], &slsr[1], scheme == 5);
  else two_wave(wl, wr, n, lr, &slsr[0], &slsr[1]);
  for (int k = 0; k < 5; ++k) {
    lr10[k] = lr[0][k];
    lr10[5 + k] = lr[1][k];
  }
}
// returns nnz blocks; row (n_elems+1), col (nnz) 1-based, v (25 nnz); cap = capacity of col
long or_be_jacobian(void* h, const int* ic, const double* dc, const int* bc_type, const double* bc_val,
                    const double* sol, double dt, int* row, int* col, double* v, long cap) {
  std::vector<int> r, c;
  std::vector<double> vv;
  g_ns_time = 0.0;
  be_jacobian(handle_mesh(h), make_cfg(ic, dc, bc_type, bc_val), sol, dt, r, c, vv);
  if ((long)c.size() > cap) return -(long)c.size();
  std::memcpy(row, r.data(), r.size() * sizeof(int));
  std::memcpy(col, c.data(), c.size() * sizeof(int));
  std::memcpy(v, vv.data(), vv.size() * sizeof(double));
  return (long)c.size();
}
void or_lu3(double* a9, double* x, const double* b) { oracle_lu3(a9, x, b); }
// the diffusion namelist entries (activate_diffusion, use_sutherland, mu_p, mu0, T0, Cv_p
// and per tag bc_type_V / bc_val_V(3) / bc_type_T / bc_val_T, kinds 1 neumann, 2 dirichlet)
void or_ns_set_diffusion(int active, int use_sutherland, const double* dc4, int n_bc, const int* bcV,
                         const double* valV, const int* bcT, const double* valT) {
  g_diff = DiffCfg();
  g_diff.active = active;
  g_diff.use_sutherland = use_sutherland;
  g_diff.mu_p = dc4[0];
  g_diff.mu0 = dc4[1];
  g_diff.T0 = dc4[2];
  g_diff.Cv_p = dc4[3];
  g_diff.prandtl = dc4[4] > 0.0 ? dc4[4] : 0.71;
  for (int i = 0; i < n_bc && i < 16; ++i) {
    g_diff.bcV[i] = bcV[i];
    g_diff.bcT[i] = bcT[i];
    g_diff.valT[i] = valT[i];
    for (int k = 0; k < 3; ++k) g_diff.valV[i][k] = valV[3 * i + k];
  }
}
// inv_lapack (dgetrf + dgetri) of the n x n column-major a, in place
void or_lapack_inverse(int n, double* a) { lapack_inverse(n, a); }
// lu_solve_inplace_lapack: a (n x n column-major) overwritten by its factors, b by x
void or_lapack_solve(int n, double* a, double* b) {
  std::vector<int> ipiv(n);
  lapack_getrf(n, a, ipiv.data());
  lapack_getrs(n, a, ipiv.data(), b);
}
// sol_potential_flow_2d / _3d at x (primitive w)
void or_potential_flow(const double* x, int three_d, double* w) { potential_flow(x, three_d != 0, w); }

}  // extern "C"
