// Explicit Euler residual path of subfvns on the GPU.
//
// Reference: src/ns/ns_euler_module.F90:151-609 (compute_euler_flux,
// compute_rhs_around_vert, add_timedisc_and_solve), src/ns/ns_euler_rs_module.F90:154-422
// (two_wave, multi_point, compute_lambdas_and_solve_nodal_velocity),
// src/ns/ns_euler_recon_module.F90:8-601 (nodal and cell gradients, limiters,
// reconstruction, boundary states, flux_limiting), src/ns/ns_euler_primitives_module.F90.
//
// Kernels of one residual evaluation (compute_rhs_ns):
//   k_ns_node        one thread per vertex: reconstruct the left/right states of its
//                    subfaces, run the 4-iteration nodal velocity solver (multi_point),
//                    evaluate the subface fluxes and sum them per corner (subcell)
//   k_ns_gather      one thread per cell: rhs = -sum of its corners' sums in ascending
//                    vertex order (the reference's scatter order), no atomics; block min
//                    of V / sum_lambda for the CFL step
//   k_ns_nodal_grad  one thread per vertex: least-squares gradient, 3x3 pseudo-inverse
//   k_ns_cell_grad   one thread per cell: method-4 weighting, physical slope limiter,
//                    relaxed maximum principle
//   (on small meshes the node kernel and both gradients run a group of lanes per
//   vertex or cell instead: k_ns_node_group, k_ns_nodal_grad_group, k_ns_cell_grad_group)
// then per stage k_ns_timedisc (flux limiting blend, diagonal solve, positivity limiter,
// residual partial sums; its last block to finish runs the stage's scalar tail) and
// k_ns_apply (batched problems: kb_ns_timedisc, kb_ns_finalize, kb_ns_apply).
//
// Plain FP64 (precision 0) follows the reference's evaluation order and is compiled
// without FMA contraction, so it reproduces the CPU restatement bit for bit, except the
// residual norms (res, res_vect), which are summed by a fixed tree of block partials.
// Precision 1 evaluates the nodal solver's wave-speed bounds (lambda, vbar) in FP32;
// precision 2 also the reconstruction, the limiters and the subface fluxes. In both the
// nodal 3x3 systems (M, R and the solve), the nodal gradient system and all sums stay
// FP64.
#include <algorithm>
#include <cstring>

#include "ns.cuh"
#include "ns_diffusion.cuh"

namespace subfv {

NsParams ns_params_from(const subfv_ns_cfg& c) {
  NsParams p{};
  p.scheme = c.scheme;
  p.second_order = c.second_order;
  p.method = c.method;
  p.bc_style = c.bc_style;
  p.b2d = c.boundary_2d;
  p.excl = c.exclude_bound_vert;
  p.lts = c.local_time_step;
  p.n_bc = c.n_bc;
  for (int i = 0; i < 16; ++i) {
    p.bc_type[i] = c.bc_type[i];
    for (int k = 0; k < 5; ++k) p.bc_val[i][k] = c.bc_val[i][k];
  }
  p.cfl = c.cfl;
  p.tmax = c.tmax;
  p.precision = c.precision;
  p.node_group = 0;
  p.diff = c.activate_diffusion;
  p.diff_kd = 0;
  return p;
}

namespace {

constexpr double G = 1.4;  // ns_global_data_module.F90:9

__device__ inline double fmax2(double a, double b) { return b > a ? b : a; }
__device__ inline double fmin2(double a, double b) { return b < a ? b : a; }
template <class T>
__device__ inline T tmax2(T a, T b) { return b > a ? b : a; }
template <class T>
__device__ inline T tmin2(T a, T b) { return b < a ? b : a; }

template <class T>
__device__ inline void p2c(const T* w, T* u) {
  u[0] = w[0];
  for (int k = 1; k < 4; ++k) u[k] = w[k] * w[0];
  u[4] = w[4] / (T)(G - 1) + (T)0.5 * w[0] * (w[1] * w[1] + w[2] * w[2] + w[3] * w[3]);
}
template <class T>
__device__ inline void c2p(const T* u, T* w) {
  w[0] = u[0];
  for (int k = 1; k < 4; ++k) w[k] = u[k] / u[0];
  w[4] = (T)(G - 1) * (u[4] - (T)0.5 * w[0] * (w[1] * w[1] + w[2] * w[2] + w[3] * w[3]));
}
template <class T>
__device__ inline T dotT(const T* a, const T* b) {
  T s = 0;
  s = s + a[0] * b[0];
  s = s + a[1] * b[1];
  s = s + a[2] * b[2];
  return s;
}
__device__ inline double sound_speed_w(const double* w) { return sqrt(G * w[4] / w[0]); }

__device__ inline void ld5(const double* U, int c, double* u) {
  const double* r = U + kRec * (size_t)c;
  for (int k = 0; k < 5; ++k) u[k] = r[k];
}

// ns_euler_primitives_module.F90:92-111
__device__ double max_omega_for_positivity(const double* U, const double* dU) {
  double omega = 1.0, US[5], WS[5];
  for (int k = 0; k < 5; ++k) US[k] = U[k] + omega * dU[k];
  c2p(US, WS);
  bool pos = WS[0] > 1e-17 && WS[4] > 1e-17;
  while (!pos && omega > 1e-6) {  // at most ~131 halvings by 0.9 before omega <= 1e-6
    omega = omega * 0.9;
    for (int k = 0; k < 5; ++k) US[k] = U[k] + omega * dU[k];
    c2p(US, WS);
    pos = WS[0] > 1e-17 && WS[4] > 1e-17;
  }
  return omega;
}

// When every singular value passes the cut, the pseudo-inverse is the inverse. The cut
// (3e-12 * sigma_max) is certainly passed when |det A| > 3e-12 ||A||_F^3, because
// sigma_min >= |det A| / sigma_max^2 and sigma_max <= ||A||_F. Then A^-1 = adj(A) / det,
// refined by one Newton step X <- X + X (I - A X); otherwise the Jacobi SVD below runs.
__device__ bool inv3_if_regular(double A[3][3]) {
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

// Pseudo-inverse of a 3x3 matrix (A[r][c] = mat(r+1, c+1)); singular values below
// 3e-12 * max discarded (the cut of pseudo_inverse_inplace_lapack,
// linear_solver_module.F90:683-715): the inverse when the cut cannot bite, else a
// one-sided Jacobi SVD of six sweeps.
__device__ __noinline__ void pinv3_jacobi(double A[3][3]);
// the Jacobi case works on a copy: an array whose address reaches an out-of-line call
// lives in local memory on every path, so the caller's matrix keeps no escaping address
__device__ inline void pinv3(double A[3][3]) {
  if (!inv3_if_regular(A)) {
    double B[3][3];
    for (int d = 0; d < 3; ++d)
      for (int e = 0; e < 3; ++e) B[d][e] = A[d][e];
    pinv3_jacobi(B);
    for (int d = 0; d < 3; ++d)
      for (int e = 0; e < 3; ++e) A[d][e] = B[d][e];
  }
}
// the rank-deficient case, out of line (rare; keeps the callers' registers low)
__device__ __noinline__ void pinv3_jacobi(double A[3][3]) {
  double U[3][3], V[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) U[i][j] = A[i][j];
  const int pr[3][2] = {{0, 1}, {0, 2}, {1, 2}};
  for (int sweep = 0; sweep < 6; ++sweep)
    for (int r = 0; r < 3; ++r) {
      const int p = pr[r][0], q = pr[r][1];
      double al = 0.0, be = 0.0, ga = 0.0;
      for (int i = 0; i < 3; ++i) {
        al = al + U[i][p] * U[i][p];
        be = be + U[i][q] * U[i][q];
        ga = ga + U[i][p] * U[i][q];
      }
      if (!(fabs(ga) > 1e-15 * sqrt(al * be))) continue;
      double zeta = (be - al) / (2.0 * ga);
      double t = 1.0 / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
      if (zeta < 0.0) t = -t;
      double c = 1.0 / sqrt(1.0 + t * t), s = c * t;
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
    sig[k] = sqrt(s);
    smax = fmax2(smax, sig[k]);
  }
  const double tol = 3 * 1e-12 * smax;
  double SUt[3][3];
  for (int k = 0; k < 3; ++k)
    for (int j = 0; j < 3; ++j) SUt[k][j] = sig[k] > tol ? (1.0 / sig[k]) * (U[j][k] / sig[k]) : 0.0;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double s = 0.0;
      for (int k = 0; k < 3; ++k) s = s + V[i][k] * SUt[k][j];
      A[i][j] = s;
    }
}

// LU with partial pivoting and the triangular solves, in the operation order of
// LAPACK dgetrf2/dgetrs with reference BLAS (lu_solve_inplace_lapack, :643-657).
__device__ void lu_solve3(double A[3][3], double* x, const double* b) {
  const double sfmin = 2.2250738585072014e-308;
  int ipiv[3];
  for (int j = 0; j < 3; ++j) {
    int p = j;
    double amax = fabs(A[j][j]);
    for (int i = j + 1; i < 3; ++i)
      if (fabs(A[i][j]) > amax) {
        amax = fabs(A[i][j]);
        p = i;
      }
    ipiv[j] = p;
    if (A[p][j] != 0.0) {
      if (p != j)
        for (int k = 0; k < 3; ++k) {
          double t = A[j][k];
          A[j][k] = A[p][k];
          A[p][k] = t;
        }
      if (fabs(A[j][j]) >= sfmin) {
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
    if (ipiv[j] != j) {
      double t = y[j];
      y[j] = y[ipiv[j]];
      y[ipiv[j]] = t;
    }
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

// Boundary semantics on the device: flr.y >= 0 is the right cell; otherwise the face's
// reference right_neigh is flr.y + 1 (0 = default wall, -tag = boundary condition tag).
__device__ inline bool is_wall(const NsParams& P, int y) {
  if (y >= 0) return false;
  if (y == -1) return true;
  return P.bc_type[-(y + 1) - 1] == 1;
}

// OI (ns_euler_recon_module.F90:322-329): gfortran's scaled NORM2 of a 3-vector, in T
template <class T>
__device__ inline T oi3(T a0, T a1, T a2) {
  const T a[3] = {a0, a1, a2};
  T scale = 1, res = 0;
  for (int i = 0; i < 3; ++i)
    if (a[i] != (T)0) {
      T ax = fabs(a[i]);
      if (ax > scale) {
        T q = scale / ax;
        res = (T)1 + res * q * q;
        scale = ax;
      } else {
        T q = ax / scale;
        res += q * q;
      }
    }
  return scale * sqrt(res);
}

// sol_potential_flow_2d / _3d (ns_euler_exact_sol_module.F90:105-170) at x, primitive.
// The 2-D routine's Mach number is a default-kind (single precision) literal, so its
// value is the float nearest 1e-4; the 3-D one is 1e-4 in double.
template <class T>
__device__ __noinline__ void potential_flow(const double4 x4, bool three_d, T* w) {
  const T x[3] = {(T)x4.x, (T)x4.y, (T)x4.z};
  const T r0 = (T)0.5, r1 = (T)5.5, rhoinf = (T)1.4, pinf = (T)1.0;
  const T mach = three_d ? (T)1e-4 : (T)1e-4f;
  const T vinf = mach * sqrt((T)G * pinf / rhoinf);
  T ux, uy, uz;
  if (!three_d) {
    const T r = sqrt(x[0] * x[0] + x[1] * x[1]);
    const T th = atan2(x[1], x[0]);
    const T c = r1 * r1 / (r1 * r1 - r0 * r0), q = (r0 / r) * (r0 / r);
    const T vr = c * ((T)1 - q) * cos(th);
    const T vt = -c * ((T)1 + q) * sin(th);
    ux = vinf * (cos(th) * vr - sin(th) * vt);
    uy = vinf * (sin(th) * vr + cos(th) * vt);
    uz = (T)0;
  } else {
    const T r = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
    const T f = r0 * r0 * r0 / ((T)2 * (r * r * r * r * r));
    ux = vinf * ((T)1 + f * (r * r - (T)3 * (x[0] * x[0])));
    uy = (T)-3 * vinf * f * x[0] * x[1];
    uz = (T)-3 * vinf * f * x[0] * x[2];
  }
  const T vmag2 = ux * ux + uy * uy + uz * uz;
  w[0] = rhoinf;
  w[1] = ux;
  w[2] = uy;
  w[3] = uz;
  w[4] = pinf + (T)0.5 * rhoinf * (vinf * vinf - vmag2);
}

// compute_right_state (:331-409): the ghost state by boundary kind (1 wall, 2 adherence
// wall, 3 freestream, 4 supersonic outflow, 5 pondered inflow, 6 double-Mach inflow /
// outflow, 7 double-Mach bottom, 8 and 9 the potential flows in 2-D and 3-D); sol_l /
// sol_r conservative, n the subface normal. The kinds that read the face centroid fx or
// the time t (of the step being evaluated) are out of line. Their arguments are values
// only: a reference to the kernel's mesh or parameter block would make every thread of
// the calling kernel copy that block into local memory.
struct BcVals {
  double v[5];
};
template <class T>
__device__ __noinline__ void right_state_ext(int kind, const BcVals bv, const double4 fx, const double t, const T* n,
                                             const T* sol_l, T* sol_r) {
  if (kind == 2) {
    for (int k = 0; k < 5; ++k) sol_r[k] = sol_l[k];
    for (int k = 1; k < 4; ++k) sol_r[k] = (T)2.0 * sol_l[0] * (T)bv.v[k] - sol_l[k];
    const T nl = oi3<T>(sol_l[1] / sol_l[0], sol_l[2] / sol_l[0], sol_l[3] / sol_l[0]);
    const T nr = oi3<T>(sol_r[1] / sol_r[0], sol_r[2] / sol_r[0], sol_r[3] / sol_r[0]);
    sol_r[4] = sol_l[4] - (T)0.5 * sol_l[0] * (nl * nl) + (T)0.5 * sol_l[0] * (nr * nr);
    return;
  }
  if (kind == 5) {
    T w[5];
    for (int k = 0; k < 5; ++k) w[k] = (T)bv.v[k];
    p2c(w, sol_r);
    if (dotT(sol_r + 1, n) > (T)0)
      for (int k = 0; k < 5; ++k) sol_r[k] = sol_l[k];
    return;
  }
  if (kind == 8 || kind == 9) {
    T w[5];
    potential_flow<T>(fx, kind == 9, w);
    p2c(w, sol_r);
    return;
  }
  const T post[5] = {(T)8.0, (T)7.145, (T)-4.125, (T)0.0, (T)116.5}, pre[5] = {(T)1.4, 0, 0, 0, (T)1.0};
  if (kind == 6) {
    p2c((T)fx.y > (T)1.732 * ((T)fx.x - (T)0.1667 - (T)10.0 * (T)t) ? post : pre, sol_r);
  } else if ((T)fx.x < (T)0.1667) {  // kind 7
    p2c(post, sol_r);
  } else {
    for (int k = 0; k < 5; ++k) sol_r[k] = sol_l[k];
    T d = dotT(sol_r + 1, n);
    for (int k = 1; k < 4; ++k) sol_r[k] = sol_r[k] - (T)2.0 * d * n[k - 1];
  }
}

template <class T>
__device__ void right_state(const DevMesh& m, const NsParams& P, int y, int sf, const T* n, const T* sol_l, T* sol_r,
                            const NsScalars* sc) {
  int kind = y == -1 ? 1 : P.bc_type[-(y + 1) - 1];
  if (kind == 1) {
    for (int k = 0; k < 5; ++k) sol_r[k] = sol_l[k];
    T d = dotT(sol_r + 1, n);
    for (int k = 1; k < 4; ++k) sol_r[k] = sol_r[k] - (T)2.0 * d * n[k - 1];
  } else if (kind == 3) {
    T w[5];
    for (int k = 0; k < 5; ++k) w[k] = (T)P.bc_val[-(y + 1) - 1][k];
    p2c(w, sol_r);
  } else if (kind == 4) {
    for (int k = 0; k < 5; ++k) sol_r[k] = sol_l[k];
  } else {
    BcVals bv;
    for (int k = 0; k < 5; ++k) bv.v[k] = P.bc_val[-(y + 1) - 1][k];
    const double4 fx = kind >= 6 ? m.fc[m.sf_face[sf]] : make_double4(0.0, 0.0, 0.0, 0.0);
    const double t = (kind == 6 && sc) ? sc->t : 0.0;
    right_state_ext<T>(kind, bv, fx, t, n, sol_l, sol_r);
  }
}

// reconstruct_lr_w (:427-451); grad records [15] with g[5*d + var] = grad(d+1, var+1)
template <class T>
__device__ void reconstruct(const DevMesh& m, const NsParams& P, const double* U, const double* grad, int v, int sf,
                            int le, int y, bool so, double* wl_out, double* wr_out, const NsScalars* sc) {
  T ul[5], wl[5], wr[5];
  double u64[5];
  ld5(U, le, u64);
  for (int k = 0; k < 5; ++k) ul[k] = (T)u64[k];
  c2p(ul, wl);
  const double4 xv = m.x[v];
  if (so) {
    const double4 cc = m.cc[le];
    const T dx[3] = {(T)(xv.x - cc.x), (T)(xv.y - cc.y), (T)(xv.z - cc.z)};
    const double* g = grad + 15 * (size_t)le;
    for (int k = 0; k < 5; ++k) {
      T s = 0;
      for (int d = 0; d < 3; ++d) s = s + (T)g[5 * d + k] * dx[d];
      wl[k] = wl[k] + s;
    }
  }
  if (y >= 0) {
    T ur[5];
    ld5(U, y, u64);
    for (int k = 0; k < 5; ++k) ur[k] = (T)u64[k];
    c2p(ur, wr);
    if (so) {
      const double4 cc = m.cc[y];
      const T dx[3] = {(T)(xv.x - cc.x), (T)(xv.y - cc.y), (T)(xv.z - cc.z)};
      const double* g = grad + 15 * (size_t)y;
      for (int k = 0; k < 5; ++k) {
        T s = 0;
        for (int d = 0; d < 3; ++d) s = s + (T)g[5 * d + k] * dx[d];
        wr[k] = wr[k] + s;
      }
    }
  } else {
    const double4 sn = m.sfn[sf];
    const T n[3] = {(T)sn.x, (T)sn.y, (T)sn.z};
    T uc[5], gh[5];
    p2c(wl, uc);
    right_state(m, P, y, sf, n, uc, gh, sc);
    c2p(gh, wr);
  }
  for (int k = 0; k < 5; ++k) {
    wl_out[k] = (double)wl[k];
    wr_out[k] = (double)wr[k];
  }
}

// two_wave (ns_euler_rs_module.F90:154-198)
template <class T>
__device__ void two_wave(const double* wl64, const double* wr64, const double* n64, double lr[2][5], double* sl_o,
                         double* sr_o) {
  T wl[5], wr[5], n[3];
  for (int k = 0; k < 5; ++k) {
    wl[k] = (T)wl64[k];
    wr[k] = (T)wr64[k];
  }
  for (int d = 0; d < 3; ++d) n[d] = (T)n64[d];
  T rhol = wl[0], vnl = dotT(wl + 1, n), pl = wl[4], al = sqrt((T)G * wl[4] / wl[0]), ul[5];
  p2c(wl, ul);
  T rhor = wr[0], vnr = dotT(wr + 1, n), pr = wr[4], ar = sqrt((T)G * wr[4] / wr[0]), ur[5];
  p2c(wr, ur);
  T fl[5], fr[5];
  fl[0] = vnl * ul[0];
  for (int k = 1; k < 4; ++k) fl[k] = vnl * ul[k] + pl * n[k - 1];
  fl[4] = (ul[4] + pl) * vnl;
  fr[0] = vnr * ur[0];
  for (int k = 1; k < 4; ++k) fr[k] = vnr * ur[k] + pr * n[k - 1];
  fr[4] = (ur[4] + pr) * vnr;
  T lam_l = tmax2(tmax2(al * rhol, sqrt(rhol * tmax2((T)0, pr - pl))), -rhol * (vnr - vnl));
  T lam_r = tmax2(tmax2(ar * rhor, sqrt(rhor * tmax2((T)0, pl - pr))), -rhor * (vnr - vnl));
  T sl = vnl - lam_l / rhol;
  T sr = vnr + lam_r / rhor;
  for (int k = 0; k < 5; ++k) {
    T et = (sr * ur[k] - sl * ul[k] - (fr[k] - fl[k])) / (sr - sl);
    T f = (T)0.5 * (fl[k] + fr[k]) - (T)0.5 * (fabs(sl) * (et - ul[k]) + fabs(sr) * (ur[k] - et));
    lr[0][k] = (double)f;
    lr[1][k] = (double)(-f);
  }
  *sl_o = (double)sl;
  *sr_o = (double)sr;
}

// three_wave (ns_euler_rs_module.F90:9-75) and modified_three_wave (:77-152): two-wave
// bounds, v* = v_bar, HLLC-type star states (the modified form averages the tangential
// velocity and carries its jump energy); arithmetic in T, results stored as double. The
// fluxes of the schemes beyond multi_point and two_wave are out of line, so the node
// kernel's register allocation for those two does not grow with them.
template <class T>
__device__ __noinline__ void three_wave(const double* wl64, const double* wr64, const double* n64, double lr[2][5],
                           double* sl_o, double* sr_o, bool modified) {
  T wl[5], wr[5], n[3];
  for (int k = 0; k < 5; ++k) {
    wl[k] = (T)wl64[k];
    wr[k] = (T)wr64[k];
  }
  for (int d = 0; d < 3; ++d) n[d] = (T)n64[d];
  const T c0 = (T)0, c1 = (T)1, ch = (T)0.5;
  T rhol = wl[0], vnl = dotT(wl + 1, n), pl = wl[4], ul[5];
  p2c(wl, ul);
  T el = ul[4] / rhol, al = sqrt((T)G * wl[4] / wl[0]);
  T rhor = wr[0], vnr = dotT(wr + 1, n), pr = wr[4], ur[5];
  p2c(wr, ur);
  T er = ur[4] / rhor, ar = sqrt((T)G * wr[4] / wr[0]);
  T fl[5], fr[5];
  fl[0] = vnl * ul[0];
  for (int k = 1; k < 4; ++k) fl[k] = vnl * ul[k] + pl * n[k - 1];
  fl[4] = (ul[4] + pl) * vnl;
  fr[0] = vnr * ur[0];
  for (int k = 1; k < 4; ++k) fr[k] = vnr * ur[k] + pr * n[k - 1];
  fr[4] = (ur[4] + pr) * vnr;
  T lam_l = tmax2(tmax2(al * rhol, sqrt(rhol * tmax2(c0, pr - pl))), -rhol * (vnr - vnl));
  T lam_r = tmax2(tmax2(ar * rhor, sqrt(rhor * tmax2(c0, pl - pr))), -rhor * (vnr - vnl));
  T v_et = (lam_l * vnl + lam_r * vnr - (pr - pl)) / (lam_r + lam_l);
  T vt_et[3] = {c0, c0, c0}, tang_energy = c0;
  if (modified) {
    T vt_l[3], vt_r[3], dvt[3];
    for (int d = 0; d < 3; ++d) {
      vt_l[d] = wl[1 + d] - vnl * n[d];
      vt_r[d] = wr[1 + d] - vnr * n[d];
    }
    for (int d = 0; d < 3; ++d) vt_et[d] = (lam_l * vt_l[d] + lam_r * vt_r[d]) / (lam_l + lam_r);
    for (int d = 0; d < 3; ++d) dvt[d] = vt_r[d] - vt_l[d];
    const T tang_coeff = -(lam_l * lam_r / (lam_l + lam_r));
    tang_energy = tang_coeff * dotT(dvt, vt_et);
  }
  T rhol_et = c1 / (c1 / rhol + (v_et - vnl) / lam_l);
  T pl_bar = pl - lam_l * (v_et - vnl);
  T rhor_et = c1 / (c1 / rhor + (vnr - v_et) / lam_r);
  T pr_bar = pr + lam_r * (v_et - vnr);
  T sle[5], sre[5];
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
  const T sl = vnl - lam_l / rhol, sr = vnr + lam_r / rhor;
  for (int k = 0; k < 5; ++k) {
    const T f = ch * (fl[k] + fr[k]) -
                ch * (fabs(sl) * (sle[k] - ul[k]) + fabs(v_et) * (sre[k] - sle[k]) + fabs(sr) * (ur[k] - sre[k]));
    lr[0][k] = (double)f;
    lr[1][k] = (double)(-f);
  }
  *sl_o = (double)sl;
  *sr_o = (double)sr;
}

// multi_point_pressure (ns_euler_rs_module.F90:555-616) and multi_point_pressure_ph
// (:618-679): star states from the nodal pressure and the nodal pressure solver's bounds.
template <class T>
__device__ __noinline__ void multi_point_pressure(const double* wl64, const double* wr64, const double* n64, double lr[2][5],
                                     double p_nodal64, double lam_l64, double lam_r64, double* sl_o, double* sr_o,
                                     bool ph) {
  T wl[5], wr[5], n[3];
  for (int k = 0; k < 5; ++k) {
    wl[k] = (T)wl64[k];
    wr[k] = (T)wr64[k];
  }
  for (int d = 0; d < 3; ++d) n[d] = (T)n64[d];
  const T lam_l = (T)lam_l64, lam_r = (T)lam_r64, p_nodal = (T)p_nodal64, c1 = (T)1, ch = (T)0.5;
  T rhol = wl[0], vnl = dotT(wl + 1, n), pl = wl[4], ul[5], vt_l[3];
  for (int d = 0; d < 3; ++d) vt_l[d] = wl[1 + d] - vnl * n[d];
  p2c(wl, ul);
  T el = ul[4] / rhol;
  T rhor = wr[0], vnr = dotT(wr + 1, n), pr = wr[4], ur[5], vt_r[3];
  for (int d = 0; d < 3; ++d) vt_r[d] = wr[1 + d] - vnr * n[d];
  p2c(wr, ur);
  T er = ur[4] / rhor;
  T fl[5], fr[5];
  fl[0] = vnl * ul[0];
  for (int k = 1; k < 4; ++k) fl[k] = vnl * ul[k] + pl * n[k - 1];
  fl[4] = (ul[4] + pl) * vnl;
  fr[0] = vnr * ur[0];
  for (int k = 1; k < 4; ++k) fr[k] = vnr * ur[k] + pr * n[k - 1];
  fr[4] = (ur[4] + pr) * vnr;
  T vn_bar = (lam_l * vnl + lam_r * vnr - (pr - pl)) / (lam_r + lam_l);
  T vn_l_et = vnl - (p_nodal - pl) / lam_l;
  T rhol_et = c1 / (c1 / rhol + (vn_bar - vnl) / lam_l);
  T sle[5], sre[5];
  sle[0] = rhol_et;
  for (int k = 1; k < 4; ++k) sle[k] = rhol_et * (vt_l[k - 1] + vn_l_et * n[k - 1]);
  sle[4] = rhol_et * (el + (pl * vnl - p_nodal * (ph ? vn_l_et : vn_bar)) / lam_l);
  T vn_r_et = vnr + (p_nodal - pr) / lam_r;
  T rhor_et = c1 / (c1 / rhor + (vnr - vn_bar) / lam_r);
  sre[0] = rhor_et;
  for (int k = 1; k < 4; ++k) sre[k] = rhor_et * (vt_r[k - 1] + vn_r_et * n[k - 1]);
  sre[4] = rhor_et * (er + (p_nodal * (ph ? vn_r_et : vn_bar) - pr * vnr) / lam_r);
  const T sl = vnl - lam_l / rhol, sr = vnr + lam_r / rhor;
  for (int k = 0; k < 5; ++k) {
    const T f = ch * (fl[k] + fr[k]) -
                ch * (fabs(sl) * (sle[k] - ul[k]) + fabs(vn_bar) * (sre[k] - sle[k]) + fabs(sr) * (ur[k] - sre[k]));
    lr[0][k] = (double)f;
    lr[1][k] = (double)(-f);
  }
  *sl_o = (double)sl;
  *sr_o = (double)sr;
}

// One subface's share of iteration `iter` of compute_lambdas_and_solve_nodal_pressure
// (ns_euler_rs_module.F90:681-758), FP64: the bounds lam_l, lam_r (updated in place),
// and the terms t1, t2 of s1 and s2 (p_node = s1 / s2). The previous iteration's p_bar
// (read at bc_style 1 walls) is recomputed from the bounds it ended with.
__device__ inline void nodal_pressure_terms(int iter, bool wall1, const double* wl, const double* wr,
                                            const double* n, double area, double p_node, double& lam_l,
                                            double& lam_r, double& t1, double& t2) {
  const double rhol = wl[0], vnl = dotT(wl + 1, n), pl = wl[4], al = sqrt(G * wl[4] / wl[0]);
  const double rhor = wr[0], vnr = dotT(wr + 1, n), pr = wr[4], ar = sqrt(G * wr[4] / wr[0]);
  auto pbar_of = [&](double ll, double lr) { return (lr * pl + ll * pr - lr * ll * (vnr - vnl)) / (lr + ll); };
  if (iter == 1) {
    lam_l = fmax2(fmax2(fmax2(lam_l, al * rhol), sqrt(rhol * fmax2(0.0, pr - pl))), -rhol * (vnr - vnl));
    lam_r = fmax2(fmax2(fmax2(lam_r, ar * rhor), sqrt(rhor * fmax2(0.0, pl - pr))), -rhor * (vnr - vnl));
    const double pb = pbar_of(lam_l, lam_r);
    lam_l = fmax2(lam_l, al * rhol + 1.5 * sqrt(fmax2(0.0, (pb - pl) * rhol)));
    lam_r = fmax2(lam_r, ar * rhor + 1.5 * sqrt(fmax2(0.0, (pb - pr) * rhor)));
  } else {
    const double pq = wall1 ? pbar_of(lam_l, lam_r) : p_node;
    lam_l = fmax2(lam_l, al * rhol + 1.5 * sqrt(fmax2(0.0, (pq - pl) * rhol)));
    lam_r = fmax2(lam_r, ar * rhor + 1.5 * sqrt(fmax2(0.0, (pq - pr) * rhor)));
  }
  const double pb = pbar_of(lam_l, lam_r);
  if (wall1) {
    t1 = (1.0 / lam_r + 1.0 / lam_l) * area * (lam_r * pl + lam_r * lam_l * vnl) / (lam_r + lam_l);
    t2 = (1.0 / lam_l) * area;
  } else {
    t1 = (1.0 / lam_r + 1.0 / lam_l) * area * pb;
    t2 = (1.0 / lam_r + 1.0 / lam_l) * area;
  }
}

// multi_point_iso's flux (ns_euler_module.F90:464-483): the multi-point (or, at an
// excluded boundary vertex, two-wave) flux blended with three_wave by
// warea = min area / area; the wave speeds sl, sr are three_wave's.
template <class T>
__device__ __noinline__ void blend_three_wave(const double* w10, const double* n, double amin, double lr[2][5], double* sl,
                                 double* sr) {
  double lr3[2][5];
  three_wave<T>(w10, w10 + 5, n, lr3, sl, sr, false);
  const double wa = amin / n[3];
  for (int q = 0; q < 2; ++q)
    for (int k = 0; k < 5; ++k) lr[q][k] = wa * lr[q][k] + (1.0 - wa) * lr3[q][k];
}

// The out-of-line fluxes called on private copies of the node kernels' arrays (the
// subface's states, its normal and area, the flux pair and wave speeds), so that those
// arrays keep no escaping address and stay in registers on the multi_point and two_wave
// paths; the called routines see the same values.
struct FluxCopy {
  double w[10], n[4], lr[2][5], sl, sr;
  __device__ void load(const double* w10, const double* n4) {
    for (int k = 0; k < 10; ++k) w[k] = w10[k];
    for (int d = 0; d < 4; ++d) n[d] = n4[d];
  }
  __device__ void store(double o[2][5], double* sl_o, double* sr_o) const {
    for (int q = 0; q < 2; ++q)
      for (int k = 0; k < 5; ++k) o[q][k] = lr[q][k];
    *sl_o = sl;
    *sr_o = sr;
  }
};
template <class T>
__device__ inline void three_wave_c(const double* w10, const double* n4, double lr[2][5], double* sl, double* sr,
                                    bool modified) {
  FluxCopy c;
  c.load(w10, n4);
  three_wave<T>(c.w, c.w + 5, c.n, c.lr, &c.sl, &c.sr, modified);
  c.store(lr, sl, sr);
}
template <class T>
__device__ inline void multi_point_pressure_c(const double* w10, const double* n4, double lr[2][5], double p_nodal,
                                              double lam_l, double lam_r, double* sl, double* sr, bool ph) {
  FluxCopy c;
  c.load(w10, n4);
  multi_point_pressure<T>(c.w, c.w + 5, c.n, c.lr, p_nodal, lam_l, lam_r, &c.sl, &c.sr, ph);
  c.store(lr, sl, sr);
}
template <class T>
__device__ inline void blend_three_wave_c(const double* w10, const double* n4, double amin, double lr[2][5],
                                          double* sl, double* sr) {
  FluxCopy c;
  c.load(w10, n4);
  for (int q = 0; q < 2; ++q)
    for (int k = 0; k < 5; ++k) c.lr[q][k] = lr[q][k];
  c.sl = *sl;
  c.sr = *sr;
  blend_three_wave<T>(c.w, c.n, amin, c.lr, &c.sl, &c.sr);
  c.store(lr, sl, sr);
}

// multi_point (ns_euler_rs_module.F90:200-286); false on a negative star density
template <class T>
__device__ bool multi_point(const double* wl64, const double* wr64, const double* n64, double lr[2][5],
                            double vn_nodal, double lam_l64, double lam_r64, double* sl_o, double* sr_o) {
  T wl[5], wr[5], n[3];
  for (int k = 0; k < 5; ++k) {
    wl[k] = (T)wl64[k];
    wr[k] = (T)wr64[k];
  }
  for (int d = 0; d < 3; ++d) n[d] = (T)n64[d];
  const T lam_l = (T)lam_l64, lam_r = (T)lam_r64;
  T rhol = wl[0], vnl = dotT(wl + 1, n), pl = wl[4], ul[5];
  p2c(wl, ul);
  T el = ul[4] / rhol;
  T rhor = wr[0], vnr = dotT(wr + 1, n), pr = wr[4], ur[5];
  p2c(wr, ur);
  T er = ur[4] / rhor;
  T fl[5], fr[5];
  fl[0] = vnl * ul[0];
  for (int k = 1; k < 4; ++k) fl[k] = vnl * ul[k] + pl * n[k - 1];
  fl[4] = (ul[4] + pl) * vnl;
  fr[0] = vnr * ur[0];
  for (int k = 1; k < 4; ++k) fr[k] = vnr * ur[k] + pr * n[k - 1];
  fr[4] = (ur[4] + pr) * vnr;
  T v_et = (T)vn_nodal;
  T rhol_et = (T)1.0 / ((T)1.0 / rhol + (v_et - vnl) / lam_l);
  T pl_bar = pl - lam_l * (v_et - vnl);
  T sle[5], sre[5];
  sle[0] = rhol_et;
  for (int k = 1; k < 4; ++k) sle[k] = rhol_et * (wl[k] + (v_et - vnl) * n[k - 1]);
  sle[4] = rhol_et * (el + (pl * vnl - pl_bar * v_et) / lam_l);
  T rhor_et = (T)1.0 / ((T)1.0 / rhor + (vnr - v_et) / lam_r);
  T pr_bar = pr + lam_r * (v_et - vnr);
  sre[0] = rhor_et;
  for (int k = 1; k < 4; ++k) sre[k] = rhor_et * (wr[k] + (v_et - vnr) * n[k - 1]);
  sre[4] = rhor_et * (er + (pr_bar * v_et - pr * vnr) / lam_r);
  bool ok = !(rhol_et < (T)0 || rhor_et < (T)0);
  T sl = vnl - lam_l / rhol;
  T sr = vnr + lam_r / rhor;
  // The pressure-jump term 0.5 (p*_r - p*_l) (0, n, v*) in FP64 whatever T is:
  // p*_r - p*_l = (lambda_l + lambda_r)(v* - vbar), so its sum over the node's subfaces
  // is M v* - R, which the FP64 nodal solve closes; with the same normal velocities and
  // pressures as vbar (the T-precision ones) the node's momentum and energy balance
  // then holds to FP64 rounding and the totals stay conserved. For T = double these
  // are the reference's expressions (:264-285) unchanged.
  const double vet64 = vn_nodal;
  const double plb64 = (double)pl - lam_l64 * (vet64 - (double)vnl);
  const double prb64 = (double)pr + lam_r64 * (vet64 - (double)vnr);
  const double e64[5] = {0.0, n64[0], n64[1], n64[2], vet64};
  for (int k = 0; k < 5; ++k) {
    T base = (T)0.5 * (fl[k] + fr[k]) -
             (T)0.5 * (fabs(sl) * (sle[k] - ul[k]) + fabs(v_et) * (sre[k] - sle[k]) + fabs(sr) * (ur[k] - sre[k]));
    const double jump = 0.5 * (prb64 - plb64) * e64[k];
    lr[0][k] = (double)base - jump;
    lr[1][k] = -((double)base + jump);
  }
  *sl_o = (double)sl;
  *sr_o = (double)sr;
  return ok;
}

// The 3x3 solve that ends each iteration of compute_lambdas_and_solve_nodal_velocity
// (ns_euler_rs_module.F90:404-421): bc_style 2 with a wall at the node imposes the wall
// pressure through B_p (pseudo-inverse of M); otherwise M v = R by LU (bc_style 2) or
// the pseudo-inverse (bc_style 0, 1). FP64. mat is overwritten.
__device__ void nodal_solve(const NsParams& P, double mat[3][3], const double* Rp, const double* Bp, double* vnode) {
  if (P.bc_style == 2) {
    double bmax = fmax2(fmax2(fabs(Bp[0]), fabs(Bp[1])), fabs(Bp[2]));
    if (bmax > 1e-8) {
      pinv3(mat);
      double mr[3], mb[3], r2[3];
      for (int d = 0; d < 3; ++d) {
        double s = 0.0, t = 0.0;
        for (int e = 0; e < 3; ++e) {
          s = s + mat[d][e] * Rp[e];
          t = t + mat[d][e] * Bp[e];
        }
        mr[d] = s;
        mb[d] = t;
      }
      double p_bound = dotT(mr, Bp) / dotT(mb, Bp);
      for (int d = 0; d < 3; ++d) r2[d] = Rp[d] - p_bound * Bp[d];
      for (int d = 0; d < 3; ++d) {
        double s = 0.0;
        for (int e = 0; e < 3; ++e) s = s + mat[d][e] * r2[e];
        vnode[d] = s;
      }
      double f = dotT(vnode, Bp) / dotT(Bp, Bp);
      for (int d = 0; d < 3; ++d) vnode[d] = vnode[d] - f * Bp[d];
    } else {
      lu_solve3(mat, vnode, Rp);
    }
  } else {
    pinv3(mat);
    for (int d = 0; d < 3; ++d) {
      double s = 0.0;
      for (int e = 0; e < 3; ++e) s = s + mat[d][e] * Rp[e];
      vnode[d] = s;
    }
  }
}

// compute_rhs_around_vert (ns_euler_module.F90:341-519) for one vertex, one thread per
// vertex; writes the corner sums of the vertex's own subcells to fs (kNsFs doubles per
// subcell). MS bounds the vertex's subfaces and subcells (8, 16 or 32).
// Per subface the thread keeps, in local arrays, only what cannot be re-read: the
// reconstructed left/right states, the sound speeds, the two wave-speed bounds and the
// subface and boundary ids; normals and areas are re-read from the mesh (read-only, so
// no local-memory write-back), and vbar is recomputed from the stored bounds when the
// next iteration needs it. The values are the reference's (the sound speeds of :322-323
// are the same expressions of the same states in every iteration).
constexpr int kNodeThreads = 256;  // the largest block of the node kernel

// vbar = (lambda_l v_l + lambda_r v_r - (p_r - p_l)) / (lambda_r + lambda_l) (:309,316),
// always in FP64 from the normal velocities and pressures the flux itself uses: with
// FP32 wave speeds the node's momentum balance sum A (p*_r - p*_l) n =
// sum A (lambda_l + lambda_r)(v* - vbar) n, which the FP64 solve of M v* = R closes,
// then holds to FP64 rounding (with an FP64 flux), so the totals stay conserved.
__device__ inline double vbar_of(double lam_l, double lam_r, double vnl, double vnr, double pl, double pr) {
  return (lam_l * vnl + lam_r * vnr - (pr - pl)) / (lam_r + lam_l);
}

// compute_lambdas_and_solve_nodal_pressure for one vertex (thread-per-vertex layout):
// ten iterations of p_node = s1 / s2, the bounds kept in L between iterations. Out of
// line, so the other schemes' register allocation does not carry it; it takes the
// subface normals' array and the walls of bc_style 1 (bit j: subface j) by value, since
// a reference to the kernel's mesh or parameter block would make every thread copy it.
template <class T, class L, int MS>
__device__ __noinline__ double nodal_pressure_vertex(const double4* __restrict__ sfn, unsigned wall1, int nsfn,
                                                     const int* sfj, const T (*wlr)[10], L (*lam)[2]) {
  double p_node = 0.0;
  for (int iter = 1; iter <= 10; ++iter) {
    double s1 = 0.0, s2 = 0.0;
    for (int j = 0; j < nsfn; ++j) {
      const double4 sn4 = sfn[sfj[j]];
      const double n[3] = {sn4.x, sn4.y, sn4.z};
      double w10[10];
      for (int k = 0; k < 10; ++k) w10[k] = (double)wlr[j][k];
      double ll = (double)lam[j][0], lr = (double)lam[j][1], t1, t2;
      nodal_pressure_terms(iter, ((wall1 >> j) & 1u) != 0, w10, w10 + 5, n, sn4.w, p_node, ll, lr, t1, t2);
      s1 = s1 + t1;
      s2 = s2 + t2;
      lam[j][0] = (L)ll;
      lam[j][1] = (L)lr;
    }
    p_node = s1 / s2;
  }
  return p_node;
}

// EXT: compiled with the schemes beyond multi_point and two_wave (2, 3, 5, 6, 8); the
// instantiation without them keeps the common path's register allocation.
template <class T, class L, int MS, bool EXT>
__device__ void ns_node_vertex(const DevMesh& m, const NsParams& P, const double* __restrict__ U,
                               const double* __restrict__ grad, double* __restrict__ fs, int so, const int v,
                               const NsScalars* sc) {
  if (v >= m.nv) return;
  const int p0 = m.vsf_off[v], nsfn = m.vsf_off[v + 1] - p0;
  const int q0 = m.vse_off[v], nsen = m.vse_off[v + 1] - q0;
  if (nsfn > MS || nsen > MS) {
    atomicOr(m.status, kErrIndex);
    return;
  }
  // Reconstructed primitive states (left then right) in the compute precision T: the
  // reconstruction already runs in T, so storing T loses nothing.
  T wlr[MS][10];
  L lam[MS][2];  // lambda_l, lambda_r
  int sfj[MS], yj[MS];
  // bit j: subface j is a slip wall (is_wall), looked up once: the kind table is indexed
  // by each subface's own tag, and inside the loops below the lookups would serialise
  unsigned wallm = 0u;
  double amin = 0.0;  // minval of the subface areas (warea of multi_point_iso, ns_euler_module.F90:386-397)
  for (int j = 0; j < nsfn; ++j) {
    const int sf = m.vsf[p0 + j];
    const int2 lr = m.flr[m.sf_face[sf]];
    sfj[j] = sf;
    yj[j] = lr.y;
    if (is_wall(P, lr.y)) wallm |= 1u << j;
    if (EXT && P.scheme == 2) amin = j == 0 ? m.sfn[sf].w : fmin2(amin, m.sfn[sf].w);
    double w10[10];
    reconstruct<T>(m, P, U, grad, v, sf, lr.x, lr.y, so != 0, w10, w10 + 5, sc);
    for (int k = 0; k < 10; ++k) wlr[j][k] = (T)w10[k];
    lam[j][0] = lam[j][1] = (L)0;
  }
  const bool excl = m.is_bound[v] && P.excl;
  const bool iso = EXT && P.scheme == 2;  // multi_point_iso: M and R without the subface areas (:424-553)
  double vn3[3] = {0.0, 0.0, 0.0};
  if (P.scheme == 1 || iso) {
    if (!excl) {  // compute_lambdas_and_solve_nodal_velocity (ns_euler_rs_module.F90:288-422)
      // wave-speed bounds and vbar in L; M, R and the 3x3 solve in FP64
      L snd[MS][2];  // left / right sound speeds
      double Bp[3] = {0.0, 0.0, 0.0};  // wall_normal (ns_euler_primitives_module.F90:162-190)
      for (int j = 0; j < nsfn; ++j) {
        const double4 sn4 = m.sfn[sfj[j]];
        const double n[4] = {sn4.x, sn4.y, sn4.z, sn4.w};
        snd[j][0] = sqrt((L)G * (L)wlr[j][4] / (L)wlr[j][0]);
        snd[j][1] = sqrt((L)G * (L)wlr[j][9] / (L)wlr[j][5]);
        if (((wallm >> j) & 1u) && !(P.b2d && fabs(n[2]) > 1e-12))
          for (int d = 0; d < 3; ++d) Bp[d] = Bp[d] + n[3] * n[d];
      }
      for (int iter = 1; iter <= 4; ++iter) {
        double M6[6] = {0, 0, 0, 0, 0, 0}, Rp[3] = {0, 0, 0};
        for (int j = 0; j < nsfn; ++j) {
          const double4 sn4 = m.sfn[sfj[j]];
          const double n[4] = {sn4.x, sn4.y, sn4.z, sn4.w};
          const double area = n[3];
          const L nt[3] = {(L)n[0], (L)n[1], (L)n[2]};
          L wl[5], wr[5];
          for (int k = 0; k < 5; ++k) {
            wl[k] = (L)wlr[j][k];
            wr[k] = (L)wlr[j][5 + k];
          }
          const L rhol = wl[0], vnl = dotT(wl + 1, nt), pl = wl[4], al = snd[j][0];
          const L rhor = wr[0], vnr = dotT(wr + 1, nt), pr = wr[4], ar = snd[j][1];
          L lam_l = lam[j][0], lam_r = lam[j][1];
          double vbar = 0.0;
          // the flux's own normal velocities and pressures (precision T), for vbar
          const T ntT[3] = {(T)n[0], (T)n[1], (T)n[2]};
          const double vnl_f = (double)dotT(wlr[j] + 1, ntT), vnr_f = (double)dotT(wlr[j] + 6, ntT);
          const double pl_f = (double)wlr[j][4], pr_f = (double)wlr[j][9];
          const bool wall = (wallm >> j) & 1u;
          const L c1 = (L)1, c15 = (L)1.5, c0 = (L)0;
          if (iter == 1) {
            lam_l = tmax2(tmax2(tmax2(lam_l, al * rhol), sqrt(rhol * tmax2(c0, pr - pl))), -rhol * (vnr - vnl));
            lam_r = tmax2(tmax2(tmax2(lam_r, ar * rhor), sqrt(rhor * tmax2(c0, pl - pr))), -rhor * (vnr - vnl));
            vbar = vbar_of((double)lam_l, (double)lam_r, vnl_f, vnr_f, pl_f, pr_f);
            lam_l = tmax2(lam_l, al * rhol * (c1 + c15 * tmax2(c0, -((L)vbar - vnl) / al)));
            lam_r = tmax2(lam_r, ar * rhor * (c1 + c15 * tmax2(c0, ((L)vbar - vnr) / ar)));
          } else if (wall && P.bc_style == 1) {
            // the previous iteration's vbar, from the bounds it ended with
            vbar = vbar_of((double)lam_l, (double)lam_r, vnl_f, vnr_f, pl_f, pr_f);
            lam_l = tmax2(lam_l, al * rhol * (c1 + c15 * tmax2(c0, -((L)vbar - vnl) / al)));
            lam_r = tmax2(lam_r, ar * rhor * (c1 + c15 * tmax2(c0, ((L)vbar - vnr) / ar)));
          } else {
            const L v_et = (L)dotT(vn3, n);
            lam_l = tmax2(lam_l, al * rhol * (c1 + c15 * tmax2(c0, -(v_et - vnl) / al)));
            lam_r = tmax2(lam_r, ar * rhor * (c1 + c15 * tmax2(c0, (v_et - vnr) / ar)));
          }
          vbar = vbar_of((double)lam_l, (double)lam_r, vnl_f, vnr_f, pl_f, pr_f);
          lam[j][0] = lam_l;
          lam[j][1] = lam_r;
          const double lsum = (double)lam_r + (double)lam_l;
          if (!wall || P.bc_style == 0 || P.bc_style == 2) {  // M += (lam_r + lam_l) A n n^T
            const double w = iso ? lsum : lsum * area;
            M6[0] = M6[0] + w * (n[0] * n[0]);
            M6[1] = M6[1] + w * (n[0] * n[1]);
            M6[2] = M6[2] + w * (n[0] * n[2]);
            M6[3] = M6[3] + w * (n[1] * n[1]);
            M6[4] = M6[4] + w * (n[1] * n[2]);
            M6[5] = M6[5] + w * (n[2] * n[2]);
          }
          if (!wall || P.bc_style == 0) {
            const double q = iso ? lsum * vbar : area * lsum * vbar;
            for (int d = 0; d < 3; ++d) Rp[d] = Rp[d] + q * n[d];
          } else if (P.bc_style == 2 && (!P.b2d || fabs(n[2]) < 1e-8)) {
            const double q = iso ? (double)pl : area * (double)pl;
            for (int d = 0; d < 3; ++d) Rp[d] = Rp[d] + q * n[d];
          }
        }
        // M is symmetric entry by entry: n_d n_e and n_e n_d are the same product
        double mat[3][3] = {{M6[0], M6[1], M6[2]}, {M6[1], M6[3], M6[4]}, {M6[2], M6[4], M6[5]}};
        nodal_solve(P, mat, Rp, Bp, vn3);
      }
    }
    m.vp[v] = make_double4(vn3[0], vn3[1], vn3[2], 0.0);
  }
  const double p_node =
      (EXT && (P.scheme == 6 || P.scheme == 8))
          ? nodal_pressure_vertex<T, L, MS>(m.sfn, P.bc_style == 1 ? wallm : 0u, nsfn, sfj, wlr, lam)
          : 0.0;
  double fsv[MS][6];  // five flux sums and the wave-speed sum per subcell
  for (int j = 0; j < nsen; ++j)
    for (int k = 0; k < 6; ++k) fsv[j][k] = 0.0;
  bool bad = false;
  for (int j = 0; j < nsfn; ++j) {
    const int sf = sfj[j];
    const int2 se = m.sf_se[sf];
    const int lse_loc = m.se_loc[se.x];
    const double4 sn4 = m.sfn[sf];
    const double n[4] = {sn4.x, sn4.y, sn4.z, sn4.w};
    double w10[10];
    for (int k = 0; k < 10; ++k) w10[k] = (double)wlr[j][k];
    double lr[2][5], sl, sr;
    if ((P.scheme == 1 || iso) && !excl) {
      const double vn = ((wallm >> j) & 1u) ? 0.0 : dotT(vn3, n);
      if (!multi_point<T>(w10, w10 + 5, n, lr, vn, (double)lam[j][0], (double)lam[j][1], &sl, &sr)) bad = true;
    } else if (EXT && (P.scheme == 3 || P.scheme == 5)) {
      three_wave_c<T>(w10, n, lr, &sl, &sr, P.scheme == 5);
    } else if (EXT && (P.scheme == 6 || P.scheme == 8)) {
      multi_point_pressure_c<T>(w10, n, lr, p_node, (double)lam[j][0], (double)lam[j][1], &sl, &sr, P.scheme == 8);
    } else {
      two_wave<T>(w10, w10 + 5, n, lr, &sl, &sr);
    }
    if (iso) blend_three_wave_c<T>(w10, n, amin, lr, &sl, &sr);
    if (m.se_vert[se.x] == v && lse_loc < nsen) {
      const double area = n[3];
      fsv[lse_loc][5] = fsv[lse_loc][5] + area * fmax2(0.0, -sl);
      for (int k = 0; k < 5; ++k) fsv[lse_loc][k] = fsv[lse_loc][k] + area * lr[0][k];
      if (se.y >= 0 && m.se_vert[se.y] == v) {
        const int rse_loc = m.se_loc[se.y];
        if (rse_loc < nsen) {
          fsv[rse_loc][5] = fsv[rse_loc][5] + area * fmax2(0.0, sr);
          for (int k = 0; k < 5; ++k) fsv[rse_loc][k] = fsv[rse_loc][k] + area * lr[1][k];
        }
      }
    }
  }
  if (bad) atomicOr(m.status, kErrNegDensity);
  for (int j = 0; j < nsen; ++j) {
    const int s = m.vse[q0 + j];
    if (m.se_vert[s] != v) continue;  // a periodic image's subcell: its sums are zero here
    double* out = fs + kNsFs * (size_t)s;
    for (int k = 0; k < 6; ++k) out[k] = fsv[j][k];
  }
}

// The same computation with a group of NG lanes per vertex (warp-per-node segmented
// reductions over the vertex-to-subface CSR): lane j owns subface j and subcell j of the
// vertex and keeps its subface's states in registers. The per-vertex sums (B_p, M, R)
// and the subcell sums are formed in shared memory by one lane per component, adding the
// subfaces' terms in subface order exactly as the thread-per-vertex kernel does, so the
// results are bit-identical to it; every lane of the group then runs the same 3x3 solve
// on the same sums. NG is 8, 16 or 32; a block of kNodeGroupThreads lanes holds
// kNodeGroupThreads / NG vertices.
constexpr int kNodeGroupThreads = 256;
constexpr int kNodeGroupMinBlocks = 2;
constexpr int kLaneVals = 12;  // per-lane scratch doubles: 9 solver terms or 12 subcell terms

template <int NG>
__device__ inline unsigned group_mask() {
  if constexpr (NG == 32) return 0xffffffffu;
  else return ((1u << NG) - 1u) << ((threadIdx.x & 31) & ~(NG - 1));
}

// sum over the group's lanes 0..n-1 of lane k's term c at slot `comp` (slots of width
// kLaneVals), adding in lane order only the terms whose lane set bit `comp` of its flag
template <int NG>
__device__ inline double group_ordered_sum(const double* __restrict__ gv, const unsigned* __restrict__ gf, int n,
                                           int comp) {
  double s = 0.0;
  for (int k = 0; k < NG; ++k)
    if (k < n && ((gf[k] >> comp) & 1u)) s = s + gv[k * kLaneVals + comp];
  return s;
}

template <class T, class L, int NG>
__device__ void ns_node_group(const DevMesh& m, const NsParams& P, const double* __restrict__ U,
                              const double* __restrict__ grad, double* __restrict__ fs, int so, const int v,
                              const bool live, double* __restrict__ gv, unsigned* __restrict__ gf,
                              double* __restrict__ gs, const NsScalars* sc) {
  const int j = threadIdx.x & (NG - 1);
  const unsigned mask = group_mask<NG>();
  int p0 = 0, nsfn = 0, q0 = 0, nsen = 0;
  bool act = live && v < m.nv;
  if (act) {
    p0 = m.vsf_off[v];
    nsfn = m.vsf_off[v + 1] - p0;
    q0 = m.vse_off[v];
    nsen = m.vse_off[v + 1] - q0;
    if (nsfn > NG || nsen > NG) {
      if (j == 0) atomicOr(m.status, kErrIndex);
      act = false;
    }
  }
  const bool mine = act && j < nsfn;  // this lane owns a subface
  T w[10];
  double n[4] = {0.0, 0.0, 0.0, 0.0};
  int sf = 0, y = 0;
  for (int k = 0; k < 10; ++k) w[k] = (T)0;
  if (mine) {
    sf = m.vsf[p0 + j];
    const int2 lr = m.flr[m.sf_face[sf]];
    y = lr.y;
    double w10[10];
    reconstruct<T>(m, P, U, grad, v, sf, lr.x, lr.y, so != 0, w10, w10 + 5, sc);
    for (int k = 0; k < 10; ++k) w[k] = (T)w10[k];
    const double4 sn = m.sfn[sf];
    n[0] = sn.x;
    n[1] = sn.y;
    n[2] = sn.z;
    n[3] = sn.w;
  }
  const bool excl = act && m.is_bound[v] && P.excl;
  double vn3[3] = {0.0, 0.0, 0.0};
  L lam_l = (L)0, lam_r = (L)0;
  const bool iso = P.scheme == 2;
  const bool solve = (P.scheme == 1 || iso) && act && !excl;
  double amin = 0.0;  // minval of the group's subface areas (exact in any order)
  if (iso) {
    amin = mine ? n[3] : (double)INFINITY;
    for (int o = NG / 2; o > 0; o >>= 1) amin = fmin2(amin, __shfl_xor_sync(mask, amin, o, NG));
  }
  if (P.scheme == 1 || iso) {  // uniform over the launch: every lane takes the same syncs
    L al = (L)0, ar = (L)0;
    if (mine) {
      al = sqrt((L)G * (L)w[4] / (L)w[0]);
      ar = sqrt((L)G * (L)w[9] / (L)w[5]);
    }
    // wall_normal: lane terms area * n
    {
      unsigned f = 0u;
      if (mine && y < 0 && !(P.b2d && fabs(n[2]) > 1e-12) && (y == -1 || P.bc_type[-(y + 1) - 1] == 1)) f = 7u;
      for (int d = 0; d < 3; ++d) gv[j * kLaneVals + d] = n[3] * n[d];
      gf[j] = f;
    }
    __syncwarp(mask);
    if (j < 3) gs[j] = group_ordered_sum<NG>(gv, gf, nsfn, j);
    __syncwarp(mask);
    const double Bp[3] = {gs[0], gs[1], gs[2]};
    __syncwarp(mask);
    const T ntT[3] = {(T)n[0], (T)n[1], (T)n[2]};
    const double vnl_f = (double)dotT(w + 1, ntT), vnr_f = (double)dotT(w + 6, ntT);
    const double pl_f = (double)w[4], pr_f = (double)w[9];
    const bool wall = is_wall(P, y);
    double vbar = 0.0;
    for (int iter = 1; iter <= 4; ++iter) {
      unsigned f = 0u;
      if (mine && solve) {
        const double area = n[3];
        const L nt[3] = {(L)n[0], (L)n[1], (L)n[2]};
        L wl[5], wr[5];
        for (int k = 0; k < 5; ++k) {
          wl[k] = (L)w[k];
          wr[k] = (L)w[5 + k];
        }
        const L rhol = wl[0], vnl = dotT(wl + 1, nt), pl = wl[4];
        const L rhor = wr[0], vnr = dotT(wr + 1, nt), pr = wr[4];
        const L c1 = (L)1, c15 = (L)1.5, c0 = (L)0;
        if (iter == 1) {
          lam_l = tmax2(tmax2(tmax2(lam_l, al * rhol), sqrt(rhol * tmax2(c0, pr - pl))), -rhol * (vnr - vnl));
          lam_r = tmax2(tmax2(tmax2(lam_r, ar * rhor), sqrt(rhor * tmax2(c0, pl - pr))), -rhor * (vnr - vnl));
          vbar = vbar_of((double)lam_l, (double)lam_r, vnl_f, vnr_f, pl_f, pr_f);
          lam_l = tmax2(lam_l, al * rhol * (c1 + c15 * tmax2(c0, -((L)vbar - vnl) / al)));
          lam_r = tmax2(lam_r, ar * rhor * (c1 + c15 * tmax2(c0, ((L)vbar - vnr) / ar)));
        } else if (wall && P.bc_style == 1) {
          lam_l = tmax2(lam_l, al * rhol * (c1 + c15 * tmax2(c0, -((L)vbar - vnl) / al)));
          lam_r = tmax2(lam_r, ar * rhor * (c1 + c15 * tmax2(c0, ((L)vbar - vnr) / ar)));
        } else {
          const L v_et = (L)dotT(vn3, n);
          lam_l = tmax2(lam_l, al * rhol * (c1 + c15 * tmax2(c0, -(v_et - vnl) / al)));
          lam_r = tmax2(lam_r, ar * rhor * (c1 + c15 * tmax2(c0, (v_et - vnr) / ar)));
        }
        vbar = vbar_of((double)lam_l, (double)lam_r, vnl_f, vnr_f, pl_f, pr_f);
        const double lsum = (double)lam_r + (double)lam_l;
        double* c = gv + j * kLaneVals;
        if (!wall || P.bc_style == 0 || P.bc_style == 2) {
          const double wgt = iso ? lsum : lsum * area;
          c[0] = wgt * (n[0] * n[0]);
          c[1] = wgt * (n[0] * n[1]);
          c[2] = wgt * (n[0] * n[2]);
          c[3] = wgt * (n[1] * n[1]);
          c[4] = wgt * (n[1] * n[2]);
          c[5] = wgt * (n[2] * n[2]);
          f |= 0x3fu;
        }
        if (!wall || P.bc_style == 0) {
          const double q = iso ? lsum * vbar : area * lsum * vbar;
          for (int d = 0; d < 3; ++d) c[6 + d] = q * n[d];
          f |= 0x1c0u;
        } else if (P.bc_style == 2 && (!P.b2d || fabs(n[2]) < 1e-8)) {
          const double q = iso ? (double)pl : area * (double)pl;
          for (int d = 0; d < 3; ++d) c[6 + d] = q * n[d];
          f |= 0x1c0u;
        }
      }
      gf[j] = f;
      __syncwarp(mask);
      for (int comp = j; comp < 9; comp += NG) gs[comp] = group_ordered_sum<NG>(gv, gf, nsfn, comp);
      __syncwarp(mask);
      if (solve) {
        double mat[3][3] = {{gs[0], gs[1], gs[2]}, {gs[1], gs[3], gs[4]}, {gs[2], gs[4], gs[5]}};
        const double Rp[3] = {gs[6], gs[7], gs[8]};
        nodal_solve(P, mat, Rp, Bp, vn3);
      }
      __syncwarp(mask);
    }
    if (act && j == 0) m.vp[v] = make_double4(vn3[0], vn3[1], vn3[2], 0.0);
  }
  const bool pres = P.scheme == 6 || P.scheme == 8;
  double p_node = 0.0;
  if (pres) {  // nodal pressure: s1 and s2 summed in subface order by lanes 0 and 1
    for (int iter = 1; iter <= 10; ++iter) {
      unsigned f = 0u;
      if (mine) {
        double w10[10];
        for (int k = 0; k < 10; ++k) w10[k] = (double)w[k];
        double ll = (double)lam_l, lr = (double)lam_r;
        nodal_pressure_terms(iter, P.bc_style == 1 && is_wall(P, y), w10, w10 + 5, n, n[3], p_node, ll, lr,
                             gv[j * kLaneVals], gv[j * kLaneVals + 1]);
        lam_l = (L)ll;
        lam_r = (L)lr;
        f = 3u;
      }
      gf[j] = f;
      __syncwarp(mask);
      if (j < 2) gs[j] = group_ordered_sum<NG>(gv, gf, nsfn, j);
      __syncwarp(mask);
      p_node = gs[0] / gs[1];
      __syncwarp(mask);
    }
  }
  // subface fluxes; lane j's terms to its left / right subcell of this vertex
  int lse = -1, rse = -1;
  unsigned f = 0u;
  if (mine) {
    const int2 se = m.sf_se[sf];
    const int lse_loc = m.se_loc[se.x];
    double w10[10];
    for (int k = 0; k < 10; ++k) w10[k] = (double)w[k];
    double lr[2][5], sl, sr;
    if (solve) {
      const double vn = is_wall(P, y) ? 0.0 : dotT(vn3, n);
      if (!multi_point<T>(w10, w10 + 5, n, lr, vn, (double)lam_l, (double)lam_r, &sl, &sr))
        atomicOr(m.status, kErrNegDensity);
    } else if (P.scheme == 3 || P.scheme == 5) {
      three_wave_c<T>(w10, n, lr, &sl, &sr, P.scheme == 5);
    } else if (P.scheme == 6 || P.scheme == 8) {
      multi_point_pressure_c<T>(w10, n, lr, p_node, (double)lam_l, (double)lam_r, &sl, &sr, P.scheme == 8);
    } else {
      two_wave<T>(w10, w10 + 5, n, lr, &sl, &sr);
    }
    if (iso) blend_three_wave_c<T>(w10, n, amin, lr, &sl, &sr);
    if (m.se_vert[se.x] == v && lse_loc < nsen) {
      const double area = n[3];
      double* c = gv + j * kLaneVals;
      lse = lse_loc;
      for (int k = 0; k < 5; ++k) c[k] = area * lr[0][k];
      c[5] = area * fmax2(0.0, -sl);
      if (se.y >= 0 && m.se_vert[se.y] == v) {
        const int rse_loc = m.se_loc[se.y];
        if (rse_loc < nsen) {
          rse = rse_loc;
          for (int k = 0; k < 5; ++k) c[6 + k] = area * lr[1][k];
          c[11] = area * fmax2(0.0, sr);
        }
      }
    }
  }
  // flag word: left subcell + 1 in bits 0-7, right subcell + 1 in bits 8-15
  f = (unsigned)(lse + 1) | ((unsigned)(rse + 1) << 8);
  gf[j] = f;
  __syncwarp(mask);
  if (act && j < nsen) {
    double acc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    for (int k = 0; k < NG; ++k) {
      if (k >= nsfn) continue;
      const unsigned fk = gf[k];
      const double* c = gv + k * kLaneVals;
      if ((int)(fk & 0xffu) == j + 1) {
        acc[5] = acc[5] + c[5];
        for (int q = 0; q < 5; ++q) acc[q] = acc[q] + c[q];
      }
      if ((int)((fk >> 8) & 0xffu) == j + 1) {
        acc[5] = acc[5] + c[11];
        for (int q = 0; q < 5; ++q) acc[q] = acc[q] + c[6 + q];
      }
    }
    const int s_id = m.vse[q0 + j];
    if (m.se_vert[s_id] == v) {  // a periodic image's subcell: its sums are zero here
      double* out = fs + kNsFs * (size_t)s_id;
      for (int k = 0; k < 6; ++k) out[k] = acc[k];
    }
  }
  __syncwarp(mask);
}

// shared scratch of the group kernels: kLaneVals doubles and a flag per lane, 12 doubles
// per group for the sums
struct NodeGroupSmem {
  double v[kNodeGroupThreads * kLaneVals];
  unsigned f[kNodeGroupThreads];
  double s[kNodeGroupThreads / 8][12];
};

template <class T, class L, int NG>
__global__ void __launch_bounds__(kNodeGroupThreads, kNodeGroupMinBlocks) k_ns_node_group(DevMesh m, NsParams P,
                                                                     const double* __restrict__ U,
                                                                     const double* __restrict__ grad,
                                                                     double* __restrict__ fs, int so,
                                                                     const NsScalars* sc) {
  if (sc && sc->done) return;
  __shared__ NodeGroupSmem sm;
  const int g = threadIdx.x / NG;
  const int v = vert_at(m, blockIdx.x * (kNodeGroupThreads / NG) + g);
  ns_node_group<T, L, NG>(m, P, U, grad, fs, so, v, true, sm.v + g * NG * kLaneVals, sm.f + g * NG, sm.s[g], sc);
}

template <class T, class L, int MS, bool EXT>
__global__ void __launch_bounds__(kNodeThreads) k_ns_node(DevMesh m, NsParams P, const double* __restrict__ U,
                                                          const double* __restrict__ grad, double* __restrict__ fs,
                                                          int so, const NsScalars* sc) {
  if (sc && sc->done) return;
  ns_node_vertex<T, L, MS, EXT>(m, P, U, grad, fs, so, vert_at(m, blockIdx.x * blockDim.x + threadIdx.x), sc);
}

__device__ inline double warp_min(double x) {
  for (int o = 16; o > 0; o >>= 1) x = fmin(x, __shfl_xor_sync(0xffffffffu, x, o));
  return x;
}
__device__ inline double warp_sum_tree(double x) {
  for (int o = 16; o > 0; o >>= 1) x = x + __shfl_down_sync(0xffffffffu, x, o);
  return x;
}

// compute_euler_flux scatter (:320-336) as a gather: rhs = 0 - corners in ascending
// vertex order; sum_lambda = 1e-12 + corners. Block min of V / sum_lambda into *dtred.
// called by every thread of a 128-thread block (block reduction inside)
__device__ void ns_gather_body(const DevMesh& m, const double* __restrict__ fs, double* __restrict__ rhs,
                               NsScalars* sc, int reduce, const int c) {
  if (sc && sc->done) return;
  double dmin = 1e10;
  if (c < m.ne) {
    double r[5] = {0.0, 0.0, 0.0, 0.0, 0.0}, sl = 1e-12;
    // the corner records of four subcells at a time loaded before their sums, which run
    // in the list's order
    constexpr int kAhead = 4;
    const int q1 = m.ev_off[c + 1];
    for (int q0 = m.ev_off[c]; q0 < q1; q0 += kAhead) {
      int id[kAhead];
#pragma unroll
      for (int i = 0; i < kAhead; ++i) id[i] = q0 + i < q1 ? m.cse_sorted[q0 + i] : 0;
      double f[kAhead][6];
#pragma unroll
      for (int i = 0; i < kAhead; ++i)
        if (q0 + i < q1)
#pragma unroll
          for (int k = 0; k < 6; ++k) f[i][k] = fs[kNsFs * (size_t)id[i] + k];
#pragma unroll
      for (int i = 0; i < kAhead; ++i)
        if (q0 + i < q1) {
#pragma unroll
          for (int k = 0; k < 5; ++k) r[k] = r[k] - f[i][k];
          sl = sl + f[i][5];
        }
    }
    double* o = rhs + kRhs * (size_t)c;
    for (int k = 0; k < 5; ++k) o[k] = r[k];
    o[5] = sl;
    dmin = m.vol[c] / sl;
  }
  if (reduce) {
    __shared__ double wm[4];
    double x = warp_min(dmin);
    if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = x;
    __syncthreads();
    if (threadIdx.x == 0) {
      x = fmin(fmin(wm[0], wm[1]), fmin(wm[2], wm[3]));
      atomic_min_pos(&sc->dtred, x);
    }
  }
}

__global__ void __launch_bounds__(128) k_ns_gather(DevMesh m, const double* __restrict__ fs, double* __restrict__ rhs,
                                                   NsScalars* sc, int reduce) {
  ns_gather_body(m, fs, rhs, sc, reduce, blockIdx.x * blockDim.x + threadIdx.x);
}

// The matrix of compute_nodal_grad (ns_euler_recon_module.F90:453-490) at vertex v,
// sum over its interior subfaces of A n (x_r - x_l)^T in subface order: it depends on
// the geometry alone.
__device__ inline void nodal_grad_matrix(const DevMesh& m, const int v, double mat[3][3]) {
  for (int d = 0; d < 3; ++d)
    for (int e = 0; e < 3; ++e) mat[d][e] = 0.0;
  for (int p = m.vsf_off[v]; p < m.vsf_off[v + 1]; ++p) {
    const int sf = m.vsf[p];
    const int2 lr = m.flr[m.sf_face[sf]];
    if (lr.y < 0) continue;
    const double4 sn = m.sfn[sf];
    const double n[3] = {sn.x, sn.y, sn.z};
    const double4 cl = m.cc[lr.x], cr = m.cc[lr.y];
    const double dxc[3] = {cr.x - cl.x, cr.y - cl.y, cr.z - cl.z};
    for (int d = 0; d < 3; ++d)
      for (int e = 0; e < 3; ++e) mat[d][e] = mat[d][e] + sn.w * (n[d] * dxc[e]);
  }
}

// The pseudo-inverse of every vertex's matrix, npinv[9 v + 3 d + e], for a mesh whose
// geometry stays put between the steps that read it: the same sums and the same pinv3
// as the per-step kernels, so a gradient formed from it has their bits.
__global__ void __launch_bounds__(128) k_ns_nodal_pinv(DevMesh m, double* __restrict__ npinv) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= m.nv) return;
  double mat[3][3];
  nodal_grad_matrix(m, v, mat);
  pinv3(mat);
  for (int d = 0; d < 3; ++d)
    for (int e = 0; e < 3; ++e) npinv[9 * (size_t)v + 3 * d + e] = mat[d][e];
}

// compute_nodal_grad (ns_euler_recon_module.F90:453-490); ng[15] = g[5*d + var]. CACHED:
// the pseudo-inverse comes from m.npinv (k_ns_nodal_pinv) instead of being formed here.
template <bool CACHED>
__device__ void ns_nodal_grad_body(const DevMesh& m, const double* __restrict__ U, double* __restrict__ ngrad,
                                   const NsScalars* sc, const int v) {
  if (sc && sc->done) return;
  if (v >= m.nv) return;
  double g[3][5] = {{0, 0, 0, 0, 0}, {0, 0, 0, 0, 0}, {0, 0, 0, 0, 0}};
  double mat[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  for (int p = m.vsf_off[v]; p < m.vsf_off[v + 1]; ++p) {
    const int sf = m.vsf[p];
    const int2 lr = m.flr[m.sf_face[sf]];
    if (lr.y < 0) continue;
    double ul[5], ur[5], wl[5], wr[5];
    ld5(U, lr.x, ul);
    ld5(U, lr.y, ur);
    c2p(ul, wl);
    c2p(ur, wr);
    const double4 sn = m.sfn[sf];
    const double n[3] = {sn.x, sn.y, sn.z};
    for (int d = 0; d < 3; ++d)
      for (int k = 0; k < 5; ++k) g[d][k] = g[d][k] + sn.w * (n[d] * (wr[k] - wl[k]));
    if (!CACHED) {
      const double4 cl = m.cc[lr.x], cr = m.cc[lr.y];
      const double dxc[3] = {cr.x - cl.x, cr.y - cl.y, cr.z - cl.z};
      for (int d = 0; d < 3; ++d)
        for (int e = 0; e < 3; ++e) mat[d][e] = mat[d][e] + sn.w * (n[d] * dxc[e]);
    }
  }
  if (CACHED) {
    for (int d = 0; d < 3; ++d)
      for (int e = 0; e < 3; ++e) mat[d][e] = m.npinv[9 * (size_t)v + 3 * d + e];
  } else {
    pinv3(mat);
  }
  const bool bnd = m.is_bound[v] != 0;
  double* o = ngrad + 15 * (size_t)v;
  for (int d = 0; d < 3; ++d)
    for (int k = 0; k < 5; ++k) {
      double s = 0.0;
      for (int e = 0; e < 3; ++e) s = s + mat[d][e] * g[e][k];
      o[5 * d + k] = bnd ? 0.0 : s;
    }
}

template <bool CACHED>
__global__ void __launch_bounds__(128) k_ns_nodal_grad(DevMesh m, const double* __restrict__ U,
                                                       double* __restrict__ ngrad, const NsScalars* sc) {
  ns_nodal_grad_body<CACHED>(m, U, ngrad, sc, vert_at(m, blockIdx.x * blockDim.x + threadIdx.x));
}

// The same nodal gradient with a group of NG lanes per vertex, lane p holding the
// vertex's p-th subface (both cells' primitives, the 15 gradient and 9 matrix terms): the
// sums run in subface order by shuffles, each lane forming the same totals and the same
// pseudo-inverse, and the lanes share the stores. Every lane of the warp reaches every
// shuffle. CACHED: the pseudo-inverse comes from m.npinv and no matrix terms are formed.
template <int NG, bool CACHED>
__device__ void ns_nodal_grad_group(const DevMesh& m, const double* __restrict__ U, double* __restrict__ ngrad,
                                    const NsScalars* sc, const int t, const int lane) {
  if (sc && sc->done) return;
  constexpr unsigned kAll = 0xffffffffu;
  const bool live = t < m.nv;
  const int v = vert_at(m, t);
  const int pb = live ? m.vsf_off[v] : 0, np = live ? m.vsf_off[v + 1] - pb : 0;
  const int nmax = __reduce_max_sync(kAll, np);
  double tg[15], tm[9];
  for (int i = 0; i < 15; ++i) tg[i] = 0.0;
  for (int i = 0; i < 9; ++i) tm[i] = 0.0;
  int in = 0;
  if (lane < np) {
    const int sf = m.vsf[pb + lane];
    const int2 lr = m.flr[m.sf_face[sf]];
    if (lr.y >= 0) {
      in = 1;
      double ul[5], ur[5], wl[5], wr[5];
      ld5(U, lr.x, ul);
      ld5(U, lr.y, ur);
      c2p(ul, wl);
      c2p(ur, wr);
      const double4 sn = m.sfn[sf];
      const double n[3] = {sn.x, sn.y, sn.z};
      for (int d = 0; d < 3; ++d)
        for (int k = 0; k < 5; ++k) tg[5 * d + k] = sn.w * (n[d] * (wr[k] - wl[k]));
      if (!CACHED) {
        const double4 cl = m.cc[lr.x], cr = m.cc[lr.y];
        const double dxc[3] = {cr.x - cl.x, cr.y - cl.y, cr.z - cl.z};
        for (int d = 0; d < 3; ++d)
          for (int e = 0; e < 3; ++e) tm[3 * d + e] = sn.w * (n[d] * dxc[e]);
      }
    }
  }
  double g[3][5] = {{0, 0, 0, 0, 0}, {0, 0, 0, 0, 0}, {0, 0, 0, 0, 0}};
  double mat[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  for (int j = 0; j < nmax; ++j) {
    const bool add = __shfl_sync(kAll, in, j, NG) != 0;
#pragma unroll
    for (int i = 0; i < 15; ++i) {
      const double x = __shfl_sync(kAll, tg[i], j, NG);
      if (add) g[i / 5][i % 5] = g[i / 5][i % 5] + x;
    }
    if (!CACHED)
#pragma unroll
      for (int i = 0; i < 9; ++i) {
        const double x = __shfl_sync(kAll, tm[i], j, NG);
        if (add) mat[i / 3][i % 3] = mat[i / 3][i % 3] + x;
      }
  }
  if (!live) return;
  if (CACHED) {
    for (int d = 0; d < 3; ++d)
      for (int e = 0; e < 3; ++e) mat[d][e] = m.npinv[9 * (size_t)v + 3 * d + e];
  } else {
    pinv3(mat);
  }
  const bool bnd = m.is_bound[v] != 0;
  double* o = ngrad + 15 * (size_t)v;
#pragma unroll
  for (int d = 0; d < 3; ++d)
#pragma unroll
    for (int k = 0; k < 5; ++k)
      if ((5 * d + k) % NG == lane) {
        double s = 0.0;
        for (int e = 0; e < 3; ++e) s = s + mat[d][e] * g[e][k];
        o[5 * d + k] = bnd ? 0.0 : s;
      }
}

template <int NG, bool CACHED>
__global__ void __launch_bounds__(128) k_ns_nodal_grad_group(DevMesh m, const double* __restrict__ U,
                                                             double* __restrict__ ngrad, const NsScalars* sc) {
  ns_nodal_grad_group<NG, CACHED>(m, U, ngrad, sc, blockIdx.x * (128 / NG) + threadIdx.x / NG,
                                  threadIdx.x % NG);
}

// compute_cell_grad_method_2..6 (:166-320) + physical_slope_limiter + relaxed_maximum_principle
template <class T>
__device__ void ns_cell_grad_body(const DevMesh& m, const NsParams& P, const double* __restrict__ U,
                                  const double* __restrict__ ngrad, double* __restrict__ grad, const NsScalars* sc,
                                  const int c) {
  if (sc && sc->done) return;
  if (c >= m.ne) return;
  double* go = grad + 15 * (size_t)c;
  if (P.method == 0 || P.method == 1) {
    for (int i = 0; i < 15; ++i) go[i] = 0.0;
    return;
  }
  const T eps = (T)1e-3, tol = (T)1e-8;
  T g[15];
  T ws[5] = {0, 0, 0, 0, 0};
  for (int i = 0; i < 15; ++i) g[i] = 0;
  const int vb = m.ev_off[c], nvc = m.ev_off[c + 1] - vb;
  if (P.method == 2) {  // dual-volume average
    T dvs = 0;
    for (int j = 0; j < nvc; ++j) {
      const int v = m.ev[vb + j];
      const double* ng = ngrad + 15 * (size_t)v;
      const T vol = (T)m.vol_v[v];
      for (int i = 0; i < 15; ++i) g[i] = g[i] + vol * (T)ng[i];
      dvs = dvs + vol;
    }
    for (int i = 0; i < 15; ++i) g[i] = g[i] / dvs;
  } else if (P.method == 3) {  // the vertex gradient of smallest norm, per variable
    const double* ng1 = ngrad + 15 * (size_t)m.ev[vb];
    for (int i = 0; i < 15; ++i) g[i] = (T)ng1[i];
    for (int j = 1; j < nvc; ++j) {
      const double* ng = ngrad + 15 * (size_t)m.ev[vb + j];
      for (int k = 0; k < 5; ++k)
        if (oi3<T>((T)ng[k], (T)ng[5 + k], (T)ng[10 + k]) < oi3<T>(g[k], g[5 + k], g[10 + k]))
          for (int d = 0; d < 3; ++d) g[5 * d + k] = (T)ng[5 * d + k];
    }
  } else {  // 4: V / (eps + |g|); 5, 6: V / (eps + |g|)^2 (6 adds the central average)
    T cg[15], cws = 0;
    for (int i = 0; i < 15; ++i) cg[i] = 0;
    for (int j = 0; j < nvc; ++j) {
      const int v = m.ev[vb + j];
      const double* ng = ngrad + 15 * (size_t)v;
      const T vol = (T)m.vol_v[v];
      for (int k = 0; k < 5; ++k) {
        const T q = eps + oi3<T>((T)ng[k], (T)ng[5 + k], (T)ng[10 + k]);
        const T w = P.method == 4 ? vol / q : vol / (q * q);
        for (int d = 0; d < 3; ++d) g[5 * d + k] = g[5 * d + k] + w * (T)ng[5 * d + k];
        ws[k] = ws[k] + w;
      }
      if (P.method == 6) {
        for (int i = 0; i < 15; ++i) cg[i] = cg[i] + vol * (T)ng[i];
        cws = cws + vol;
      }
    }
    if (P.method == 6) {  // OI of the (3, 5) central gradient: the norm of its first column
      for (int i = 0; i < 15; ++i) cg[i] = cg[i] / cws;
      const T q = eps + oi3<T>(cg[0], cg[5], cg[10]);
      const T wc = cws / (q * q);
      for (int i = 0; i < 15; ++i) g[i] = g[i] + wc * cg[i];
      for (int k = 0; k < 5; ++k) ws[k] = ws[k] + wc;
    }
    for (int k = 0; k < 5; ++k)
      for (int d = 0; d < 3; ++d) g[5 * d + k] = g[5 * d + k] / ws[k];
  }
  double u0[5];
  ld5(U, c, u0);
  T uu[5], w0[5];
  for (int k = 0; k < 5; ++k) uu[k] = (T)u0[k];
  c2p(uu, w0);
  const double4 ce = m.cc[c];
  T omega = 1;
  for (int j = 0; j < nvc; ++j) {  // physical_slope_limiter
    const double4 xv = m.x[m.ev[vb + j]];
    const T dx[3] = {(T)(xv.x - ce.x), (T)(xv.y - ce.y), (T)(xv.z - ce.z)};
    T dw0 = 0, dw4 = 0;
    for (int d = 0; d < 3; ++d) dw0 = dw0 + g[5 * d] * dx[d];
    for (int d = 0; d < 3; ++d) dw4 = dw4 + g[5 * d + 4] * dx[d];
    if (dw0 < (T)0) omega = tmin2(omega, tmax2((T)0, w0[0] / (tol - dw0)));
    if (dw4 < (T)0) omega = tmin2(omega, tmax2((T)0, w0[4] / (tol - dw4)));
  }
  for (int i = 0; i < 15; ++i) g[i] = omega * g[i];
  T rmin = (T)1e100, rmax = 0, pmin = (T)1e100, pmax = 0;  // relaxed_maximum_principle
  if (sizeof(T) == 4) rmin = pmin = (T)3.0e38f;
  for (int j = 0; j < nvc; ++j) {
    const int v = m.ev[vb + j];
    for (int q = m.vel_off[v]; q < m.vel_off[v + 1]; ++q) {
      double un[5];
      ld5(U, m.vel[q], un);
      T ut[5], w[5];
      for (int k = 0; k < 5; ++k) ut[k] = (T)un[k];
      c2p(ut, w);
      pmin = tmin2(pmin, w[4]);
      pmax = tmax2(pmax, w[4]);
      rmin = tmin2(rmin, w[0]);
      rmax = tmax2(rmax, w[0]);
    }
  }
  pmin = ((T)1.0 - (T)1e-2) * pmin;
  rmin = ((T)1.0 - (T)1e-2) * rmin;
  pmax = ((T)1.0 + (T)1e-2) * pmax;
  rmax = ((T)1.0 + (T)1e-2) * rmax;
  omega = 1;
  for (int j = 0; j < nvc; ++j) {
    const double4 xv = m.x[m.ev[vb + j]];
    const T dx[3] = {(T)(xv.x - ce.x), (T)(xv.y - ce.y), (T)(xv.z - ce.z)};
    T dw0 = 0, dw4 = 0;
    for (int d = 0; d < 3; ++d) dw0 = dw0 + g[5 * d] * dx[d];
    for (int d = 0; d < 3; ++d) dw4 = dw4 + g[5 * d + 4] * dx[d];
    if (dw0 < (T)0)
      omega = tmin2(omega, tmax2((T)0, (w0[0] - rmin) / (tol - dw0)));
    else
      omega = tmin2(omega, tmax2((T)0, -(w0[0] - rmax) / (tol + dw0)));
    if (dw4 < (T)0)
      omega = tmin2(omega, tmax2((T)0, (w0[4] - pmin) / (tol - dw4)));
    else
      omega = tmin2(omega, tmax2((T)0, -(w0[4] - pmax) / (tol + dw4)));
  }
  for (int i = 0; i < 15; ++i) go[i] = (double)(omega * g[i]);
}

template <class T>
__global__ void __launch_bounds__(128) k_ns_cell_grad(DevMesh m, NsParams P, const double* __restrict__ U,
                                                      const double* __restrict__ ngrad, double* __restrict__ grad,
                                                      const NsScalars* sc) {
  ns_cell_grad_body<T>(m, P, U, ngrad, grad, sc, blockIdx.x * blockDim.x + threadIdx.x);
}

// The same cell gradient with a group of kCellLanes lanes per cell, lane j holding the
// cell's j-th vertex, for small meshes where a thread per cell leaves most SMs idle and
// each cell's chain sets the kernel's length. Per-vertex terms (weights, their products,
// the limiters' candidates, the neighbour states' primitives) are formed in parallel;
// every sum is taken in vertex order by shuffles, each lane forming the same totals from
// the same operands, so the sums have the thread-per-cell kernel's bits. The min / max
// folds (tmin2, tmax2) run over each lane's own list from the initial value, then over
// the lanes' results in vertex order: a fold keeps the first occurrence of its extreme
// among the values strictly past the initial one and never takes a NaN, so the two-level
// fold returns the single fold's bits. Every lane of the warp reaches every shuffle.
template <class T>
__device__ void ns_cell_grad_group(const DevMesh& m, const NsParams& P, const double* __restrict__ U,
                                   const double* __restrict__ ngrad, double* __restrict__ grad,
                                   const NsScalars* sc, const int c, const int lane) {
  if (sc && sc->done) return;
  const bool live = c < m.ne;
  if (P.method == 0 || P.method == 1) {
    if (live)
      for (int i = lane; i < 15; i += kCellLanes) grad[15 * (size_t)c + i] = 0.0;
    return;
  }
  constexpr unsigned kAll = 0xffffffffu;
  const T eps = (T)1e-3, tol = (T)1e-8;
  const int vb = live ? m.ev_off[c] : 0, nvc = live ? m.ev_off[c + 1] - vb : 0;
  const int nmax = __reduce_max_sync(kAll, nvc);
  const bool own = lane < nvc;
  const int v = own ? m.ev[vb + lane] : 0;
  T ng[15], vol = 0;
  for (int i = 0; i < 15; ++i) ng[i] = 0;
  if (own) {
    const double* src = ngrad + 15 * (size_t)v;
    for (int i = 0; i < 15; ++i) ng[i] = (T)src[i];
    vol = (T)m.vol_v[v];
  }
  // relaxed_maximum_principle, this lane's part: the states of the cells around its
  // vertex do not depend on the gradient, so their folds run first, their loads issued
  // four cells at a time (the folds in the list's order)
  T lrmin = (T)1e100, lrmax = 0, lpmin = (T)1e100, lpmax = 0;
  if (sizeof(T) == 4) lrmin = lpmin = (T)3.0e38f;
  if (own) {
    constexpr int kAhead = 4;
    const int qb = m.vel_off[v + 1];
    for (int q0 = m.vel_off[v]; q0 < qb; q0 += kAhead) {
      int id[kAhead];
#pragma unroll
      for (int i = 0; i < kAhead; ++i) id[i] = q0 + i < qb ? m.vel[q0 + i] : 0;
      double un[kAhead][5];
#pragma unroll
      for (int i = 0; i < kAhead; ++i)
        if (q0 + i < qb) ld5(U, id[i], un[i]);
#pragma unroll
      for (int i = 0; i < kAhead; ++i)
        if (q0 + i < qb) {
          T ut[5], w[5];
          for (int k = 0; k < 5; ++k) ut[k] = (T)un[i][k];
          c2p(ut, w);
          lpmin = tmin2(lpmin, w[4]);
          lpmax = tmax2(lpmax, w[4]);
          lrmin = tmin2(lrmin, w[0]);
          lrmax = tmax2(lrmax, w[0]);
        }
    }
  }
  // the cell's primitive state and this lane's vertex offset, for both limiters
  T w0[5] = {0, 0, 0, 0, 0}, dx[3] = {0, 0, 0};
  if (live) {
    double u0[5];
    ld5(U, c, u0);
    T uu[5];
    for (int k = 0; k < 5; ++k) uu[k] = (T)u0[k];
    c2p(uu, w0);
  }
  if (own) {
    const double4 ce = m.cc[c], xv = m.x[v];
    dx[0] = (T)(xv.x - ce.x);
    dx[1] = (T)(xv.y - ce.y);
    dx[2] = (T)(xv.z - ce.z);
  }
  T g[15], ws[5] = {0, 0, 0, 0, 0};
  for (int i = 0; i < 15; ++i) g[i] = 0;
  if (P.method == 2) {  // dual-volume average
    T t[15], dvs = 0;
    for (int i = 0; i < 15; ++i) t[i] = vol * ng[i];
    for (int j = 0; j < nmax; ++j) {
      const bool in = j < nvc;
      for (int i = 0; i < 15; ++i) {
        const T x = __shfl_sync(kAll, t[i], j, kCellLanes);
        if (in) g[i] = g[i] + x;
      }
      const T x = __shfl_sync(kAll, vol, j, kCellLanes);
      if (in) dvs = dvs + x;
    }
    for (int i = 0; i < 15; ++i) g[i] = g[i] / dvs;
  } else if (P.method == 3) {  // the vertex gradient of smallest norm, per variable
    for (int k = 0; k < 5; ++k) {
      const T o = oi3<T>(ng[k], ng[5 + k], ng[10 + k]);
      T best = __shfl_sync(kAll, o, 0, kCellLanes);
      int sel = 0;
      for (int j = 1; j < nmax; ++j) {
        const T x = __shfl_sync(kAll, o, j, kCellLanes);
        if (j < nvc && x < best) {
          best = x;
          sel = j;
        }
      }
      for (int d = 0; d < 3; ++d) g[5 * d + k] = __shfl_sync(kAll, ng[5 * d + k], sel, kCellLanes);
    }
  } else {  // 4: V / (eps + |g|); 5, 6: V / (eps + |g|)^2 (6 adds the central average)
    T w[5], t[15];
    for (int k = 0; k < 5; ++k) {
      const T q = eps + oi3<T>(ng[k], ng[5 + k], ng[10 + k]);
      w[k] = P.method == 4 ? vol / q : vol / (q * q);
      for (int d = 0; d < 3; ++d) t[5 * d + k] = w[k] * ng[5 * d + k];
    }
    for (int j = 0; j < nmax; ++j) {
      const bool in = j < nvc;
      for (int i = 0; i < 15; ++i) {
        const T x = __shfl_sync(kAll, t[i], j, kCellLanes);
        if (in) g[i] = g[i] + x;
      }
      for (int k = 0; k < 5; ++k) {
        const T x = __shfl_sync(kAll, w[k], j, kCellLanes);
        if (in) ws[k] = ws[k] + x;
      }
    }
    if (P.method == 6) {  // OI of the (3, 5) central gradient: the norm of its first column
      T cg[15], cws = 0;
      for (int i = 0; i < 15; ++i) {
        cg[i] = 0;
        t[i] = vol * ng[i];
      }
      for (int j = 0; j < nmax; ++j) {
        const bool in = j < nvc;
        for (int i = 0; i < 15; ++i) {
          const T x = __shfl_sync(kAll, t[i], j, kCellLanes);
          if (in) cg[i] = cg[i] + x;
        }
        const T x = __shfl_sync(kAll, vol, j, kCellLanes);
        if (in) cws = cws + x;
      }
      for (int i = 0; i < 15; ++i) cg[i] = cg[i] / cws;
      const T q = eps + oi3<T>(cg[0], cg[5], cg[10]);
      const T wc = cws / (q * q);
      for (int i = 0; i < 15; ++i) g[i] = g[i] + wc * cg[i];
      for (int k = 0; k < 5; ++k) ws[k] = ws[k] + wc;
    }
    for (int k = 0; k < 5; ++k)
      for (int d = 0; d < 3; ++d) g[5 * d + k] = g[5 * d + k] / ws[k];
  }
  T om = 1;  // physical_slope_limiter: this lane's vertex
  {
    T dw0 = 0, dw4 = 0;
    for (int d = 0; d < 3; ++d) dw0 = dw0 + g[5 * d] * dx[d];
    for (int d = 0; d < 3; ++d) dw4 = dw4 + g[5 * d + 4] * dx[d];
    if (dw0 < (T)0) om = tmin2(om, tmax2((T)0, w0[0] / (tol - dw0)));
    if (dw4 < (T)0) om = tmin2(om, tmax2((T)0, w0[4] / (tol - dw4)));
  }
  T omega = 1;
  for (int j = 0; j < nmax; ++j) {
    const T x = __shfl_sync(kAll, om, j, kCellLanes);
    if (j < nvc) omega = tmin2(omega, x);
  }
  for (int i = 0; i < 15; ++i) g[i] = omega * g[i];
  T rmin = (T)1e100, rmax = 0, pmin = (T)1e100, pmax = 0;  // relaxed_maximum_principle
  if (sizeof(T) == 4) rmin = pmin = (T)3.0e38f;
  for (int j = 0; j < nmax; ++j) {
    const T a = __shfl_sync(kAll, lpmin, j, kCellLanes), b = __shfl_sync(kAll, lpmax, j, kCellLanes);
    const T e = __shfl_sync(kAll, lrmin, j, kCellLanes), f = __shfl_sync(kAll, lrmax, j, kCellLanes);
    if (j < nvc) {
      pmin = tmin2(pmin, a);
      pmax = tmax2(pmax, b);
      rmin = tmin2(rmin, e);
      rmax = tmax2(rmax, f);
    }
  }
  pmin = ((T)1.0 - (T)1e-2) * pmin;
  rmin = ((T)1.0 - (T)1e-2) * rmin;
  pmax = ((T)1.0 + (T)1e-2) * pmax;
  rmax = ((T)1.0 + (T)1e-2) * rmax;
  om = 1;
  {
    T dw0 = 0, dw4 = 0;
    for (int d = 0; d < 3; ++d) dw0 = dw0 + g[5 * d] * dx[d];
    for (int d = 0; d < 3; ++d) dw4 = dw4 + g[5 * d + 4] * dx[d];
    if (dw0 < (T)0)
      om = tmin2(om, tmax2((T)0, (w0[0] - rmin) / (tol - dw0)));
    else
      om = tmin2(om, tmax2((T)0, -(w0[0] - rmax) / (tol + dw0)));
    if (dw4 < (T)0)
      om = tmin2(om, tmax2((T)0, (w0[4] - pmin) / (tol - dw4)));
    else
      om = tmin2(om, tmax2((T)0, -(w0[4] - pmax) / (tol + dw4)));
  }
  omega = 1;
  for (int j = 0; j < nmax; ++j) {
    const T x = __shfl_sync(kAll, om, j, kCellLanes);
    if (j < nvc) omega = tmin2(omega, x);
  }
  if (live)
#pragma unroll
    for (int i = 0; i < 15; ++i)
      if (i % kCellLanes == lane) grad[15 * (size_t)c + i] = (double)(omega * g[i]);
}

template <class T>
__global__ void __launch_bounds__(128) k_ns_cell_grad_group(DevMesh m, NsParams P, const double* __restrict__ U,
                                                            const double* __restrict__ ngrad,
                                                            double* __restrict__ grad, const NsScalars* sc) {
  const int c = blockIdx.x * (blockDim.x / kCellLanes) + threadIdx.x / kCellLanes;
  ns_cell_grad_group<T>(m, P, U, ngrad, grad, sc, c, threadIdx.x % kCellLanes);
}

constexpr int kTdBlock = 128;

// flux_limiting (ns_euler_recon_module.F90:560-601) and the per-cell part of
// add_timedisc_and_solve (ns_euler_module.F90:546-580). U_rhs: the state the residual
// was evaluated at; U_td: the state being advanced. Writes delta, per-block omega min
// (atomic on the bit pattern) and per-block residual partial sums (res, res_vect(5)).
// called by every thread of a kTdBlock-thread block; blk is the block's index within
// its problem (it selects the slot of the residual partial sums)
// With diffusion the cell's terms go onto the limited residual and into its 5x5 block,
// and the cell solves (block + s I) x = rhs + s U by LU (out of line: rare). The
// out-of-line solve takes the five mesh arrays it reads by value: a reference to the
// kernel's mesh would make every thread copy the whole mesh block into local memory.
struct DiffCellView {
  const int *ev_off, *cse_sorted, *se_vert, *dse_off;
  const int4* se_sf;
};
__device__ __noinline__ void diffusion_cell_solve(const DiffCellView m, int c, const double* __restrict__ dterm,
                                                  int kd, double* r, double* rv, const double* u, double s,
                                                  double* d5) {
  double D[25];
  for (int k = 0; k < 25; ++k) D[k] = 0.0;
  apply_diffusion_terms(m, c, dterm, kd, r, D);
  for (int k = 0; k < 5; ++k) rv[k] = r[k] * r[k];
  for (int a = 0; a < 5; ++a)
    for (int b = 0; b < 5; ++b) D[a + 5 * b] = D[a + 5 * b] + s * (a == b ? 1.0 : 0.0);
  double x[5];
  for (int k = 0; k < 5; ++k) x[k] = r[k] + s * u[k];
  lu_solve5(D, x);
  for (int k = 0; k < 5; ++k) d5[k] = x[k] - u[k];
}

template <bool DIFF = false>
__device__ void ns_timedisc_body(const DevMesh& m, const NsParams& P, const double* __restrict__ U_rhs,
                                 const double* __restrict__ rhs1, const double* __restrict__ rhs2,
                                 const double* __restrict__ U_td, double* __restrict__ delta,
                                 double* __restrict__ partial, NsScalars* sc, double a1, double a2, const int blk,
                                 const double* __restrict__ dterm = nullptr) {
  if (sc->done) return;
  const int c = blk * kTdBlock + threadIdx.x;
  const double dt_fl = P.cfl * sc->dtred;
  double dt = P.cfl * sc->dtred;
  if (!P.lts) dt = fmin2(sc->tmax - sc->t + 1e-12, dt);
  double om = 1.0, rn = 0.0, rv[5] = {0, 0, 0, 0, 0};
  if (c < m.ne) {
    const double V = m.vol[c];
    const double* r1 = rhs1 + kRhs * (size_t)c;
    double r[5];
    for (int k = 0; k < 5; ++k) r[k] = r1[k];
    if (rhs2) {
      const double* r2 = rhs2 + kRhs * (size_t)c;
      const double den = V / dt_fl + r1[5];
      double us[5], Ub[5], dU[5];
      ld5(U_rhs, c, us);
      for (int k = 0; k < 5; ++k) {
        Ub[k] = us[k] + r[k] / den;
        dU[k] = (r2[k] - r[k]) / den;
      }
      const double w = fmin2(1.0, max_omega_for_positivity(Ub, dU));
      for (int k = 0; k < 5; ++k) r[k] = r[k] + w * (r2[k] - r[k]);
    }
    double u[5], d5[5], ad[5];
    ld5(U_td, c, u);
    const double s = a1 * (V / dt + 0.0);  // sum_lambda is zeroed once dt is known
    if (DIFF) {
      diffusion_cell_solve({m.ev_off, m.cse_sorted, m.se_vert, m.dse_off, m.se_sf}, c, dterm, P.diff_kd, r, rv, u, s,
                           d5);
      for (int k = 0; k < 5; ++k) ad[k] = a2 * d5[k];
    } else {
      for (int k = 0; k < 5; ++k) rv[k] = r[k] * r[k];
      for (int k = 0; k < 5; ++k) {
        const double rr = r[k] + s * u[k];
        d5[k] = rr / s - u[k];
        ad[k] = a2 * d5[k];
      }
    }
    om = max_omega_for_positivity(u, ad);
    {  // norm2(delta): gfortran's scaled sum of squares
      double scale = 1.0, res = 0.0;
      for (int k = 0; k < 5; ++k)
        if (d5[k] != 0.0) {
          double ax = fabs(d5[k]);
          if (ax > scale) {
            double q = scale / ax;
            res = 1.0 + res * q * q;
            scale = ax;
          } else {
            double q = ax / scale;
            res += q * q;
          }
        }
      rn = scale * sqrt(res);
    }
    double* dl = delta + 5 * (size_t)c;
    for (int k = 0; k < 5; ++k) dl[k] = d5[k];
  }
  __shared__ double sh[6][kTdBlock / 32];
  __shared__ double shm[kTdBlock / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  double x = warp_min(om);
  if (lane == 0) shm[wid] = x;
  double vals[6] = {rn, rv[0], rv[1], rv[2], rv[3], rv[4]};
  for (int i = 0; i < 6; ++i) {
    double y = warp_sum_tree(vals[i]);
    if (lane == 0) sh[i][wid] = y;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double mn = shm[0];
    for (int w = 1; w < kTdBlock / 32; ++w) mn = fmin(mn, shm[w]);
    atomic_min_pos(&sc->omega, mn);
    for (int i = 0; i < 6; ++i) {
      double s = sh[i][0];
      for (int w = 1; w < kTdBlock / 32; ++w) s = s + sh[i][w];
      partial[6 * (size_t)blk + i] = s;
    }
  }
}


// scalar tail of add_timedisc_and_solve (:582-608); last_stage also advances t
__device__ void ns_finalize_body(NsScalars* sc, const NsParams& P, const double* __restrict__ partial, int nblocks,
                                 unsigned* status, int last_stage) {
  if (sc->done) {
    sc->skip = 1;
    return;
  }
  double dt = P.cfl * sc->dtred;
  if (!P.lts) dt = fmin2(sc->tmax - sc->t + 1e-12, dt);
  // the partial sums in block order, the loads of eight blocks issued before their adds
  double res = 0.0, rv[5] = {0, 0, 0, 0, 0};
  constexpr int kAhead = 8;
  for (int b0 = 0; b0 < nblocks; b0 += kAhead) {
    double buf[kAhead][6];
#pragma unroll
    for (int i = 0; i < kAhead; ++i)
      if (b0 + i < nblocks)
#pragma unroll
        for (int k = 0; k < 6; ++k) buf[i][k] = __ldcg(partial + 6 * (size_t)(b0 + i) + k);
#pragma unroll
    for (int i = 0; i < kAhead; ++i)
      if (b0 + i < nblocks) {
        res = res + buf[i][0];
#pragma unroll
        for (int k = 0; k < 5; ++k) rv[k] = rv[k] + buf[i][1 + k];
      }
  }
  const double omega = __ldcg(&sc->omega);
  sc->omega_step = omega;  // for the update; the next stage's limiter starts afresh
  sc->omega = 1.0;
  if (omega <= 1e-6) atomicOr(status, kErrBadOmega);
  if (!P.lts && omega < 1.0) dt = (1.0 - omega) * dt;
  sc->res = res;
  for (int k = 0; k < 5; ++k) sc->resv[k] = sqrt(rv[k]);
  sc->dt = dt;
  sc->skip = 0;
  sc->dtred = 1e10;  // the next stage's reductions start afresh
  if (last_stage) {
    sc->t = sc->t + dt;
    sc->steps += 1;
    sc->done = ((!P.lts && sc->t >= sc->tmax) || !(res > sc->final_res)) ? 1 : 0;
  }
}

// The time discretisation of one problem with the stage's scalar tail folded in: each
// block publishes its partial sums and limiter minimum, then counts itself in, and the
// block that arrives last runs ns_finalize_body over all the blocks' partial sums (in
// block order, whichever block that is, reading them from L2) and clears the count. No
// block waits for another.
template <bool DIFF>
__global__ void __launch_bounds__(kTdBlock) k_ns_timedisc(DevMesh m, NsParams P, const double* __restrict__ U_rhs,
                                                          const double* __restrict__ rhs1,
                                                          const double* __restrict__ rhs2,
                                                          const double* __restrict__ U_td,
                                                          double* __restrict__ delta, double* __restrict__ partial,
                                                          NsScalars* sc, double a1, double a2,
                                                          const double* __restrict__ dterm, int last_stage) {
  ns_timedisc_body<DIFF>(m, P, U_rhs, rhs1, rhs2, U_td, delta, partial, sc, a1, a2, blockIdx.x, dterm);
  __shared__ int last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();  // this block's partial sums and limiter minimum before its arrival
    last = atomicAdd(&sc->arrive, 1u) == gridDim.x - 1 ? 1 : 0;
  }
  __syncthreads();
  if (last && threadIdx.x == 0) {
    __threadfence();
    ns_finalize_body(sc, P, partial, gridDim.x, m.status, last_stage);
    sc->arrive = 0u;
  }
}

// sol = sol + a2*omega*delta (:608); U_out may be U_td
__device__ void ns_apply_body(const DevMesh& m, const double* __restrict__ U_td, const double* __restrict__ delta,
                              double* __restrict__ U_out, NsScalars* sc, double a2, const int c) {
  if (sc->skip) return;
  if (c >= m.ne) return;
  const double omega = sc->omega_step;
  const double* u = U_td + kRec * (size_t)c;
  double* o = U_out + kRec * (size_t)c;
  const double* d = delta + 5 * (size_t)c;
  bool fin = true;
  for (int k = 0; k < 5; ++k) {
    o[k] = u[k] + a2 * omega * d[k];
    fin = fin && isfinite(o[k]);
  }
  if (!fin) atomicOr(m.status, kErrNonFinite);
  if (!(o[0] > 0.0)) atomicOr(m.status, kErrNegDensity);
}

__global__ void k_ns_apply(DevMesh m, const double* __restrict__ U_td, const double* __restrict__ delta,
                           double* __restrict__ U_out, NsScalars* sc, double a2) {
  ns_apply_body(m, U_td, delta, U_out, sc, a2, blockIdx.x * blockDim.x + threadIdx.x);
}


// ---------------------------------------------------------------------------------
// Batched launches over a table of problems. A persistent grid walks the work blocks of
// all problems (vertex kernels: blockDim.x vertices per work block, cell kernels: 128
// cells); each block finds its problem by binary search in the prefix table, so every
// per-problem reduction sees exactly the blocks of a solo run and the results are the
// solo results bit for bit. hdr[0] is the number of problems, read on the device so
// that a captured step loop stays valid while problems join and leave.

__device__ inline int item_of(const int* __restrict__ wofs, int n, int w) {
  int lo = 0, hi = n;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (wofs[mid] <= w) lo = mid;
    else hi = mid;
  }
  return lo;
}

// which: the state the phase reads (0: U0, 1: U1)
template <class T, class L, int MS, bool EXT>
__global__ void __launch_bounds__(kNodeThreads) kb_ns_node(const NsItem* __restrict__ it, const int* __restrict__ wv,
                                                           const int* __restrict__ hdr, NsParams P, int which,
                                                           int so) {
  const int n = hdr[0];
  for (int w = blockIdx.x; w < wv[n]; w += gridDim.x) {
    const int p = item_of(wv, n, w);
    const NsItem& I = it[p];
    if (I.sc->done) continue;
    ns_node_vertex<T, L, MS, EXT>(I.m, P, which ? I.U1 : I.U0, I.grad, I.fs, so,
                                  vert_at(I.m, (w - wv[p]) * blockDim.x + threadIdx.x), I.sc);
  }
}
// the group variant: a work block of block_v vertices is walked kNodeGroupThreads / NG
// vertices at a time
template <class T, class L, int NG>
__global__ void __launch_bounds__(kNodeGroupThreads, kNodeGroupMinBlocks) kb_ns_node_group(const NsItem* __restrict__ it,
                                                                      const int* __restrict__ wv,
                                                                      const int* __restrict__ hdr, NsParams P,
                                                                      int which, int so, int block_v) {
  __shared__ NodeGroupSmem sm;
  constexpr int VPB = kNodeGroupThreads / NG;
  const int g = threadIdx.x / NG;
  const int n = hdr[0];
  for (int w = blockIdx.x; w < wv[n]; w += gridDim.x) {
    const int p = item_of(wv, n, w);
    const NsItem& I = it[p];
    if (I.sc->done) continue;
    for (int c = 0; c < block_v; c += VPB)
      ns_node_group<T, L, NG>(I.m, P, which ? I.U1 : I.U0, I.grad, I.fs, so, vert_at(I.m, (w - wv[p]) * block_v + c + g), true,
                             sm.v + g * NG * kLaneVals, sm.f + g * NG, sm.s[g], I.sc);
  }
}
__global__ void __launch_bounds__(128) kb_ns_gather(const NsItem* __restrict__ it, const int* __restrict__ wc,
                                                    const int* __restrict__ hdr, int second) {
  const int n = hdr[0];
  for (int w = blockIdx.x; w < wc[n]; w += gridDim.x) {
    const int p = item_of(wc, n, w);
    const NsItem& I = it[p];
    ns_gather_body(I.m, I.fs, second ? I.rhs2 : I.rhs1, I.sc, second ? 0 : 1, (w - wc[p]) * 128 + threadIdx.x);
    __syncthreads();  // the block-reduction scratch is reused by the next work block
  }
}
__global__ void __launch_bounds__(256) kb_ns_nodal_grad(const NsItem* __restrict__ it, const int* __restrict__ wv,
                                                        const int* __restrict__ hdr, int which) {
  const int n = hdr[0];
  for (int w = blockIdx.x; w < wv[n]; w += gridDim.x) {
    const int p = item_of(wv, n, w);
    const NsItem& I = it[p];
    ns_nodal_grad_body<false>(I.m, which ? I.U1 : I.U0, I.ngrad, I.sc, vert_at(I.m, (w - wv[p]) * blockDim.x + threadIdx.x));
  }
}
template <class T>
__global__ void __launch_bounds__(128) kb_ns_cell_grad(const NsItem* __restrict__ it, const int* __restrict__ wc,
                                                       const int* __restrict__ hdr, NsParams P, int which) {
  const int n = hdr[0];
  for (int w = blockIdx.x; w < wc[n]; w += gridDim.x) {
    const int p = item_of(wc, n, w);
    const NsItem& I = it[p];
    ns_cell_grad_body<T>(I.m, P, which ? I.U1 : I.U0, I.ngrad, I.grad, I.sc, (w - wc[p]) * 128 + threadIdx.x);
  }
}
// stage: 0 first stage of two (rhs at U0, advance U0 -> U1), 1 second stage (rhs at U1,
// advance U0 in place), 2 the single first-order stage (rhs at U0, U0 in place)
__global__ void __launch_bounds__(kTdBlock) kb_ns_timedisc(const NsItem* __restrict__ it, const int* __restrict__ wc,
                                                           const int* __restrict__ hdr, NsParams P, int stage,
                                                           double a1, double a2) {
  const int n = hdr[0];
  for (int w = blockIdx.x; w < wc[n]; w += gridDim.x) {
    const int p = item_of(wc, n, w);
    const NsItem& I = it[p];
    const double* Ur = stage == 1 ? I.U1 : I.U0;
    ns_timedisc_body(I.m, P, Ur, I.rhs1, P.second_order ? I.rhs2 : nullptr, I.U0, I.delta, I.partial, I.sc, a1, a2,
                     w - wc[p]);
    __syncthreads();
  }
}
__global__ void kb_ns_finalize(const NsItem* __restrict__ it, const int* __restrict__ hdr, NsParams P,
                               int last_stage) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= hdr[0]) return;
  const NsItem& I = it[p];
  ns_finalize_body(I.sc, P, I.partial, (I.m.ne + kTdBlock - 1) / kTdBlock, I.m.status, last_stage);
}
__global__ void __launch_bounds__(128) kb_ns_apply(const NsItem* __restrict__ it, const int* __restrict__ wc,
                                                   const int* __restrict__ hdr, int stage, double a2) {
  const int n = hdr[0];
  for (int w = blockIdx.x; w < wc[n]; w += gridDim.x) {
    const int p = item_of(wc, n, w);
    const NsItem& I = it[p];
    ns_apply_body(I.m, I.U0, I.delta, stage == 0 ? I.U1 : I.U0, I.sc, a2, (w - wc[p]) * 128 + threadIdx.x);
  }
}

// ---------------------------------------------------------------------------------
// Backward-Euler Jacobian (no counterpart in the reference): A = V/dt I - d rhs/dU of
// the first-order two-wave residual with sl, sr frozen. One thread per block row, which
// owns all of its blocks, so the assembly needs no atomics and is deterministic.

// dF.n/dU for the Euler flux, conservative variables
__device__ void euler_jac(const double* U, const double* n, double A[5][5]) {
  const double rho = U[0];
  const double u[3] = {U[1] / rho, U[2] / rho, U[3] / rho};
  const double q2 = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
  const double p = (G - 1) * (U[4] - 0.5 * rho * q2);
  const double vn = dotT(u, n);
  const double H = (U[4] + p) / rho;
  const double phi = 0.5 * (G - 1) * q2;
  A[0][0] = 0.0;
  for (int mm = 0; mm < 3; ++mm) A[0][mm + 1] = n[mm];
  A[0][4] = 0.0;
  for (int k = 0; k < 3; ++k) {
    A[k + 1][0] = phi * n[k] - u[k] * vn;
    for (int mm = 0; mm < 3; ++mm) {
      const double a = u[k] * n[mm] - (G - 1) * u[mm] * n[k];
      A[k + 1][mm + 1] = k == mm ? a + vn : a;
    }
    A[k + 1][4] = (G - 1) * n[k];
  }
  A[4][0] = vn * (phi - H);
  for (int mm = 0; mm < 3; ++mm) A[4][mm + 1] = H * n[mm] - (G - 1) * u[mm] * vn;
  A[4][4] = G * vn;
}

__device__ void two_wave_jac(const double* wl, const double* wr, const double* n, double JL[5][5],
                             double JR[5][5]) {
  const double rhol = wl[0], vnl = dotT(wl + 1, n), pl = wl[4], al = sound_speed_w(wl);
  const double rhor = wr[0], vnr = dotT(wr + 1, n), pr = wr[4], ar = sound_speed_w(wr);
  double ul[5], ur[5];
  p2c(wl, ul);
  p2c(wr, ur);
  const double lam_l = fmax2(fmax2(al * rhol, sqrt(rhol * fmax2(0.0, pr - pl))), -rhol * (vnr - vnl));
  const double lam_r = fmax2(fmax2(ar * rhor, sqrt(rhor * fmax2(0.0, pl - pr))), -rhor * (vnr - vnl));
  const double sl = vnl - lam_l / rhol, sr = vnr + lam_r / rhor;
  double AL[5][5], AR[5][5];
  euler_jac(ul, n, AL);
  euler_jac(ur, n, AR);
  const double den = sr - sl, asl = fabs(sl), asr = fabs(sr), d = asl - asr;
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

// The Euler flux Jacobian d(F.n)/dU of euler_jac one entry at a time, from the same
// intermediate values and with the same operations, so that a caller can consume the
// 5x5 matrix entry by entry without holding it.
struct EulerJacScalars {
  double u[3], vn, H, phi;
};
__device__ inline void euler_jac_scalars(const double* U, const double* n, EulerJacScalars& e) {
  const double rho = U[0];
  e.u[0] = U[1] / rho;
  e.u[1] = U[2] / rho;
  e.u[2] = U[3] / rho;
  const double q2 = e.u[0] * e.u[0] + e.u[1] * e.u[1] + e.u[2] * e.u[2];
  const double p = (G - 1) * (U[4] - 0.5 * rho * q2);
  e.vn = dotT(e.u, n);
  e.H = (U[4] + p) / rho;
  e.phi = 0.5 * (G - 1) * q2;
}
__device__ inline double euler_jac_entry(const EulerJacScalars& e, const double* n, int r, int c) {
  if (r == 0) return (c == 0 || c == 4) ? 0.0 : n[c - 1];
  if (r == 4) {
    if (c == 0) return e.vn * (e.phi - e.H);
    if (c == 4) return G * e.vn;
    return e.H * n[c - 1] - (G - 1) * e.u[c - 1] * e.vn;
  }
  const int k = r - 1;
  if (c == 0) return e.phi * n[k] - e.u[k] * e.vn;
  if (c == 4) return (G - 1) * n[k];
  const int mm = c - 1;
  const double a = e.u[k] * n[mm] - (G - 1) * e.u[mm] * n[k];
  return k == mm ? a + e.vn : a;
}

// A boundary subface's term of the diagonal block, area (J_L + J_R M), column-major:
// the ghost state U_R(U_L) enters through M = dU_R/dU_L (wall, and the double-Mach
// bottom past x = 0.1667: momentum reflection; outflow, and pondered inflow leaving the
// domain: I; adherence wall: the derivative of its reflection about the wall velocity;
// imposed states: 0). fx0 is the face centroid's x. Out of line: rare, and it holds
// three full matrices.
// kind: the boundary kind of the face, bc its values (by value: a reference to the
// kernel's parameter block would make every thread copy it into local memory)
__device__ __noinline__ void ghost_block(int kind, const BcVals bc, const double* wl, const double* wr,
                                         const double* n, double area, double fx0, double* g) {
  double JL[5][5], JR[5][5];
  two_wave_jac(wl, wr, n, JL, JR);
  double M[5][5];
  for (int a = 0; a < 5; ++a)
    for (int b = 0; b < 5; ++b) M[a][b] = 0.0;
  const double* bv = bc.v;
  if (kind == 1 || (kind == 7 && !(fx0 < 0.1667))) {
    M[0][0] = M[4][4] = 1.0;
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) M[a + 1][b + 1] = (a == b ? 1.0 : 0.0) - 2.0 * n[a] * n[b];
  } else if (kind == 4) {
    for (int a = 0; a < 5; ++a) M[a][a] = 1.0;
  } else if (kind == 5) {
    double ub[5];
    p2c(bv, ub);
    if (dotT(ub + 1, n) > 0.0)
      for (int a = 0; a < 5; ++a) M[a][a] = 1.0;
  } else if (kind == 2) {
    // rho_r = rho, m_r = 2 rho b - m, E_r = E - |m|^2/(2 rho) + |m_r|^2/(2 rho); with
    // u = m / rho and r = 2 b - u: dE_r/drho = |u|^2/2 + 2 r.b - |r|^2/2, dE_r/dm = -2 b
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
    for (int cc = 0; cc < 5; ++cc) {
      double t = 0.0;
      for (int k = 0; k < 5; ++k) t = t + JR[r][k] * M[k][cc];
      g[r + 5 * cc] = area * (JL[r][cc] + t);
    }
}

// jq: per cell its subfaces (2*sf + side) in ascending id; jblk: the block of the other
// cell (-1 for a boundary); row_off/dblk: the row's first block and its diagonal block.
// One thread per block row. The diagonal block and the block of the current neighbour
// are accumulated in registers, entry by entry in subface order (the order of the
// reference-style accumulation into the stored matrix), and each block is stored once
// per run of subfaces that share a neighbour; the two-wave Jacobian is formed entry by
// entry from the scalars of two_wave_jac. Boundary subfaces (the ghost-state chain rule)
// take the full-matrix path.
__global__ void __launch_bounds__(64) k_be_assemble(DevMesh m, NsParams P, const double* __restrict__ U,
                                                    const int* __restrict__ jq_off, const int* __restrict__ jq,
                                                    const int* __restrict__ jblk, const int* __restrict__ row_off,
                                                    const int* __restrict__ dblk, double* __restrict__ v, double dt,
                                                    const NsScalars* sc) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= m.ne) return;
  const int rb = row_off[c], re = row_off[c + 1], db = dblk[c];
  const bool small = re - rb <= 64;  // first-touch bits for the row's blocks
  if (!small)
    for (size_t q = (size_t)25 * rb; q < (size_t)25 * re; ++q) v[q] = 0.0;
  unsigned long long touched = 0ull;
  double D[25], O[25];
  const double vdt = m.vol[c] / dt;
#pragma unroll
  for (int e = 0; e < 25; ++e) {
    D[e] = e % 6 == 0 ? vdt : 0.0;
    O[e] = 0.0;
  }
  int ob = -1;  // the block O holds
  auto flush = [&]() {
    if (ob >= 0) {
      double* dst = v + (size_t)25 * ob;
#pragma unroll
      for (int e = 0; e < 25; ++e) dst[e] = O[e];
    }
  };
  for (int q = jq_off[c]; q < jq_off[c + 1]; ++q) {
    const int e0 = jq[q];
    const int sf = e0 >> 1, side = e0 & 1;
    const int2 lr = m.flr[m.sf_face[sf]];
    const double4 sn = m.sfn[sf];
    const double n[3] = {sn.x, sn.y, sn.z};
    const double area = sn.w;
    double wl[5], wr[5];
    reconstruct<double>(m, P, U, nullptr, m.sf_vert[sf], sf, lr.x, lr.y, false, wl, wr, sc);
    if (side == 0 && lr.y < 0) {
      double g[25];
      const int kind = lr.y == -1 ? 1 : P.bc_type[-(lr.y + 1) - 1];
      BcVals bc{{0.0, 0.0, 0.0, 0.0, 0.0}};
      if (lr.y != -1)
        for (int k = 0; k < 5; ++k) bc.v[k] = P.bc_val[-(lr.y + 1) - 1][k];
      ghost_block(kind, bc, wl, wr, n, area, m.fc[m.sf_face[sf]].x, g);
#pragma unroll
      for (int e = 0; e < 25; ++e) D[e] = D[e] + g[e];
      continue;
    }
    // the other cell's block: registers O (a new run loads what earlier runs stored)
    const int tb = jblk[q];
    const bool selfb = tb == db;  // a cell that neighbours itself through a periodic face
    if (!selfb && tb != ob) {
      flush();
      const int bit = tb - rb;
      if (!small || ((touched >> bit) & 1ull)) {
        const double* src = v + (size_t)25 * tb;
#pragma unroll
        for (int e = 0; e < 25; ++e) O[e] = src[e];
      } else {
#pragma unroll
        for (int e = 0; e < 25; ++e) O[e] = 0.0;
      }
      if (small) touched |= 1ull << bit;
      ob = tb;
    }
    // two_wave_jac's scalars
    const double rhol = wl[0], vnl = dotT(wl + 1, n), pl = wl[4], al = sound_speed_w(wl);
    const double rhor = wr[0], vnr = dotT(wr + 1, n), pr = wr[4], ar = sound_speed_w(wr);
    double ul[5], ur[5];
    p2c(wl, ul);
    p2c(wr, ur);
    const double lam_l = fmax2(fmax2(al * rhol, sqrt(rhol * fmax2(0.0, pr - pl))), -rhol * (vnr - vnl));
    const double lam_r = fmax2(fmax2(ar * rhor, sqrt(rhor * fmax2(0.0, pl - pr))), -rhor * (vnr - vnl));
    const double sl = vnl - lam_l / rhol, sr = vnr + lam_r / rhor;
    EulerJacScalars eL, eR;
    euler_jac_scalars(ul, n, eL);
    euler_jac_scalars(ur, n, eR);
    const double den = sr - sl, asl = fabs(sl), asr = fabs(sr), d = asl - asr;
    const double rden = 1.0 / den;
#pragma unroll
    for (int r = 0; r < 5; ++r)
#pragma unroll
      for (int cc = 0; cc < 5; ++cc) {
        const bool I = r == cc;
        const double AL = euler_jac_entry(eL, n, r, cc), AR = euler_jac_entry(eR, n, r, cc);
        const double dL = (AL - (I ? sl : 0.0)) * rden;
        const double dR = ((I ? sr : 0.0) - AR) * rden;
        const double JL = 0.5 * AL - 0.5 * (d * dL - (I ? asl : 0.0));
        const double JR = 0.5 * AR - 0.5 * (d * dR + (I ? asr : 0.0));
        const int e = r + 5 * cc;
        if (side == 0) {
          D[e] = D[e] + area * JL;
          if (selfb) D[e] = D[e] + area * JR;
          else O[e] = O[e] + area * JR;
        } else {
          D[e] = D[e] - area * JR;
          if (selfb) D[e] = D[e] - area * JL;
          else O[e] = O[e] - area * JL;
        }
      }
  }
  flush();
  double* dst = v + (size_t)25 * db;
#pragma unroll
  for (int e = 0; e < 25; ++e) dst[e] = D[e];
  if (small)  // blocks no subface reached (none in a pattern built from the subfaces)
    for (int b = rb; b < re; ++b)
      if (b != db && !((touched >> (b - rb)) & 1ull))
        for (int e = 0; e < 25; ++e) v[(size_t)25 * b + e] = 0.0;
}

// b = rhs (the first five entries of each residual record), and U += x after the solve
__global__ void k_be_pack_rhs(int ne, const double* __restrict__ rhs, double* __restrict__ b) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ne) return;
  for (int k = 0; k < 5; ++k) b[5 * (size_t)c + k] = rhs[kRhs * (size_t)c + k];
}
__global__ void k_be_update(DevMesh m, double* __restrict__ U, const double* __restrict__ x) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= m.ne) return;
  bool fin = true;
  for (int k = 0; k < 5; ++k) {
    U[kRec * (size_t)c + k] = U[kRec * (size_t)c + k] + x[5 * (size_t)c + k];
    fin = fin && isfinite(U[kRec * (size_t)c + k]);
  }
  if (!fin) atomicOr(m.status, kErrNonFinite);
  if (!(U[kRec * (size_t)c] > 0.0)) atomicOr(m.status, kErrNegDensity);
}

// flux_limiting alone (ns_euler_recon_module.F90:560-601): rhs1 <- blend(rhs1, rhs2)
__global__ void k_ns_flux_limiting(DevMesh m, NsParams P, const double* __restrict__ U, double* __restrict__ rhs1,
                                   const double* __restrict__ rhs2, const NsScalars* sc) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= m.ne) return;
  const double dt_fl = P.cfl * sc->dtred;
  double* r1 = rhs1 + kRhs * (size_t)c;
  const double* r2 = rhs2 + kRhs * (size_t)c;
  const double den = m.vol[c] / dt_fl + r1[5];
  double us[5], Ub[5], dU[5];
  ld5(U, c, us);
  for (int k = 0; k < 5; ++k) {
    Ub[k] = us[k] + r1[k] / den;
    dU[k] = (r2[k] - r1[k]) / den;
  }
  const double w = fmin2(1.0, max_omega_for_positivity(Ub, dU));
  for (int k = 0; k < 5; ++k) r1[k] = r1[k] + w * (r2[k] - r1[k]);
}

__global__ void k_ns_pack(int n, const double* __restrict__ s5, double* __restrict__ U) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  double* r = U + kRec * (size_t)c;
  for (int k = 0; k < 5; ++k) r[k] = s5[5 * (size_t)c + k];
  r[5] = r[6] = r[7] = 0.0;
}

}  // namespace

int ns_partial_blocks(const DevMesh& m) { return grid_for(m.ne, kTdBlock); }

// the schemes compiled only into the extended node kernels
bool ns_scheme_ext(const NsParams& P) { return !(P.scheme == 1 || P.scheme == 4); }

template <class T, class L>
void launch_kb_node_tl(const NsTable& t, const NsParams& P, cudaStream_t s, int which, int so) {
  const int gv = t.grid_v, bv = t.block_v;
  if (P.node_group) {
    const int nt = kNodeGroupThreads, g = std::max(t.group, P.node_group);
    if (g == 8) kb_ns_node_group<T, L, 8><<<gv, nt, 0, s>>>(t.items, t.wv, t.hdr, P, which, so, bv);
    else if (g == 16) kb_ns_node_group<T, L, 16><<<gv, nt, 0, s>>>(t.items, t.wv, t.hdr, P, which, so, bv);
    else kb_ns_node_group<T, L, 32><<<gv, nt, 0, s>>>(t.items, t.wv, t.hdr, P, which, so, bv);
    return;
  }
  if (ns_scheme_ext(P)) {
    if (t.group == 8) kb_ns_node<T, L, 8, true><<<gv, bv, 0, s>>>(t.items, t.wv, t.hdr, P, which, so);
    else if (t.group == 16) kb_ns_node<T, L, 16, true><<<gv, bv, 0, s>>>(t.items, t.wv, t.hdr, P, which, so);
    else kb_ns_node<T, L, 32, true><<<gv, bv, 0, s>>>(t.items, t.wv, t.hdr, P, which, so);
    return;
  }
  if (t.group == 8) kb_ns_node<T, L, 8, false><<<gv, bv, 0, s>>>(t.items, t.wv, t.hdr, P, which, so);
  else if (t.group == 16) kb_ns_node<T, L, 16, false><<<gv, bv, 0, s>>>(t.items, t.wv, t.hdr, P, which, so);
  else kb_ns_node<T, L, 32, false><<<gv, bv, 0, s>>>(t.items, t.wv, t.hdr, P, which, so);
}
// precision 0: FP64 throughout; 1: FP32 wave-speed bounds; 2: FP32 wave speeds, flux and
// reconstruction
void launch_kb_node(const NsTable& t, const NsParams& P, cudaStream_t s, int which, int so) {
  if (P.precision == 2) launch_kb_node_tl<float, float>(t, P, s, which, so);
  else if (P.precision == 1) launch_kb_node_tl<double, float>(t, P, s, which, so);
  else launch_kb_node_tl<double, double>(t, P, s, which, so);
}

void launch_ns_batch_step(const NsTable& t, const NsParams& P, cudaStream_t s) {
  const int gv = t.grid_v, gc = t.grid_c, nb = t.block_v, gp = grid_for(t.cap, 128);
  auto node = [&](int which, int so) { launch_kb_node(t, P, s, which, so); };
  auto rhs = [&](int which) {
    node(which, 0);
    kb_ns_gather<<<gc, 128, 0, s>>>(t.items, t.wc, t.hdr, 0);
    if (P.second_order) {
      kb_ns_nodal_grad<<<gv, nb, 0, s>>>(t.items, t.wv, t.hdr, which);
      if (P.precision == 2) kb_ns_cell_grad<float><<<gc, 128, 0, s>>>(t.items, t.wc, t.hdr, P, which);
      else kb_ns_cell_grad<double><<<gc, 128, 0, s>>>(t.items, t.wc, t.hdr, P, which);
      node(which, 1);
      kb_ns_gather<<<gc, 128, 0, s>>>(t.items, t.wc, t.hdr, 1);
    }
  };
  auto stage = [&](int st, double a1, double a2, int last) {
    kb_ns_timedisc<<<gc, kTdBlock, 0, s>>>(t.items, t.wc, t.hdr, P, st, a1, a2);
    kb_ns_finalize<<<gp, 128, 0, s>>>(t.items, t.hdr, P, last);
    kb_ns_apply<<<gc, 128, 0, s>>>(t.items, t.wc, t.hdr, st, a2);
  };
  if (P.second_order) {
    rhs(0);
    stage(0, 2.0, 1.0, 0);
    rhs(1);
    stage(1, 1.0, 1.0, 1);
  } else {
    rhs(0);
    stage(2, 1.0, 1.0, 1);
  }
}

void launch_ns_flux_limiting(const DevMesh& m, const NsParams& P, const double* U, double* rhs1, const double* rhs2,
                             const NsScalars* sc) {
  k_ns_flux_limiting<<<grid_for(m.ne, 128), 128, 0, m.stream>>>(m, P, U, rhs1, rhs2, sc);
}

void launch_be_assemble(const DevMesh& m, const NsParams& P, const double* U, const int* jq_off, const int* jq,
                        const int* jblk, const int* row_off, const int* dblk, double* v, double dt,
                        const NsScalars* sc) {
  k_be_assemble<<<grid_for(m.ne, 64), 64, 0, m.stream>>>(m, P, U, jq_off, jq, jblk, row_off, dblk, v, dt, sc);
}
void launch_be_pack_rhs(const DevMesh& m, const double* rhs, double* b) {
  k_be_pack_rhs<<<grid_for(m.ne, 256), 256, 0, m.stream>>>(m.ne, rhs, b);
}
// The diffusion terms in the backward-Euler system: the reference's point-implicit
// blocks (add_timedisc_and_solve solves (mat_diag + a1 V/dt I) U^{n+1} = rhs + a1 V/dt U^n,
// ns_euler_module.F90:565-576) go onto the diagonal blocks, and the right-hand side
// becomes rhs - mat_diag U (the same system written for the increment).
__global__ void k_be_add_diffusion(int ne, const int* __restrict__ dblk, const double* __restrict__ diag25,
                                   const double* __restrict__ U, double* __restrict__ v, double* __restrict__ b) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ne) return;
  const double* D = diag25 + 25 * (size_t)c;
  double* blk = v + 25 * (size_t)dblk[c];
  for (int e = 0; e < 25; ++e) blk[e] = blk[e] + D[e];
  const double* u = U + kRec * (size_t)c;
  for (int a = 0; a < 5; ++a) {
    double s = 0.0;
    for (int k = 0; k < 5; ++k) s = s + D[a + 5 * k] * u[k];
    b[5 * (size_t)c + a] = b[5 * (size_t)c + a] - s;
  }
}
void launch_be_add_diffusion(const DevMesh& m, const int* dblk, const double* diag25, const double* U, double* v,
                             double* b) {
  k_be_add_diffusion<<<grid_for(m.ne, 128), 128, 0, m.stream>>>(m.ne, dblk, diag25, U, v, b);
}
void launch_be_update(const DevMesh& m, double* U, const double* x) {
  k_be_update<<<grid_for(m.ne, 256), 256, 0, m.stream>>>(m, U, x);
}

void launch_ns_pack(const DevMesh& m, const double* s5, double* U) {
  k_ns_pack<<<grid_for(m.ne, 256), 256, 0, m.stream>>>(m.ne, s5, U);
}

int ns_node_lanes(const DevMesh& m) {
  const int k = std::max(m.max_vsf, m.max_vse);
  return k <= 8 ? 8 : k <= 16 ? 16 : k <= 32 ? 32 : 0;
}

template <class T, class L>
void launch_node_tl(const DevMesh& m, const NsParams& P, const double* U, const double* grad, double* fs, int so,
                    const NsScalars* sc) {
  int ms = std::max(8, ns_node_lanes(m));  // a mesh beyond 32 is flagged by the kernel
  if (P.node_group) {
    ms = std::max(ms, P.node_group);
    const int nt = kNodeGroupThreads;
    if (ms == 8)
      k_ns_node_group<T, L, 8><<<grid_for(m.nv, nt / 8), nt, 0, m.stream>>>(m, P, U, grad, fs, so, sc);
    else if (ms == 16)
      k_ns_node_group<T, L, 16><<<grid_for(m.nv, nt / 16), nt, 0, m.stream>>>(m, P, U, grad, fs, so, sc);
    else
      k_ns_node_group<T, L, 32><<<grid_for(m.nv, nt / 32), nt, 0, m.stream>>>(m, P, U, grad, fs, so, sc);
    return;
  }
  const int grid = grid_for(m.nv, 128);
  if (ns_scheme_ext(P)) {
    if (ms == 8) k_ns_node<T, L, 8, true><<<grid, 128, 0, m.stream>>>(m, P, U, grad, fs, so, sc);
    else if (ms == 16) k_ns_node<T, L, 16, true><<<grid, 128, 0, m.stream>>>(m, P, U, grad, fs, so, sc);
    else k_ns_node<T, L, 32, true><<<grid, 128, 0, m.stream>>>(m, P, U, grad, fs, so, sc);
    return;
  }
  if (ms == 8) k_ns_node<T, L, 8, false><<<grid, 128, 0, m.stream>>>(m, P, U, grad, fs, so, sc);
  else if (ms == 16) k_ns_node<T, L, 16, false><<<grid, 128, 0, m.stream>>>(m, P, U, grad, fs, so, sc);
  else k_ns_node<T, L, 32, false><<<grid, 128, 0, m.stream>>>(m, P, U, grad, fs, so, sc);
}
void launch_node(const DevMesh& m, const NsParams& P, const double* U, const double* grad, double* fs, int so,
                 const NsScalars* sc) {
  if (P.precision == 2) launch_node_tl<float, float>(m, P, U, grad, fs, so, sc);
  else if (P.precision == 1) launch_node_tl<double, float>(m, P, U, grad, fs, so, sc);
  else launch_node_tl<double, double>(m, P, U, grad, fs, so, sc);
}

// The nodal gradient: a group of 8, 16 or 32 lanes per vertex (the fewest that hold
// every vertex's subfaces) along with the grouped node kernel, else a thread per vertex.
template <bool CACHED>
void launch_nodal_grad_t(const DevMesh& m, const NsParams& P, const double* U, double* ngrad, const NsScalars* sc) {
  const int k = m.max_vsf, ng = k <= 8 ? 8 : k <= 16 ? 16 : k <= 32 ? 32 : 0;
  if (P.node_group && ng) {
    const int g = grid_for(m.nv, 128 / ng);
    if (ng == 8) k_ns_nodal_grad_group<8, CACHED><<<g, 128, 0, m.stream>>>(m, U, ngrad, sc);
    else if (ng == 16) k_ns_nodal_grad_group<16, CACHED><<<g, 128, 0, m.stream>>>(m, U, ngrad, sc);
    else k_ns_nodal_grad_group<32, CACHED><<<g, 128, 0, m.stream>>>(m, U, ngrad, sc);
    return;
  }
  k_ns_nodal_grad<CACHED><<<grid_for(m.nv, 128), 128, 0, m.stream>>>(m, U, ngrad, sc);
}
// with the mesh's cached pseudo-inverses when they belong to its current geometry
void launch_nodal_grad(const DevMesh& m, const NsParams& P, const double* U, double* ngrad, const NsScalars* sc) {
  if (m.npinv && m.npinv_epoch == m.geom_epoch) launch_nodal_grad_t<true>(m, P, U, ngrad, sc);
  else launch_nodal_grad_t<false>(m, P, U, ngrad, sc);
}

int ensure_nodal_pinv(DevMesh* m) {
  if (m->moving || m->nv == 0) return 0;
  if (m->npinv && m->npinv_epoch == m->geom_epoch) return 0;
  if (!m->npinv) {
    SUBFV_CUDA(cudaMallocAsync((void**)&m->npinv, 9 * (size_t)m->nv * sizeof(double), m->stream));
    m->bytes += 9 * (size_t)m->nv * sizeof(double);
  }
  k_ns_nodal_pinv<<<grid_for(m->nv, 128), 128, 0, m->stream>>>(*m, m->npinv);
  SUBFV_CUDA(cudaGetLastError());
  m->npinv_epoch = m->geom_epoch;
  return 0;
}

// The cell gradient: a group of kCellLanes lanes per cell along with the grouped node
// kernel when every cell has at most kCellLanes vertices, else a thread per cell (same
// results either way).
void launch_cell_grad(const DevMesh& m, const NsParams& P, const double* U, const double* ngrad, double* grad,
                      const NsScalars* sc) {
  if (P.node_group && m.max_evc > 0 && m.max_evc <= kCellLanes) {
    const int g = grid_for(m.ne, 128 / kCellLanes);
    if (P.precision == 2)
      k_ns_cell_grad_group<float><<<g, 128, 0, m.stream>>>(m, P, U, ngrad, grad, sc);
    else
      k_ns_cell_grad_group<double><<<g, 128, 0, m.stream>>>(m, P, U, ngrad, grad, sc);
    return;
  }
  const int g = grid_for(m.ne, 128);
  if (P.precision == 2)
    k_ns_cell_grad<float><<<g, 128, 0, m.stream>>>(m, P, U, ngrad, grad, sc);
  else
    k_ns_cell_grad<double><<<g, 128, 0, m.stream>>>(m, P, U, ngrad, grad, sc);
}

void launch_ns_rhs(const DevMesh& m, const NsParams& P, const double* U, double* fs, double* rhs1, double* rhs2,
                   double* ngrad, double* grad, NsScalars* sc) {
  const int gc = grid_for(m.ne, 128);
  launch_node(m, P, U, grad, fs, 0, sc);
  k_ns_gather<<<gc, 128, 0, m.stream>>>(m, fs, rhs1, sc, sc ? 1 : 0);
  if (P.second_order) {
    launch_nodal_grad(m, P, U, ngrad, sc);
    launch_cell_grad(m, P, U, ngrad, grad, sc);
    launch_node(m, P, U, grad, fs, 1, sc);
    k_ns_gather<<<gc, 128, 0, m.stream>>>(m, fs, rhs2, sc, 0);
  }
}

void launch_ns_timedisc(const DevMesh& m, const NsParams& P, const double* U_rhs, const double* rhs1,
                        const double* rhs2, const double* U_td, double* U_out, double* delta, double* partial,
                        NsScalars* sc, double a1, double a2, int last_stage, const double* dterm) {
  const int nb = ns_partial_blocks(m);
  if (P.diff && dterm)
    k_ns_timedisc<true><<<nb, kTdBlock, 0, m.stream>>>(m, P, U_rhs, rhs1, P.second_order ? rhs2 : nullptr, U_td,
                                                       delta, partial, sc, a1, a2, dterm, last_stage);
  else
    k_ns_timedisc<false><<<nb, kTdBlock, 0, m.stream>>>(m, P, U_rhs, rhs1, P.second_order ? rhs2 : nullptr, U_td,
                                                        delta, partial, sc, a1, a2, nullptr, last_stage);
  k_ns_apply<<<grid_for(m.ne, 256), 256, 0, m.stream>>>(m, U_td, delta, U_out, sc, a2);
}


// ---------------------------------------------------------------------------------
// The reference's module procedures one at a time, for the host-buffer C entries of
// ns_procs.cu (ns_main's loop calls them in turn). Arrays in the reference's layouts:
// sol5 / rhs5 / delta5 five doubles per cell, diag25 the column-major 5 x 5 block.

// compute_euler_flux (ns_euler_module.F90:151-339) at state U with the cell gradients
// grad (read when second_order): corner sums by the node kernel, then the cell gather;
// rhs records hold the five residuals and sum_lambda (started at 1e-12)
void launch_ns_euler_flux(const DevMesh& m, const NsParams& P, const double* U, const double* grad, double* fs,
                          double* rhs, int second_order, NsScalars* sc) {
  launch_node(m, P, U, grad, fs, second_order ? 1 : 0, sc);
  k_ns_gather<<<grid_for(m.ne, 128), 128, 0, m.stream>>>(m, fs, rhs, sc, 0);
}

// compute_cell_grad_from_nodal_grad (ns_euler_recon_module.F90:8-59)
void launch_ns_cell_grads(const DevMesh& m, const NsParams& P, const double* U, double* ngrad, double* grad,
                          NsScalars* sc) {
  launch_nodal_grad(m, P, U, ngrad, sc);
  launch_cell_grad(m, P, U, ngrad, grad, sc);
}

namespace {

// dt = min(1e10, min_i V_i / sum_lambda_i): the first loop of flux_limiting
// (ns_euler_recon_module.F90:575-580) and add_timedisc_and_solve (ns_euler_module.F90:
// 546-551), before the factor cfl; the minimum of non-negative doubles is exact in any
// order (atomicMin on the bit pattern)
__global__ void __launch_bounds__(128) k_proc_dtmin(DevMesh m, const double* __restrict__ sl, double* slot) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  double x = 1e10;
  if (c < m.ne) x = fmin2(x, m.vol[c] / sl[c]);
  __shared__ double wm[4];
  x = warp_min(x);
  if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = x;
  __syncthreads();
  if (threadIdx.x == 0) atomic_min_pos(slot, fmin(fmin(wm[0], wm[1]), fmin(wm[2], wm[3])));
}

// flux_limiting's cell loop (:582-590)
__global__ void __launch_bounds__(128) k_proc_flux_limiting(DevMesh m, const double* __restrict__ sol5,
                                                            double* __restrict__ rhs5,
                                                            const double* __restrict__ rhso2_5,
                                                            const double* __restrict__ sl, double dt) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= m.ne) return;
  double* r = rhs5 + 5 * (size_t)c;
  const double* r2 = rhso2_5 + 5 * (size_t)c;
  const double* u = sol5 + 5 * (size_t)c;
  const double den = m.vol[c] / dt + sl[c];
  double Ub[5], dU[5];
  for (int k = 0; k < 5; ++k) {
    Ub[k] = u[k] + r[k] / den;
    dU[k] = (r2[k] - r[k]) / den;
  }
  const double w = fmin2(1.0, max_omega_for_positivity(Ub, dU));
  for (int k = 0; k < 5; ++k) r[k] = r[k] + w * (r2[k] - r[k]);
}

// add_timedisc_and_solve's cell loop (:559-574) with the global time step (sum_lambda
// already zeroed): rsq = rhs^2 (for res_vect), diag += a1 V/dt I, rhs += a1 V/dt sol,
// the 5 x 5 solve (dgetrf + dgetrs, factors left in diag; without diag the block is
// a1 V/dt I and the solve a division), delta, the positivity limiter's omega (atomic
// minimum) and norm2(delta) (gfortran's scaled sum of squares)
__global__ void __launch_bounds__(128) k_proc_timedisc(DevMesh m, const double* __restrict__ sol5,
                                                       double* __restrict__ rhs5, double* __restrict__ diag25,
                                                       double* __restrict__ delta5, double* __restrict__ rn,
                                                       double* __restrict__ rsq, double a1, double a2, double dt,
                                                       double* omega_slot) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  double om = 1.0;
  if (c < m.ne) {
    const double* u = sol5 + 5 * (size_t)c;
    double* r = rhs5 + 5 * (size_t)c;
    double x[5], d5[5], ad[5];
    for (int k = 0; k < 5; ++k) rsq[5 * (size_t)c + k] = r[k] * r[k];
    const double s = a1 * (m.vol[c] / dt + 0.0);
    for (int k = 0; k < 5; ++k) {
      r[k] = r[k] + s * u[k];
      x[k] = r[k];
    }
    if (diag25) {
      double D[25];
      double* dg = diag25 + 25 * (size_t)c;
      for (int k = 0; k < 25; ++k) D[k] = dg[k];
      for (int a = 0; a < 5; ++a)
        for (int b = 0; b < 5; ++b) D[a + 5 * b] = D[a + 5 * b] + s * (a == b ? 1.0 : 0.0);
      lu_solve5(D, x);
      for (int k = 0; k < 25; ++k) dg[k] = D[k];
    } else {
      for (int k = 0; k < 5; ++k) x[k] = x[k] / s;
    }
    for (int k = 0; k < 5; ++k) {
      d5[k] = x[k] - u[k];
      delta5[5 * (size_t)c + k] = d5[k];
      ad[k] = a2 * d5[k];
    }
    om = max_omega_for_positivity(u, ad);
    double scale = 1.0, res = 0.0;
    for (int k = 0; k < 5; ++k)
      if (d5[k] != 0.0) {
        const double ax = fabs(d5[k]);
        if (ax > scale) {
          const double q = scale / ax;
          res = 1.0 + res * q * q;
          scale = ax;
        } else {
          const double q = ax / scale;
          res += q * q;
        }
      }
    rn[c] = scale * sqrt(res);
  }
  __shared__ double wm[4];
  om = warp_min(om);
  if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = om;
  __syncthreads();
  if (threadIdx.x == 0) atomic_min_pos(omega_slot, fmin(fmin(wm[0], wm[1]), fmin(wm[2], wm[3])));
}

// res = sum_i norm2(delta_i) and res_vect(k) = sum_i rhs(k, i)^2 in cell order, as the
// reference's loop adds them (one thread: the order is the result)
__global__ void k_proc_ordered_sums(int n, const double* __restrict__ rn, const double* __restrict__ rsq,
                                    double* out6) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  double res = 0.0, rv[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  for (int c = 0; c < n; ++c) {
    res = res + rn[c];
    for (int k = 0; k < 5; ++k) rv[k] = rv[k] + rsq[5 * (size_t)c + k];
  }
  out6[0] = res;
  for (int k = 0; k < 5; ++k) out6[1 + k] = rv[k];
}

// sol = sol + a2 omega delta (:608), aw = a2 * omega
__global__ void k_proc_apply(int n5, double* __restrict__ sol5, const double* __restrict__ delta5, double aw) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n5) sol5[i] = sol5[i] + aw * delta5[i];
}

}  // namespace

void launch_proc_dtmin(const DevMesh& m, const double* sl, double* slot) {
  k_proc_dtmin<<<grid_for(m.ne, 128), 128, 0, m.stream>>>(m, sl, slot);
}
void launch_proc_flux_limiting(const DevMesh& m, const double* sol5, double* rhs5, const double* rhso2_5,
                               const double* sl, double dt) {
  k_proc_flux_limiting<<<grid_for(m.ne, 128), 128, 0, m.stream>>>(m, sol5, rhs5, rhso2_5, sl, dt);
}
void launch_proc_timedisc(const DevMesh& m, const double* sol5, double* rhs5, double* diag25, double* delta5,
                          double* rn, double* rsq, double a1, double a2, double dt, double* omega_slot,
                          double* sums6) {
  k_proc_timedisc<<<grid_for(m.ne, 128), 128, 0, m.stream>>>(m, sol5, rhs5, diag25, delta5, rn, rsq, a1, a2, dt,
                                                               omega_slot);
  k_proc_ordered_sums<<<1, 32, 0, m.stream>>>(m.ne, rn, rsq, sums6);
}
void launch_proc_apply(const DevMesh& m, double* sol5, const double* delta5, double aw) {
  k_proc_apply<<<grid_for(5 * m.ne, 256), 256, 0, m.stream>>>(5 * m.ne, sol5, delta5, aw);
}

}  // namespace subfv
