// Test infrastructure only (oracle). Restatement of the subfv Lagrangian hydro step:
// src/lagrange/lagrange_module.F90 (compute_rhs_lagrange, compute_dt, init_sol,
// pressure, move_mesh; the "sidil" scheme's compute_rhs_lagrange_sidil, nodal velocity,
// nodal pressure, compute_length, boundary_normal, corner_normal, lag_to_primit),
// src/linear_algebra/linear_solver_module.F90 (inverse_3_by_3)
// and the time loop of src/lagrange/lagrange_main.F90:81-127.
// PARITY UNPINNED (no Fortran compiler here; the reference tests hold no golden data).
#include "oracle.h"
#include <cmath>

namespace oracle {

static const double kGamma = 7.0 / 5.0;  // lagrange_module.F90:12

// lagrange_module.F90:429-436; u is 0-based (tau, u, v, w, e)
static double pressure(const double* u) {
  double n = fnorm2(u + 1, 3);
  return (kGamma - 1.0) / u[0] * (u[4] - 0.5 * (n * n));
}

static double det2(double a, double b, double c, double d) { return a * d - c * b; }

// linear_solver_module.F90:125-172; M[i][j] = mat(i+1, j+1)
void inverse_3_by_3(const double M[3][3], double Inv[3][3]) {
  double T[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) T[i][j] = M[j][i];
  double A[3][3];
  A[0][0] = det2(T[1][1], T[1][2], T[2][1], T[2][2]);
  A[0][1] = -det2(T[1][0], T[1][2], T[2][0], T[2][2]);
  A[0][2] = det2(T[1][0], T[1][1], T[2][0], T[2][1]);
  A[1][0] = -det2(T[0][1], T[0][2], T[2][1], T[2][2]);
  A[1][1] = det2(T[0][0], T[0][2], T[2][0], T[2][2]);
  A[1][2] = -det2(T[0][0], T[0][1], T[2][0], T[2][1]);
  A[2][0] = det2(T[0][1], T[0][2], T[1][1], T[1][2]);
  A[2][1] = -det2(T[0][0], T[0][2], T[1][0], T[1][2]);
  A[2][2] = det2(T[0][0], T[0][1], T[1][0], T[1][1]);
  double det = M[0][0] * A[0][0] + M[0][1] * A[1][0] + M[0][2] * A[2][0];
  double inv = 1.0 / det;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) Inv[i][j] = inv * A[i][j];
}

static void matvec3(const double M[3][3], const double* x, double* y) {
  for (int i = 0; i < 3; ++i) {
    double s = 0.0;
    for (int k = 0; k < 3; ++k) s = s + M[i][k] * x[k];
    y[i] = s;
  }
}
static double dot3(const double* a, const double* b) {
  double s = 0.0;
  for (int k = 0; k < 3; ++k) s = s + a[k] * b[k];
  return s;
}

// lagrange_module.F90:14-147. sol/rhs: [5*n_elems] Fortran sol(5,n) column-major;
// vp: [3*n_vert]; mass: [n_elems].
void compute_rhs_lagrange(const Mesh& m, const double* sol, double* vp, double* rhs, bool b2d,
                          const double* mass) {
  for (int i = 0; i < 5 * m.n_elems; ++i) rhs[i] = 0.0;
  for (int i = 0; i < 3 * m.n_vert; ++i) vp[i] = 0.0;
  std::vector<double> lam1, lam2;
  for (int i = 1; i <= m.n_vert; ++i) {
    const Vert& v = m.vert[i];
    int nsfn = v.n_sub_faces_neigh;
    lam1.assign(nsfn + 1, 0.0);
    lam2.assign(nsfn + 1, 0.0);
    double Bp[3] = {0, 0, 0}, Rp[3] = {0, 0, 0}, Mp[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    for (int j = 1; j <= nsfn; ++j) {
      int sf = v.sub_face_neigh[j];
      const Face& f = m.face[m.sub_face[sf].mesh_face];
      const double* n = &f.norm[1];
      double area = m.sub_face[sf].area;
      int idl = f.left_neigh, idr = f.right_neigh;
      const double* ul = sol + 5 * (idl - 1);
      double pl = pressure(ul);
      double vl = dot3(ul + 1, n);
      if (idr > 0) {
        const double* ur = sol + 5 * (idr - 1);
        double pr = pressure(ur);
        double vr = dot3(ur + 1, n);
        double a = std::sqrt(kGamma * pl * ul[0]) / ul[0];
        double b = std::sqrt(std::max(0.0, pr - pl) / ul[0]);
        double c = -(vr - vl) / ul[0];
        lam1[j] = std::max(std::max(a, b), c);
        a = std::sqrt(kGamma * pr * ur[0]) / ur[0];
        b = std::sqrt(std::max(0.0, pl - pr) / ur[0]);
        c = -(vr - vl) / ur[0];
        lam2[j] = std::max(std::max(a, b), c);
        double v_bar = (lam1[j] * vl + lam2[j] * vr - (pr - pl)) / (lam2[j] + lam1[j]);
        double w = area * (lam1[j] + lam2[j]);
        for (int r = 0; r < 3; ++r)
          for (int s = 0; s < 3; ++s) Mp[r][s] = Mp[r][s] + w * (n[r] * n[s]);
        for (int r = 0; r < 3; ++r) Rp[r] = Rp[r] + w * n[r] * v_bar;
      } else if (b2d && std::fabs(n[2]) > 1e-8) {
        lam1[j] = std::sqrt(kGamma * pl * ul[0]) / ul[0];
        double w = area * 2 * lam1[j];
        for (int r = 0; r < 3; ++r)
          for (int s = 0; s < 3; ++s) Mp[r][s] = Mp[r][s] + w * (n[r] * n[s]);
      } else {
        lam1[j] = std::sqrt(kGamma * pl * ul[0]) / ul[0];
        for (int r = 0; r < 3; ++r) Bp[r] = Bp[r] + area * n[r];
        double w = area * lam1[j];
        for (int r = 0; r < 3; ++r)
          for (int s = 0; s < 3; ++s) Mp[r][s] = Mp[r][s] + w * (n[r] * n[s]);
        double q = area * (pl + lam1[j] * vl);
        for (int r = 0; r < 3; ++r) Rp[r] = Rp[r] + q * n[r];
      }
    }
    double Minv[3][3], out[3];
    double bmax = std::max(std::max(std::fabs(Bp[0]), std::fabs(Bp[1])), std::fabs(Bp[2]));
    inverse_3_by_3(Mp, Minv);
    if (bmax > 1e-8) {
      double mb[3], rb[3];
      matvec3(Minv, Bp, mb);
      double Pp = dot3(Rp, mb) / dot3(Bp, mb);
      for (int r = 0; r < 3; ++r) rb[r] = Rp[r] - Pp * Bp[r];
      matvec3(Minv, rb, out);
    } else {
      matvec3(Minv, Rp, out);
    }
    for (int r = 0; r < 3; ++r) vp[3 * (i - 1) + r] = out[r];
    for (int j = 1; j <= nsfn; ++j) {
      int sf = v.sub_face_neigh[j];
      const Face& f = m.face[m.sub_face[sf].mesh_face];
      const double* n = &f.norm[1];
      double area = m.sub_face[sf].area;
      int idl = f.left_neigh, idr = f.right_neigh;
      const double* ul = sol + 5 * (idl - 1);
      double v_et = dot3(out, n);
      double vl = dot3(ul + 1, n);
      double pl = pressure(ul);
      double pl_et = pl - lam1[j] * (v_et - vl);
      double flux[5] = {-v_et, pl_et * n[0], pl_et * n[1], pl_et * n[2], pl_et * v_et};
      double am = area / mass[idl - 1];
      for (int k = 0; k < 5; ++k) rhs[5 * (idl - 1) + k] = rhs[5 * (idl - 1) + k] - am * flux[k];
      if (idr > 0) {
        const double* ur = sol + 5 * (idr - 1);
        double vr = dot3(ur + 1, n);
        double pr = pressure(ur);
        double pr_et = pr + lam2[j] * (v_et - vr);
        double fr[5] = {-v_et, pr_et * n[0], pr_et * n[1], pr_et * n[2], pr_et * v_et};
        double ar = area / mass[idr - 1];
        for (int k = 0; k < 5; ++k) rhs[5 * (idr - 1) + k] = rhs[5 * (idr - 1) + k] + ar * fr[k];
      }
    }
  }
}

// ---------------------------------------------------------------- scheme "sidil"
// lagrange_module.F90:802-809 (lag_to_primit): (1/tau, u, v, w, p)
static void lag_to_primit(const double* u, double* w) {
  w[0] = 1.0 / u[0];
  for (int d = 1; d < 4; ++d) w[d] = u[d];
  w[4] = pressure(u);
}

// the primitive states either side of face f: the neighbour's, or at a boundary the
// left state with its velocity mirrored in the face normal (:568-576, :643-651)
static void sidil_lr(const Mesh& m, const double* sol, const Face& f, double* wl, double* wr) {
  const double* ul = sol + 5 * (f.left_neigh - 1);
  double ur[5];
  if (f.right_neigh > 0) {
    for (int k = 0; k < 5; ++k) ur[k] = sol[5 * (f.right_neigh - 1) + k];
  } else {
    for (int k = 0; k < 5; ++k) ur[k] = ul[k];
    const double d = dot3(ur + 1, &f.norm[1]);
    for (int k = 1; k < 4; ++k) ur[k] = ur[k] - 2.0 * d * f.norm[k];
  }
  lag_to_primit(ul, wl);
  lag_to_primit(ur, wr);
}

// compute_length (:680-711) with corner_normal (:730-757): method scales V_p / sum |n_c|
static double sidil_length(const Mesh& m, int v, int method, bool b2d) {
  const Vert& vv = m.vert[v];
  double area_sum = 0.0;
  for (int j = 1; j <= vv.n_sub_elems_neigh; ++j) {
    const SubElem& se = m.sub_elem[vv.sub_elem_neigh[j]];
    double nc[3] = {0.0, 0.0, 0.0};
    for (int k = 1; k <= se.n_sub_faces; ++k) {
      const SubFace& s = m.sub_face[se.sub_face[k]];
      const Face& f = m.face[s.mesh_face];
      if (!b2d || std::fabs(f.norm[3]) < 1e-12) {
        if (f.left_neigh == se.mesh_elem)
          for (int d = 0; d < 3; ++d) nc[d] = nc[d] + s.area * f.norm[d + 1];
        else
          for (int d = 0; d < 3; ++d) nc[d] = nc[d] - s.area * f.norm[d + 1];
      }
    }
    area_sum = area_sum + fnorm2(nc, 3);
  }
  const double c = method == 0 ? 0.0 : method == 1 ? 1.0 : method == 2 ? 2.0 : method == 3 ? 4.0 : 8.0;
  return c * vv.volume / area_sum;
}

// compute_nodal_velocity_sidil (:538-612) and compute_nodal_pressure_sidil (:614-678)
// for vertex v; returns false on a negative nodal pressure (the reference stops)
static bool sidil_node(const Mesh& m, const double* sol, int v, int method, bool b2d, double* vp, double* pp_out) {
  const Vert& vv = m.vert[v];
  double w[5], wl[5], wr[5];
  double rho_p = 0.0, a_p = 0.0, pp = 0.0;
  vp[0] = vp[1] = vp[2] = 0.0;
  for (int j = 1; j <= vv.n_sub_elems_neigh; ++j) {
    const SubElem& se = m.sub_elem[vv.sub_elem_neigh[j]];
    lag_to_primit(sol + 5 * (se.mesh_elem - 1), w);
    for (int d = 0; d < 3; ++d) vp[d] = vp[d] + se.volume * w[1 + d];
    rho_p = rho_p + se.volume * w[0];
    a_p = a_p + se.volume * std::sqrt(kGamma * w[4] / w[0]);
    pp = pp + se.volume * w[4];
  }
  rho_p = rho_p / vv.volume;
  a_p = a_p / vv.volume;
  for (int d = 0; d < 3; ++d) vp[d] = vp[d] / vv.volume;
  pp = pp / vv.volume;
  double grad_p[3] = {0.0, 0.0, 0.0}, div_v = 0.0;
  for (int j = 1; j <= vv.n_sub_faces_neigh; ++j) {
    const SubFace& s = m.sub_face[vv.sub_face_neigh[j]];
    const Face& f = m.face[s.mesh_face];
    sidil_lr(m, sol, f, wl, wr);
    for (int d = 0; d < 3; ++d) grad_p[d] = grad_p[d] + (wr[4] - wl[4]) * s.area * f.norm[d + 1];
    double dv[3], an[3];
    for (int d = 0; d < 3; ++d) {
      dv[d] = wr[1 + d] - wl[1 + d];
      an[d] = s.area * f.norm[d + 1];
    }
    div_v = div_v + dot3(dv, an);
  }
  for (int d = 0; d < 3; ++d) grad_p[d] = grad_p[d] / vv.volume;
  div_v = div_v / vv.volume;
  if (vv.is_bound) {  // boundary_normal (:713-728), normalised
    double Bp[3] = {0.0, 0.0, 0.0};
    for (int j = 1; j <= vv.n_sub_faces_neigh; ++j) {
      const SubFace& s = m.sub_face[vv.sub_face_neigh[j]];
      const Face& f = m.face[s.mesh_face];
      if (f.right_neigh <= 0)
        for (int d = 0; d < 3; ++d) Bp[d] = Bp[d] + s.area * f.norm[d + 1];
    }
    const double nb = fnorm2(Bp, 3);
    for (int d = 0; d < 3; ++d) Bp[d] = Bp[d] / nb;
    const double gb = dot3(grad_p, Bp);
    for (int d = 0; d < 3; ++d) grad_p[d] = grad_p[d] - gb * Bp[d];
  }
  const double h_p = sidil_length(m, v, method, b2d);
  for (int d = 0; d < 3; ++d) vp[d] = vp[d] - 0.5 * h_p / (rho_p * a_p) * grad_p[d];
  pp = pp - 0.5 * h_p * rho_p * a_p * div_v;
  *pp_out = pp;
  return !(pp < 0.0);
}

// compute_rhs_lagrange_sidil (:149-223); returns 4 (negative nodal pressure) or 0
int compute_rhs_lagrange_sidil(const Mesh& m, const double* sol, double* vp, double* rhs, bool b2d,
                               const double* mass, int method) {
  for (int i = 0; i < 5 * m.n_elems; ++i) rhs[i] = 0.0;
  for (int i = 0; i < 3 * m.n_vert; ++i) vp[i] = 0.0;
  int status = 0;
  for (int v = 1; v <= m.n_vert; ++v) {
    double* vpv = vp + 3 * (v - 1);
    double pp = 0.0;
    if (!sidil_node(m, sol, v, method, b2d, vpv, &pp)) status |= 4;
    const Vert& vv = m.vert[v];
    for (int j = 1; j <= vv.n_sub_faces_neigh; ++j) {
      const SubFace& s = m.sub_face[vv.sub_face_neigh[j]];
      const Face& f = m.face[s.mesh_face];
      const double* n = &f.norm[1];
      const double v_et = dot3(vpv, n);
      const double fl[5] = {-v_et, pp * n[0], pp * n[1], pp * n[2], pp * v_et};
      const int idl = f.left_neigh, idr = f.right_neigh;
      const double al = s.area / mass[idl - 1];
      for (int k = 0; k < 5; ++k) rhs[5 * (idl - 1) + k] = rhs[5 * (idl - 1) + k] - al * fl[k];
      if (idr > 0) {
        const double ar = s.area / mass[idr - 1];
        for (int k = 0; k < 5; ++k) rhs[5 * (idr - 1) + k] = rhs[5 * (idr - 1) + k] + ar * fl[k];
      }
    }
  }
  return status;
}

// lagrange_module.F90:240-283 (keeps the reference's sub_elem(i) with i a cell index)
double compute_dt(const Mesh& m, const double* sol, double cfl, const double* vp) {
  const double CV = 0.8;
  double dt = 1e6;
  for (int i = 1; i <= m.n_elems; ++i) {
    const double* u = sol + 5 * (i - 1);
    double c = std::sqrt(kGamma * pressure(u) * u[0]);
    const Elem& e = m.elem[i];
    for (int j = 1; j <= e.n_sub_elems; ++j) {
      const SubElem& se = m.sub_elem[e.sub_elem[j]];
      for (int k = 1; k <= se.n_sub_faces; ++k) {
        const SubFace& s = m.sub_face[se.sub_face[k]];
        const Face& f = m.face[s.mesh_face];
        double n[3];
        for (int d = 0; d < 3; ++d) n[d] = f.left_neigh == i ? f.norm[d + 1] : -f.norm[d + 1];
        dt = std::min(dt, m.sub_elem[i].volume / (s.area * c));
        double vn = dot3(vp + 3 * (s.mesh_vert - 1), n);
        dt = std::min(dt, CV * se.volume / (1e-8 + std::fabs(vn) * f.area));
      }
    }
  }
  return cfl * dt;
}

// lagrange_module.F90:772-784
void move_mesh(Mesh& m, const double* vp, double dt) {
  for (int i = 1; i <= m.n_vert; ++i)
    for (int d = 1; d <= 3; ++d) m.vert[i].coord[d] = m.vert[i].coord[d] + dt * vp[3 * (i - 1) + d - 1];
}

// lagrange_module.F90:318-356 (init = 1): Sedov energy spike. sel_mode 0 selects
// cells whose centroid radius (x,y) is < r_sedov (the reference); sel_mode 1 uses the
// caller's mask (cells touching the origin in the benchmark configuration).
int init_sedov(const Mesh& m, double* sol, double r_sedov, double e_total, const int* mask) {
  double tot_vol = 0.0;
  auto sel = [&](int i) {
    if (mask) return mask[i - 1] != 0;
    const double* c = &m.elem[i].coord[1];
    return std::sqrt(c[0] * c[0] + c[1] * c[1]) < r_sedov;
  };
  for (int i = 1; i <= m.n_elems; ++i)
    if (sel(i)) tot_vol = tot_vol + m.elem[i].volume;
  if (tot_vol < 1e-10) return 1;
  for (int i = 1; i <= m.n_elems; ++i) {
    double* u = sol + 5 * (i - 1);
    u[0] = 1.0;
    u[1] = u[2] = u[3] = 0.0;
    u[4] = sel(i) ? e_total / tot_vol : 1e-8 / (kGamma - 1.0);
  }
  return 0;
}

// lagrange_main.F90:81-127, scheme "classic" (scheme 0) or "sidil" (scheme 1, with
// method_length). Runs until t >= t_max or max_steps. Returns the number of steps taken
// (negated on a negative sidil nodal pressure); *t_io is updated.
int lagrange_run(Mesh& m, double* sol, double* vp, double* rhs, const double* mass, double cfl,
                 double t_max, int max_steps, bool b2d, double* t_io, double* last_dt, int scheme, int method) {
  double t = *t_io;
  int iter = 0;
  std::vector<double> new_sol(5 * m.n_elems);
  while (t < t_max && iter < max_steps) {
    if (scheme == 1) {
      if (compute_rhs_lagrange_sidil(m, sol, vp, rhs, b2d, mass, method)) {
        *t_io = t;
        return -iter - 1;
      }
    } else {
      compute_rhs_lagrange(m, sol, vp, rhs, b2d, mass);
    }
    double dt = compute_dt(m, sol, cfl, vp);
    if (t + dt > t_max) dt = t_max - t;
    move_mesh(m, vp, dt);
    compute_geometry_mesh(m, b2d);
    for (int k = 0; k < 5 * m.n_elems; ++k) new_sol[k] = sol[k] + dt * rhs[k];
    for (int k = 0; k < 5 * m.n_elems; ++k) sol[k] = new_sol[k];
    t = t + dt;
    *last_dt = dt;
    iter++;
  }
  *t_io = t;
  return iter;
}

}  // namespace oracle
