// Test infrastructure only (oracle): a flat C interface over the restatement so the
// CPU tests can drive it through ctypes. PARITY UNPINNED.
#include "oracle.h"
#include <cstring>
#include <string>

namespace oracle {
void compute_rhs_lagrange(const Mesh& m, const double* sol, double* vp, double* rhs, bool b2d,
                          const double* mass);
double compute_dt(const Mesh& m, const double* sol, double cfl, const double* vp);
void move_mesh(Mesh& m, const double* vp, double dt);
int init_sedov(const Mesh& m, double* sol, double r_sedov, double e_total, const int* mask);
int lagrange_run(Mesh& m, double* sol, double* vp, double* rhs, const double* mass, double cfl,
                 double t_max, int max_steps, bool b2d, double* t_io, double* last_dt, int scheme, int method);
int compute_rhs_lagrange_sidil(const Mesh& m, const double* sol, double* vp, double* rhs, bool b2d,
                               const double* mass, int method);
void inverse_3_by_3(const double M[3][3], double Inv[3][3]);
}  // namespace oracle

using namespace oracle;

struct OHandle {
  Mesh m;
  std::map<std::string, std::vector<int32_t>> topo;
};

namespace oracle {
Mesh& handle_mesh(void* h) { return ((OHandle*)h)->m; }
}  // namespace oracle

extern "C" {

void* or_mesh_new_ex(int n_vert, const double* coords, int n_elems, const int* kind, const int* ev_off,
                     const int* ev, int n_bf, const int* bf_off, const int* bf_vert, const int* bf_tag,
                     int b2d, int periodic, int renumber) {
  OHandle* h = new OHandle();
  try {
    read_raw(h->m, n_vert, coords, n_elems, kind, ev_off, ev, n_bf, bf_off, bf_vert, bf_tag);
    build_mesh(h->m, true, b2d != 0, periodic != 0, renumber);
    h->topo = export_topology(h->m);
    compute_geometry_mesh(h->m, b2d != 0);
  } catch (...) {
    delete h;
    return nullptr;
  }
  return h;
}

void* or_mesh_new(int n_vert, const double* coords, int n_elems, const int* kind, const int* ev_off, const int* ev,
                  int n_bf, const int* bf_off, const int* bf_vert, const int* bf_tag, int b2d, int periodic) {
  return or_mesh_new_ex(n_vert, coords, n_elems, kind, ev_off, ev, n_bf, bf_off, bf_vert, bf_tag, b2d, periodic, 0);
}

void or_mesh_free(void* p) { delete (OHandle*)p; }

int or_topo_len(void* p, const char* name) {
  OHandle* h = (OHandle*)p;
  auto it = h->topo.find(name);
  return it == h->topo.end() ? -1 : (int)it->second.size();
}
int or_topo_get(void* p, const char* name, int32_t* out) {
  OHandle* h = (OHandle*)p;
  auto it = h->topo.find(name);
  if (it == h->topo.end()) return -1;
  std::memcpy(out, it->second.data(), it->second.size() * sizeof(int32_t));
  return 0;
}
// is_bound after geometry (find_if_vert_is_bound with real normals)
void or_vert_is_bound(void* p, int32_t* out) {
  Mesh& m = ((OHandle*)p)->m;
  for (int i = 1; i <= m.n_vert; ++i) out[i - 1] = m.vert[i].is_bound ? 1 : 0;
}

int or_geometry(void* p, int b2d) {
  Mesh& m = ((OHandle*)p)->m;
  compute_geometry_mesh(m, b2d != 0);
  return m.geometry_ok ? 0 : 1;
}
int or_geometry_ok(void* p) { return ((OHandle*)p)->m.geometry_ok ? 1 : 0; }

void or_set_coords(void* p, const double* c) {
  Mesh& m = ((OHandle*)p)->m;
  for (int i = 1; i <= m.n_vert; ++i)
    for (int d = 1; d <= 3; ++d) m.vert[i].coord[d] = c[3 * (i - 1) + d - 1];
}

// name in {vert_coord, vert_volume, face_coord, face_norm, face_area, sub_face_norm,
//          sub_face_area, elem_coord, elem_volume, sub_elem_volume}
int or_geom_get(void* p, const char* name, double* out) {
  Mesh& m = ((OHandle*)p)->m;
  std::string n(name);
  if (n == "vert_coord") {
    for (int i = 1; i <= m.n_vert; ++i) for (int d = 0; d < 3; ++d) out[3 * (i - 1) + d] = m.vert[i].coord[d + 1];
  } else if (n == "vert_volume") {
    for (int i = 1; i <= m.n_vert; ++i) out[i - 1] = m.vert[i].volume;
  } else if (n == "face_coord") {
    for (int i = 1; i <= m.n_faces; ++i) for (int d = 0; d < 3; ++d) out[3 * (i - 1) + d] = m.face[i].coord[d + 1];
  } else if (n == "face_norm") {
    for (int i = 1; i <= m.n_faces; ++i) for (int d = 0; d < 3; ++d) out[3 * (i - 1) + d] = m.face[i].norm[d + 1];
  } else if (n == "face_area") {
    for (int i = 1; i <= m.n_faces; ++i) out[i - 1] = m.face[i].area;
  } else if (n == "sub_face_norm") {
    for (int i = 1; i <= m.n_sub_faces; ++i) for (int d = 0; d < 3; ++d) out[3 * (i - 1) + d] = m.sub_face[i].norm[d + 1];
  } else if (n == "sub_face_area") {
    for (int i = 1; i <= m.n_sub_faces; ++i) out[i - 1] = m.sub_face[i].area;
  } else if (n == "elem_coord") {
    for (int i = 1; i <= m.n_elems; ++i) for (int d = 0; d < 3; ++d) out[3 * (i - 1) + d] = m.elem[i].coord[d + 1];
  } else if (n == "elem_volume") {
    for (int i = 1; i <= m.n_elems; ++i) out[i - 1] = m.elem[i].volume;
  } else if (n == "sub_elem_volume") {
    for (int i = 1; i <= m.n_sub_elems; ++i) out[i - 1] = m.sub_elem[i].volume;
  } else {
    return -1;
  }
  return 0;
}

void or_lag_rhs(void* p, const double* sol, double* vp, double* rhs, int b2d, const double* mass) {
  compute_rhs_lagrange(((OHandle*)p)->m, sol, vp, rhs, b2d != 0, mass);
}
double or_lag_dt(void* p, const double* sol, double cfl, const double* vp) {
  return compute_dt(((OHandle*)p)->m, sol, cfl, vp);
}
void or_lag_move(void* p, const double* vp, double dt) { move_mesh(((OHandle*)p)->m, vp, dt); }
int or_sedov_init(void* p, double* sol, double r_sedov, double e_total, const int* mask) {
  return init_sedov(((OHandle*)p)->m, sol, r_sedov, e_total, mask);
}
int or_lag_run(void* p, double* sol, double* vp, double* rhs, const double* mass, double cfl,
               double t_max, int max_steps, int b2d, double* t_io, double* last_dt) {
  return lagrange_run(((OHandle*)p)->m, sol, vp, rhs, mass, cfl, t_max, max_steps, b2d != 0, t_io,
                      last_dt, 0, 0);
}
int or_lag_run_scheme(void* p, double* sol, double* vp, double* rhs, const double* mass, double cfl,
                      double t_max, int max_steps, int b2d, double* t_io, double* last_dt, int scheme, int method) {
  return lagrange_run(((OHandle*)p)->m, sol, vp, rhs, mass, cfl, t_max, max_steps, b2d != 0, t_io,
                      last_dt, scheme, method);
}
int or_lag_rhs_sidil(void* p, const double* sol, double* vp, double* rhs, int b2d, const double* mass,
                     int method) {
  return compute_rhs_lagrange_sidil(((OHandle*)p)->m, sol, vp, rhs, b2d != 0, mass, method);
}
void or_inverse_3_by_3(const double* m9, double* inv9) {
  double M[3][3], I[3][3];
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) M[i][j] = m9[3 * i + j];
  inverse_3_by_3(M, I);
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) inv9[3 * i + j] = I[i][j];
}
double or_fnorm2(const double* a, int n) { return fnorm2(a, n); }

}  // extern "C"
