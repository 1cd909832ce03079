// C-ABI entry points (include/subfv.h): topology, device mesh, Lagrangian hydro.
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/subfv.h"
#include "common.cuh"
#include "handles.cuh"
#include "lagrange.cuh"
#include "mesh_dev.cuh"
#include "topology.h"

namespace subfv {
namespace {
thread_local std::string g_err;
}
void set_error(const std::string& msg) { g_err = msg; }
const char* last_error() { return g_err.c_str(); }
}  // namespace subfv

using namespace subfv;

struct subfv_topology {
  Topology t;
};


struct subfv_lag_state {
  subfv_mesh* m = nullptr;
  double* sol6 = nullptr;
  double* rhs6 = nullptr;
  LagScalars* sc = nullptr;
  double* host_stage = nullptr;  // pinned staging for the host-buffer step
  double* dev_stage = nullptr;
  int precision = 0;
  int scheme = 0, method = 0;  // 0 "classic"; 1 "sidil" with method_length
  cudaGraphExec_t graph = nullptr;
  int graph_steps = 0;
  cudaStream_t side = nullptr;  // the host-buffer step's copy back, beside move and geometry
  cudaEvent_t updated = nullptr;
};

namespace subfv {
const DevMesh& mesh_device_view(const subfv_mesh* m) { return m->d; }
}  // namespace subfv

namespace {
int check_status(DevMesh& d);
int clear_status(DevMesh& d);
int ensure_scratch(subfv_mesh* m);
int ensure_full_geometry(DevMesh& d);
int ensure_lag_arrays(DevMesh& d);
}  // namespace

namespace subfv {
int handle_check_status(DevMesh& d) { return check_status(d); }
int handle_clear_status(DevMesh& d) { return clear_status(d); }
int handle_ensure_scratch(subfv_mesh* m) { return ensure_scratch(m); }
int handle_ensure_full_geometry(DevMesh& d) { return ensure_full_geometry(d); }
int handle_ensure_lag_arrays(DevMesh& d) { return ensure_lag_arrays(d); }
}  // namespace subfv

namespace {

int check_status(DevMesh& d) {
  unsigned st = 0;
  SUBFV_CUDA(cudaMemcpyAsync(&st, d.status, sizeof(unsigned), cudaMemcpyDeviceToHost, d.stream));
  SUBFV_CUDA(cudaStreamSynchronize(d.stream));
  return (int)st;
}
int clear_status(DevMesh& d) {
  SUBFV_CUDA(cudaMemsetAsync(d.status, 0, sizeof(unsigned), d.stream));
  return 0;
}
int ensure_scratch(subfv_mesh* m) {
  if (m->stage) return 0;
  size_t n = std::max<size_t>(5 * (size_t)m->d.ne, 3 * (size_t)m->d.nv);
  SUBFV_CUDA(cudaMalloc(&m->stage, n * sizeof(double)));
  SUBFV_CUDA(cudaMalloc(&m->sol6, kRec * (size_t)m->d.ne * sizeof(double)));
  SUBFV_CUDA(cudaMalloc(&m->rhs6, 6 * (size_t)m->d.ne * sizeof(double)));
  SUBFV_CUDA(cudaMalloc(&m->mass, (size_t)m->d.ne * sizeof(double)));
  SUBFV_CUDA(cudaMalloc(&m->sc, sizeof(LagScalars)));
  return ensure_lag_arrays(m->d);
}
// The Lagrangian step's per-mesh arrays (face records, cell entries, face subface sums),
// stream-ordered on the mesh's stream and released with the mesh.
int ensure_lag_arrays(DevMesh& d) {
  if (d.frec) return 0;
  SUBFV_CUDA(cudaMallocAsync((void**)&d.frec, 6 * (size_t)d.nf * sizeof(double), d.stream));
  SUBFV_CUDA(cudaMallocAsync((void**)&d.centry, std::max<size_t>(d.ncsf, 1) * sizeof(int4), d.stream));
  SUBFV_CUDA(cudaMallocAsync((void**)&d.fS, (size_t)d.nf * sizeof(double4), d.stream));
  SUBFV_CUDA(cudaMallocAsync((void**)&d.gface, 8 * (size_t)d.ne * sizeof(uint16_t), d.stream));
  SUBFV_CUDA(cudaMallocAsync((void**)&d.gsub, (size_t)d.nse * sizeof(uint32_t), d.stream));
  d.bytes += 6 * (size_t)d.nf * sizeof(double) + std::max<size_t>(d.ncsf, 1) * sizeof(int4) +
             (size_t)d.nf * sizeof(double4) + 8 * (size_t)d.ne * sizeof(uint16_t) + (size_t)d.nse * sizeof(uint32_t);
  launch_build_cell_entries(d);
  launch_build_geom_codes(d);
  SUBFV_CUDA(cudaGetLastError());
  return 0;
}
// After Lagrangian steps (which refresh only what the next step reads), recompute every
// geometric array from the current coordinates; check_mesh's verdict on this geometry
// was already reported by the step that produced it.
int ensure_full_geometry(DevMesh& d) {
  if (!d.geom_partial) return 0;
  launch_geometry(d, 1);
  launch_vert_is_bound(d);
  launch_vert_volume(d);
  SUBFV_CUDA(cudaStreamSynchronize(d.stream));
  SUBFV_CUDA(cudaGetLastError());
  d.geom_partial = 0;
  return 0;
}
int load_sol(subfv_mesh* m, const double* sol, const double* mass) {
  DevMesh& d = m->d;
  SUBFV_CUDA(cudaMemcpyAsync(m->stage, sol, 5 * (size_t)d.ne * sizeof(double), cudaMemcpyHostToDevice, d.stream));
  if (mass) SUBFV_CUDA(cudaMemcpyAsync(m->mass, mass, (size_t)d.ne * sizeof(double), cudaMemcpyHostToDevice, d.stream));
  launch_pack6(d, d.ne, m->stage, mass ? m->mass : nullptr, m->sol6);
  return 0;
}

}  // namespace

extern "C" {

const char* subfv_last_error(void) { return subfv::last_error(); }
int subfv_version(void) { return 1; }

// ------------------------------------------------------------------- topology
int subfv_topology_build(int n_vert, const double* coords, int n_elems, const int32_t* elem_kind,
                         const int32_t* elem_vert_off, const int32_t* elem_vert, int n_bfaces,
                         const int32_t* bface_off, const int32_t* bface_vert, const int32_t* bface_tag,
                         int b2d, int periodic, subfv_topology** out) {
  return subfv_topology_build_ex(n_vert, coords, n_elems, elem_kind, elem_vert_off, elem_vert, n_bfaces, bface_off,
                                 bface_vert, bface_tag, b2d, periodic, 0, out);
}
int subfv_topology_build_ex(int n_vert, const double* coords, int n_elems, const int32_t* elem_kind,
                            const int32_t* elem_vert_off, const int32_t* elem_vert, int n_bfaces,
                            const int32_t* bface_off, const int32_t* bface_vert, const int32_t* bface_tag,
                            int b2d, int periodic, int renumber, subfv_topology** out) {
  if (!out || !coords || !elem_kind || !elem_vert_off || !elem_vert) {
    set_error("subfv_topology_build: null argument");
    return -2;
  }
  if (renumber != 0 && renumber != 1) {
    set_error("subfv_topology_build_ex: renumber must be 0 (breadth-first) or 1 (Hilbert curve)");
    return -2;
  }
  RawMeshView in{n_vert, coords, n_elems, elem_kind, elem_vert_off, elem_vert,
                 n_bfaces, bface_off, bface_vert, bface_tag, b2d, periodic, renumber};
  auto* t = new subfv_topology();
  std::string err;
  int rc = build_topology(in, t->t, &err);
  if (rc) {
    delete t;
    set_error("subfv_topology_build: " + err);
    return -3;
  }
  *out = t;
  return 0;
}
int64_t subfv_topology_array_len(const subfv_topology* t, const char* name) {
  auto it = t->t.arr.find(name);
  return it == t->t.arr.end() ? -1 : (int64_t)it->second.size();
}
int subfv_topology_array_get(const subfv_topology* t, const char* name, int32_t* out) {
  auto it = t->t.arr.find(name);
  if (it == t->t.arr.end()) {
    set_error(std::string("unknown topology array ") + name);
    return -2;
  }
  std::memcpy(out, it->second.data(), it->second.size() * sizeof(int32_t));
  return 0;
}
int subfv_topology_coords(const subfv_topology* t, double* out) {
  std::memcpy(out, t->t.vert_coord.data(), t->t.vert_coord.size() * sizeof(double));
  return 0;
}
void subfv_topology_destroy(subfv_topology* t) { delete t; }

// ------------------------------------------------------------------- mesh
int subfv_mesh_create(const subfv_mesh_desc* desc, subfv_mesh** out) {
  if (!desc || !out) {
    set_error("subfv_mesh_create: null argument");
    return -2;
  }
  auto* m = new subfv_mesh();
  int rc = devmesh_create(desc, &m->d);
  if (rc) {
    devmesh_free(&m->d);
    delete m;
    return rc;
  }
  *out = m;
  return 0;
}

int subfv_mesh_create_from_topology(const subfv_topology* tp, int b2d, subfv_mesh** out) {
  const Topology& t = tp->t;
  subfv_mesh_desc d{};
  d.n_vert = t.n_vert;
  d.n_elems = t.n_elems;
  d.n_faces = t.n_faces;
  d.n_sub_faces = t.n_sub_faces;
  d.n_sub_elems = t.n_sub_elems;
  d.b2d = b2d;
  d.vert_coord = t.vert_coord.data();
  d.elem_kind = t.a("elem_kind").data();
  d.elem_vert_off = t.a("elem_vert_off").data();
  d.elem_vert = t.a("elem_vert").data();
  d.elem_sub_elem = t.a("elem_sub_elem").data();
  d.elem_face_off = t.a("elem_face_off").data();
  d.elem_face = t.a("elem_face").data();
  d.face_vert_off = t.a("face_vert_off").data();
  d.face_vert = t.a("face_vert").data();
  d.face_sub_face = t.a("face_sub_face").data();
  d.face_left = t.a("face_left").data();
  d.face_right = t.a("face_right").data();
  d.sub_face_vert = t.a("sub_face_vert").data();
  d.sub_face_face = t.a("sub_face_face").data();
  d.sub_face_left_sub_elem = t.a("sub_face_left_sub_elem").data();
  d.sub_face_right_sub_elem = t.a("sub_face_right_sub_elem").data();
  d.sub_face_loc = t.a("sub_face_loc").data();
  d.sub_elem_elem = t.a("sub_elem_elem").data();
  d.sub_elem_vert = t.a("sub_elem_vert").data();
  d.sub_elem_loc = t.a("sub_elem_loc").data();
  d.sub_elem_sub_face_off = t.a("sub_elem_sub_face_off").data();
  d.sub_elem_sub_face = t.a("sub_elem_sub_face").data();
  d.vert_sub_face_off = t.a("vert_sub_face_off").data();
  d.vert_sub_face = t.a("vert_sub_face").data();
  d.vert_sub_elem_off = t.a("vert_sub_elem_off").data();
  d.vert_sub_elem = t.a("vert_sub_elem").data();
  d.vert_is_bound = t.a("vert_is_bound").data();
  d.vert_elem_off = t.a("vert_elem_off").data();
  d.vert_elem = t.a("vert_elem").data();
  return subfv_mesh_create(&d, out);
}

int subfv_mesh_destroy(subfv_mesh* m) {
  if (!m) return 0;
  // scratch of the stateless calls (allocated on first use only); a mesh that never
  // needed it is released without any device-wide synchronisation
  void* scratch[] = {m->stage, m->sol6, m->rhs6, m->mass, m->sc};
  for (void* p : scratch)
    if (p) cudaFree(p);
  if (m->imp_pattern && m->imp_pattern_free) m->imp_pattern_free(m->imp_pattern);
  devmesh_free(&m->d);
  delete m;
  return 0;
}

int64_t subfv_mesh_device_bytes(const subfv_mesh* m) { return (int64_t)m->d.bytes; }

int subfv_mesh_set_coords(subfv_mesh* m, const double* c) {
  DevMesh& d = m->d;
  std::vector<double4> x(d.nv);
  for (int i = 0; i < d.nv; ++i) x[i] = make_double4(c[3 * i], c[3 * i + 1], c[3 * i + 2], 0.0);
  SUBFV_CUDA(cudaMemcpyAsync(d.x, x.data(), x.size() * sizeof(double4), cudaMemcpyHostToDevice, d.stream));
  SUBFV_CUDA(cudaStreamSynchronize(d.stream));
  ++d.geom_epoch;
  return 0;
}
int subfv_mesh_get_coords(subfv_mesh* m, double* c) {
  DevMesh& d = m->d;
  std::vector<double4> x(d.nv);
  SUBFV_CUDA(cudaMemcpyAsync(x.data(), d.x, x.size() * sizeof(double4), cudaMemcpyDeviceToHost, d.stream));
  SUBFV_CUDA(cudaStreamSynchronize(d.stream));
  for (int i = 0; i < d.nv; ++i) {
    c[3 * i] = x[i].x;
    c[3 * i + 1] = x[i].y;
    c[3 * i + 2] = x[i].z;
  }
  return 0;
}

int subfv_mesh_get_geometry(subfv_mesh* m, const char* name, double* out) {
  DevMesh& d = m->d;
  if (ensure_full_geometry(d)) return -1;
  std::string n(name);
  auto get4 = [&](const double4* src, int cnt, int ncomp, int first) -> int {
    std::vector<double4> h(cnt);
    SUBFV_CUDA(cudaMemcpyAsync(h.data(), src, cnt * sizeof(double4), cudaMemcpyDeviceToHost, d.stream));
    SUBFV_CUDA(cudaStreamSynchronize(d.stream));
    for (int i = 0; i < cnt; ++i) {
      const double v[4] = {h[i].x, h[i].y, h[i].z, h[i].w};
      for (int k = 0; k < ncomp; ++k) out[(size_t)ncomp * i + k] = v[first + k];
    }
    return 0;
  };
  auto get1 = [&](const double* src, int cnt) -> int {
    SUBFV_CUDA(cudaMemcpyAsync(out, src, cnt * sizeof(double), cudaMemcpyDeviceToHost, d.stream));
    SUBFV_CUDA(cudaStreamSynchronize(d.stream));
    return 0;
  };
  if (n == "face_coord") return get4(d.fc, d.nf, 3, 0);
  if (n == "face_norm") return get4(d.fn, d.nf, 3, 0);
  if (n == "face_area") return get4(d.fn, d.nf, 1, 3);
  if (n == "sub_face_norm") return get4(d.sfn, d.nsf, 3, 0);
  if (n == "sub_face_area") return get4(d.sfn, d.nsf, 1, 3);
  if (n == "elem_coord") return get4(d.cc, d.ne, 3, 0);
  if (n == "elem_volume") return get1(d.vol, d.ne);
  if (n == "sub_elem_volume") return get1(d.vol_se, d.nse);
  if (n == "vert_volume") return get1(d.vol_v, d.nv);
  if (n == "vert_is_bound") {
    std::vector<int8_t> h(d.nv);
    SUBFV_CUDA(cudaMemcpyAsync(h.data(), d.is_bound, d.nv, cudaMemcpyDeviceToHost, d.stream));
    SUBFV_CUDA(cudaStreamSynchronize(d.stream));
    for (int i = 0; i < d.nv; ++i) out[i] = h[i];
    return 0;
  }
  set_error("subfv_mesh_get_geometry: unknown array " + n);
  return -2;
}

int subfv_compute_geometry_mesh(subfv_mesh* m) {
  DevMesh& d = m->d;
  ++d.geom_epoch;
  if (clear_status(d)) return -1;
  launch_geometry(d, 1);
  launch_vert_is_bound(d);
  launch_vert_volume(d);
  SUBFV_CUDA(cudaGetLastError());
  d.geom_partial = 0;
  return check_status(d);
}

// ------------------------------------------------------------------- Lagrange (stateless)
int subfv_compute_rhs_lagrange(subfv_mesh* m, const double* sol, double* vp, double* rhs, int b2d,
                               const double* mass) {
  DevMesh& d = m->d;
  if (ensure_scratch(m) || clear_status(d)) return -1;
  d.b2d = b2d;
  if (load_sol(m, sol, mass)) return -1;
  launch_lag_node(d, m->sol6, nullptr, 0);
  launch_lag_cell(d, m->sol6, m->rhs6, nullptr, nullptr, 0, 1);
  launch_unpack6(d, d.ne, kRhs, m->rhs6, m->stage);
  SUBFV_CUDA(cudaMemcpyAsync(rhs, m->stage, 5 * (size_t)d.ne * sizeof(double), cudaMemcpyDeviceToHost, d.stream));
  std::vector<double4> h(d.nv);
  SUBFV_CUDA(cudaMemcpyAsync(h.data(), d.vp, d.nv * sizeof(double4), cudaMemcpyDeviceToHost, d.stream));
  SUBFV_CUDA(cudaStreamSynchronize(d.stream));
  for (int i = 0; i < d.nv; ++i) {
    vp[3 * i] = h[i].x;
    vp[3 * i + 1] = h[i].y;
    vp[3 * i + 2] = h[i].z;
  }
  SUBFV_CUDA(cudaGetLastError());
  return check_status(d);
}

int subfv_compute_rhs_lagrange_sidil(subfv_mesh* m, const double* sol, double* vp, double* rhs, int b2d,
                                     const double* mass, int method_length) {
  if (!m || !sol || !vp || !rhs || !mass || method_length < 0 || method_length > 4) {
    set_error("subfv_compute_rhs_lagrange_sidil: null argument or method_length outside 0..4");
    return -2;
  }
  DevMesh& d = m->d;
  if (ensure_scratch(m) || ensure_full_geometry(d) || clear_status(d)) return -1;
  d.b2d = b2d;
  if (load_sol(m, sol, mass)) return -1;
  launch_lag_sidil_node(d, m->sol6, nullptr, method_length);
  launch_lag_cell(d, m->sol6, m->rhs6, nullptr, nullptr, 0, 5);
  launch_unpack6(d, d.ne, kRhs, m->rhs6, m->stage);
  SUBFV_CUDA(cudaMemcpyAsync(rhs, m->stage, 5 * (size_t)d.ne * sizeof(double), cudaMemcpyDeviceToHost, d.stream));
  std::vector<double4> h(d.nv);
  SUBFV_CUDA(cudaMemcpyAsync(h.data(), d.vp, d.nv * sizeof(double4), cudaMemcpyDeviceToHost, d.stream));
  SUBFV_CUDA(cudaStreamSynchronize(d.stream));
  for (int i = 0; i < d.nv; ++i) {
    vp[3 * i] = h[i].x;
    vp[3 * i + 1] = h[i].y;
    vp[3 * i + 2] = h[i].z;
  }
  SUBFV_CUDA(cudaGetLastError());
  return check_status(d);
}

int subfv_lag_state_set_scheme(subfv_lag_state* s, int scheme, int method_length) {
  if (!s || scheme < 0 || scheme > 1 || method_length < 0 || method_length > 4) {
    set_error("subfv_lag_state_set_scheme: scheme 0 (classic) or 1 (sidil), method_length 0..4");
    return -2;
  }
  if (s->scheme != scheme || s->method != method_length) {
    s->scheme = scheme;
    s->method = method_length;
    if (s->graph) {  // the captured step loop holds the old scheme
      SUBFV_CUDA(cudaStreamSynchronize(s->m->d.stream));
      cudaGraphExecDestroy(s->graph);
      s->graph = nullptr;
      s->graph_steps = 0;
    }
  }
  return 0;
}

int subfv_compute_dt(subfv_mesh* m, const double* sol, double cfl, const double* vp, double* dt) {
  DevMesh& d = m->d;
  if (ensure_scratch(m) || clear_status(d)) return -1;
  if (load_sol(m, sol, nullptr)) return -1;
  SUBFV_CUDA(cudaMemcpyAsync(m->stage, vp, 3 * (size_t)d.nv * sizeof(double), cudaMemcpyHostToDevice, d.stream));
  launch_vp_in(d, m->stage);
  double* slot = &m->sc->dtmin;
  launch_set_scalar(d, slot, 1e6);
  launch_lag_cell(d, m->sol6, nullptr, nullptr, slot, 0, 2);
  double h = 0;
  SUBFV_CUDA(cudaMemcpyAsync(&h, slot, sizeof(double), cudaMemcpyDeviceToHost, d.stream));
  SUBFV_CUDA(cudaStreamSynchronize(d.stream));
  SUBFV_CUDA(cudaGetLastError());
  *dt = cfl * h;
  return check_status(d);
}

int subfv_move_mesh(subfv_mesh* m, const double* vp, double dt) {
  DevMesh& d = m->d;
  ++d.geom_epoch;
  if (ensure_scratch(m)) return -1;
  SUBFV_CUDA(cudaMemcpyAsync(m->stage, vp, 3 * (size_t)d.nv * sizeof(double), cudaMemcpyHostToDevice, d.stream));
  launch_vp_in(d, m->stage);
  launch_lag_move(d, nullptr, dt);
  SUBFV_CUDA(cudaStreamSynchronize(d.stream));
  SUBFV_CUDA(cudaGetLastError());
  return 0;
}

// ------------------------------------------------------------------- Lagrange (device-resident)
int subfv_lag_state_create(subfv_mesh* m, const double* sol, const double* mass, double cfl, double t0,
                           double t_max, int precision, subfv_lag_state** out) {
  if (!m || !sol || !mass || !out || (precision != 0 && precision != 1)) {
    set_error("subfv_lag_state_create: bad argument");
    return -2;
  }
  DevMesh& d = m->d;
  d.moving = 1;
  if (ensure_scratch(m)) return -1;
  auto* s = new subfv_lag_state();
  s->m = m;
  s->precision = precision;
  SUBFV_CUDA(cudaMalloc(&s->sol6, kRec * (size_t)d.ne * sizeof(double)));
  SUBFV_CUDA(cudaMalloc(&s->rhs6, 6 * (size_t)d.ne * sizeof(double)));
  SUBFV_CUDA(cudaMalloc(&s->sc, sizeof(LagScalars)));
  SUBFV_CUDA(cudaMallocHost(&s->host_stage, 5 * (size_t)d.ne * sizeof(double)));
  SUBFV_CUDA(cudaMalloc(&s->dev_stage, 5 * (size_t)d.ne * sizeof(double)));
  SUBFV_CUDA(cudaMemsetAsync(s->rhs6, 0, 6 * (size_t)d.ne * sizeof(double), d.stream));
  LagScalars h{};
  h.dtmin = 1e6;
  h.t = t0;
  h.t_max = t_max;
  h.cfl = cfl;
  h.done = (t0 < t_max) ? 0 : 1;
  SUBFV_CUDA(cudaMemcpyAsync(s->sc, &h, sizeof(h), cudaMemcpyHostToDevice, d.stream));
  SUBFV_CUDA(cudaMemcpyAsync(s->dev_stage, sol, 5 * (size_t)d.ne * sizeof(double), cudaMemcpyHostToDevice, d.stream));
  SUBFV_CUDA(cudaMemcpyAsync(m->mass, mass, (size_t)d.ne * sizeof(double), cudaMemcpyHostToDevice, d.stream));
  launch_pack6(d, d.ne, s->dev_stage, m->mass, s->sol6);
  SUBFV_CUDA(cudaStreamSynchronize(d.stream));
  SUBFV_CUDA(cudaGetLastError());
  *out = s;
  return 0;
}

int subfv_lag_state_destroy(subfv_lag_state* s) {
  if (!s) return 0;
  if (s->graph) cudaGraphExecDestroy(s->graph);
  if (s->updated) cudaEventDestroy(s->updated);
  if (s->side) cudaStreamDestroy(s->side);
  cudaFree(s->sol6);
  cudaFree(s->rhs6);
  cudaFree(s->sc);
  cudaFree(s->dev_stage);
  cudaFreeHost(s->host_stage);
  delete s;
  return 0;
}

namespace {
// Captures `steps` consecutive steps into one graph (reused while `steps` is unchanged).
int lag_graph(subfv_lag_state* s, int steps) {
  if (s->graph && s->graph_steps == steps) return 0;
  if (s->graph) {
    cudaGraphExecDestroy(s->graph);
    s->graph = nullptr;
  }
  DevMesh& d = s->m->d;
  cudaGraph_t g;
  SUBFV_CUDA(cudaStreamBeginCapture(d.stream, cudaStreamCaptureModeThreadLocal));
  for (int i = 0; i < steps; ++i) enqueue_lag_step(d, s->sol6, s->rhs6, s->sc, s->precision, s->scheme, s->method);
  SUBFV_CUDA(cudaStreamEndCapture(d.stream, &g));
  cudaError_t e = cudaGraphInstantiate(&s->graph, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    set_error(std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
    return -1;
  }
  s->graph_steps = steps;
  return 0;
}
}  // namespace

constexpr int kLagGraphSteps = 16;  // steps per captured graph

int subfv_lag_prepare(subfv_lag_state* s) {
  if (!s) return -2;
  return lag_graph(s, kLagGraphSteps) ? -1 : 0;
}

int subfv_lag_advance_async(subfv_lag_state* s, int n_steps) {
  DevMesh& d = s->m->d;
  if (n_steps > 0) d.geom_partial = 1;
  const int chunk = kLagGraphSteps;
  if (n_steps >= chunk) {
    if (lag_graph(s, chunk)) return -1;
    for (int i = 0; i + chunk <= n_steps; i += chunk) SUBFV_CUDA(cudaGraphLaunch(s->graph, d.stream));
  }
  for (int i = 0; i < n_steps % chunk; ++i)
    enqueue_lag_step(d, s->sol6, s->rhs6, s->sc, s->precision, s->scheme, s->method);
  SUBFV_CUDA(cudaGetLastError());
  return 0;
}

int subfv_lag_sync(subfv_lag_state* s, int* steps_done, double* t) {
  DevMesh& d = s->m->d;
  LagScalars h{};
  SUBFV_CUDA(cudaMemcpyAsync(&h, s->sc, sizeof(h), cudaMemcpyDeviceToHost, d.stream));
  int st = check_status(d);
  if (st < 0) return st;
  if (steps_done) *steps_done = (int)h.steps;
  if (t) *t = h.t;
  return st;
}

int subfv_lag_advance(subfv_lag_state* s, int n_steps, int* steps_done, double* t) {
  if (subfv_lag_advance_async(s, n_steps)) return -1;
  return subfv_lag_sync(s, steps_done, t);
}

int subfv_lag_get_sol(subfv_lag_state* s, double* sol) {
  DevMesh& d = s->m->d;
  launch_unpack6(d, d.ne, kRec, s->sol6, s->dev_stage);
  SUBFV_CUDA(cudaMemcpyAsync(sol, s->dev_stage, 5 * (size_t)d.ne * sizeof(double), cudaMemcpyDeviceToHost, d.stream));
  SUBFV_CUDA(cudaStreamSynchronize(d.stream));
  return 0;
}
int subfv_lag_set_sol(subfv_lag_state* s, const double* sol) {
  DevMesh& d = s->m->d;
  SUBFV_CUDA(cudaMemcpyAsync(s->dev_stage, sol, 5 * (size_t)d.ne * sizeof(double), cudaMemcpyHostToDevice, d.stream));
  launch_pack6(d, d.ne, s->dev_stage, nullptr, s->sol6);
  SUBFV_CUDA(cudaStreamSynchronize(d.stream));
  return 0;
}
int subfv_lag_get_vp(subfv_lag_state* s, double* vp) {
  DevMesh& d = s->m->d;
  std::vector<double4> h(d.nv);
  SUBFV_CUDA(cudaMemcpyAsync(h.data(), d.vp, d.nv * sizeof(double4), cudaMemcpyDeviceToHost, d.stream));
  SUBFV_CUDA(cudaStreamSynchronize(d.stream));
  for (int i = 0; i < d.nv; ++i) {
    vp[3 * i] = h[i].x;
    vp[3 * i + 1] = h[i].y;
    vp[3 * i + 2] = h[i].z;
  }
  return 0;
}
int subfv_lag_last_dt(subfv_lag_state* s, double* dt) {
  DevMesh& d = s->m->d;
  LagScalars h{};
  SUBFV_CUDA(cudaMemcpyAsync(&h, s->sc, sizeof(h), cudaMemcpyDeviceToHost, d.stream));
  SUBFV_CUDA(cudaStreamSynchronize(d.stream));
  *dt = h.dt;
  return 0;
}

// Host-buffer step: pinned staging, one H2D of the state, one step, one D2H.
int subfv_lag_step_host(subfv_lag_state* s, double* sol_inout) {
  DevMesh& d = s->m->d;
  size_t bytes = 5 * (size_t)d.ne * sizeof(double);
  // a page-locked caller buffer is copied to and from directly; a pageable one goes
  // through the state's pinned staging buffer
  cudaPointerAttributes attr{};
  const bool pinned = cudaPointerGetAttributes(&attr, sol_inout) == cudaSuccess && attr.type == cudaMemoryTypeHost;
  cudaGetLastError();  // a pageable pointer is not an error here
  double* hbuf = pinned ? sol_inout : s->host_stage;
  if (!pinned) std::memcpy(s->host_stage, sol_inout, bytes);
  if (!s->side) {
    SUBFV_CUDA(cudaStreamCreateWithFlags(&s->side, cudaStreamNonBlocking));
    SUBFV_CUDA(cudaEventCreateWithFlags(&s->updated, cudaEventDisableTiming));
  }
  SUBFV_CUDA(cudaMemcpyAsync(s->dev_stage, hbuf, bytes, cudaMemcpyHostToDevice, d.stream));
  launch_pack6(d, d.ne, s->dev_stage, nullptr, s->sol6);
  // the state is final once updated: its copy back runs on the side stream while the
  // main stream moves the mesh and recomputes the geometry (which read neither sol6 nor
  // the staging buffer)
  enqueue_lag_step_head(d, s->sol6, s->rhs6, s->sc, s->precision, s->scheme, s->method);
  launch_lag_update(d, s->sol6, s->rhs6, s->sc);
  SUBFV_CUDA(cudaEventRecord(s->updated, d.stream));
  SUBFV_CUDA(cudaStreamWaitEvent(s->side, s->updated, 0));
  DevMesh ds = d;
  ds.stream = s->side;
  launch_unpack6(ds, d.ne, kRec, s->sol6, s->dev_stage);
  SUBFV_CUDA(cudaMemcpyAsync(hbuf, s->dev_stage, bytes, cudaMemcpyDeviceToHost, s->side));
  launch_lag_move(d, s->sc, 0.0);
  launch_geometry(d, 0, nullptr, nullptr, s->sc);
  d.geom_partial = 1;
  SUBFV_CUDA(cudaStreamSynchronize(s->side));
  SUBFV_CUDA(cudaStreamSynchronize(d.stream));
  if (!pinned) std::memcpy(sol_inout, s->host_stage, bytes);
  return check_status(d);
}

}  // extern "C"

extern "C" {

void* subfv_mesh_stream(subfv_mesh* m) { return (void*)m->d.stream; }

int subfv_lag_profile_steps(subfv_lag_state* s, int n_steps, double* kernel_ms) {
  DevMesh& d = s->m->d;
  const int K = 7;
  cudaEvent_t ev[K + 1];
  for (int k = 0; k <= K; ++k) SUBFV_CUDA(cudaEventCreate(&ev[k]));
  for (int k = 0; k < K; ++k) kernel_ms[k] = 0.0;
  for (int i = 0; i < n_steps; ++i) {
    SUBFV_CUDA(cudaEventRecord(ev[0], d.stream));
    launch_lag_face_only(d, s->sol6, s->sc, s->precision);
    SUBFV_CUDA(cudaEventRecord(ev[1], d.stream));
    launch_lag_node_only(d, s->sc, s->precision);
    SUBFV_CUDA(cudaEventRecord(ev[2], d.stream));
    launch_lag_cell(d, s->sol6, s->rhs6, s->sc, &s->sc->dtmin, s->precision, 3);
    SUBFV_CUDA(cudaEventRecord(ev[3], d.stream));
    launch_lag_finalize(d, s->sc);
    SUBFV_CUDA(cudaEventRecord(ev[4], d.stream));
    launch_lag_move(d, s->sc, 0.0);
    SUBFV_CUDA(cudaEventRecord(ev[5], d.stream));
    launch_face_geometry_step(d, s->sc);
    SUBFV_CUDA(cudaEventRecord(ev[6], d.stream));
    launch_cell_geometry_step(d, s->sol6, s->rhs6, s->sc);
    SUBFV_CUDA(cudaEventRecord(ev[7], d.stream));
    SUBFV_CUDA(cudaEventSynchronize(ev[7]));
    for (int k = 0; k < K; ++k) {
      float ms = 0.f;
      SUBFV_CUDA(cudaEventElapsedTime(&ms, ev[k], ev[k + 1]));
      kernel_ms[k] += ms;
    }
  }
  for (int k = 0; k <= K; ++k) cudaEventDestroy(ev[k]);
  SUBFV_CUDA(cudaGetLastError());
  return check_status(d);
}

}  // extern "C"
