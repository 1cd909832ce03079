// C-ABI of the explicit Euler path (include/subfv.h, subfv_ns_*).
#include <cmath>
#include <cstring>
#include <vector>

#include <algorithm>

#include "bcsr.cuh"
#include "handles.cuh"
#include "ns.cuh"
#include "ns_diffusion.cuh"

using namespace subfv;

// Backward-Euler context: the Jacobian's BCSR pattern on the mesh's cell adjacency and
// the GMRES workspace.
struct ImplicitCtx {
  DevBcsr A;
  GmresWork W;
  int *jq_off = nullptr, *jq = nullptr, *jblk = nullptr, *row_off = nullptr, *dblk = nullptr;
  double *b = nullptr, *x = nullptr;
  double* ddiag = nullptr;      // the diffusion blocks (25 per cell) when the state has diffusion
  std::vector<int> row1, col1;  // 1-based pattern (bcsr_matrix_type)
  int krylov = 0;
};

struct subfv_ns_state {
  subfv_mesh* m = nullptr;
  NsParams P{};
  double *U0 = nullptr, *U1 = nullptr, *fs = nullptr, *rhs1 = nullptr, *rhs2 = nullptr;
  double *ngrad = nullptr, *grad = nullptr, *delta = nullptr, *partial = nullptr, *stage = nullptr;
  NsScalars* sc = nullptr;
  cudaGraphExec_t graph = nullptr;
  int graph_steps = 0;
  ImplicitCtx* imp = nullptr;
  DiffParams D{};                                // diffusion parameters (P.diff)
  double *dterm = nullptr, *mu0c = nullptr;      // corner records, mu0corr
  unsigned long long seen_epoch = 0;             // the mesh geometry the state last ran on
  int geom_seen = 0;
};

namespace {

constexpr int kSmallMeshVertices = 32768;

int check_cfg(const subfv_ns_cfg* c) {
  if (!c || (c->scheme < 1 || c->scheme > 8 || c->scheme == 7) || (c->method < 0 || c->method > 6) ||
      c->local_time_step != 0 || c->n_bc < 0 || c->n_bc > 16 || (c->precision < 0 || c->precision > 2)) {
    set_error("subfv_ns: unsupported configuration (scheme 1-6 or 8, method 0-6, global time step, n_bc <= 16)");
    return -2;
  }
  // compute_right_state's select case stops on a kind it does not know
  for (int i = 0; i < c->n_bc; ++i)
    if (c->bc_type[i] < 1 || c->bc_type[i] > 9) {
      set_error("subfv_ns: boundary kind not recognized (1-9)");
      return -2;
    }
  if (c->activate_diffusion) {  // bc_type_V / bc_type_T: "" or neumann, dirichlet
    for (int i = 0; i < c->n_bc; ++i)
      if (c->bc_type_V[i] < 0 || c->bc_type_V[i] > 2 || c->bc_type_T[i] < 0 || c->bc_type_T[i] > 2) {
        set_error("subfv_ns: diffusion boundary kind not recognized (0/1 neumann, 2 dirichlet)");
        return -2;
      }
    if (!(c->Cv_p > 0.0) || !(c->mu_p >= 0.0) || (c->use_sutherland && !(c->mu0 > 0.0 && c->T0 > 0.0)) ||
        !(c->prandtl >= 0.0)) {
      set_error("subfv_ns: diffusion parameters out of range");
      return -2;
    }
  }
  return 0;
}

// zeroed on the stream that later fills the buffer (the mesh's non-blocking stream does
// not order against the legacy default stream)
template <class T>
int dalloc(T** p, size_t n, cudaStream_t s) {
  SUBFV_CUDA(cudaMalloc((void**)p, std::max<size_t>(n, 1) * sizeof(T)));
  SUBFV_CUDA(cudaMemsetAsync(*p, 0, std::max<size_t>(n, 1) * sizeof(T), s));
  return 0;
}

// One iteration of ns_main.F90:83-107 (graph-capturable).
void enqueue_ns_step(subfv_ns_state* s) {
  const DevMesh& d = s->m->d;
  const NsParams& P = s->P;
  auto rhs = [&](const double* U) {
    launch_ns_rhs(d, P, U, s->fs, s->rhs1, s->rhs2, s->ngrad, s->grad, s->sc);
    if (P.diff) launch_ns_diffusion(d, s->D, U, s->dterm, s->mu0c);
  };
  if (P.second_order) {
    rhs(s->U0);
    launch_ns_timedisc(d, P, s->U0, s->rhs1, s->rhs2, s->U0, s->U1, s->delta, s->partial, s->sc, 2.0, 1.0, 0,
                       s->dterm);
    rhs(s->U1);
    launch_ns_timedisc(d, P, s->U1, s->rhs1, s->rhs2, s->U0, s->U0, s->delta, s->partial, s->sc, 1.0, 1.0, 1,
                       s->dterm);
  } else {
    rhs(s->U0);
    launch_ns_timedisc(d, P, s->U0, s->rhs1, nullptr, s->U0, s->U0, s->delta, s->partial, s->sc, 1.0, 1.0, 1,
                       s->dterm);
  }
}

// The caches that belong to the mesh geometry (the nodal-gradient pseudo-inverses, the
// diffusion arrays) are filled for the state's first steps and refilled once the mesh's
// geometry has changed since the state last ran; the captured step loop, which holds the
// kernels chosen for the old caches, is then dropped.
int ns_sync_geometry(subfv_ns_state* s) {
  DevMesh& d = s->m->d;
  if (s->geom_seen && s->seen_epoch == d.geom_epoch) return 0;
  if (s->P.second_order && ensure_nodal_pinv(&d)) return -1;
  if (s->geom_seen && s->P.diff && diffusion_cache_build(&d, s->D, s->U0, s->dterm, s->mu0c)) return -1;
  if (s->graph) {
    SUBFV_CUDA(cudaStreamSynchronize(d.stream));
    cudaGraphExecDestroy(s->graph);
    s->graph = nullptr;
    s->graph_steps = 0;
  }
  s->seen_epoch = d.geom_epoch;
  s->geom_seen = 1;
  return 0;
}

int ns_graph(subfv_ns_state* s, int steps) {
  if (ns_sync_geometry(s)) return -1;
  if (s->graph && s->graph_steps == steps) return 0;
  if (s->graph) {
    cudaGraphExecDestroy(s->graph);
    s->graph = nullptr;
  }
  DevMesh& d = s->m->d;
  cudaGraph_t g;
  SUBFV_CUDA(cudaStreamBeginCapture(d.stream, cudaStreamCaptureModeThreadLocal));
  for (int i = 0; i < steps; ++i) enqueue_ns_step(s);
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

extern "C" {

int subfv_ns_init_gresho(subfv_mesh* m, double mach, double* sol) {
  DevMesh& d = m->d;
  std::vector<double4> cc(d.ne);
  SUBFV_CUDA(cudaMemcpyAsync(cc.data(), d.cc, d.ne * sizeof(double4), cudaMemcpyDeviceToHost, d.stream));
  SUBFV_CUDA(cudaStreamSynchronize(d.stream));
  const double G = 1.4;
  for (int i = 0; i < d.ne; ++i) {
    const double x0 = cc[i].x, x1 = cc[i].y;
    double w[5];
    const double wg = 0.2, pg = 1.0 / (G * (mach * mach));
    // norm2(coord2(:2)): gfortran's scaled sum of squares
    double scale = 1.0, ss = 0.0;
    const double a[2] = {x0, x1};
    for (int k = 0; k < 2; ++k)
      if (a[k] != 0.0) {
        double ax = std::fabs(a[k]);
        if (ax > scale) {
          double q = scale / ax;
          ss = 1.0 + ss * q * q;
          scale = ax;
        } else {
          double q = ax / scale;
          ss += q * q;
        }
      }
    const double r = scale * std::sqrt(ss);
    if (r < wg) {
      w[0] = 1.0;
      w[1] = -5.0 * x1;
      w[2] = 5.0 * x0;
      w[3] = 0.0;
      w[4] = pg + 12.5 * (r * r);
    } else if (r > 1.0 * wg && r < 2.0 * wg) {
      w[0] = 1.0;
      w[1] = (5.0 - 2.0 / r) * x1;
      w[2] = (-5.0 + 2.0 / r) * x0;
      w[3] = 0.0;
      w[4] = pg + 12.5 * (r * r) + 4.0 - 20.0 * r + 4.0 * std::log(5.0 * r);
    } else {
      w[0] = 1.0;
      w[1] = w[2] = w[3] = 0.0;
      w[4] = pg - 2.0 + 4.0 * std::log(2.0);
    }
    double* u = sol + 5 * (size_t)i;  // primit_to_conserv
    u[0] = w[0];
    for (int k = 1; k < 4; ++k) u[k] = w[k] * w[0];
    u[4] = w[4] / (G - 1) + 0.5 * w[0] * (w[1] * w[1] + w[2] * w[2] + w[3] * w[3]);
  }
  return 0;
}

int subfv_ns_state_create(subfv_mesh* m, const subfv_ns_cfg* cfg, const double* sol, double t0,
                          subfv_ns_state** out) {
  if (!m || !sol || !out || check_cfg(cfg)) return -2;
  DevMesh& d = m->d;
  if (handle_ensure_full_geometry(d)) return -1;
  auto* s = new subfv_ns_state();
  s->m = m;
  s->P = ns_params_from(*cfg);
  // a small mesh leaves most of the GPU idle with one thread per vertex: a group of lanes
  // per vertex (one per subface) shortens each vertex's serial chain (Gresho 64x64: 0.39
  // against 0.48 ms per iteration); subfv_ns_state_set_node_kernel overrides it
  if (d.nv < kSmallMeshVertices) s->P.node_group = 1;
  const size_t ne = d.ne, nv = d.nv, nse = d.nse;
  cudaStream_t q = d.stream;
  if (dalloc(&s->U0, kRec * ne, q) || dalloc(&s->U1, kRec * ne, q) || dalloc(&s->fs, kNsFs * nse, q) ||
      dalloc(&s->rhs1, kRhs * ne, q) || dalloc(&s->rhs2, kRhs * ne, q) || dalloc(&s->ngrad, 15 * nv, q) ||
      dalloc(&s->grad, 15 * ne, q) || dalloc(&s->delta, 5 * ne, q) ||
      dalloc(&s->partial, 6 * (size_t)ns_partial_blocks(d), q) || dalloc(&s->stage, 5 * ne, q) ||
      dalloc(&s->sc, 1, q)) {
    subfv_ns_state_destroy(s);
    return -1;
  }
  if (s->P.diff) {
    // periodic nodes use the union stencil of their images (mesh_dev.cuh)
    if (ensure_diffusion_stencil(&d)) {
      subfv_ns_state_destroy(s);
      return -1;
    }
    const size_t smem = diffusion_smem_bytes(d);
    if (!d.dstencil_ok || smem > 200 * 1024 || d.max_dsf > 32) {
      set_error(!d.dstencil_ok ? "subfv_ns: a periodic node's diffusion stencil is incomplete"
                               : "subfv_ns: a vertex's diffusion system exceeds shared memory");
      subfv_ns_state_destroy(s);
      return -2;
    }
    s->D = diff_params_from(*cfg, d);
    s->P.diff_kd = s->D.kd;
    if (diffusion_prepare(smem) || dalloc(&s->dterm, (size_t)s->D.kd * nse, q) || dalloc(&s->mu0c, 1, q)) {
      subfv_ns_state_destroy(s);
      return -1;
    }
  }
  NsScalars h{};
  h.dtred = 1e10;
  h.omega = 1.0;
  h.t = t0;
  h.final_res = -1.0;
  h.tmax = s->P.tmax;
  h.done = (t0 < s->P.tmax) ? 0 : 1;
  SUBFV_CUDA(cudaMemcpyAsync(s->sc, &h, sizeof(h), cudaMemcpyHostToDevice, d.stream));
  SUBFV_CUDA(cudaMemcpyAsync(s->stage, sol, 5 * ne * sizeof(double), cudaMemcpyHostToDevice, d.stream));
  launch_ns_pack(d, s->stage, s->U0);
  SUBFV_CUDA(cudaStreamSynchronize(d.stream));
  SUBFV_CUDA(cudaGetLastError());
  if ((s->P.diff && diffusion_cache_build(&d, s->D, s->U0, s->dterm, s->mu0c)) || ns_sync_geometry(s)) {
    subfv_ns_state_destroy(s);
    return -1;
  }
  *out = s;
  return 0;
}

int subfv_ns_state_set_node_kernel(subfv_ns_state* s, int lanes) {
  if (!s || (lanes != 0 && lanes != 1 && lanes != 8 && lanes != 16 && lanes != 32)) {
    set_error("subfv_ns_state_set_node_kernel: lanes must be 0, 1, 8, 16 or 32");
    return -2;
  }
  if (s->P.node_group != lanes) {
    s->P.node_group = lanes;
    if (s->graph) {  // the captured step loop holds the old kernel
      SUBFV_CUDA(cudaStreamSynchronize(s->m->d.stream));
      cudaGraphExecDestroy(s->graph);
      s->graph = nullptr;
      s->graph_steps = 0;
    }
  }
  return 0;
}

int subfv_ns_state_destroy(subfv_ns_state* s) {
  if (!s) return 0;
  if (s->imp) {
    ImplicitCtx* c = s->imp;
    int* ip[] = {c->jq_off, c->jq, c->jblk, c->row_off, c->dblk};
    for (int* p : ip) cudaFree(p);
    cudaFree(c->b);
    cudaFree(c->ddiag);
    cudaFree(c->x);
    gmres_work_free(&c->W);
    bcsr_free(&c->A);
    delete c;
  }
  if (s->graph) cudaGraphExecDestroy(s->graph);
  double* bufs[] = {s->U0, s->U1, s->fs, s->rhs1, s->rhs2, s->ngrad, s->grad, s->delta, s->partial, s->stage};
  for (double* b : bufs) cudaFree(b);
  cudaFree(s->sc);
  cudaFree(s->dterm);
  cudaFree(s->mu0c);
  delete s;
  return 0;
}

constexpr int kNsGraphSteps = 8;  // steps per captured graph

int subfv_ns_prepare(subfv_ns_state* s) {
  if (!s) return -2;
  return ns_graph(s, kNsGraphSteps) ? -1 : 0;
}

int subfv_ns_advance_async(subfv_ns_state* s, int n_steps) {
  DevMesh& d = s->m->d;
  if (ns_sync_geometry(s)) return -1;
  const int chunk = kNsGraphSteps;
  if (n_steps >= chunk) {
    if (ns_graph(s, chunk)) return -1;
    for (int i = 0; i + chunk <= n_steps; i += chunk) SUBFV_CUDA(cudaGraphLaunch(s->graph, d.stream));
  }
  for (int i = 0; i < n_steps % chunk; ++i) enqueue_ns_step(s);
  SUBFV_CUDA(cudaGetLastError());
  return 0;
}

int subfv_ns_sync(subfv_ns_state* s, int* steps_done, double* t) {
  DevMesh& d = s->m->d;
  NsScalars h{};
  SUBFV_CUDA(cudaMemcpyAsync(&h, s->sc, sizeof(h), cudaMemcpyDeviceToHost, d.stream));
  int st = handle_check_status(d);
  if (st < 0) return st;
  if (steps_done) *steps_done = (int)h.steps;
  if (t) *t = h.t;
  return st;
}

int subfv_ns_advance(subfv_ns_state* s, int n_steps, int* steps_done, double* t) {
  if (subfv_ns_advance_async(s, n_steps)) return -1;
  return subfv_ns_sync(s, steps_done, t);
}

int subfv_ns_get_sol(subfv_ns_state* s, double* sol) {
  DevMesh& d = s->m->d;
  std::vector<double> rec(kRec * (size_t)d.ne);
  SUBFV_CUDA(cudaMemcpyAsync(rec.data(), s->U0, rec.size() * sizeof(double), cudaMemcpyDeviceToHost, d.stream));
  SUBFV_CUDA(cudaStreamSynchronize(d.stream));
  for (int c = 0; c < d.ne; ++c)
    for (int k = 0; k < 5; ++k) sol[5 * (size_t)c + k] = rec[kRec * (size_t)c + k];
  return 0;
}

int subfv_ns_residuals(subfv_ns_state* s, double* res, double* res_vect, double* dt) {
  DevMesh& d = s->m->d;
  NsScalars h{};
  SUBFV_CUDA(cudaMemcpyAsync(&h, s->sc, sizeof(h), cudaMemcpyDeviceToHost, d.stream));
  SUBFV_CUDA(cudaStreamSynchronize(d.stream));
  if (res) *res = h.res;
  if (res_vect)
    for (int k = 0; k < 5; ++k) res_vect[k] = h.resv[k];
  if (dt) *dt = h.dt;
  return 0;
}

}  // extern "C"

namespace {

template <class T>
int up(T** d, const std::vector<T>& h, cudaStream_t s) {
  SUBFV_CUDA(cudaMalloc((void**)d, std::max<size_t>(h.size(), 1) * sizeof(T)));
  if (!h.empty()) SUBFV_CUDA(cudaMemcpyAsync(*d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, s));
  return 0;
}

// The Jacobian's pattern on one mesh (host arrays), built once and kept with the mesh.
struct ImplicitPattern {
  std::vector<int> jq_off, jq, jblk, row_off, dblk;
  std::vector<int> row1, col1;  // 1-based (bcsr_matrix_type)
  int ncs = 0;                  // greedy colouring of the rows for the LU-SGS preconditioner
  std::vector<int> color;
};

int build_pattern(DevMesh& d, ImplicitPattern& P) {
  std::vector<int2> flr(d.nf), sse(d.nsf);
  std::vector<int> sff(d.nsf), sfv(d.nsf), sev(d.nse);
  SUBFV_CUDA(cudaMemcpyAsync(flr.data(), d.flr, d.nf * sizeof(int2), cudaMemcpyDeviceToHost, d.stream));
  SUBFV_CUDA(cudaMemcpyAsync(sse.data(), d.sf_se, d.nsf * sizeof(int2), cudaMemcpyDeviceToHost, d.stream));
  SUBFV_CUDA(cudaMemcpyAsync(sff.data(), d.sf_face, d.nsf * sizeof(int), cudaMemcpyDeviceToHost, d.stream));
  SUBFV_CUDA(cudaMemcpyAsync(sfv.data(), d.sf_vert, d.nsf * sizeof(int), cudaMemcpyDeviceToHost, d.stream));
  SUBFV_CUDA(cudaMemcpyAsync(sev.data(), d.se_vert, d.nse * sizeof(int), cudaMemcpyDeviceToHost, d.stream));
  SUBFV_CUDA(cudaStreamSynchronize(d.stream));
  const int ne = d.ne;
  std::vector<int>& jq_off = P.jq_off;
  jq_off.assign(ne + 1, 0);
  auto owns_right = [&](int sf) { return sse[sf].y >= 0 && sev[sse[sf].y] == sfv[sf]; };
  for (int sf = 0; sf < d.nsf; ++sf) {
    const int2 lr = flr[sff[sf]];
    jq_off[lr.x + 1]++;
    if (lr.y >= 0 && owns_right(sf)) jq_off[lr.y + 1]++;
  }
  for (int i = 0; i < ne; ++i) jq_off[i + 1] += jq_off[i];
  std::vector<int>& jq = P.jq;
  jq.assign(jq_off[ne], 0);
  std::vector<int> other(jq_off[ne]);
  {
    std::vector<int> fill(jq_off.begin(), jq_off.end() - 1);
    for (int sf = 0; sf < d.nsf; ++sf) {
      const int2 lr = flr[sff[sf]];
      other[fill[lr.x]] = lr.y;
      jq[fill[lr.x]++] = 2 * sf;
      if (lr.y >= 0 && owns_right(sf)) {
        other[fill[lr.y]] = lr.x;
        jq[fill[lr.y]++] = 2 * sf + 1;
      }
    }
  }
  std::vector<int>& row_off = P.row_off;
  std::vector<int> col;
  row_off.assign(ne + 1, 0);
  P.dblk.assign(ne, 0);
  P.jblk.assign(jq.size(), -1);
  std::vector<int> cs;
  for (int i = 0; i < ne; ++i) {
    cs.assign(1, i);
    for (int q = jq_off[i]; q < jq_off[i + 1]; ++q)
      if (other[q] >= 0) cs.push_back(other[q]);
    std::sort(cs.begin(), cs.end());
    cs.erase(std::unique(cs.begin(), cs.end()), cs.end());
    for (int q = jq_off[i]; q < jq_off[i + 1]; ++q)
      if (other[q] >= 0) P.jblk[q] = row_off[i] + (int)(std::lower_bound(cs.begin(), cs.end(), other[q]) - cs.begin());
    P.dblk[i] = row_off[i] + (int)(std::lower_bound(cs.begin(), cs.end(), i) - cs.begin());
    col.insert(col.end(), cs.begin(), cs.end());
    row_off[i + 1] = (int)col.size();
  }
  P.row1.resize(ne + 1);
  P.col1.resize(col.size());
  for (int i = 0; i <= ne; ++i) P.row1[i] = row_off[i] + 1;
  for (size_t j = 0; j < col.size(); ++j) P.col1[j] = col[j] + 1;
  // rows in order, each the smallest colour not taken by a coupled row of lower index
  // (the pattern is symmetric: cell adjacency)
  P.color.assign(ne, 0);
  P.ncs = 0;
  std::vector<int> seen;
  for (int i = 0; i < ne; ++i) {
    seen.assign(P.ncs + 2, 0);
    for (int j = row_off[i]; j < row_off[i + 1]; ++j)
      if (col[j] < i) seen[P.color[col[j]]] = 1;
    int k = 1;
    while (seen[k]) ++k;
    P.color[i] = k;
    P.ncs = std::max(P.ncs, k);
  }
  return 0;
}

void free_pattern(void* p) { delete static_cast<ImplicitPattern*>(p); }

// Pattern: row i holds i and the other cells of its subfaces, ascending. A cell's
// subfaces are those of elem%sub_face: every subface it is left of, and those it is right
// of through its own subcell at the subface's vertex (not a periodic image's). The
// host pattern is cached on the mesh; each state uploads its own copy.
int implicit_setup(subfv_ns_state* s, int krylov) {
  if (s->imp && s->imp->krylov == krylov) return 0;
  DevMesh& d = s->m->d;
  if (!s->imp) {
    if (!s->m->imp_pattern) {
      auto* P = new ImplicitPattern();
      if (build_pattern(d, *P)) {
        delete P;
        return -1;
      }
      s->m->imp_pattern = P;
      s->m->imp_pattern_free = free_pattern;
    }
    const ImplicitPattern& P = *static_cast<const ImplicitPattern*>(s->m->imp_pattern);
    auto* c = new ImplicitCtx();
    s->imp = c;
    c->row1 = P.row1;
    c->col1 = P.col1;
    const int ne = d.ne;
    if (bcsr_upload(&c->A, ne, 5, c->row1.data(), c->col1.data(), nullptr, d.stream) ||
        bcsr_set_colors(&c->A, P.ncs, P.color.data()))
      return -1;
    if (up(&c->jq_off, P.jq_off, d.stream) || up(&c->jq, P.jq, d.stream) || up(&c->jblk, P.jblk, d.stream) ||
        up(&c->row_off, P.row_off, d.stream) || up(&c->dblk, P.dblk, d.stream))
      return -1;
    SUBFV_CUDA(cudaMalloc(&c->b, 5 * (size_t)ne * sizeof(double)));
    SUBFV_CUDA(cudaMalloc(&c->x, 5 * (size_t)ne * sizeof(double)));
    if (s->P.diff) SUBFV_CUDA(cudaMalloc(&c->ddiag, 25 * (size_t)ne * sizeof(double)));
  }
  ImplicitCtx* c = s->imp;
  gmres_work_free(&c->W);
  if (gmres_work_alloc(&c->W, 5L * d.ne, krylov)) return -1;
  c->krylov = krylov;
  return 0;
}

NsParams implicit_params(const NsParams& P) {
  NsParams q = P;
  q.scheme = 4;  // the implicit residual: first-order two-wave
  q.second_order = 0;
  q.precision = 0;
  return q;
}

// residual at U0, dt = cfl_implicit * min V/sum_lambda (host), Jacobian at U0
int implicit_assemble(subfv_ns_state* s, double cfl_implicit, double dt_force, double* dt_out) {
  DevMesh& d = s->m->d;
  ImplicitCtx* c = s->imp;
  const NsParams Q = implicit_params(s->P);
  NsScalars h{};
  SUBFV_CUDA(cudaMemcpyAsync(&h, s->sc, sizeof(h), cudaMemcpyDeviceToHost, d.stream));
  SUBFV_CUDA(cudaStreamSynchronize(d.stream));
  h.dtred = 1e10;
  h.omega = 1.0;
  h.done = 0;
  SUBFV_CUDA(cudaMemcpyAsync(s->sc, &h, sizeof(h), cudaMemcpyHostToDevice, d.stream));
  launch_ns_rhs(d, Q, s->U0, s->fs, s->rhs1, s->rhs2, s->ngrad, s->grad, s->sc);
  double dtred = 0.0;
  SUBFV_CUDA(cudaMemcpyAsync(&dtred, &s->sc->dtred, sizeof(double), cudaMemcpyDeviceToHost, d.stream));
  SUBFV_CUDA(cudaStreamSynchronize(d.stream));
  const double dt = dt_force > 0.0 ? dt_force : cfl_implicit * dtred;
  launch_be_assemble(d, Q, s->U0, c->jq_off, c->jq, c->jblk, c->row_off, c->dblk, c->A.v, dt, s->sc);
  if (s->P.diff) {  // the viscous and heat terms at U0, with their point-implicit blocks
    launch_ns_diffusion(d, s->D, s->U0, s->dterm, s->mu0c);
    launch_ns_diffusion_apply(d, s->dterm, s->D.kd, s->rhs1, c->ddiag);
  }
  launch_be_pack_rhs(d, s->rhs1, c->b);
  if (s->P.diff) launch_be_add_diffusion(d, c->dblk, c->ddiag, s->U0, c->A.v, c->b);
  if (bcsr_set_values(&c->A, c->A.v, true)) return -1;
  *dt_out = dt;
  return 0;
}

}  // namespace

extern "C" {

int subfv_ns_implicit_step(subfv_ns_state* s, double cfl_implicit, int krylov, double rel_tol, int refine_fp32,
                           subfv_implicit_stats* out) {
  return subfv_ns_implicit_step_ex(s, cfl_implicit, krylov, rel_tol, refine_fp32, 1, out);
}

int subfv_ns_implicit_step_ex(subfv_ns_state* s, double cfl_implicit, int krylov, double rel_tol, int refine_fp32,
                              int precond, subfv_implicit_stats* out) {
  if (!s || krylov < 1 || krylov > 200 || !(rel_tol > 0.0) || (precond != 1 && precond != 2)) {
    set_error("subfv_ns_implicit_step: bad argument");
    return -2;
  }
  DevMesh& d = s->m->d;
  if (handle_clear_status(d) || implicit_setup(s, krylov)) return -1;
  ImplicitCtx* c = s->imp;
  cudaEvent_t e[4];
  for (auto& q : e) SUBFV_CUDA(cudaEventCreate(&q));
  SUBFV_CUDA(cudaEventRecord(e[0], d.stream));
  double dt = 0.0;
  if (implicit_assemble(s, cfl_implicit, 0.0, &dt)) return -1;
  SUBFV_CUDA(cudaEventRecord(e[1], d.stream));
  GmresStats st;
  const double bnorm = device_norm2(c->A, c->W, c->b, 5L * d.ne);
  if (bnorm < 0.0) return -1;
  if (refine_fp32) {
    if (gmres_refine_device(c->A, c->W, c->x, c->b, rel_tol, 1e-3, 30, &st, precond)) return -1;
  } else {
    if (gmres_device(c->A, c->W, c->x, c->b, rel_tol * bnorm, precond, false, precond == kPrecondDiag ? 40 : 20,
                     &st, nullptr))
      return -1;
  }
  SUBFV_CUDA(cudaEventRecord(e[2], d.stream));
  launch_be_update(d, s->U0, c->x);
  {  // t += dt
    NsScalars h{};
    SUBFV_CUDA(cudaMemcpyAsync(&h, s->sc, sizeof(h), cudaMemcpyDeviceToHost, d.stream));
    SUBFV_CUDA(cudaStreamSynchronize(d.stream));
    h.t = h.t + dt;
    h.dt = dt;
    h.steps += 1;
    h.dtred = 1e10;
    h.omega = 1.0;
    SUBFV_CUDA(cudaMemcpyAsync(s->sc, &h, sizeof(h), cudaMemcpyHostToDevice, d.stream));
  }
  SUBFV_CUDA(cudaEventRecord(e[3], d.stream));
  SUBFV_CUDA(cudaEventSynchronize(e[3]));
  float ms[3];
  for (int k = 0; k < 3; ++k) SUBFV_CUDA(cudaEventElapsedTime(&ms[k], e[k], e[k + 1]));
  for (auto& q : e) cudaEventDestroy(q);
  if (out) {
    out->dt = dt;
    out->conv = st.conv;
    out->restarts = refine_fp32 ? st.inner_total : st.restarts;
    out->outer = st.outer;
    out->b_norm = bnorm;
    out->res_norm = st.rho;
    out->ms_assemble = ms[0];
    out->ms_solve = ms[1];
    out->ms_update = ms[2];
    out->nnz_blocks = c->A.nnz;
  }
  int stbits = handle_check_status(d);
  if (stbits < 0) return stbits;
  return stbits | (st.conv ? 0 : SUBFV_ERR_GMRES);
}

int subfv_ns_be_jacobian(subfv_ns_state* s, double dt, int32_t* row, int32_t* col, double* v, int64_t cap) {
  if (implicit_setup(s, 4)) return -1;
  ImplicitCtx* c = s->imp;
  if ((int64_t)c->col1.size() > cap) {
    set_error("subfv_ns_be_jacobian: capacity too small");
    return -2;
  }
  double dto = 0.0;
  if (implicit_assemble(s, 1.0, dt, &dto)) return -1;
  DevMesh& d = s->m->d;
  std::memcpy(row, c->row1.data(), c->row1.size() * sizeof(int32_t));
  std::memcpy(col, c->col1.data(), c->col1.size() * sizeof(int32_t));
  SUBFV_CUDA(cudaMemcpyAsync(v, c->A.v, (size_t)25 * c->A.nnz * sizeof(double), cudaMemcpyDeviceToHost, d.stream));
  SUBFV_CUDA(cudaStreamSynchronize(d.stream));
  return (int)c->col1.size();
}

int subfv_compute_rhs_ns(subfv_mesh* m, const subfv_ns_cfg* cfg, const double* sol, double* rhs, double* sum_lambda,
                         double* vp, double* cell_grad) {
  return subfv_compute_rhs_ns_ex(m, cfg, sol, rhs, sum_lambda, vp, cell_grad, nullptr);
}

int subfv_compute_rhs_ns_ex(subfv_mesh* m, const subfv_ns_cfg* cfg, const double* sol, double* rhs,
                            double* sum_lambda, double* vp, double* cell_grad, double* mat_diag) {
  if (!m || !sol || !rhs || !sum_lambda || check_cfg(cfg)) return -2;
  subfv_ns_state* s = nullptr;
  int rc = subfv_ns_state_create(m, cfg, sol, 0.0, &s);
  if (rc) return rc;
  DevMesh& d = m->d;
  int st = 0;
  do {
    if (handle_clear_status(d)) {
      st = -1;
      break;
    }
    NsScalars h{};
    h.dtred = 1e10;
    h.omega = 1.0;
    h.t = 0.0;
    h.tmax = s->P.tmax;
    if (cudaMemcpyAsync(s->sc, &h, sizeof(h), cudaMemcpyHostToDevice, d.stream) != cudaSuccess) {
      st = -1;
      break;
    }
    launch_ns_rhs(d, s->P, s->U0, s->fs, s->rhs1, s->rhs2, s->ngrad, s->grad, s->sc);
    if (s->P.second_order) launch_ns_flux_limiting(d, s->P, s->U0, s->rhs1, s->rhs2, s->sc);
    double* ddiag = nullptr;
    if (s->P.diff) {
      launch_ns_diffusion(d, s->D, s->U0, s->dterm, s->mu0c);
      if (mat_diag && cudaMallocAsync(&ddiag, 25 * sizeof(double) * d.ne, d.stream) != cudaSuccess) {
        st = -1;
        break;
      }
      launch_ns_diffusion_apply(d, s->dterm, s->D.kd, s->rhs1, ddiag);
    }
    std::vector<double> r(kRhs * (size_t)d.ne);
    if (cudaMemcpyAsync(r.data(), s->rhs1, r.size() * sizeof(double), cudaMemcpyDeviceToHost, d.stream) !=
        cudaSuccess) {
      st = -1;
      break;
    }
    std::vector<double> g(cell_grad ? 15 * (size_t)d.ne : 0);
    if (cell_grad) cudaMemcpyAsync(g.data(), s->grad, g.size() * sizeof(double), cudaMemcpyDeviceToHost, d.stream);
    std::vector<double4> vph(vp ? d.nv : 0);
    if (vp) cudaMemcpyAsync(vph.data(), d.vp, vph.size() * sizeof(double4), cudaMemcpyDeviceToHost, d.stream);
    if (mat_diag) {  // mat_diag(5, 5, n): the diffusion blocks (zero without diffusion)
      if (ddiag) cudaMemcpyAsync(mat_diag, ddiag, 25 * sizeof(double) * d.ne, cudaMemcpyDeviceToHost, d.stream);
      else std::memset(mat_diag, 0, 25 * sizeof(double) * d.ne);
    }
    if (ddiag) cudaFreeAsync(ddiag, d.stream);
    st = handle_check_status(d);
    for (int c = 0; c < d.ne; ++c) {
      for (int k = 0; k < 5; ++k) rhs[5 * (size_t)c + k] = r[kRhs * (size_t)c + k];
      sum_lambda[c] = r[kRhs * (size_t)c + 5];
    }
    if (cell_grad)  // device g[5*d + var] -> Fortran grad(3, 5, n): index d + 3*var
      for (int c = 0; c < d.ne; ++c)
        for (int dd = 0; dd < 3; ++dd)
          for (int k = 0; k < 5; ++k) cell_grad[15 * (size_t)c + dd + 3 * k] = g[15 * (size_t)c + 5 * dd + k];
    if (vp)
      for (int v = 0; v < d.nv; ++v) {
        vp[3 * (size_t)v] = vph[v].x;
        vp[3 * (size_t)v + 1] = vph[v].y;
        vp[3 * (size_t)v + 2] = vph[v].z;
      }
  } while (0);
  subfv_ns_state_destroy(s);
  return st;
}

}  // extern "C"

// ---- the reference's module procedures one at a time, on host buffers in the
// reference's layouts, for a shim that keeps ns_main's loop as it is (ns_main.F90:83-107
// calls compute_rhs_ns, whose compute_euler_flux / compute_cell_grad_from_nodal_grad /
// flux_limiting are below, and add_timedisc_and_solve). Each call uploads its inputs,
// runs the kernels on the mesh's stream and downloads its outputs; FP64 (the precision
// field of cfg applies to compute_euler_flux and the gradients as in the state loop).

namespace {

struct StateHold {
  subfv_ns_state* s = nullptr;
  ~StateHold() {
    if (s) subfv_ns_state_destroy(s);
  }
};

int reset_scalars(subfv_ns_state* s) {
  DevMesh& d = s->m->d;
  NsScalars h{};
  h.dtred = 1e10;
  h.omega = 1.0;
  h.t = 0.0;
  h.final_res = -1.0;
  h.tmax = s->P.tmax;
  SUBFV_CUDA(cudaMemcpyAsync(s->sc, &h, sizeof(h), cudaMemcpyHostToDevice, d.stream));
  return handle_clear_status(d);
}

// grad(3, 5, n) of the reference <-> the kernels' 15 doubles per entity, g[5 d + var]
void grad_from_ref(const double* f, double* g, size_t n) {
  for (size_t c = 0; c < n; ++c)
    for (int dd = 0; dd < 3; ++dd)
      for (int k = 0; k < 5; ++k) g[15 * c + 5 * dd + k] = f[15 * c + dd + 3 * k];
}
void grad_to_ref(const double* g, double* f, size_t n) {
  for (size_t c = 0; c < n; ++c)
    for (int dd = 0; dd < 3; ++dd)
      for (int k = 0; k < 5; ++k) f[15 * c + dd + 3 * k] = g[15 * c + 5 * dd + k];
}

// device scratch of one call, released on the mesh's stream
struct Scratch {
  cudaStream_t q;
  std::vector<void*> ptrs;
  explicit Scratch(cudaStream_t s) : q(s) {}
  ~Scratch() {
    for (void* p : ptrs) cudaFreeAsync(p, q);
  }
  template <class T>
  T* get(size_t n) {
    void* p = nullptr;
    if (cudaMallocAsync(&p, std::max<size_t>(n, 1) * sizeof(T), q) != cudaSuccess) return nullptr;
    ptrs.push_back(p);
    return static_cast<T*>(p);
  }
};

}  // namespace

extern "C" {

int subfv_compute_euler_flux(subfv_mesh* m, const subfv_ns_cfg* cfg, const double* sol, double* rhs,
                             const double* grad, double* sum_lambda, int second_order, double* vp) {
  if (!m || !sol || !rhs || !sum_lambda || (second_order && !grad)) {
    set_error("subfv_compute_euler_flux: null argument");
    return -2;
  }
  StateHold h;
  int rc = subfv_ns_state_create(m, cfg, sol, 0.0, &h.s);
  if (rc) return rc;
  DevMesh& d = m->d;
  if (reset_scalars(h.s)) return -1;
  std::vector<double> g;
  if (second_order) {
    g.resize(15 * (size_t)d.ne);
    grad_from_ref(grad, g.data(), d.ne);
    SUBFV_CUDA(cudaMemcpyAsync(h.s->grad, g.data(), g.size() * sizeof(double), cudaMemcpyHostToDevice, d.stream));
  }
  launch_ns_euler_flux(d, h.s->P, h.s->U0, h.s->grad, h.s->fs, h.s->rhs1, second_order, h.s->sc);
  std::vector<double> r(kRhs * (size_t)d.ne);
  SUBFV_CUDA(cudaMemcpyAsync(r.data(), h.s->rhs1, r.size() * sizeof(double), cudaMemcpyDeviceToHost, d.stream));
  std::vector<double4> vph(vp ? d.nv : 0);
  if (vp) SUBFV_CUDA(cudaMemcpyAsync(vph.data(), d.vp, vph.size() * sizeof(double4), cudaMemcpyDeviceToHost, d.stream));
  const int st = handle_check_status(d);
  SUBFV_CUDA(cudaGetLastError());
  for (int c = 0; c < d.ne; ++c) {
    for (int k = 0; k < 5; ++k) rhs[5 * (size_t)c + k] = r[kRhs * (size_t)c + k];
    sum_lambda[c] = r[kRhs * (size_t)c + 5];
  }
  for (int v = 0; vp && v < d.nv; ++v) {
    vp[3 * (size_t)v] = vph[v].x;
    vp[3 * (size_t)v + 1] = vph[v].y;
    vp[3 * (size_t)v + 2] = vph[v].z;
  }
  return st;
}

int subfv_compute_cell_grad_from_nodal_grad(subfv_mesh* m, const subfv_ns_cfg* cfg, const double* sol, double* grad,
                                            double* nodal_grad) {
  if (!m || !sol || !grad) {
    set_error("subfv_compute_cell_grad_from_nodal_grad: null argument");
    return -2;
  }
  StateHold h;
  int rc = subfv_ns_state_create(m, cfg, sol, 0.0, &h.s);
  if (rc) return rc;
  DevMesh& d = m->d;
  if (reset_scalars(h.s)) return -1;
  launch_ns_cell_grads(d, h.s->P, h.s->U0, h.s->ngrad, h.s->grad, h.s->sc);
  std::vector<double> g(15 * (size_t)d.ne), ng(nodal_grad ? 15 * (size_t)d.nv : 0);
  SUBFV_CUDA(cudaMemcpyAsync(g.data(), h.s->grad, g.size() * sizeof(double), cudaMemcpyDeviceToHost, d.stream));
  if (nodal_grad)
    SUBFV_CUDA(cudaMemcpyAsync(ng.data(), h.s->ngrad, ng.size() * sizeof(double), cudaMemcpyDeviceToHost, d.stream));
  const int st = handle_check_status(d);
  SUBFV_CUDA(cudaGetLastError());
  grad_to_ref(g.data(), grad, d.ne);
  if (nodal_grad) grad_to_ref(ng.data(), nodal_grad, d.nv);
  return st;
}

int subfv_flux_limiting(subfv_mesh* m, const double* sol, double* rhs, const double* rhs_o2, const double* sum_lambda,
                        double cfl) {
  if (!m || !sol || !rhs || !rhs_o2 || !sum_lambda) {
    set_error("subfv_flux_limiting: null argument");
    return -2;
  }
  DevMesh& d = m->d;
  if (handle_ensure_full_geometry(d)) return -1;
  const size_t n = d.ne;
  Scratch w(d.stream);
  double *u = w.get<double>(5 * n), *r = w.get<double>(5 * n), *r2 = w.get<double>(5 * n), *sl = w.get<double>(n),
         *slot = w.get<double>(1);
  if (!u || !r || !r2 || !sl || !slot) {
    set_error("subfv_flux_limiting: device allocation failed");
    return -1;
  }
  const double big = 1e10;
  SUBFV_CUDA(cudaMemcpyAsync(u, sol, 5 * n * sizeof(double), cudaMemcpyHostToDevice, d.stream));
  SUBFV_CUDA(cudaMemcpyAsync(r, rhs, 5 * n * sizeof(double), cudaMemcpyHostToDevice, d.stream));
  SUBFV_CUDA(cudaMemcpyAsync(r2, rhs_o2, 5 * n * sizeof(double), cudaMemcpyHostToDevice, d.stream));
  SUBFV_CUDA(cudaMemcpyAsync(sl, sum_lambda, n * sizeof(double), cudaMemcpyHostToDevice, d.stream));
  SUBFV_CUDA(cudaMemcpyAsync(slot, &big, sizeof(double), cudaMemcpyHostToDevice, d.stream));
  launch_proc_dtmin(d, sl, slot);
  double dtmin = 0.0;
  SUBFV_CUDA(cudaMemcpyAsync(&dtmin, slot, sizeof(double), cudaMemcpyDeviceToHost, d.stream));
  SUBFV_CUDA(cudaStreamSynchronize(d.stream));
  launch_proc_flux_limiting(d, u, r, r2, sl, cfl * dtmin);
  SUBFV_CUDA(cudaMemcpyAsync(rhs, r, 5 * n * sizeof(double), cudaMemcpyDeviceToHost, d.stream));
  SUBFV_CUDA(cudaStreamSynchronize(d.stream));
  SUBFV_CUDA(cudaGetLastError());
  return 0;
}

int subfv_add_timedisc_and_solve(subfv_mesh* m, double* sol, double* rhs, double* diag, double* sum_lambda,
                                 double* delta_sol, double* res, double* res_vect, double a1, double a2, double cfl,
                                 double t, double tmax, double* dt) {
  if (!m || !sol || !rhs || !sum_lambda || !delta_sol || !res || !res_vect || !dt) {
    set_error("subfv_add_timedisc_and_solve: null argument");
    return -2;
  }
  DevMesh& d = m->d;
  if (handle_ensure_full_geometry(d)) return -1;
  const size_t n = d.ne;
  Scratch w(d.stream);
  double *u = w.get<double>(5 * n), *r = w.get<double>(5 * n), *dl = w.get<double>(5 * n),
         *rsq = w.get<double>(5 * n), *rn = w.get<double>(n), *sl = w.get<double>(n), *slots = w.get<double>(8);
  double* dg = diag ? w.get<double>(25 * n) : nullptr;
  if (!u || !r || !dl || !rsq || !rn || !sl || !slots || (diag && !dg)) {
    set_error("subfv_add_timedisc_and_solve: device allocation failed");
    return -1;
  }
  // slots: [0] min V / sum_lambda, [1] omega, [2..7] res and the five sums of squares
  const double init[2] = {1e10, 1.0};
  SUBFV_CUDA(cudaMemcpyAsync(u, sol, 5 * n * sizeof(double), cudaMemcpyHostToDevice, d.stream));
  SUBFV_CUDA(cudaMemcpyAsync(r, rhs, 5 * n * sizeof(double), cudaMemcpyHostToDevice, d.stream));
  SUBFV_CUDA(cudaMemcpyAsync(sl, sum_lambda, n * sizeof(double), cudaMemcpyHostToDevice, d.stream));
  if (diag) SUBFV_CUDA(cudaMemcpyAsync(dg, diag, 25 * n * sizeof(double), cudaMemcpyHostToDevice, d.stream));
  SUBFV_CUDA(cudaMemcpyAsync(slots, init, sizeof(init), cudaMemcpyHostToDevice, d.stream));
  launch_proc_dtmin(d, sl, slots);
  double dtmin = 0.0;
  SUBFV_CUDA(cudaMemcpyAsync(&dtmin, slots, sizeof(double), cudaMemcpyDeviceToHost, d.stream));
  SUBFV_CUDA(cudaStreamSynchronize(d.stream));
  // dt = cfl min(...); global time step: dt = min(tmax - t + 1e-12, dt), sum_lambda = 0
  double dtv = cfl * dtmin;
  const double cap = tmax - t + 1e-12;
  dtv = dtv < cap ? dtv : cap;
  launch_proc_timedisc(d, u, r, dg, dl, rn, rsq, a1, a2, dtv, slots + 1, slots + 2);
  double hs[7];
  SUBFV_CUDA(cudaMemcpyAsync(hs, slots + 1, sizeof(hs), cudaMemcpyDeviceToHost, d.stream));
  SUBFV_CUDA(cudaStreamSynchronize(d.stream));
  const double omega = hs[0];
  int st = 0;
  if (omega <= 1e-6) st |= SUBFV_ERR_BAD_OMEGA;  // the reference prints BAD OMEGA and stops
  if (omega < 1.0) dtv = (1.0 - omega) * dtv;
  if (!st) launch_proc_apply(d, u, dl, a2 * omega);
  SUBFV_CUDA(cudaMemcpyAsync(sol, u, 5 * n * sizeof(double), cudaMemcpyDeviceToHost, d.stream));
  SUBFV_CUDA(cudaMemcpyAsync(rhs, r, 5 * n * sizeof(double), cudaMemcpyDeviceToHost, d.stream));
  SUBFV_CUDA(cudaMemcpyAsync(delta_sol, dl, 5 * n * sizeof(double), cudaMemcpyDeviceToHost, d.stream));
  if (diag) SUBFV_CUDA(cudaMemcpyAsync(diag, dg, 25 * n * sizeof(double), cudaMemcpyDeviceToHost, d.stream));
  SUBFV_CUDA(cudaStreamSynchronize(d.stream));
  SUBFV_CUDA(cudaGetLastError());
  for (size_t c = 0; c < n; ++c) sum_lambda[c] = 0.0;
  *res = hs[1];
  for (int k = 0; k < 5; ++k) res_vect[k] = std::sqrt(hs[2 + k]);
  *dt = dtv;
  return st;
}

}  // extern "C"
