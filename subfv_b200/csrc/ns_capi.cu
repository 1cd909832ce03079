// C-ABI of the explicit Euler path (include/subfv.h, subfv_ns_*).
#include <cmath>
#include <cstring>
#include <vector>

#include "handles.cuh"
#include "ns.cuh"

using namespace subfv;

struct subfv_ns_state {
  subfv_mesh* m = nullptr;
  NsParams P{};
  double *U0 = nullptr, *U1 = nullptr, *fs = nullptr, *rhs1 = nullptr, *rhs2 = nullptr;
  double *ngrad = nullptr, *grad = nullptr, *delta = nullptr, *partial = nullptr, *stage = nullptr;
  NsScalars* sc = nullptr;
  cudaGraphExec_t graph = nullptr;
  int graph_steps = 0;
};

namespace {

int check_cfg(const subfv_ns_cfg* c) {
  if (!c || (c->scheme != 1 && c->scheme != 4) || (c->method != 0 && c->method != 1 && c->method != 4) ||
      c->local_time_step != 0 || c->n_bc < 0 || c->n_bc > 16 || (c->precision != 0 && c->precision != 1)) {
    set_error("subfv_ns: unsupported configuration (scheme 1/4, method 0/1/4, global time step, n_bc <= 16)");
    return -2;
  }
  return 0;
}

template <class T>
int dalloc(T** p, size_t n) {
  SUBFV_CUDA(cudaMalloc((void**)p, std::max<size_t>(n, 1) * sizeof(T)));
  SUBFV_CUDA(cudaMemset(*p, 0, std::max<size_t>(n, 1) * sizeof(T)));
  return 0;
}

// One iteration of ns_main.F90:83-107 (graph-capturable).
void enqueue_ns_step(subfv_ns_state* s) {
  const DevMesh& d = s->m->d;
  const NsParams& P = s->P;
  if (P.second_order) {
    launch_ns_rhs(d, P, s->U0, s->fs, s->rhs1, s->rhs2, s->ngrad, s->grad, s->sc);
    launch_ns_timedisc(d, P, s->U0, s->rhs1, s->rhs2, s->U0, s->U1, s->delta, s->partial, s->sc, 2.0, 1.0, 0);
    launch_ns_rhs(d, P, s->U1, s->fs, s->rhs1, s->rhs2, s->ngrad, s->grad, s->sc);
    launch_ns_timedisc(d, P, s->U1, s->rhs1, s->rhs2, s->U0, s->U0, s->delta, s->partial, s->sc, 1.0, 1.0, 1);
  } else {
    launch_ns_rhs(d, P, s->U0, s->fs, s->rhs1, s->rhs2, s->ngrad, s->grad, s->sc);
    launch_ns_timedisc(d, P, s->U0, s->rhs1, nullptr, s->U0, s->U0, s->delta, s->partial, s->sc, 1.0, 1.0, 1);
  }
}

int ns_graph(subfv_ns_state* s, int steps) {
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
  auto* s = new subfv_ns_state();
  s->m = m;
  s->P = ns_params_from(*cfg);
  const size_t ne = d.ne, nv = d.nv, nse = d.nse;
  if (dalloc(&s->U0, kRec * ne) || dalloc(&s->U1, kRec * ne) || dalloc(&s->fs, kNsFs * nse) ||
      dalloc(&s->rhs1, kRhs * ne) || dalloc(&s->rhs2, kRhs * ne) || dalloc(&s->ngrad, 15 * nv) ||
      dalloc(&s->grad, 15 * ne) || dalloc(&s->delta, 5 * ne) || dalloc(&s->partial, 6 * (size_t)ns_partial_blocks(d)) ||
      dalloc(&s->stage, 5 * ne) || dalloc(&s->sc, 1)) {
    subfv_ns_state_destroy(s);
    return -1;
  }
  NsScalars h{};
  h.dtred = 1e10;
  h.omega = 1.0;
  h.t = t0;
  h.final_res = -1.0;
  h.done = (t0 < s->P.tmax) ? 0 : 1;
  SUBFV_CUDA(cudaMemcpyAsync(s->sc, &h, sizeof(h), cudaMemcpyHostToDevice, d.stream));
  SUBFV_CUDA(cudaMemcpyAsync(s->stage, sol, 5 * ne * sizeof(double), cudaMemcpyHostToDevice, d.stream));
  launch_ns_pack(d, s->stage, s->U0);
  SUBFV_CUDA(cudaStreamSynchronize(d.stream));
  SUBFV_CUDA(cudaGetLastError());
  *out = s;
  return 0;
}

int subfv_ns_state_destroy(subfv_ns_state* s) {
  if (!s) return 0;
  if (s->graph) cudaGraphExecDestroy(s->graph);
  double* bufs[] = {s->U0, s->U1, s->fs, s->rhs1, s->rhs2, s->ngrad, s->grad, s->delta, s->partial, s->stage};
  for (double* b : bufs) cudaFree(b);
  cudaFree(s->sc);
  delete s;
  return 0;
}

int subfv_ns_advance_async(subfv_ns_state* s, int n_steps) {
  DevMesh& d = s->m->d;
  const int chunk = 8;
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

int subfv_compute_rhs_ns(subfv_mesh* m, const subfv_ns_cfg* cfg, const double* sol, double* rhs, double* sum_lambda,
                         double* vp, double* cell_grad) {
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
    if (cudaMemcpyAsync(s->sc, &h, sizeof(h), cudaMemcpyHostToDevice, d.stream) != cudaSuccess) {
      st = -1;
      break;
    }
    launch_ns_rhs(d, s->P, s->U0, s->fs, s->rhs1, s->rhs2, s->ngrad, s->grad, s->sc);
    if (s->P.second_order) launch_ns_flux_limiting(d, s->P, s->U0, s->rhs1, s->rhs2, s->sc);
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
