// Batched and served Lagrangian hydro (include/subfv.h, subfv_lag_batch_*): many
// independent problems, each on its own device mesh (moved by its steps), advanced
// together in shared persistent launches (launch_lag_batch_step) with the step loop
// captured once in a CUDA graph. No counterpart in the reference, whose
// lagrange_main.F90:89-127 loop advances one mesh per process. The slot, snapshot and
// table machinery is the explicit Euler batch's (ns_batch.cu).
//
// Concurrency model. All step work runs on the batch stream. Admission work (state
// allocation, upload, packing) runs on the admitted mesh's own stream and is joined to
// the batch stream by an event, so a request can be admitted while earlier chunks are
// still running. The table of in-flight problems lives in device memory and is rewritten
// in stream order; the captured graph reads its size from the device, so it stays valid
// as problems join and leave. Removed slots are reused only after the batch stream has
// passed the point where they left the table; their memory is freed stream-ordered.
#include <algorithm>
#include <cstring>
#include <deque>
#include <vector>

#include "handles.cuh"
#include "lagrange.cuh"

using namespace subfv;

namespace {

struct Slot {
  subfv_mesh* mesh = nullptr;
  int owns_mesh = 0;
  int live = 0;            // holds a problem (in the table or waiting to be removed)
  cudaEvent_t free_ev = nullptr;  // recorded on the batch stream when the slot left the table
  double *sol6 = nullptr, *rhs6 = nullptr;
  int64_t bytes = 0;       // state + mesh bytes charged against the budget
  unsigned long long first_snap = 0;  // the first snapshot that includes this problem
  double t0 = 0.0;
};

struct Snapshot {
  LagScalars* sc = nullptr;  // pinned
  unsigned* status = nullptr;
  cudaEvent_t ev = nullptr;
  int pending = 0;
  unsigned long long seq = 0;  // snapshots are numbered in enqueue order from 1
};

// The per-problem state: cell records and residual records.
int64_t state_bytes(const DevMesh& d) { return 8 * (int64_t)(kRec + kRhs) * d.ne; }

}  // namespace

struct subfv_lag_batch {
  int precision = 0;
  cudaStream_t stream = nullptr;
  int cap = 0;
  int64_t budget = 0, used = 0;
  LagScalars* sc = nullptr;  // device [cap]
  unsigned* status = nullptr;  // device [cap]
  std::vector<Slot> slots;
  std::vector<int> order;  // live slots in table order
  // device table and its pinned host staging (double-buffered staging)
  LagTable tab{};
  LagItem* h_items[2] = {nullptr, nullptr};
  int* h_w[2] = {nullptr, nullptr};  // [wf (cap+1) | wv (cap+1) | wc (cap+1) | hdr (4)]
  cudaEvent_t stage_ev[2] = {nullptr, nullptr};
  int stage_cur = 0;
  bool dirty = true;
  cudaGraphExec_t graph = nullptr;
  int graph_steps = 0;
  Snapshot snap[2];
  std::deque<int> outstanding;  // snapshot indices in enqueue order
  int snap_next = 0;
  // the latest completed snapshot, copied out of the pinned ring
  std::vector<LagScalars> last_sc;
  std::vector<unsigned> last_status;
  bool have_last = false;
  unsigned long long last_seq = 0, snap_count = 0;
  std::vector<int> retiring;    // removed slots whose memory is freed at the next table rewrite
};

namespace {

template <class T>
int dalloc_async(T** p, size_t n, cudaStream_t s) {
  SUBFV_CUDA(cudaMallocAsync((void**)p, std::max<size_t>(n, 1) * sizeof(T), s));
  SUBFV_CUDA(cudaMemsetAsync(*p, 0, std::max<size_t>(n, 1) * sizeof(T), s));
  return 0;
}

void slot_free_state(Slot& q, cudaStream_t s) {
  if (q.sol6) cudaFreeAsync(q.sol6, s);
  if (q.rhs6) cudaFreeAsync(q.rhs6, s);
  q.sol6 = q.rhs6 = nullptr;
}

int graph_for(subfv_lag_batch* b, int steps) {
  if (b->graph && b->graph_steps == steps) return 0;
  if (b->graph) {
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
  }
  cudaGraph_t g;
  SUBFV_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
  for (int i = 0; i < steps; ++i) launch_lag_batch_step(b->tab, b->precision, b->stream);
  SUBFV_CUDA(cudaStreamEndCapture(b->stream, &g));
  cudaError_t e = cudaGraphInstantiate(&b->graph, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    set_error(std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
    return -1;
  }
  b->graph_steps = steps;
  return 0;
}

// Rewrite the device table from the live slots (stream-ordered on the batch stream).
int table_upload(subfv_lag_batch* b) {
  if (!b->dirty) return 0;
  const int k = b->stage_cur;
  SUBFV_CUDA(cudaEventSynchronize(b->stage_ev[k]));  // the staging copy issued two updates ago
  LagItem* it = b->h_items[k];
  int* wf = b->h_w[k];
  int* wv = wf + (b->cap + 1);
  int* wc = wv + (b->cap + 1);
  int* hdr = wc + (b->cap + 1);
  const int n = (int)b->order.size();
  wf[0] = wv[0] = wc[0] = 0;
  for (int i = 0; i < n; ++i) {
    Slot& q = b->slots[b->order[i]];
    LagItem& I = it[i];
    I.m = q.mesh->d;
    I.m.status = b->status + b->order[i];
    I.sol6 = q.sol6;
    I.rhs6 = q.rhs6;
    I.sc = b->sc + b->order[i];
    wf[i + 1] = wf[i] + (I.m.nf + kLagFaceBlock - 1) / kLagFaceBlock;
    wv[i + 1] = wv[i] + (I.m.nv + kLagVertBlock - 1) / kLagVertBlock;
    wc[i + 1] = wc[i] + (I.m.ne + kLagCellBlock - 1) / kLagCellBlock;
  }
  hdr[0] = n;
  if (n) SUBFV_CUDA(cudaMemcpyAsync(b->tab.items, it, n * sizeof(LagItem), cudaMemcpyHostToDevice, b->stream));
  SUBFV_CUDA(cudaMemcpyAsync(b->tab.wf, wf, 3 * (size_t)(b->cap + 1) * sizeof(int) + sizeof(int),
                             cudaMemcpyHostToDevice, b->stream));
  SUBFV_CUDA(cudaEventRecord(b->stage_ev[k], b->stream));
  b->stage_cur ^= 1;
  b->dirty = false;
  // slots that left the table: their frees are stream-ordered after the rewrite
  for (int r : b->retiring) {
    Slot& q = b->slots[r];
    slot_free_state(q, b->stream);
    SUBFV_CUDA(cudaEventRecord(q.free_ev, b->stream));
    if (q.owns_mesh && q.mesh) {
      SUBFV_CUDA(cudaStreamWaitEvent(q.mesh->d.stream, q.free_ev, 0));
      subfv_mesh_destroy(q.mesh);
    }
    q.mesh = nullptr;
  }
  b->retiring.clear();
  return 0;
}

void snapshot_take(subfv_lag_batch* b, Snapshot& s) {
  s.pending = 0;
  b->outstanding.pop_front();
  std::memcpy(b->last_sc.data(), s.sc, b->cap * sizeof(LagScalars));
  std::memcpy(b->last_status.data(), s.status, b->cap * sizeof(unsigned));
  b->have_last = true;
  b->last_seq = s.seq;
}

int snapshot_enqueue(subfv_lag_batch* b) {
  const int k = b->snap_next;
  Snapshot& s = b->snap[k];
  if (s.pending) {  // both buffers in flight: retire the older one first
    SUBFV_CUDA(cudaEventSynchronize(s.ev));
    snapshot_take(b, s);
  }
  SUBFV_CUDA(cudaMemcpyAsync(s.sc, b->sc, b->cap * sizeof(LagScalars), cudaMemcpyDeviceToHost, b->stream));
  SUBFV_CUDA(cudaMemcpyAsync(s.status, b->status, b->cap * sizeof(unsigned), cudaMemcpyDeviceToHost, b->stream));
  SUBFV_CUDA(cudaEventRecord(s.ev, b->stream));
  s.pending = 1;
  s.seq = ++b->snap_count;
  b->outstanding.push_back(k);
  b->snap_next ^= 1;
  return 0;
}

}  // namespace

extern "C" {

int subfv_lag_batch_create(int precision, int capacity, int64_t budget_bytes, subfv_lag_batch** out) {
  if (!out || capacity < 1 || capacity > (1 << 20) || budget_bytes <= 0 || (precision != 0 && precision != 1)) {
    set_error("subfv_lag_batch_create: bad argument");
    return -2;
  }
  auto* b = new subfv_lag_batch();
  b->precision = precision;
  b->cap = capacity;
  b->budget = budget_bytes;
  b->slots.resize(capacity);
  b->last_sc.resize(capacity);
  b->last_status.resize(capacity);
  auto fail = [&]() {
    subfv_lag_batch_destroy(b);
    return -1;
  };
  if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) return fail();
  const size_t nw = 3 * (size_t)(capacity + 1) + 4;
  if (cudaMalloc(&b->sc, capacity * sizeof(LagScalars)) != cudaSuccess ||
      cudaMalloc(&b->status, capacity * sizeof(unsigned)) != cudaSuccess ||
      cudaMalloc(&b->tab.items, capacity * sizeof(LagItem)) != cudaSuccess ||
      cudaMalloc(&b->tab.wf, nw * sizeof(int)) != cudaSuccess)
    return fail();
  cudaMemsetAsync(b->sc, 0, capacity * sizeof(LagScalars), b->stream);
  cudaMemsetAsync(b->status, 0, capacity * sizeof(unsigned), b->stream);
  cudaMemsetAsync(b->tab.wf, 0, nw * sizeof(int), b->stream);
  b->tab.wv = b->tab.wf + (capacity + 1);
  b->tab.wc = b->tab.wv + (capacity + 1);
  b->tab.hdr = b->tab.wc + (capacity + 1);
  b->tab.cap = capacity;
  b->tab.grid = 148 * 8;
  for (int k = 0; k < 2; ++k) {
    if (cudaHostAlloc((void**)&b->h_items[k], capacity * sizeof(LagItem), cudaHostAllocDefault) != cudaSuccess ||
        cudaHostAlloc((void**)&b->h_w[k], nw * sizeof(int), cudaHostAllocDefault) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->stage_ev[k], cudaEventDisableTiming) != cudaSuccess ||
        cudaHostAlloc((void**)&b->snap[k].sc, capacity * sizeof(LagScalars), cudaHostAllocDefault) != cudaSuccess ||
        cudaHostAlloc((void**)&b->snap[k].status, capacity * sizeof(unsigned), cudaHostAllocDefault) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->snap[k].ev, cudaEventDisableTiming) != cudaSuccess)
      return fail();
    std::memset(b->snap[k].sc, 0, capacity * sizeof(LagScalars));
    std::memset(b->snap[k].status, 0, capacity * sizeof(unsigned));
  }
  for (auto& q : b->slots)
    if (cudaEventCreateWithFlags(&q.free_ev, cudaEventDisableTiming) != cudaSuccess) return fail();
  if (cudaDeviceSynchronize() != cudaSuccess) return fail();
  *out = b;
  return 0;
}

int subfv_lag_batch_destroy(subfv_lag_batch* b) {
  if (!b) return 0;
  if (b->stream) cudaStreamSynchronize(b->stream);
  for (auto& q : b->slots) {
    if (q.live || q.mesh) {
      slot_free_state(q, b->stream);
      if (q.owns_mesh) subfv_mesh_destroy(q.mesh);
    }
    if (q.free_ev) cudaEventDestroy(q.free_ev);
  }
  if (b->stream) cudaStreamSynchronize(b->stream);
  if (b->graph) cudaGraphExecDestroy(b->graph);
  cudaFree(b->sc);
  cudaFree(b->status);
  cudaFree(b->tab.items);
  cudaFree(b->tab.wf);
  for (int k = 0; k < 2; ++k) {
    cudaFreeHost(b->h_items[k]);
    cudaFreeHost(b->h_w[k]);
    if (b->stage_ev[k]) cudaEventDestroy(b->stage_ev[k]);
    cudaFreeHost(b->snap[k].sc);
    cudaFreeHost(b->snap[k].status);
    if (b->snap[k].ev) cudaEventDestroy(b->snap[k].ev);
  }
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return 0;
}

int64_t subfv_lag_batch_state_bytes(const subfv_lag_batch* b, const subfv_mesh* m) {
  return (b && m) ? state_bytes(m->d) : -2;
}

int64_t subfv_lag_batch_free_bytes(const subfv_lag_batch* b) { return b ? b->budget - b->used : -2; }

int subfv_lag_batch_add(subfv_lag_batch* b, subfv_mesh* m, int take_mesh, const double* sol, const double* mass,
                        double cfl, double t0, double t_max, int* slot) {
  if (!b || !m || !sol || !mass || !slot) {
    set_error("subfv_lag_batch_add: null argument");
    return -2;
  }
  if (handle_ensure_full_geometry(m->d) || handle_ensure_lag_arrays(m->d)) return -1;
  m->d.moving = 1;
  const DevMesh& d = m->d;
  const int64_t need = state_bytes(d) + (int64_t)d.bytes;
  int k = -1;
  for (int i = 0; i < b->cap && k < 0; ++i) {
    Slot& q = b->slots[i];
    if (!q.live && !q.mesh && cudaEventQuery(q.free_ev) == cudaSuccess) k = i;
  }
  if (k < 0 || b->used + need > b->budget) {
    set_error("subfv_lag_batch_add: no free slot or HBM budget exhausted");
    return SUBFV_BATCH_FULL;
  }
  Slot& q = b->slots[k];
  cudaStream_t s = d.stream;
  const size_t ne = d.ne;
  double *stage = nullptr, *mstage = nullptr;
  if (cudaMallocAsync((void**)&q.sol6, kRec * ne * sizeof(double), s) != cudaSuccess ||
      cudaMallocAsync((void**)&q.rhs6, kRhs * ne * sizeof(double), s) != cudaSuccess ||
      cudaMallocAsync((void**)&stage, 5 * ne * sizeof(double), s) != cudaSuccess ||
      cudaMallocAsync((void**)&mstage, ne * sizeof(double), s) != cudaSuccess) {
    slot_free_state(q, s);
    set_error("subfv_lag_batch_add: device allocation failed");
    return -1;
  }
  SUBFV_CUDA(cudaMemsetAsync(q.rhs6, 0, kRhs * ne * sizeof(double), s));
  LagScalars h{};  // as subfv_lag_state_create
  h.dtmin = 1e6;
  h.t = t0;
  h.t_max = t_max;
  h.cfl = cfl;
  h.done = (t0 < t_max) ? 0 : 1;
  const unsigned zero = 0;
  SUBFV_CUDA(cudaMemcpyAsync(stage, sol, 5 * ne * sizeof(double), cudaMemcpyHostToDevice, s));
  SUBFV_CUDA(cudaMemcpyAsync(mstage, mass, ne * sizeof(double), cudaMemcpyHostToDevice, s));
  SUBFV_CUDA(cudaMemcpyAsync(b->sc + k, &h, sizeof(h), cudaMemcpyHostToDevice, s));
  SUBFV_CUDA(cudaMemcpyAsync(b->status + k, &zero, sizeof(zero), cudaMemcpyHostToDevice, s));
  launch_pack6(d, (int)ne, stage, mstage, q.sol6);
  SUBFV_CUDA(cudaFreeAsync(stage, s));
  SUBFV_CUDA(cudaFreeAsync(mstage, s));
  cudaEvent_t ready;
  SUBFV_CUDA(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
  SUBFV_CUDA(cudaEventRecord(ready, s));
  SUBFV_CUDA(cudaStreamWaitEvent(b->stream, ready, 0));
  cudaEventDestroy(ready);
  SUBFV_CUDA(cudaGetLastError());
  m->d.geom_partial = 1;  // the batch's steps refresh only the step's geometry
  q.mesh = m;
  q.owns_mesh = take_mesh ? 1 : 0;
  q.live = 1;
  q.bytes = need;
  q.first_snap = b->snap_count + 1;
  q.t0 = t0;
  b->used += need;
  b->order.push_back(k);
  b->dirty = true;
  *slot = k;
  return 0;
}

int subfv_lag_batch_remove(subfv_lag_batch* b, int slot) {
  if (!b || slot < 0 || slot >= b->cap || !b->slots[slot].live) {
    set_error("subfv_lag_batch_remove: bad slot");
    return -2;
  }
  Slot& q = b->slots[slot];
  auto it = std::find(b->order.begin(), b->order.end(), slot);
  if (it != b->order.end()) b->order.erase(it);
  b->used -= q.bytes;
  q.bytes = 0;
  q.live = 0;
  b->retiring.push_back(slot);  // freed after the table rewrite that drops it
  b->dirty = true;
  return 0;
}

int subfv_lag_batch_set_grid(subfv_lag_batch* b, int grid) {
  if (!b || grid < 1) {
    set_error("subfv_lag_batch_set_grid: the grid must be positive");
    return -2;
  }
  if (grid != b->tab.grid) {
    b->tab.grid = grid;
    if (b->graph) {
      SUBFV_CUDA(cudaStreamSynchronize(b->stream));
      cudaGraphExecDestroy(b->graph);
      b->graph = nullptr;
    }
  }
  return 0;
}

int subfv_lag_batch_advance(subfv_lag_batch* b, int n_steps) {
  if (!b || n_steps < 0) {
    set_error("subfv_lag_batch_advance: bad argument");
    return -2;
  }
  if (table_upload(b)) return -1;
  const int chunk = 8;
  if (n_steps >= chunk) {
    if (graph_for(b, chunk)) return -1;
    for (int i = 0; i + chunk <= n_steps; i += chunk) SUBFV_CUDA(cudaGraphLaunch(b->graph, b->stream));
  }
  for (int i = 0; i < n_steps % chunk; ++i) launch_lag_batch_step(b->tab, b->precision, b->stream);
  SUBFV_CUDA(cudaGetLastError());
  return snapshot_enqueue(b);
}

int subfv_lag_batch_time_steps(subfv_lag_batch* b, int n_steps, double* ms) {
  if (!b || n_steps < 1 || !ms) {
    set_error("subfv_lag_batch_time_steps: bad argument");
    return -2;
  }
  if (table_upload(b)) return -1;
  cudaEvent_t e0, e1;
  SUBFV_CUDA(cudaEventCreate(&e0));
  SUBFV_CUDA(cudaEventCreate(&e1));
  SUBFV_CUDA(cudaEventRecord(e0, b->stream));
  if (subfv_lag_batch_advance(b, n_steps)) return -1;
  SUBFV_CUDA(cudaEventRecord(e1, b->stream));
  SUBFV_CUDA(cudaEventSynchronize(e1));
  float f = 0.f;
  SUBFV_CUDA(cudaEventElapsedTime(&f, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *ms = f;
  return 0;
}

int subfv_lag_batch_poll(subfv_lag_batch* b, int wait) {
  if (!b) return -2;
  if (b->outstanding.empty()) {
    if (!wait) return b->have_last ? 0 : 1;
    if (snapshot_enqueue(b)) return -1;
  }
  Snapshot& s = b->snap[b->outstanding.front()];
  if (!wait) {
    cudaError_t e = cudaEventQuery(s.ev);
    if (e == cudaErrorNotReady) return 1;
    SUBFV_CUDA(e);
  } else {
    SUBFV_CUDA(cudaEventSynchronize(s.ev));
  }
  snapshot_take(b, s);
  return 0;
}

int subfv_lag_batch_sync(subfv_lag_batch* b) {
  if (!b) return -2;
  if (snapshot_enqueue(b)) return -1;
  while (!b->outstanding.empty())
    if (subfv_lag_batch_poll(b, 1)) return -1;
  return 0;
}

int subfv_lag_batch_slot_info(const subfv_lag_batch* b, int slot, double* t, int64_t* steps, int* done,
                             unsigned* status) {
  if (!b || slot < 0 || slot >= b->cap) return -2;
  const Slot& q = b->slots[slot];
  if (!q.live || b->last_seq < q.first_snap) {  // not yet seen by a completed snapshot
    if (t) *t = q.t0;
    if (steps) *steps = 0;
    if (done) *done = 0;
    if (status) *status = 0;
    return q.live ? 1 : -2;
  }
  const LagScalars& h = b->last_sc[slot];
  if (t) *t = h.t;
  if (steps) *steps = (int64_t)h.steps;
  if (done) *done = h.done;
  if (status) *status = b->last_status[slot];
  return 0;
}

int subfv_lag_batch_get_sol(subfv_lag_batch* b, int slot, double* sol) {
  if (!b || !sol || slot < 0 || slot >= b->cap || !b->slots[slot].live) {
    set_error("subfv_lag_batch_get_sol: bad slot");
    return -2;
  }
  Slot& q = b->slots[slot];
  const DevMesh& d = q.mesh->d;
  // A problem that a completed snapshot shows done is final: the step kernels no longer
  // write its state, so the copy need not wait for the chunks still queued. Otherwise
  // the copy is ordered after everything enqueued so far on the batch stream.
  if (!(b->last_seq >= q.first_snap && b->last_sc[slot].done)) {
    cudaEvent_t e;
    SUBFV_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    SUBFV_CUDA(cudaEventRecord(e, b->stream));
    SUBFV_CUDA(cudaStreamWaitEvent(d.stream, e, 0));
    cudaEventDestroy(e);
  }
  std::vector<double> rec(kRec * (size_t)d.ne);
  SUBFV_CUDA(cudaMemcpyAsync(rec.data(), q.sol6, rec.size() * sizeof(double), cudaMemcpyDeviceToHost, d.stream));
  SUBFV_CUDA(cudaStreamSynchronize(d.stream));
  for (int c = 0; c < d.ne; ++c)
    for (int k = 0; k < 5; ++k) sol[5 * (size_t)c + k] = rec[kRec * (size_t)c + k];
  return 0;
}

int subfv_lag_batch_size(const subfv_lag_batch* b, int* n_live, int64_t* used_bytes) {
  if (!b) return -2;
  if (n_live) *n_live = (int)b->order.size();
  if (used_bytes) *used_bytes = b->used;
  return 0;
}

}  // extern "C"
