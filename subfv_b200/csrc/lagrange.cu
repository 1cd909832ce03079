// Lagrangian hydro step, scheme "classic" (src/lagrange/lagrange_module.F90:14-147,
// 240-283, 772-784; time loop src/lagrange/lagrange_main.F90:89-127) on the GPU.
//
// Per step, all in HBM, no host round trip:
//   k_lag_face     one thread per face: the wave speeds of the face's two sides
//                  (:68-73 and the boundary branches) and the normal velocities, once
//                  per face; the node and cell kernels read them from the face record
//   k_lag_node     one thread per vertex: nodal 3x3 system (Mp, Rp, Bp) over the
//                  vertex's subfaces, inverse_3_by_3, vp
//   k_lag_cell     one thread per cell: deterministic gather of the subface fluxes in
//                  the reference's scatter order (no float atomics) -> rhs, and the
//                  cell's CFL terms -> block min -> one atomicMin on the bit pattern
//   k_lag_finalize one thread: dt = cfl*min, clip to t_max, t += dt
//   k_lag_move     x += dt*vp
//   k_geom<0>      geometry of the moved mesh, one thread per cell (mesh_dev.cu), fused
//                  with sol += dt*rhs
//
// precision 0 (plain FP64) evaluates every expression in the reference's order and is
// compiled without FMA contraction: bit-identical to the CPU restatement.
// precision 1 (mixed) evaluates the per-face wave speeds and the subface fluxes in
// FP32 and keeps the nodal 3x3 solve, positions, volumes and the residual sums in FP64.
#include <vector>

#include "../../include/subfv.h"
#include "common.cuh"
#include "geom_body.cuh"
#include "lagrange.cuh"
#include "mesh_dev.cuh"

namespace subfv {

namespace {

struct U5 {
  double t, u, v, w, e, p;
};
// cell record: (tau, u, v, w, e, mass, p, -)
__device__ inline U5 ld_u(const double* sol6, int c) {
  const double2* q = reinterpret_cast<const double2*>(sol6 + kRec * (size_t)c);
  double2 a = q[0], b = q[1], d = q[2], g = q[3];
  return {a.x, a.y, b.x, b.y, d.x, g.x};
}
__device__ inline double ld_mass(const double* sol6, int c) { return sol6[kRec * (size_t)c + 5]; }

template <int P>
struct Flt;
template <>
struct Flt<0> {
  using T = double;
};
template <>
struct Flt<1> {
  using T = float;
};

// Wave speed of one side (lagrange_module.F90:68-73), in the precision of P.
template <int P>
__device__ inline double lam_side(double p_me, double p_ot, double tau_me, double vdiff) {
  using T = typename Flt<P>::T;
  T tm = (T)tau_me;
  T a = sqrt((T)kGamma * (T)p_me * tm) / tm;
  T mx = (T)p_ot - (T)p_me;
  T b = sqrt((mx > (T)0 ? mx : (T)0) / tm);
  T c = -(T)vdiff / tm;
  T r = a;
  if (b > r) r = b;
  if (c > r) r = c;
  return (double)r;
}
template <int P>
__device__ inline double lam_wall(double p_me, double tau_me) {
  using T = typename Flt<P>::T;
  T tm = (T)tau_me;
  return (double)(sqrt((T)kGamma * (T)p_me * tm) / tm);
}

// Face record (6 doubles): l1, l2 (the left / right wave speeds lambda of :68-73; l2 = 0
// on a boundary), vl, vr (the left / right normal velocities), xb, kind. kind 0
// interior (xb = v_bar of :75), 1 a z-face of a one-layer slab (b2d), 2 a wall
// (xb = p_l + l1 v_l).
constexpr int kFrec = 6;
constexpr int kNodeChunk = 4, kCellChunk = 2;

template <int P>
__device__ inline void lag_face_body(const DevMesh& m, const double* __restrict__ sol6, const int f) {
  if (f >= m.nf) return;
  const int2 lr = m.flr[f];
  const double4 fn = m.fn[f];
  const double n0 = fn.x, n1 = fn.y, n2 = fn.z;
  const U5 ul = ld_u(sol6, lr.x);
  const double pl = ul.p;
  const double vl = dot3(ul.u, ul.v, ul.w, n0, n1, n2);
  double l1, l2 = 0.0, vr = 0.0, xb = 0.0, kind;
  if (lr.y >= 0) {
    const U5 ur = ld_u(sol6, lr.y);
    const double pr = ur.p;
    vr = dot3(ur.u, ur.v, ur.w, n0, n1, n2);
    l1 = lam_side<P>(pl, pr, ul.t, vr - vl);
    l2 = lam_side<P>(pr, pl, ur.t, vr - vl);
    xb = (l1 * vl + l2 * vr - (pr - pl)) / (l2 + l1);
    kind = 0.0;
  } else if (m.b2d && fabs(n2) > 1e-8) {
    l1 = lam_wall<P>(pl, ul.t);
    kind = 1.0;
  } else {
    l1 = lam_wall<P>(pl, ul.t);
    xb = pl + l1 * vl;
    kind = 2.0;
  }
  double2* r = reinterpret_cast<double2*>(m.frec + kFrec * (size_t)f);
  r[0] = make_double2(l1, l2);
  r[1] = make_double2(vl, vr);
  r[2] = make_double2(xb, kind);
}
template <int P>
__global__ void __launch_bounds__(128) k_lag_face(DevMesh m, const double* __restrict__ sol6, const LagScalars* sc) {
  if (sc && sc->done) return;
  lag_face_body<P>(m, sol6, blockIdx.x * blockDim.x + threadIdx.x);
}

template <int P>
__device__ inline void lag_node_body(const DevMesh& m, const int v) {
  if (v >= m.nv) return;
  double M00 = 0, M01 = 0, M02 = 0, M10 = 0, M11 = 0, M12 = 0, M20 = 0, M21 = 0, M22 = 0;
  double R0 = 0, R1 = 0, R2 = 0, B0 = 0, B1 = 0, B2 = 0;
  const int p0 = m.vsf_off[v], p1 = m.vsf_off[v + 1];
  // entries in chunks of kNodeChunk: the chunk's loads are issued together, then the
  // sums run in entry order
  for (int p = p0; p < p1; p += kNodeChunk) {
    double4 fnc[kNodeChunk];
    double2 llc[kNodeChunk], xkc[kNodeChunk];
    double arc[kNodeChunk];
    int fc[kNodeChunk];
#pragma unroll
    for (int u = 0; u < kNodeChunk; ++u)
      if (p + u < p1) {
        const int sf = m.vsf_identity ? p + u : m.vsf[p + u];
        fc[u] = m.sf_face[sf];
        arc[u] = m.sfa[sf];
      }
#pragma unroll
    for (int u = 0; u < kNodeChunk; ++u)
      if (p + u < p1) {
        fnc[u] = m.fn[fc[u]];
        const double2* fr = reinterpret_cast<const double2*>(m.frec + kFrec * (size_t)fc[u]);
        llc[u] = fr[0];
        xkc[u] = fr[2];
      }
#pragma unroll
    for (int u = 0; u < kNodeChunk; ++u) {
      if (p + u >= p1) break;
      const double n0 = fnc[u].x, n1 = fnc[u].y, n2 = fnc[u].z;
      const double area = arc[u];
      const double2 ll = llc[u], xk = xkc[u];
      double w;
      if (xk.y == 0.0) {  // interior face
        const double v_bar = xk.x;
        w = area * (ll.x + ll.y);
        R0 = R0 + w * n0 * v_bar;
        R1 = R1 + w * n1 * v_bar;
        R2 = R2 + w * n2 * v_bar;
      } else if (xk.y == 1.0) {
        w = area * 2 * ll.x;
      } else {
        B0 = B0 + area * n0;
        B1 = B1 + area * n1;
        B2 = B2 + area * n2;
        w = area * ll.x;
        const double q = area * xk.x;
        R0 = R0 + q * n0;
        R1 = R1 + q * n1;
        R2 = R2 + q * n2;
      }
      M00 = M00 + w * (n0 * n0); M01 = M01 + w * (n0 * n1); M02 = M02 + w * (n0 * n2);
      M10 = M10 + w * (n1 * n0); M11 = M11 + w * (n1 * n1); M12 = M12 + w * (n1 * n2);
      M20 = M20 + w * (n2 * n0); M21 = M21 + w * (n2 * n1); M22 = M22 + w * (n2 * n2);
    }
  }
  // inverse_3_by_3 (linear_solver_module.F90:134-172): adjugate of the transpose
  double A00 = M11 * M22 - M12 * M21;
  double A01 = -(M01 * M22 - M02 * M21);
  double A02 = M01 * M12 - M02 * M11;
  double A10 = -(M10 * M22 - M20 * M12);
  double A11 = M00 * M22 - M20 * M02;
  double A12 = -(M00 * M12 - M10 * M02);
  double A20 = M10 * M21 - M20 * M11;
  double A21 = -(M00 * M21 - M20 * M01);
  double A22 = M00 * M11 - M10 * M01;
  double det = M00 * A00 + M01 * A10 + M02 * A20;
  double id = 1.0 / det;
  double I00 = id * A00, I01 = id * A01, I02 = id * A02;
  double I10 = id * A10, I11 = id * A11, I12 = id * A12;
  double I20 = id * A20, I21 = id * A21, I22 = id * A22;
  double b0 = R0, b1 = R1, b2 = R2;
  double bmax = fmax(fmax(fabs(B0), fabs(B1)), fabs(B2));
  if (bmax > 1e-8) {
    double mb0 = 0.0 + I00 * B0 + I01 * B1 + I02 * B2;
    double mb1 = 0.0 + I10 * B0 + I11 * B1 + I12 * B2;
    double mb2 = 0.0 + I20 * B0 + I21 * B1 + I22 * B2;
    double Pp = dot3(R0, R1, R2, mb0, mb1, mb2) / dot3(B0, B1, B2, mb0, mb1, mb2);
    b0 = R0 - Pp * B0;
    b1 = R1 - Pp * B1;
    b2 = R2 - Pp * B2;
  }
  double v0 = 0.0 + I00 * b0 + I01 * b1 + I02 * b2;
  double v1 = 0.0 + I10 * b0 + I11 * b1 + I12 * b2;
  double v2 = 0.0 + I20 * b0 + I21 * b1 + I22 * b2;
  m.vp[v] = make_double4(v0, v1, v2, 0.0);
}
template <int P>
__global__ void __launch_bounds__(128) k_lag_node(DevMesh m, const LagScalars* sc) {
  if (sc && sc->done) return;
  lag_node_body<P>(m, blockIdx.x * blockDim.x + threadIdx.x);
}

__device__ inline double warp_min(double x) {
  for (int o = 16; o > 0; o >>= 1) x = fmin(x, __shfl_xor_sync(0xffffffffu, x, o));
  return x;
}

// mode bit 1: rhs, bit 2: CFL terms; every thread of the block calls (block reduction)
template <int P>
__device__ inline void lag_cell_body(const DevMesh& m, const double* __restrict__ sol6, double* __restrict__ rhs6,
                                     double* dt_slot, const int mode, const int c) {
  using T = typename Flt<P>::T;
  double dtloc = 1e6;
  if (c < m.ne) {
    U5 me = ld_u(sol6, c);
    double mass = ld_mass(sol6, c);
    double pme = me.p;
    double csnd = sqrt(kGamma * pme * me.t);
    double r0 = 0, r1 = 0, r2 = 0, r3 = 0, r4 = 0;
    bool bad = false;
    const double vse_c = m.vol_se[c < m.nse ? c : 0];  // sub_elem(i) with i the cell (reference quirk)
    const int q1 = m.csf_off[c + 1];
    // entries in chunks of kCellChunk: the chunk's loads are issued together, then the
    // sums run in entry order
    for (int q = m.csf_off[c]; q < q1; q += kCellChunk) {
      int4 Ec[kCellChunk];
#pragma unroll
      for (int u = 0; u < kCellChunk; ++u)
        if (q + u < q1) Ec[u] = m.centry[q + u];
      double4 fnc[kCellChunk], vpc[kCellChunk];
      double2 llc[kCellChunk], vvc[kCellChunk];
      double arc[kCellChunk], vsub[kCellChunk];
#pragma unroll
      for (int u = 0; u < kCellChunk; ++u)
        if (q + u < q1) {
          const int4 E = Ec[u];
          const int node = E.z & 0x3fffffff;
          fnc[u] = m.fn[E.y];
          arc[u] = m.sfa[E.x];
          vpc[u] = m.vp[node];
          if (mode & 1) {
            const double2* fr = reinterpret_cast<const double2*>(m.frec + kFrec * (size_t)E.y);
            llc[u] = fr[0];
            vvc[u] = fr[1];
          }
          if (mode & 2) vsub[u] = E.w >= 0 ? m.vol_se[E.w] : 0.0;
        }
#pragma unroll
      for (int u = 0; u < kCellChunk; ++u) {
        if (q + u >= q1) break;
        const int side = (Ec[u].z >> 30) & 1;
        const double4 fn = fnc[u];
        const double area = arc[u];
        if (mode & 1) {
          const double4 vpn = vpc[u];
          double v_et = dot3(vpn.x, vpn.y, vpn.z, fn.x, fn.y, fn.z);
          double am = area / mass;
          const double2 ll = llc[u], vv = vvc[u];
          if (side == 0) {  // this cell is the face's left neighbour: lambda of its side, v.n
            double lam = ll.x, vme = vv.x;
            if (P == 0) {
              double ps = pme - lam * (v_et - vme);
              r0 = r0 - am * (-v_et);
              r1 = r1 - am * (ps * fn.x);
              r2 = r2 - am * (ps * fn.y);
              r3 = r3 - am * (ps * fn.z);
              r4 = r4 - am * (ps * v_et);
            } else {
              T ps = (T)pme - (T)lam * ((T)v_et - (T)vme);
              r0 = r0 - am * (double)(-(T)v_et);
              r1 = r1 - am * (double)(ps * (T)fn.x);
              r2 = r2 - am * (double)(ps * (T)fn.y);
              r3 = r3 - am * (double)(ps * (T)fn.z);
              r4 = r4 - am * (double)(ps * (T)v_et);
            }
          } else {  // right neighbour
            double lam = ll.y, vme = vv.y;
            if (P == 0) {
              double ps = pme + lam * (v_et - vme);
              r0 = r0 + am * (-v_et);
              r1 = r1 + am * (ps * fn.x);
              r2 = r2 + am * (ps * fn.y);
              r3 = r3 + am * (ps * fn.z);
              r4 = r4 + am * (ps * v_et);
            } else {
              T ps = (T)pme + (T)lam * ((T)v_et - (T)vme);
              r0 = r0 + am * (double)(-(T)v_et);
              r1 = r1 + am * (double)(ps * (T)fn.x);
              r2 = r2 + am * (double)(ps * (T)fn.y);
              r3 = r3 + am * (double)(ps * (T)fn.z);
              r4 = r4 + am * (double)(ps * (T)v_et);
            }
          }
        }
        if (mode & 2) {  // compute_dt terms for (cell, subface)
          double sg = side == 0 ? 1.0 : -1.0;
          // the subface's own vertex (the owning node unless the node list is a periodic extension)
          const double4 vps = m.vsf_identity ? vpc[u] : m.vp[m.sf_vert[Ec[u].x]];
          double t1 = vse_c / (area * csnd);
          double vn = dot3(vps.x, vps.y, vps.z, sg * fn.x, sg * fn.y, sg * fn.z);
          double t2 = Ec[u].w >= 0 ? 0.8 * vsub[u] / (1e-8 + fabs(vn) * fn.w) : 1e6;
          if (t1 < dtloc) dtloc = t1;
          if (t2 < dtloc) dtloc = t2;
          bad = bad || !(t1 >= 0.0) || !(t2 >= 0.0);
        }
      }
    }
    if (mode & 1) {
      double2* r = reinterpret_cast<double2*>(rhs6 + kRhs * (size_t)c);
      r[0] = make_double2(r0, r1);
      r[1] = make_double2(r2, r3);
      r[2] = make_double2(r4, 0.0);
    }
    if (bad) atomicOr(m.status, kErrNonFinite);
  }
  if (mode & 2) {
    __shared__ double wmin[32];
    double x = warp_min(dtloc);
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) wmin[wid] = x;
    __syncthreads();
    if (wid == 0) {
      int nw = (blockDim.x + 31) >> 5;
      x = lane < nw ? wmin[lane] : 1e6;
      x = warp_min(x);
      if (lane == 0) atomic_min_pos(dt_slot, x);
    }
  }
}
template <int P>
__global__ void __launch_bounds__(128) k_lag_cell(DevMesh m, const double* __restrict__ sol6, double* __restrict__ rhs6,
                                                  LagScalars* sc, double* dt_slot, int mode) {
  if (sc && sc->done) return;
  lag_cell_body<P>(m, sol6, rhs6, dt_slot, mode, blockIdx.x * blockDim.x + threadIdx.x);
}

// dt = cfl*dt; if (t + dt > t_max) dt = t_max - t; t = t + dt (lagrange_main.F90:102-116)
__device__ inline void lag_finalize_body(LagScalars* sc) {
  if (sc->done) {
    sc->skip = 1;
    return;
  }
  double dt = sc->cfl * sc->dtmin;
  if (sc->t + dt > sc->t_max) dt = sc->t_max - sc->t;
  sc->dt = dt;
  sc->t = sc->t + dt;
  sc->steps += 1;
  sc->dtmin = 1e6;  // compute_dt starts from dt = 1e6
  sc->done = (sc->t < sc->t_max) ? 0 : 1;
  sc->skip = 0;
}
__global__ void k_lag_finalize(LagScalars* sc) { lag_finalize_body(sc); }

__device__ inline void lag_move_body(const DevMesh& m, const double dt, const int v) {
  if (v >= m.nv) return;
  double4 x = m.x[v], vp = m.vp[v];
  m.x[v] = make_double4(x.x + dt * vp.x, x.y + dt * vp.y, x.z + dt * vp.z, 0.0);
}
__global__ void k_lag_move(DevMesh m, const LagScalars* sc, double dt_host) {
  if (sc && sc->skip) return;
  lag_move_body(m, sc ? sc->dt : dt_host, blockIdx.x * blockDim.x + threadIdx.x);
}

// ---------------------------------------------------------------------------------
// Batched step over a table of problems (one mesh, state and scalars each): persistent
// grids walk the work blocks of all problems, each block finds its problem in the
// prefix table, so every per-problem result equals the solo run's bit for bit (the only
// cross-block reduction, the CFL minimum, is exact).

__device__ inline int lag_item_of(const int* __restrict__ wofs, int n, int w) {
  int lo = 0, hi = n;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (wofs[mid] <= w) lo = mid;
    else hi = mid;
  }
  return lo;
}

template <int P>
__global__ void __launch_bounds__(kLagFaceBlock) kb_lag_face(const LagItem* __restrict__ it,
                                                             const int* __restrict__ wf, const int* __restrict__ hdr) {
  const int n = hdr[0];
  for (int w = blockIdx.x; w < wf[n]; w += gridDim.x) {
    const int p = lag_item_of(wf, n, w);
    const LagItem& I = it[p];
    if (I.sc->done) continue;
    lag_face_body<P>(I.m, I.sol6, (w - wf[p]) * kLagFaceBlock + threadIdx.x);
  }
}
template <int P>
__global__ void __launch_bounds__(kLagVertBlock) kb_lag_node(const LagItem* __restrict__ it,
                                                             const int* __restrict__ wv, const int* __restrict__ hdr) {
  const int n = hdr[0];
  for (int w = blockIdx.x; w < wv[n]; w += gridDim.x) {
    const int p = lag_item_of(wv, n, w);
    const LagItem& I = it[p];
    if (I.sc->done) continue;
    lag_node_body<P>(I.m, (w - wv[p]) * kLagVertBlock + threadIdx.x);
  }
}
template <int P>
__global__ void __launch_bounds__(kLagCellBlock) kb_lag_cell(const LagItem* __restrict__ it,
                                                             const int* __restrict__ wc, const int* __restrict__ hdr) {
  const int n = hdr[0];
  for (int w = blockIdx.x; w < wc[n]; w += gridDim.x) {
    const int p = lag_item_of(wc, n, w);
    const LagItem& I = it[p];
    if (I.sc->done) continue;
    lag_cell_body<P>(I.m, I.sol6, I.rhs6, &I.sc->dtmin, 3, (w - wc[p]) * kLagCellBlock + threadIdx.x);
    __syncthreads();  // the block-reduction scratch is reused by the next work block
  }
}
__global__ void kb_lag_finalize(const LagItem* __restrict__ it, const int* __restrict__ hdr) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < hdr[0]) lag_finalize_body(it[p].sc);
}
__global__ void __launch_bounds__(kLagVertBlock) kb_lag_move(const LagItem* __restrict__ it,
                                                             const int* __restrict__ wv, const int* __restrict__ hdr) {
  const int n = hdr[0];
  for (int w = blockIdx.x; w < wv[n]; w += gridDim.x) {
    const int p = lag_item_of(wv, n, w);
    const LagItem& I = it[p];
    if (I.sc->skip) continue;
    lag_move_body(I.m, I.sc->dt, (w - wv[p]) * kLagVertBlock + threadIdx.x);
  }
}
__global__ void __launch_bounds__(kLagFaceBlock) kb_face_geom(const LagItem* __restrict__ it,
                                                              const int* __restrict__ wf, const int* __restrict__ hdr) {
  const int n = hdr[0];
  for (int w = blockIdx.x; w < wf[n]; w += gridDim.x) {
    const int p = lag_item_of(wf, n, w);
    const LagItem& I = it[p];
    if (I.sc->skip) continue;
    geo::face_geom_body<0>(I.m, (w - wf[p]) * kLagFaceBlock + threadIdx.x);
  }
}
__global__ void __launch_bounds__(geo::kGeoBlock) kb_geom_step(const LagItem* __restrict__ it,
                                                               const int* __restrict__ wc,
                                                               const int* __restrict__ hdr) {
  static_assert(geo::kGeoBlock == kLagCellBlock, "cell work blocks");
  const int n = hdr[0];
  for (int w = blockIdx.x; w < wc[n]; w += gridDim.x) {
    const int p = lag_item_of(wc, n, w);
    const LagItem& I = it[p];
    if (I.sc->skip) continue;
    geo::geom_step_body(I.m, I.sol6, I.rhs6, I.sc->dt, (w - wc[p]) * kLagCellBlock + threadIdx.x);
  }
}

// (5, n) host layout <-> [n][6] device records; mass goes to slot 5
__global__ void k_pack6(int n, const double* __restrict__ s5, const double* __restrict__ mass, double* __restrict__ s6) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  double* r = s6 + kRec * (size_t)c;
  const double* u = s5 + 5 * (size_t)c;
  for (int k = 0; k < 5; ++k) r[k] = u[k];
  if (mass) r[5] = mass[c];
  r[6] = lag_pressure(u[0], u[1], u[2], u[3], u[4]);
  r[7] = 0.0;
}
__global__ void k_unpack6(int n, int stride, const double* __restrict__ s6, double* __restrict__ s5) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  for (int k = 0; k < 5; ++k) s5[5 * (size_t)c + k] = s6[stride * (size_t)c + k];
}
__global__ void k_vp_out(int n, const double4* __restrict__ vp, double* __restrict__ out) {
  int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n) return;
  double4 a = vp[v];
  out[3 * (size_t)v] = a.x;
  out[3 * (size_t)v + 1] = a.y;
  out[3 * (size_t)v + 2] = a.z;
}
__global__ void k_vp_in(int n, const double* __restrict__ in, double4* __restrict__ vp) {
  int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n) return;
  vp[v] = make_double4(in[3 * (size_t)v], in[3 * (size_t)v + 1], in[3 * (size_t)v + 2], 0.0);
}
__global__ void k_set_scalar(double* p, double v) { *p = v; }

// Per cell-CSR entry (csf = 2p + side): the subface, its face, the node that owns
// position p (bit 30: side) and the cell's subcell on the subface; one 16-byte record
// instead of four dependent lookups in k_lag_cell.
__global__ void k_build_cell_entries(DevMesh m) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= m.ncsf) return;
  const int e = m.csf[q];
  const int p = e >> 1, side = e & 1;
  const int sf = m.vsf_identity ? p : m.vsf[p];
  const int node = m.vsf_identity ? m.sf_vert[sf] : m.p_node[p];
  const int2 se = m.sf_se[sf];
  m.centry[q] = make_int4(sf, m.sf_face[sf], node | (side << 30), side == 0 ? se.x : se.y);
}

}  // namespace

constexpr int kBlkNode = 128, kBlkCell = 128, kBlkVert = 256;

void launch_lag_node(const DevMesh& m, const double* sol6, const LagScalars* sc, int precision) {
  if (precision == 1) {
    k_lag_face<1><<<grid_for(m.nf, kBlkNode), kBlkNode, 0, m.stream>>>(m, sol6, sc);
    k_lag_node<1><<<grid_for(m.nv, kBlkNode), kBlkNode, 0, m.stream>>>(m, sc);
  } else {
    k_lag_face<0><<<grid_for(m.nf, kBlkNode), kBlkNode, 0, m.stream>>>(m, sol6, sc);
    k_lag_node<0><<<grid_for(m.nv, kBlkNode), kBlkNode, 0, m.stream>>>(m, sc);
  }
}
void launch_lag_face_only(const DevMesh& m, const double* sol6, const LagScalars* sc, int precision) {
  if (precision == 1) k_lag_face<1><<<grid_for(m.nf, kBlkNode), kBlkNode, 0, m.stream>>>(m, sol6, sc);
  else k_lag_face<0><<<grid_for(m.nf, kBlkNode), kBlkNode, 0, m.stream>>>(m, sol6, sc);
}
void launch_lag_node_only(const DevMesh& m, const LagScalars* sc, int precision) {
  if (precision == 1) k_lag_node<1><<<grid_for(m.nv, kBlkNode), kBlkNode, 0, m.stream>>>(m, sc);
  else k_lag_node<0><<<grid_for(m.nv, kBlkNode), kBlkNode, 0, m.stream>>>(m, sc);
}
void launch_lag_cell(const DevMesh& m, const double* sol6, double* rhs6, LagScalars* sc, double* dt_slot,
                     int precision, int mode) {
  if (precision == 1)
    k_lag_cell<1><<<grid_for(m.ne, kBlkCell), kBlkCell, 0, m.stream>>>(m, sol6, rhs6, sc, dt_slot, mode);
  else
    k_lag_cell<0><<<grid_for(m.ne, kBlkCell), kBlkCell, 0, m.stream>>>(m, sol6, rhs6, sc, dt_slot, mode);
}
void launch_lag_finalize(const DevMesh& m, LagScalars* sc) { k_lag_finalize<<<1, 1, 0, m.stream>>>(sc); }
void launch_lag_move(const DevMesh& m, const LagScalars* sc, double dt_host) {
  k_lag_move<<<grid_for(m.nv, kBlkVert), kBlkVert, 0, m.stream>>>(m, sc, dt_host);
}
void launch_pack6(const DevMesh& m, int n, const double* s5, const double* mass, double* s6) {
  k_pack6<<<grid_for(n, 256), 256, 0, m.stream>>>(n, s5, mass, s6);
}
void launch_unpack6(const DevMesh& m, int n, int stride, const double* s6, double* s5) {
  k_unpack6<<<grid_for(n, 256), 256, 0, m.stream>>>(n, stride, s6, s5);
}
void launch_vp_out(const DevMesh& m, double* out) { k_vp_out<<<grid_for(m.nv, 256), 256, 0, m.stream>>>(m.nv, m.vp, out); }
void launch_vp_in(const DevMesh& m, const double* in) { k_vp_in<<<grid_for(m.nv, 256), 256, 0, m.stream>>>(m.nv, in, m.vp); }
void launch_set_scalar(const DevMesh& m, double* p, double v) { k_set_scalar<<<1, 1, 0, m.stream>>>(p, v); }
void launch_build_cell_entries(const DevMesh& m) {
  k_build_cell_entries<<<grid_for(m.ncsf, 256), 256, 0, m.stream>>>(m);
}

void launch_lag_batch_step(const LagTable& t, int precision, cudaStream_t s) {
  const int g = t.grid, gp = grid_for(t.cap, 128);
  if (precision == 1) {
    kb_lag_face<1><<<g, kLagFaceBlock, 0, s>>>(t.items, t.wf, t.hdr);
    kb_lag_node<1><<<g, kLagVertBlock, 0, s>>>(t.items, t.wv, t.hdr);
    kb_lag_cell<1><<<g, kLagCellBlock, 0, s>>>(t.items, t.wc, t.hdr);
  } else {
    kb_lag_face<0><<<g, kLagFaceBlock, 0, s>>>(t.items, t.wf, t.hdr);
    kb_lag_node<0><<<g, kLagVertBlock, 0, s>>>(t.items, t.wv, t.hdr);
    kb_lag_cell<0><<<g, kLagCellBlock, 0, s>>>(t.items, t.wc, t.hdr);
  }
  kb_lag_finalize<<<gp, 128, 0, s>>>(t.items, t.hdr);
  kb_lag_move<<<g, kLagVertBlock, 0, s>>>(t.items, t.wv, t.hdr);
  kb_face_geom<<<g, kLagFaceBlock, 0, s>>>(t.items, t.wf, t.hdr);
  kb_geom_step<<<g, geo::kGeoBlock, 0, s>>>(t.items, t.wc, t.hdr);
}

// One full time step of lagrange_main.F90:89-127 (graph-capturable: no host sync).
void enqueue_lag_step(const DevMesh& m, double* sol6, double* rhs6, LagScalars* sc, int precision) {
  launch_lag_node(m, sol6, sc, precision);
  launch_lag_cell(m, sol6, rhs6, sc, &sc->dtmin, precision, 3);
  launch_lag_finalize(m, sc);
  launch_lag_move(m, sc, 0.0);
  launch_geometry(m, 0, sol6, rhs6, sc);
}

}  // namespace subfv
