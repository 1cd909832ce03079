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
// precision 1 (mixed) evaluates the per-face wave speeds (the acoustic and shock bounds
// of :68-73, square roots and divisions) in FP32 and keeps the nodal 3x3 solve, the star
// pressures and fluxes, positions, volumes and the residual sums in FP64, so the totals
// are conserved to FP64 rounding.
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
  // sums run in entry order; the next chunk's subface ids and areas are loaded while
  // they run
  int fc[kNodeChunk];
  double arc[kNodeChunk];
#pragma unroll
  for (int u = 0; u < kNodeChunk; ++u)
    if (p0 + u < p1) {
      const int sf = m.vsf_identity ? p0 + u : m.vsf[p0 + u];
      fc[u] = m.sf_face[sf];
      arc[u] = m.sfa[sf];
    }
  for (int p = p0; p < p1; p += kNodeChunk) {
    double4 fnc[kNodeChunk];
    double2 llc[kNodeChunk], xkc[kNodeChunk];
#pragma unroll
    for (int u = 0; u < kNodeChunk; ++u)
      if (p + u < p1) {
        fnc[u] = m.fn[fc[u]];
        const double2* fr = reinterpret_cast<const double2*>(m.frec + kFrec * (size_t)fc[u]);
        llc[u] = fr[0];
        xkc[u] = fr[2];
      }
    int fn_next[kNodeChunk];
    double ar_next[kNodeChunk];
#pragma unroll
    for (int u = 0; u < kNodeChunk; ++u)
      if (p + kNodeChunk + u < p1) {
        const int sf = m.vsf_identity ? p + kNodeChunk + u : m.vsf[p + kNodeChunk + u];
        fn_next[u] = m.sf_face[sf];
        ar_next[u] = m.sfa[sf];
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
#pragma unroll
    for (int u = 0; u < kNodeChunk; ++u) {
      fc[u] = fn_next[u];
      arc[u] = ar_next[u];
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

// Scheme "sidil" (lagrange_module.F90:149-223, 538-809), one thread per vertex, FP64:
// nodal velocity and pressure from the volume-weighted averages of the vertex's subcells
// (lag_to_primit: 1/tau, u, p), corrected by the subface jumps of p (velocity) and of
// u.n (pressure) over the vertex's subfaces, the pressure gradient projected off the
// boundary normal at boundary vertices, with h_p = c V_p / sum |corner normal| of
// compute_length (c = 0, 1, 2, 4, 8 for method 0..4). vp[v] = (velocity, nodal p).
// Across a boundary face the right state is the left one with its velocity mirrored.
__device__ inline void lag_sidil_node_body(const DevMesh& m, const double* __restrict__ sol6, int method,
                                           const int v) {
  if (v >= m.nv) return;
  double vx = 0.0, vy = 0.0, vz = 0.0, rho_p = 0.0, a_p = 0.0, pp = 0.0;
  for (int q = m.vse_off[v]; q < m.vse_off[v + 1]; ++q) {
    const int se = m.vse[q];
    const U5 u = ld_u(sol6, m.se_elem[se]);
    const double vol = m.vol_se[se], w0 = 1.0 / u.t;
    vx = vx + vol * u.u;
    vy = vy + vol * u.v;
    vz = vz + vol * u.w;
    rho_p = rho_p + vol * w0;
    a_p = a_p + vol * sqrt(kGamma * u.p / w0);
    pp = pp + vol * u.p;
  }
  const double V = m.vol_v[v];
  rho_p = rho_p / V;
  a_p = a_p / V;
  vx = vx / V;
  vy = vy / V;
  vz = vz / V;
  pp = pp / V;
  double g0 = 0.0, g1 = 0.0, g2 = 0.0, div_v = 0.0, b0 = 0.0, b1 = 0.0, b2 = 0.0;
  for (int q = m.vsf_off[v]; q < m.vsf_off[v + 1]; ++q) {
    const int sf = m.vsf[q], f = m.sf_face[sf];
    const int2 lr = m.flr[f];
    const double4 fn = m.fn[f];
    const double area = m.sfa[sf];
    const U5 ul = ld_u(sol6, lr.x);
    double r1, r2, r3, rp;
    if (lr.y >= 0) {
      const U5 ur = ld_u(sol6, lr.y);
      r1 = ur.u;
      r2 = ur.v;
      r3 = ur.w;
      rp = ur.p;
    } else {
      const double d = dot3(ul.u, ul.v, ul.w, fn.x, fn.y, fn.z);
      r1 = ul.u - 2.0 * d * fn.x;
      r2 = ul.v - 2.0 * d * fn.y;
      r3 = ul.w - 2.0 * d * fn.z;
      rp = lag_pressure(ul.t, r1, r2, r3, ul.e);
      b0 = b0 + area * fn.x;  // boundary_normal: the faces with right_neigh <= 0
      b1 = b1 + area * fn.y;
      b2 = b2 + area * fn.z;
    }
    g0 = g0 + (rp - ul.p) * area * fn.x;
    g1 = g1 + (rp - ul.p) * area * fn.y;
    g2 = g2 + (rp - ul.p) * area * fn.z;
    div_v = div_v + dot3(r1 - ul.u, r2 - ul.v, r3 - ul.w, area * fn.x, area * fn.y, area * fn.z);
  }
  g0 = g0 / V;
  g1 = g1 / V;
  g2 = g2 / V;
  div_v = div_v / V;
  if (m.is_bound[v]) {
    const double nb = fnorm2_3(b0, b1, b2);
    b0 = b0 / nb;
    b1 = b1 / nb;
    b2 = b2 / nb;
    const double gb = dot3(g0, g1, g2, b0, b1, b2);
    g0 = g0 - gb * b0;
    g1 = g1 - gb * b1;
    g2 = g2 - gb * b2;
  }
  double area_sum = 0.0;  // compute_length over corner_normal of each subcell
  for (int q = m.vse_off[v]; q < m.vse_off[v + 1]; ++q) {
    const int se = m.vse[q], c = m.se_elem[se];
    const int4 ss = m.se_sf[se];
    const int sfs[4] = {ss.x, ss.y, ss.z, ss.w};
    double n0 = 0.0, n1 = 0.0, n2 = 0.0;
    for (int k = 0; k < 4; ++k) {
      if (sfs[k] < 0) break;
      const int f = m.sf_face[sfs[k]];
      const double4 fn = m.fn[f];
      const double a = m.sfa[sfs[k]];
      if (!m.b2d || fabs(fn.z) < 1e-12) {
        if (m.flr[f].x == c) {
          n0 = n0 + a * fn.x;
          n1 = n1 + a * fn.y;
          n2 = n2 + a * fn.z;
        } else {
          n0 = n0 - a * fn.x;
          n1 = n1 - a * fn.y;
          n2 = n2 - a * fn.z;
        }
      }
    }
    area_sum = area_sum + fnorm2_3(n0, n1, n2);
  }
  const double cm = method == 0 ? 0.0 : method == 1 ? 1.0 : method == 2 ? 2.0 : method == 3 ? 4.0 : 8.0;
  const double h_p = cm * V / area_sum;
  vx = vx - 0.5 * h_p / (rho_p * a_p) * g0;
  vy = vy - 0.5 * h_p / (rho_p * a_p) * g1;
  vz = vz - 0.5 * h_p / (rho_p * a_p) * g2;
  pp = pp - 0.5 * h_p * rho_p * a_p * div_v;
  if (pp < 0.0) atomicOr(m.status, kErrNegDensity);  // "Neg prex in sidil nodal" (:674-676)
  m.vp[v] = make_double4(vx, vy, vz, pp);
}
__global__ void __launch_bounds__(128) k_lag_sidil_node(DevMesh m, const double* __restrict__ sol6,
                                                        const LagScalars* sc, int method) {
  if (sc && sc->done) return;
  lag_sidil_node_body(m, sol6, method, blockIdx.x * blockDim.x + threadIdx.x);
}

__device__ inline double warp_min(double x) {
  for (int o = 16; o > 0; o >>= 1) x = fmin(x, __shfl_xor_sync(0xffffffffu, x, o));
  return x;
}

// mode bit 1: rhs, bit 2: CFL terms, bit 4: the rhs of scheme "sidil" (the nodal
// pressure vp.w in place of the face's star pressures); every thread of the block calls
// (block reduction)
template <int P>
__device__ inline void lag_cell_body(const DevMesh& m, const double* __restrict__ sol6, double* __restrict__ rhs6,
                                     double* dt_slot, const int mode, const int c) {
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
    // sums run in entry order; the next chunk's entries are loaded while they run
    int q = m.csf_off[c];
    int4 Ec[kCellChunk];
#pragma unroll
    for (int u = 0; u < kCellChunk; ++u)
      if (q + u < q1) Ec[u] = m.centry[q + u];
    for (; q < q1; q += kCellChunk) {
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
          if ((mode & 1) && !(mode & 4)) {
            const double2* fr = reinterpret_cast<const double2*>(m.frec + kFrec * (size_t)E.y);
            llc[u] = fr[0];
            vvc[u] = fr[1];
          }
          if (mode & 2) vsub[u] = E.w >= 0 ? m.vol_se[E.w] : 0.0;
        }
      int4 En[kCellChunk];
#pragma unroll
      for (int u = 0; u < kCellChunk; ++u)
        if (q + kCellChunk + u < q1) En[u] = m.centry[q + kCellChunk + u];
#pragma unroll
      for (int u = 0; u < kCellChunk; ++u) {
        if (q + u >= q1) break;
        const int side = (Ec[u].z >> 30) & 1;
        const double4 fn = fnc[u];
        const double area = arc[u];
        if ((mode & 5) == 5) {  // sidil: flux (-v.n, pp n, pp v.n) of the vertex
          const double4 vpn = vpc[u];
          const double v_et = dot3(vpn.x, vpn.y, vpn.z, fn.x, fn.y, fn.z);
          const double am = area / mass, ps = vpn.w;
          if (side == 0) {
            r0 = r0 - am * (-v_et);
            r1 = r1 - am * (ps * fn.x);
            r2 = r2 - am * (ps * fn.y);
            r3 = r3 - am * (ps * fn.z);
            r4 = r4 - am * (ps * v_et);
          } else {
            r0 = r0 + am * (-v_et);
            r1 = r1 + am * (ps * fn.x);
            r2 = r2 + am * (ps * fn.y);
            r3 = r3 + am * (ps * fn.z);
            r4 = r4 + am * (ps * v_et);
          }
        } else if (mode & 1) {
          const double4 vpn = vpc[u];
          double v_et = dot3(vpn.x, vpn.y, vpn.z, fn.x, fn.y, fn.z);
          double am = area / mass;
          const double2 ll = llc[u], vv = vvc[u];
          // The star pressures and the flux in FP64 at every precision: at precision 1
          // lambda is the FP32 wave speed (stored as a double), the same value the nodal
          // solve used, so sum over a node of A (p*_L - p*_R) n = R - M v* closes to FP64
          // rounding and the totals stay conserved.
          if (side == 0) {  // this cell is the face's left neighbour: lambda of its side, v.n
            double lam = ll.x, vme = vv.x;
            double ps = pme - lam * (v_et - vme);
            r0 = r0 - am * (-v_et);
            r1 = r1 - am * (ps * fn.x);
            r2 = r2 - am * (ps * fn.y);
            r3 = r3 - am * (ps * fn.z);
            r4 = r4 - am * (ps * v_et);
          } else {  // right neighbour
            double lam = ll.y, vme = vv.y;
            double ps = pme + lam * (v_et - vme);
            r0 = r0 + am * (-v_et);
            r1 = r1 + am * (ps * fn.x);
            r2 = r2 + am * (ps * fn.y);
            r3 = r3 + am * (ps * fn.z);
            r4 = r4 + am * (ps * v_et);
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
#pragma unroll
      for (int u = 0; u < kCellChunk; ++u) Ec[u] = En[u];
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
    geo::face_geom_body<0>(I.m, face_at(I.m, (w - wf[p]) * kLagFaceBlock + threadIdx.x));
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
void launch_lag_sidil_node(const DevMesh& m, const double* sol6, const LagScalars* sc, int method) {
  launch_vert_volume(m);  // V_p of the current (moved) mesh
  k_lag_sidil_node<<<grid_for(m.nv, kBlkNode), kBlkNode, 0, m.stream>>>(m, sol6, sc, method);
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

// One full time step of lagrange_main.F90:89-127 (graph-capturable: no host sync);
// scheme 0 "classic", 1 "sidil" (FP64, method_length `method`).
void enqueue_lag_step_head(const DevMesh& m, double* sol6, double* rhs6, LagScalars* sc, int precision, int scheme,
                           int method) {
  if (scheme == 1) {
    launch_lag_sidil_node(m, sol6, sc, method);
    launch_lag_cell(m, sol6, rhs6, sc, &sc->dtmin, 0, 7);
  } else {
    launch_lag_node(m, sol6, sc, precision);
    launch_lag_cell(m, sol6, rhs6, sc, &sc->dtmin, precision, 3);
  }
  launch_lag_finalize(m, sc);
}

void enqueue_lag_step(const DevMesh& m, double* sol6, double* rhs6, LagScalars* sc, int precision, int scheme,
                      int method) {
  enqueue_lag_step_head(m, sol6, rhs6, sc, precision, scheme, method);
  launch_lag_move(m, sc, 0.0);
  launch_geometry(m, 0, sol6, rhs6, sc);
}

}  // namespace subfv
