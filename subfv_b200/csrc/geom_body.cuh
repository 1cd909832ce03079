// Geometry of compute_geometry_mesh (src/mesh/mesh_geometry_module.F90) as per-entity
// device functions, shared by the solo kernels (mesh_dev.cu) and the batched Lagrangian
// kernels (lagrange.cu).
#pragma once
#include "common.cuh"
#include "mesh_dev.cuh"

namespace subfv {
namespace geo {

struct V3 {
  double x, y, z;
};
__device__ inline V3 ld3(const double4* a, int i) {
  double4 v = a[i];
  return {v.x, v.y, v.z};
}
__device__ inline V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ inline V3 cross(V3 a, V3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ inline double dot(V3 a, V3 b) { return dot3(a.x, a.y, a.z, b.x, b.y, b.z); }
__device__ inline V3 half_sum(V3 a, V3 b) { return {0.5 * (a.x + b.x), 0.5 * (a.y + b.y), 0.5 * (a.z + b.z)}; }

__device__ inline V3 pick4(const V3 (&P)[4], int i) { return i == 0 ? P[0] : i == 1 ? P[1] : i == 2 ? P[2] : P[3]; }

// s / nvc, the vertex average of compute_elem_centroid: exact shortcuts for the usual
// vertex counts (a power of two scales exactly; div6 is exact), the division otherwise
__device__ inline V3 vertex_mean(V3 s, int nvc) {
  if (nvc == 8) return {s.x * 0.125, s.y * 0.125, s.z * 0.125};
  if (nvc == 4) return {s.x * 0.25, s.y * 0.25, s.z * 0.25};
  if (nvc == 6) return {div6(s.x), div6(s.y), div6(s.z)};
  return {s.x / nvc, s.y / nvc, s.z / nvc};
}

// compute_face_centroid + compute_subface_norm + compute_face_norm (:177-271), one thread
// per face. Also fS[f] = sum over the face's subfaces (in face%sub_face order) of
// area * unit normal, which the Lagrangian step's cell kernel uses for check_mesh's
// subface closure. FULL = 0 (the Lagrangian step) skips the subface unit normals, which
// the step does not read.
template <int FULL>
__device__ inline void face_geom_body(const DevMesh& m, const int f) {
  if (f >= m.nf) return;
  const int4 fv = m.fvert[f];
  const int vid[4] = {fv.x, fv.y, fv.z, fv.w};
  const int n = fv.w < 0 ? 3 : 4;
  V3 P[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) P[k] = k < n ? ld3(m.x, vid[k]) : V3{0.0, 0.0, 0.0};
  V3 cg = {0.0, 0.0, 0.0};
#pragma unroll
  for (int k = 0; k < 4; ++k)
    if (k < n) cg = {cg.x + P[k].x, cg.y + P[k].y, cg.z + P[k].z};
  cg = n == 4 ? V3{cg.x * 0.25, cg.y * 0.25, cg.z * 0.25} : V3{div3(cg.x), div3(cg.y), div3(cg.z)};
  V3 c = {0.0, 0.0, 0.0};
  double sum_area = 0.0;
#pragma unroll
  for (int j = 0; j < 4; ++j)
    if (j < n) {
      const V3 pj = P[j], pp = pick4(P, j + 1 == n ? 0 : j + 1);
      const V3 x = cross(sub(pj, cg), sub(pp, cg));
      const double area = 0.5 * fnorm2_3(x.x, x.y, x.z);
      c.x = c.x + div3(area * (pj.x + pp.x + cg.x));
      c.y = c.y + div3(area * (pj.y + pp.y + cg.y));
      c.z = c.z + div3(area * (pj.z + pp.z + cg.z));
      sum_area = sum_area + area;
    }
  c = {c.x / sum_area, c.y / sum_area, c.z / sum_area};
  m.fc[f] = make_double4(c.x, c.y, c.z, 0.0);
  const int4 fs = m.fsf[f];
  const int sfi[4] = {fs.x, fs.y, fs.z, fs.w};
  const unsigned fp = m.fpos[f];
  V3 fnrm = {0.0, 0.0, 0.0}, S = {0.0, 0.0, 0.0};
#pragma unroll
  for (int k = 0; k < 4; ++k)
    if (k < n) {
      const int sf = sfi[k];
      const int j = (fp >> (2 * k)) & 3;  // the subface's vertex slot in the face
      const V3 cp = pick4(P, j);
      const V3 cpm = half_sum(pick4(P, j == 0 ? n - 1 : j - 1), cp), cpp = half_sum(pick4(P, j + 1 == n ? 0 : j + 1), cp);
      const V3 a = cross(sub(cpm, c), sub(cp, c));
      const V3 b = cross(sub(cp, c), sub(cpp, c));
      const V3 nr = {0.5 * (a.x + b.x), 0.5 * (a.y + b.y), 0.5 * (a.z + b.z)};
      const double area = fnorm2_3(nr.x, nr.y, nr.z);
      if (FULL) {
        const V3 un = {nr.x / area, nr.y / area, nr.z / area};
        m.sfn[sf] = make_double4(un.x, un.y, un.z, area);
        S = {S.x + area * un.x, S.y + area * un.y, S.z + area * un.z};
      } else {
        // the step keeps no unit normals: the closure sum takes the area vector itself
        // (A n of the check, up to rounding), which only feeds check_mesh's threshold
        S = {S.x + nr.x, S.y + nr.y, S.z + nr.z};
      }
      m.sfa[sf] = area;
      fnrm = {fnrm.x + nr.x, fnrm.y + nr.y, fnrm.z + nr.z};
    }
  const double fa = fnorm2_3(fnrm.x, fnrm.y, fnrm.z);
  m.fn[f] = make_double4(fnrm.x / fa, fnrm.y / fa, fnrm.z / fa, fa);
  if (m.fS) m.fS[f] = make_double4(S.x, S.y, S.z, 0.0);
}

// The cell part of compute_geometry_mesh for the Lagrangian step, one cell per thread,
// after k_face_geom<0>: compute_elem_centroid (:59-110), compute_subelem_volume
// (:112-160), compute_elem_volume (:162-175) and check_mesh (:374-411), then
// sol += dt * rhs (lagrange_main.F90:110). The cell's vertex coordinates and face
// centroids are cached in shared memory (one column per thread), so each is loaded once
// per cell. The local topology comes from the static codes gface / gsub (built once by
// build_geom_codes below): no id is searched and no face or subface index array is read
// per step. check_mesh_subface_closed adds each face's subface sum S as a whole: the same
// total as the subface-by-subface sum up to rounding, and the test is a 1e-14 threshold
// on its norm. Every face vertex must be a vertex of the cell (no periodic faces);
// otherwise the cell reports SUBFV_ERR_INDEX.
constexpr int kGeoMaxV = 8, kGeoMaxF = 8, kGeoBlock = 64;
// faces of a cell the step kernel stages (hexahedra have 6, prisms and pyramids 5,
// tetrahedra 4): with a face-centroid cache of 6 rather than 8 slots the kernel's shared
// memory no longer limits it below the 9 blocks its registers allow
constexpr int kGeoCellFaces = 6;

// gface[8 c + j], face slot j of cell c (ef8 order): bits 3k..3k+2 the local index (in
// the cell's vertex order) of the face's k-th vertex, bit 12 quadrilateral, bit 13 the
// cell is the face's left neighbour, bit 14 valid (every face vertex found among the
// cell's vertices). gsub[s], subcell s = (cell, local vertex k): bits 0..2 the number of
// its subfaces, then per subface (sub_elem order) 5 bits: the face slot j (3 bits) and
// the position kk of the vertex in that face's vertex order (2 bits).
constexpr unsigned kGfQuad = 1u << 12, kGfLeft = 1u << 13, kGfValid = 1u << 14;

// check_mesh's closure tests (mesh_geometry_module.F90:374-411) compare a norm2 with
// 1e-14. With every component at most 1 in magnitude gfortran's NORM2 is the correctly
// rounded sqrt(a*a + b*b + c*c), and rounding sqrt to nearest is monotone, so the test
// holds exactly when the sum is below the smallest double whose rounded square root
// reaches 1e-14; a component above 1 (or a NaN) fails both forms. The step's cell kernel
// takes this form and skips the two square roots.
constexpr double kClosedSumSq = 0x1.fb0f6be506018p-94;  // 9.999999999999999e-29
__device__ inline bool norm2_below_1em14(double a0, double a1, double a2) {
  return fabs(a0) <= 1.0 && fabs(a1) <= 1.0 && fabs(a2) <= 1.0 && (a0 * a0 + a1 * a1 + a2 * a2) < kClosedSumSq;
}

// The codes of cell c, by the same searches the per-step kernel used to run: a face
// vertex's local index is its first match among the cell's vertices; a subface's face
// slot is the first slot holding its face (else the last slot) and its vertex position
// the first match in that face (else the last position).
__device__ inline void build_geom_codes(const DevMesh& m, const int c) {
  if (c >= m.ne) return;
  const int vb = m.ev_off[c], nvc = m.ev_off[c + 1] - vb;
  if (nvc > kGeoMaxV) {
    for (int j = 0; j < kGeoMaxF; ++j) m.gface[8 * (size_t)c + j] = 0;
    return;
  }
  int vid[kGeoMaxV], fid[kGeoMaxF];
  unsigned code[kGeoMaxF];
  for (int k = 0; k < nvc; ++k) vid[k] = m.ev[vb + k];
  int nfc = 0;
  for (int k = 0; k < kGeoMaxF; ++k) {
    const int f = m.ef8[8 * (size_t)c + k];
    if (f < 0) break;
    fid[nfc++] = f;
  }
  for (int j = 0; j < kGeoMaxF; ++j) {
    unsigned w = 0;
    if (j < nfc) {
      const int f = fid[j];
      const int4 fv = m.fvert[f];
      const int gid[4] = {fv.x, fv.y, fv.z, fv.w};
      const int n = fv.w < 0 ? 3 : 4;
      bool ok = true;
      for (int k = 0; k < n; ++k) {
        int q = 0;
        while (q < nvc - 1 && vid[q] != gid[k]) ++q;
        if (vid[q] != gid[k]) ok = false;
        w |= (unsigned)q << (3 * k);
      }
      if (n == 4) w |= kGfQuad;
      if (m.flr[f].x == c) w |= kGfLeft;
      if (ok) w |= kGfValid;
    }
    code[j] = w;
    m.gface[8 * (size_t)c + j] = (uint16_t)w;
  }
  for (int k = 0; k < nvc; ++k) {
    const int4 q4 = m.se_sf[vb + k];
    const int q[4] = {q4.x, q4.y, q4.z, q4.w};
    unsigned g = 0;
    int cnt = 0;
    for (int jj = 0; jj < 4; ++jj) {
      if (q[jj] < 0) break;
      const int f = m.sf_face[q[jj]], vert = m.sf_vert[q[jj]];
      int j = 0;
      while (j < nfc - 1 && fid[j] != f) ++j;
      const int n = 3 + ((code[j] & kGfQuad) ? 1 : 0);
      int kk = 0;
      while (kk < n - 1 && vid[(code[j] >> (3 * kk)) & 7] != vert) ++kk;
      g |= (unsigned)(j | (kk << 3)) << (3 + 5 * jj);
      ++cnt;
    }
    m.gsub[vb + k] = g | (unsigned)cnt;
  }
}

// c: this thread's cell; every thread of a kGeoBlock-thread block calls (the caches are
// indexed by threadIdx.x); dt: the step's time step for the update (with sol6)
// lagrange_main.F90:110: new_sol = sol + dt*rhs, and the cell's pressure record
__device__ inline void state_update(const DevMesh& m, double* sol6, const double* rhs6, const double dt,
                                    const int c) {
  double* u = sol6 + kRec * (size_t)c;
  const double* r = rhs6 + kRhs * (size_t)c;
  bool fin = true;
  for (int k = 0; k < 5; ++k) {
    u[k] = u[k] + dt * r[k];
    fin = fin && isfinite(u[k]);
  }
  u[6] = lag_pressure(u[0], u[1], u[2], u[3], u[4]);
  if (!fin) atomicOr(m.status, kErrNonFinite);
  if (!(u[0] > 0.0)) atomicOr(m.status, kErrNegDensity);
}

// the 16-bit code of face slot j (0..7) from the cell's four code words
__device__ inline unsigned gface_code(const unsigned (&gw)[4], const int j) {
  const unsigned w = (j >> 1) == 0 ? gw[0] : (j >> 1) == 1 ? gw[1] : (j >> 1) == 2 ? gw[2] : gw[3];
  return (w >> (16 * (j & 1))) & 0xffffu;
}

__device__ inline void geom_step_body(const DevMesh& m, double* sol6, const double* rhs6, const double dt,
                                      const int c) {
  __shared__ double sX[kGeoMaxV][3][kGeoBlock];
  __shared__ double sCF[kGeoCellFaces][3][kGeoBlock];
  const int t = threadIdx.x;
  if (c >= m.ne) return;
  const int vb = m.ev_off[c], nvc = m.ev_off[c + 1] - vb;
  if (nvc > kGeoMaxV) {
    atomicOr(m.status, kErrIndex);
    return;
  }
  const uint4 g4 = reinterpret_cast<const uint4*>(m.gface)[c];
  const unsigned gw[4] = {g4.x, g4.y, g4.z, g4.w};
  const int4 e0 = reinterpret_cast<const int4*>(m.ef8)[2 * (size_t)c];
  const int4 e1 = reinterpret_cast<const int4*>(m.ef8)[2 * (size_t)c + 1];
  const int fid[kGeoMaxF] = {e0.x, e0.y, e0.z, e0.w, e1.x, e1.y, e1.z, e1.w};
  int nfc = 0;
#pragma unroll
  for (int j = 0; j < kGeoMaxF; ++j)
    if (fid[j] >= 0 && nfc == j) nfc = j + 1;
  if (nfc > kGeoCellFaces) {
    atomicOr(m.status, kErrIndex);
    return;
  }
  // Every global load of the cell first: vertex coordinates, then per face its
  // centroid, normal and subface sum (the check terms are formed as they arrive, in face
  // order), then the subcells' codes. What follows reads shared memory and registers.
  V3 ce = {0.0, 0.0, 0.0};
  for (int k = 0; k < nvc; ++k) {
    const V3 x = ld3(m.x, m.ev[vb + k]);
    sX[k][0][t] = x.x;
    sX[k][1][t] = x.y;
    sX[k][2][t] = x.z;
    ce = {ce.x + x.x, ce.y + x.y, ce.z + x.z};
  }
  double vdiv = 0.0;
  V3 nt = {0.0, 0.0, 0.0}, ns = {0.0, 0.0, 0.0};
  bool valid = true;
#pragma unroll
  for (int j = 0; j < kGeoCellFaces; ++j)
    if (j < nfc) {
      const int f = fid[j];
      const unsigned code = gface_code(gw, j);
      valid = valid && (code & kGfValid);
      const V3 cf = ld3(m.fc, f);
      const double4 fn = m.fn[f];
      const double4 S = m.fS[f];
      sCF[j][0][t] = cf.x;
      sCF[j][1][t] = cf.y;
      sCF[j][2][t] = cf.z;
      // check_mesh_elem_volume / _closed / _subface_closed terms of this face (the
      // subface closure sums the face's own subface sum S, formed in face%sub_face order)
      const double sg = (code & kGfLeft) ? 1.0 : -1.0;
      const V3 nn = {sg * fn.x, sg * fn.y, sg * fn.z};
      const V3 an = {fn.w * nn.x, fn.w * nn.y, fn.w * nn.z};
      vdiv = vdiv + dot(cf, an);
      nt = {nt.x + an.x, nt.y + an.y, nt.z + an.z};
      ns = {ns.x + sg * S.x, ns.y + sg * S.y, ns.z + sg * S.z};
    }
  unsigned gs[kGeoMaxV];
#pragma unroll
  for (int k = 0; k < kGeoMaxV; ++k) gs[k] = k < nvc ? m.gsub[vb + k] : 0u;
  if (!valid) {
    atomicOr(m.status, kErrIndex);
    return;
  }
  ce = vertex_mean(ce, nvc);
  // compute_elem_centroid: tetrahedra (edge, face centroid, vertex centroid)
  V3 cen = {0.0, 0.0, 0.0};
  double sum_vol = 0.0;
  for (int j = 0; j < nfc; ++j) {
    const unsigned code = gface_code(gw, j);
    const int n = (code & kGfQuad) ? 4 : 3;
    const bool left = (code & kGfLeft) != 0;
    const V3 cf = {sCF[j][0][t], sCF[j][1][t], sCF[j][2][t]};
    const V3 fe = sub(cf, ce);
    int q = code & 7;
    V3 cp = {sX[q][0][t], sX[q][1][t], sX[q][2][t]};
    const V3 c0 = cp;
    for (int k = 0; k < n; ++k) {
      V3 cpp = c0;
      if (k + 1 < n) {
        q = (code >> (3 * (k + 1))) & 7;
        cpp = {sX[q][0][t], sX[q][1][t], sX[q][2][t]};
      }
      const V3 x = left ? cross(sub(cp, cf), sub(cpp, cf)) : cross(sub(cpp, cf), sub(cp, cf));
      const double vol = div6(dot(x, fe));
      cen.x = cen.x + vol * (cp.x + cpp.x + cf.x + ce.x) * 0.25;
      cen.y = cen.y + vol * (cp.y + cpp.y + cf.y + ce.y) * 0.25;
      cen.z = cen.z + vol * (cp.z + cpp.z + cf.z + ce.z) * 0.25;
      sum_vol = sum_vol + vol;
      cp = cpp;
    }
  }
  cen = {cen.x / sum_vol, cen.y / sum_vol, cen.z / sum_vol};
  // compute_subelem_volume: subcell k is (cell, vertex k); its subfaces in sub_elem order
  bool ok = true;
  double vcell = 0.0;
#pragma unroll
  for (int k = 0; k < kGeoMaxV; ++k) {
    if (k >= nvc) break;
    const unsigned g = gs[k];
    const int cnt = g & 7;
    double vol = 0.0;
    for (int jj = 0; jj < cnt; ++jj) {
      const unsigned slot = (g >> (3 + 5 * jj)) & 31u;
      const int j = slot & 7, kk = slot >> 3;
      const unsigned code = gface_code(gw, j);
      const int n = (code & kGfQuad) ? 4 : 3;
      const int lc = (code >> (3 * kk)) & 7;
      const int lm = (code >> (3 * (kk == 0 ? n - 1 : kk - 1))) & 7;
      const int lp = (code >> (3 * (kk + 1 == n ? 0 : kk + 1))) & 7;
      const V3 cp = {sX[lc][0][t], sX[lc][1][t], sX[lc][2][t]};
      const V3 cpm = half_sum({sX[lm][0][t], sX[lm][1][t], sX[lm][2][t]}, cp);
      const V3 cpp = half_sum({sX[lp][0][t], sX[lp][1][t], sX[lp][2][t]}, cp);
      const V3 cf = {sCF[j][0][t], sCF[j][1][t], sCF[j][2][t]};
      const V3 fe = sub(cf, cen);
      const V3 a = sub(cpm, cf), b = sub(cp, cf), cc3 = sub(cpp, cf);
      V3 x1, x2;
      if (code & kGfLeft) {
        x1 = cross(a, b);
        x2 = cross(b, cc3);
      } else {
        x1 = cross(cc3, b);
        x2 = cross(b, a);
      }
      vol = vol + div6(dot(x1, fe)) + div6(dot(x2, fe));
    }
    m.vol_se[vb + k] = vol;
    ok = ok && (vol > 0.0);
    vcell = vcell + vol;
  }
  m.vol[c] = vcell;
  vdiv = div3(vdiv);
  ok = ok && (fabs(vcell - vdiv) < 1e-14);
  ok = ok && norm2_below_1em14(nt.x, nt.y, nt.z);
  ok = ok && norm2_below_1em14(ns.x, ns.y, ns.z);
  if (!ok) atomicOr(m.status, kErrMeshCheck);
  if (sol6) state_update(m, sol6, rhs6, dt, c);
}

}  // namespace geo
}  // namespace subfv
