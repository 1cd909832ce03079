// Host-side mesh topology (see topology.h). Every pass is a counting sort or a
// per-group scan, so building a 40M-cell batch takes seconds, while the numbering
// matches the reference's build_mesh (src/mesh/mesh_connectivity_module.F90:12-59)
// id for id.
#include "topology.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <unordered_map>

namespace subfv {
namespace {

// gmsh face tables (1-based local vertices), src/mesh/mesh_reading_module.F90:1163-1316.
// A face of three vertices has 0 in the last slot.
const int kTetF[4][4] = {{1, 3, 2, 0}, {1, 2, 4, 0}, {1, 4, 3, 0}, {2, 3, 4, 0}};
const int kHexF[6][4] = {{1, 4, 3, 2}, {3, 4, 8, 7}, {7, 8, 5, 6}, {1, 2, 6, 5}, {1, 5, 8, 4}, {2, 3, 7, 6}};
const int kPriF[5][4] = {{1, 3, 2, 0}, {4, 5, 6, 0}, {1, 2, 5, 4}, {2, 3, 6, 5}, {1, 4, 6, 3}};
const int kPyrF[5][4] = {{1, 4, 3, 2}, {1, 2, 5, 0}, {2, 3, 5, 0}, {3, 4, 5, 0}, {1, 5, 4, 0}};

int kind_nv(int k) { return k == 4 ? 4 : k == 5 ? 8 : k == 6 ? 6 : k == 7 ? 5 : -1; }
int kind_nf(int k) { return k == 4 ? 4 : k == 5 ? 6 : (k == 6 || k == 7) ? 5 : -1; }
const int (*kind_tab(int k))[4] { return k == 4 ? kTetF : k == 5 ? kHexF : k == 6 ? kPriF : kPyrF; }

using V = std::vector<int32_t>;

// CSR from (owner, value) pairs emitted in the order the reference appends them.
struct Csr {
  V off, val;
};
template <class Emit>
Csr bucket(int n_owner, int64_t n_items, Emit emit) {
  Csr c;
  c.off.assign(n_owner + 1, 0);
  emit([&](int owner, int32_t) { c.off[owner]++; });
  for (int i = 1; i <= n_owner; ++i) c.off[i] += c.off[i - 1];  // owner k spans [off[k-1], off[k])
  c.val.assign((size_t)n_items, 0);
  V fill(c.off.begin(), c.off.end() - 1);
  emit([&](int owner, int32_t v) { c.val[fill[owner - 1]++] = v; });
  return c;
}

struct FaceKey {
  std::array<int32_t, 4> s;  // sorted vertex ids, 0-padded
  int n;
  bool operator==(const FaceKey& o) const { return n == o.n && s == o.s; }
};
FaceKey make_key(const int32_t* v, int n) {
  FaceKey k{{0, 0, 0, 0}, n};
  for (int i = 0; i < n; ++i) k.s[i] = v[i];
  for (int i = 1; i < n; ++i)  // insertion sort of at most four ids
    for (int j = i; j > 0 && k.s[j - 1] > k.s[j]; --j) std::swap(k.s[j - 1], k.s[j]);
  return k;
}

bool near(double a, double b) { return a < b + 1e-12 && a > b - 1e-12; }

// Index of the grid point X (n coordinates of b bits) along the n-dimensional Hilbert
// curve, by Skilling's transpose method (J. Skilling, "Programming the Hilbert curve",
// AIP Conf. Proc. 707, 381 (2004)): undo the excess rotations level by level, Gray-code
// the transposed index, then read its bits most significant first across the axes.
uint64_t hilbert_index(uint32_t* X, int n, int b) {
  const uint32_t M = 1u << (b - 1);
  for (uint32_t Q = M; Q > 1; Q >>= 1) {
    const uint32_t P = Q - 1;
    for (int i = 0; i < n; ++i) {
      if (X[i] & Q) {
        X[0] ^= P;
      } else {
        const uint32_t t = (X[0] ^ X[i]) & P;
        X[0] ^= t;
        X[i] ^= t;
      }
    }
  }
  for (int i = 1; i < n; ++i) X[i] ^= X[i - 1];
  uint32_t t = 0;
  for (uint32_t Q = M; Q > 1; Q >>= 1)
    if (X[n - 1] & Q) t ^= Q - 1;
  for (int i = 0; i < n; ++i) X[i] ^= t;
  uint64_t key = 0;
  for (int bit = b - 1; bit >= 0; --bit)
    for (int i = 0; i < n; ++i) key = (key << 1) | ((X[i] >> bit) & 1u);
  return key;
}

}  // namespace

void hilbert_vertex_order(int nv, const double* c, int b2d, std::vector<int32_t>& otn, std::vector<int32_t>& nto) {
  const int dims = b2d ? 2 : 3, bits = b2d ? 31 : 21;
  double lo[3], hi[3];
  for (int d = 0; d < 3; ++d) lo[d] = hi[d] = c[d];
  for (int i = 1; i < nv; ++i)
    for (int d = 0; d < 3; ++d) {
      lo[d] = std::min(lo[d], c[3 * i + d]);
      hi[d] = std::max(hi[d], c[3 * i + d]);
    }
  double ext = 0.0;
  for (int d = 0; d < dims; ++d) ext = std::max(ext, hi[d] - lo[d]);
  const double top = (double)((1u << bits) - 1u);
  const double scale = ext > 0.0 ? top / ext : 0.0;
  std::vector<std::pair<uint64_t, int32_t>> key(nv);
  for (int i = 0; i < nv; ++i) {
    uint32_t X[3] = {0, 0, 0};
    for (int d = 0; d < dims; ++d) {
      double q = (c[3 * i + d] - lo[d]) * scale;
      q = q < 0.0 ? 0.0 : (q > top ? top : q);
      X[d] = (uint32_t)q;
    }
    key[i] = {hilbert_index(X, dims, bits), i + 1};
  }
  std::sort(key.begin(), key.end());
  otn.assign(nv + 1, -1);
  nto.assign(nv + 1, -1);
  for (int k = 0; k < nv; ++k) {
    nto[k + 1] = key[k].second;
    otn[key[k].second] = k + 1;
  }
}

int build_topology(const RawMeshView& in, Topology& T, std::string* err) {
  const int nv = in.n_vert, ne = in.n_elems;
  auto fail = [&](const char* m) {
    if (err) *err = m;
    return 1;
  };
  if (nv <= 0 || ne <= 0) return fail("empty mesh");
  for (int e = 0; e < ne; ++e) {
    int k = in.elem_kind[e];
    if (kind_nv(k) < 0 || in.elem_vert_off[e + 1] - in.elem_vert_off[e] != kind_nv(k))
      return fail("unsupported element kind or vertex count");
    for (int q = in.elem_vert_off[e]; q < in.elem_vert_off[e + 1]; ++q)
      if (in.elem_vert[q] < 1 || in.elem_vert[q] > nv) return fail("vertex id out of range");
  }

  // -- vertex -> element lists in element order (:475-509)
  Csr ve0 = bucket(nv, in.elem_vert_off[ne], [&](auto put) {
    for (int e = 0; e < ne; ++e)
      for (int q = in.elem_vert_off[e]; q < in.elem_vert_off[e + 1]; ++q) put(in.elem_vert[q], e + 1);
  });

  // -- BFS vertex renumbering (:851-926): a FIFO over the new numbering, restarted at
  // the lowest unnumbered vertex when a component is exhausted. Or, as an option, the
  // vertices along a Hilbert curve; everything below follows whichever order is chosen.
  V otn_v(nv + 1, -1), nto_v(nv + 1, -1);
  if (in.renumber == 1) {
    hilbert_vertex_order(nv, in.coords, in.b2d, otn_v, nto_v);
  } else {
    int iloc = 1, head = 1, scan = 1;
    otn_v[1] = 1;
    nto_v[1] = 1;
    iloc = 2;
    while (iloc <= nv) {
      if (head >= iloc) {
        while (otn_v[scan] >= 0) ++scan;
        otn_v[scan] = iloc;
        nto_v[iloc] = scan;
        ++iloc;
      }
      int v = nto_v[head++];
      for (int q = ve0.off[v - 1]; q < ve0.off[v]; ++q) {
        int e = ve0.val[q] - 1;
        for (int r = in.elem_vert_off[e]; r < in.elem_vert_off[e + 1]; ++r) {
          int w = in.elem_vert[r];
          if (otn_v[w] < 0) {
            otn_v[w] = iloc;
            nto_v[iloc] = w;
            ++iloc;
          }
        }
      }
    }
  }

  // -- cell renumbering by first touch over the new vertex order (:752-849)
  V otn_e(ne + 1, -1), nto_e(ne + 1, -1);
  {
    int iloc = 1;
    for (int vn = 1; vn <= nv; ++vn) {
      int vo = nto_v[vn];
      for (int q = ve0.off[vo - 1]; q < ve0.off[vo]; ++q) {
        int e = ve0.val[q];
        if (otn_e[e] <= 0) {
          otn_e[e] = iloc;
          nto_e[iloc] = e;
          ++iloc;
        }
      }
    }
    if (iloc != ne + 1) return fail("mesh has elements not reachable from any vertex");
  }

  T.n_vert = nv;
  T.n_elems = ne;
  T.vert_coord.assign(3 * (size_t)nv, 0.0);
  for (int i = 1; i <= nv; ++i)
    for (int d = 0; d < 3; ++d) T.vert_coord[3 * (otn_v[i] - 1) + d] = in.coords[3 * (i - 1) + d];

  V& ekind = T.arr["elem_kind"];
  V& ev_off = T.arr["elem_vert_off"];
  V& ev = T.arr["elem_vert"];
  ekind.resize(ne);
  ev_off.assign(ne + 1, 0);
  for (int en = 1; en <= ne; ++en) {
    int eo = nto_e[en] - 1;
    ekind[en - 1] = in.elem_kind[eo];
    ev_off[en] = ev_off[en - 1] + kind_nv(in.elem_kind[eo]);
  }
  ev.resize(ev_off[ne]);
  for (int en = 1; en <= ne; ++en) {
    int eo = nto_e[en] - 1;
    int b = in.elem_vert_off[eo];
    for (int j = 0; j < ev_off[en] - ev_off[en - 1]; ++j) ev[ev_off[en - 1] + j] = otn_v[in.elem_vert[b + j]];
  }
  // vertex -> element lists, renumbered, order kept (:828-832)
  V& vel_off = T.arr["vert_elem_off"];
  V& vel = T.arr["vert_elem"];
  vel_off.assign(nv + 1, 0);
  for (int vn = 1; vn <= nv; ++vn) vel_off[vn] = vel_off[vn - 1] + (ve0.off[nto_v[vn]] - ve0.off[nto_v[vn] - 1]);
  vel.resize(vel_off[nv]);
  for (int vn = 1; vn <= nv; ++vn) {
    int vo = nto_v[vn];
    int p = vel_off[vn - 1];
    for (int q = ve0.off[vo - 1]; q < ve0.off[vo]; ++q) vel[p++] = otn_e[ve0.val[q]];
  }

  // -- minimal faces in file order (reader), vertex ids renumbered
  int64_t nmf = 0;
  for (int e = 0; e < ne; ++e) nmf += kind_nf(in.elem_kind[e]);
  V mf_nv(nmf), mf_left(nmf), mf_lf(nmf), mf_min(nmf);
  std::vector<std::array<int32_t, 4>> mf_v(nmf);
  {
    int64_t f = 0;
    for (int e = 0; e < ne; ++e) {
      int k = in.elem_kind[e];
      const int(*tab)[4] = kind_tab(k);
      int b = in.elem_vert_off[e];
      for (int j = 0; j < kind_nf(k); ++j, ++f) {
        int n = tab[j][3] ? 4 : 3;
        mf_nv[f] = n;
        mf_left[f] = otn_e[e + 1];
        mf_lf[f] = j + 1;
        int mn = 1 << 30;
        for (int q = 0; q < 4; ++q) {
          mf_v[f][q] = q < n ? otn_v[in.elem_vert[b + tab[j][q] - 1]] : 0;
          if (q < n) mn = std::min(mn, mf_v[f][q]);
        }
        mf_min[f] = mn;
      }
    }
  }

  // -- face deduplication grouped by smallest vertex id (:61-211)
  struct Slot {
    FaceKey key;
    int64_t src;  // minimal face that created it
    int right, rface;
  };
  int id_glob_max = 0;
  for (int64_t f = 0; f < nmf; ++f) id_glob_max = std::max(id_glob_max, (int)mf_min[f]);
  V grp_off(id_glob_max + 2, 0);
  for (int64_t f = 0; f < nmf; ++f) grp_off[mf_min[f] + 1]++;
  for (int g = 1; g <= id_glob_max + 1; ++g) grp_off[g] += grp_off[g - 1];
  std::vector<int64_t> grp(nmf);
  {
    V fill(grp_off.begin(), grp_off.end());
    for (int64_t f = 0; f < nmf; ++f) grp[fill[mf_min[f]]++] = f;
  }
  // boundary faces by group
  std::unordered_map<int, std::vector<int>> bf_by_min;
  for (int j = 0; j < in.n_bfaces; ++j) {
    int mn = 1 << 30;
    for (int q = in.bface_off[j]; q < in.bface_off[j + 1]; ++q) mn = std::min(mn, (int)otn_v[in.bface_vert[q]]);
    bf_by_min[mn].push_back(j);
  }
  V& f_off = T.arr["face_vert_off"];
  V fv_tmp, fl_tmp, fr_tmp, flf_tmp, frf_tmp;
  f_off.assign(1, 0);
  std::vector<Slot> slots;
  for (int g = 1; g <= id_glob_max; ++g) {
    slots.clear();
    for (int q = grp_off[g]; q < grp_off[g + 1]; ++q) {
      int64_t f = grp[q];
      FaceKey k = make_key(mf_v[f].data(), mf_nv[f]);
      bool found = false;
      for (Slot& s : slots)
        if (s.key == k) {
          s.right = mf_left[f];
          s.rface = mf_lf[f];
          found = true;
          break;
        }
      if (!found) slots.push_back(Slot{k, f, 0, 0});
    }
    auto it = bf_by_min.find(g);
    if (it != bf_by_min.end())
      for (int j : it->second) {
        int n = in.bface_off[j + 1] - in.bface_off[j];
        int32_t tmp[4] = {0, 0, 0, 0};
        for (int q = 0; q < n && q < 4; ++q) tmp[q] = otn_v[in.bface_vert[in.bface_off[j] + q]];
        if (n > 4) continue;
        FaceKey k = make_key(tmp, n);
        for (Slot& s : slots)
          if (s.key == k) {
            if (s.right <= 0) {
              s.right = -(in.bface_tag ? in.bface_tag[j] : 0);
              s.rface = 0;
            }
            break;
          }
      }
    for (const Slot& s : slots) {
      for (int q = 0; q < mf_nv[s.src]; ++q) fv_tmp.push_back(mf_v[s.src][q]);
      f_off.push_back((int32_t)fv_tmp.size());
      fl_tmp.push_back(mf_left[s.src]);
      flf_tmp.push_back(mf_lf[s.src]);
      fr_tmp.push_back(s.right);
      frf_tmp.push_back(s.rface);
    }
  }
  const int nf = (int)fl_tmp.size();

  // -- vertex -> face lists in face order (:299-333), then first-touch face order (:928-974)
  Csr vf0 = bucket(nv, f_off[nf], [&](auto put) {
    for (int f = 0; f < nf; ++f)
      for (int q = f_off[f]; q < f_off[f + 1]; ++q) put(fv_tmp[q], f + 1);
  });
  V otn_f(nf + 1, -1), nto_f(nf + 1, -1);
  {
    int iloc = 1;
    for (int v = 0; v < (int)vf0.val.size(); ++v) {
      int f = vf0.val[v];
      if (otn_f[f] < 0) {
        otn_f[f] = iloc;
        nto_f[iloc] = f;
        ++iloc;
      }
    }
  }
  T.n_faces = nf;
  V& fvo = T.arr["face_vert_off"];
  V& fv = T.arr["face_vert"];
  V& fl = T.arr["face_left"];
  V& fr = T.arr["face_right"];
  V& flf = T.arr["face_left_face"];
  V& frf = T.arr["face_right_face"];
  {
    V new_off(nf + 1, 0);
    for (int fn = 1; fn <= nf; ++fn) {
      int fo = nto_f[fn] - 1;
      new_off[fn] = new_off[fn - 1] + (f_off[fo + 1] - f_off[fo]);
    }
    fv.resize(new_off[nf]);
    fl.resize(nf);
    fr.resize(nf);
    flf.resize(nf);
    frf.resize(nf);
    for (int fn = 1; fn <= nf; ++fn) {
      int fo = nto_f[fn] - 1;
      std::copy(fv_tmp.begin() + f_off[fo], fv_tmp.begin() + f_off[fo + 1], fv.begin() + new_off[fn - 1]);
      fl[fn - 1] = fl_tmp[fo];
      fr[fn - 1] = fr_tmp[fo];
      flf[fn - 1] = flf_tmp[fo];
      frf[fn - 1] = frf_tmp[fo];
    }
    fvo = new_off;
  }
  V& vfo = T.arr["vert_face_off"];
  V& vfl = T.arr["vert_face"];
  vfo = vf0.off;
  vfl.resize(vf0.val.size());
  for (size_t q = 0; q < vf0.val.size(); ++q) vfl[q] = otn_f[vf0.val[q]];

  // element -> face (by local face index)
  V& efo = T.arr["elem_face_off"];
  V& ef = T.arr["elem_face"];
  efo.assign(ne + 1, 0);
  for (int e = 1; e <= ne; ++e) efo[e] = efo[e - 1] + kind_nf(ekind[e - 1]);
  ef.assign(efo[ne], 0);
  for (int f = 1; f <= nf; ++f) {
    ef[efo[fl[f - 1] - 1] + flf[f - 1] - 1] = f;
    if (fr[f - 1] > 0) ef[efo[fr[f - 1] - 1] + frf[f - 1] - 1] = f;
  }

  // -- subfaces (:335-402): vertex by vertex over each vertex's face list
  V& esfo = T.arr["elem_sub_face_off"];
  V& esf = T.arr["elem_sub_face"];
  esfo.assign(ne + 1, 0);
  for (int e = 1; e <= ne; ++e) {
    int s = 0;
    for (int q = efo[e - 1]; q < efo[e]; ++q) s += fvo[ef[q]] - fvo[ef[q] - 1];
    esfo[e] = esfo[e - 1] + s;
  }
  esf.assign(esfo[ne], -1);
  const int nsf = fvo[nf];
  T.n_sub_faces = nsf;
  V& fsf = T.arr["face_sub_face"];
  T.arr["face_sub_face_off"] = fvo;
  fsf.assign(nsf, -1);
  V& sfv = T.arr["sub_face_vert"];
  V& sff = T.arr["sub_face_face"];
  V& sfl = T.arr["sub_face_left_elem"];
  V& sfr = T.arr["sub_face_right_elem"];
  sfv.resize(nsf);
  sff.resize(nsf);
  sfl.resize(nsf);
  sfr.resize(nsf);
  {
    V ffill(fvo.begin(), fvo.end() - 1), efill(esfo.begin(), esfo.end() - 1);
    int id = 1;
    for (int v = 1; v <= nv; ++v)
      for (int q = vfo[v - 1]; q < vfo[v]; ++q, ++id) {
        int f = vfl[q];
        fsf[ffill[f - 1]++] = id;
        sff[id - 1] = f;
        sfv[id - 1] = v;
        sfl[id - 1] = fl[f - 1];
        sfr[id - 1] = fr[f - 1];
        esf[efill[fl[f - 1] - 1]++] = id;
        if (fr[f - 1] > 0) esf[efill[fr[f - 1] - 1]++] = id;
      }
  }

  // -- subelements (:404-452): one per (cell, vertex), in cell then vertex order
  const int nse = ev_off[ne];
  T.n_sub_elems = nse;
  V& ese = T.arr["elem_sub_elem"];
  T.arr["elem_sub_elem_off"] = ev_off;
  ese.resize(nse);
  V& see = T.arr["sub_elem_elem"];
  V& sev = T.arr["sub_elem_vert"];
  V& sesfo = T.arr["sub_elem_sub_face_off"];
  V& sesf = T.arr["sub_elem_sub_face"];
  see.resize(nse);
  sev.resize(nse);
  sesfo.assign(nse + 1, 0);
  sesf.clear();
  sesf.reserve(3 * (size_t)nse);
  std::vector<int32_t> lv;  // the cell's subfaces' vertices, gathered once per cell
  for (int e = 1; e <= ne; ++e) {
    const int q0 = esfo[e - 1], q1 = esfo[e];
    lv.resize(q1 - q0);
    for (int q = q0; q < q1; ++q) lv[q - q0] = sfv[esf[q] - 1];
    for (int j = ev_off[e - 1]; j < ev_off[e]; ++j) {
      int id = j + 1;
      ese[j] = id;
      see[j] = e;
      sev[j] = 0;
      for (int q = q0; q < q1; ++q)
        if (lv[q - q0] == ev[j]) {
          sev[j] = lv[q - q0];
          sesf.push_back(esf[q]);
        }
      sesfo[id] = (int32_t)sesf.size();
    }
  }
  // (:454-473)
  V& sfls = T.arr["sub_face_left_sub_elem"];
  V& sfrs = T.arr["sub_face_right_sub_elem"];
  sfls.assign(nsf, 0);
  sfrs.assign(nsf, 0);
  for (int s = 1; s <= nse; ++s)
    for (int q = sesfo[s - 1]; q < sesfo[s]; ++q) {
      int sf = sesf[q];
      if (sfl[sf - 1] == see[s - 1]) sfls[sf - 1] = s;
      if (sfr[sf - 1] == see[s - 1]) sfrs[sf - 1] = s;
    }

  // -- vertex -> subface / subelement lists in id order (:511-556)
  {
    Csr c = bucket(nv, nsf, [&](auto put) {
      for (int s = 1; s <= nsf; ++s) put(sfv[s - 1], s);
    });
    T.arr["vert_sub_face_off"] = c.off;
    T.arr["vert_sub_face"] = c.val;
    V& loc = T.arr["sub_face_loc"];
    loc.resize(nsf);
    for (int v = 1; v <= nv; ++v)
      for (int q = c.off[v - 1]; q < c.off[v]; ++q) loc[c.val[q] - 1] = q - c.off[v - 1] + 1;
    Csr d = bucket(nv, nse, [&](auto put) {
      for (int s = 1; s <= nse; ++s) put(sev[s - 1], s);
    });
    T.arr["vert_sub_elem_off"] = d.off;
    T.arr["vert_sub_elem"] = d.val;
    V& sl = T.arr["sub_elem_loc"];
    sl.resize(nse);
    for (int v = 1; v <= nv; ++v)
      for (int q = d.off[v - 1]; q < d.off[v]; ++q) sl[d.val[q] - 1] = q - d.off[v - 1] + 1;
  }

  // -- max subfaces per vertex, before any periodic extension (:581-593)
  {
    int mx = 0;
    const V& o = T.a("vert_sub_face_off");
    for (int v = 1; v <= nv; ++v) mx = std::max(mx, o[v] - o[v - 1]);
    T.n_max_sub_faces_around_node = mx;
  }
  // -- cell tags (:558-579)
  V& etag = T.arr["elem_tag"];
  etag.assign(ne, -1);
  for (int f = 1; f <= nf; ++f)
    if (fr[f - 1] < 0) {
      int tag = -fr[f - 1];
      int32_t& t = etag[fl[f - 1] - 1];
      if (t < 0 || t > tag) t = tag;
    }

  // -- neighbours by vertex, first occurrence kept (:595-654)
  {
    V& no = T.arr["elem_neigh_by_vert_off"];
    V& nb = T.arr["elem_neigh_by_vert"];
    no.assign(ne + 1, 0);
    nb.clear();
    V stamp(ne + 1, 0);
    for (int e = 1; e <= ne; ++e) {
      for (int j = ev_off[e - 1]; j < ev_off[e]; ++j) {
        int v = ev[j];
        for (int q = vel_off[v - 1]; q < vel_off[v]; ++q) {
          int o = vel[q];
          if (o != e && stamp[o] != e) {
            stamp[o] = e;
            nb.push_back(o);
          }
        }
      }
      no[e] = (int32_t)nb.size();
    }
  }

  // -- periodic stitching (:976-1073) and stencil extension (:1075-1328)
  if (in.periodic) {
    const double lo = -0.5, hi = 0.5;
    std::vector<double> fc(3 * (size_t)nf, 0.0);
    for (int f = 1; f <= nf; ++f) {
      double c[3] = {0, 0, 0};
      int n = fvo[f] - fvo[f - 1];
      for (int q = fvo[f - 1]; q < fvo[f]; ++q)
        for (int d = 0; d < 3; ++d) c[d] = c[d] + T.vert_coord[3 * (fv[q] - 1) + d];
      for (int d = 0; d < 3; ++d) fc[3 * (f - 1) + d] = c[d] / (double)n;
    }
    // match planes by hashing the two in-plane coordinates on a 1e-9 grid
    auto match_planes = [&](const double* pc, int npts, auto on_pair) {
      for (int d = 0; d < 3; ++d) {
        int a = d == 0 ? 1 : 0, b = d == 2 ? 1 : 2;
        std::vector<int> L, R;
        for (int i = 0; i < npts; ++i) {
          if (near(pc[3 * i + d], lo)) L.push_back(i);
          if (near(pc[3 * i + d], hi)) R.push_back(i);
        }
        if (L.size() != R.size()) return false;
        std::unordered_map<int64_t, std::vector<int>> h;
        auto key = [](double x, double y) {
          return (int64_t)std::llround(x * 1e9) * 1000003LL + (int64_t)std::llround(y * 1e9);
        };
        for (int j : R) h[key(pc[3 * j + a], pc[3 * j + b])].push_back(j);
        for (int i : L) {
          std::vector<int> cand;
          for (int dx = -1; dx <= 1; ++dx)
            for (int dy = -1; dy <= 1; ++dy) {
              auto it = h.find(key(pc[3 * i + a] + dx * 1e-9, pc[3 * i + b] + dy * 1e-9));
              if (it != h.end()) cand.insert(cand.end(), it->second.begin(), it->second.end());
            }
          std::sort(cand.begin(), cand.end());
          cand.erase(std::unique(cand.begin(), cand.end()), cand.end());
          for (int j : cand) {
            double da = pc[3 * i + a] - pc[3 * j + a], db = pc[3 * i + b] - pc[3 * j + b];
            if (std::sqrt(da * da + db * db) < 1e-12) on_pair(d, i, j);
          }
        }
      }
      return true;
    };
    bool ok = match_planes(fc.data(), nf, [&](int, int i, int j) {
      fr[i] = fl[j];
      fr[j] = fl[i];
    });
    if (!ok) return fail("Error periodic boundaries !");
    for (int s = 1; s <= nsf; ++s) {
      sfl[s - 1] = fl[sff[s - 1] - 1];
      sfr[s - 1] = fr[sff[s - 1] - 1];
    }
    // stencil extension works on per-vertex lists
    std::vector<V> vsf(nv + 1), vse(nv + 1);
    {
      const V& o = T.a("vert_sub_face_off");
      const V& l = T.a("vert_sub_face");
      const V& o2 = T.a("vert_sub_elem_off");
      const V& l2 = T.a("vert_sub_elem");
      for (int v = 1; v <= nv; ++v) {
        vsf[v].assign(l.begin() + o[v - 1], l.begin() + o[v]);
        vse[v].assign(l2.begin() + o2[v - 1], l2.begin() + o2[v]);
      }
    }
    auto sf_match = [&](int p, int q) {
      return (sfl[p - 1] == sfr[q - 1] && sfr[p - 1] == sfl[q - 1]) ||
             (sfl[p - 1] == sfl[q - 1] && sfr[p - 1] == sfr[q - 1]);
    };
    auto process_pair = [&](int v1, int v2) {
      for (int sf : vsf[v1]) {
        int re = sfr[sf - 1];
        if (re > 0 && sfrs[sf - 1] == 0)
          for (int se : vse[v2])
            if (see[se - 1] == re) {
              sfrs[sf - 1] = se;
              break;
            }
      }
      int nm = 0;
      for (int a : vsf[v1])
        for (int b : vsf[v2])
          if (sf_match(a, b)) ++nm;
      int n1 = (int)vsf[v1].size();
      int st = n1 + (int)vsf[v2].size() - nm;
      vsf[v1].resize(st, -1);
      for (int ki = 0; ki < st; ++ki) {
        if (vsf[v1][ki] >= 0) continue;
        for (int b : vsf[v2]) {
          bool found = false;
          for (int p = 0; p < ki; ++p) {
            int sp = vsf[v1][p];
            if (sp < 0) continue;
            if (sf_match(sp, b)) found = true;
          }
          if (!found) {
            vsf[v1][ki] = b;
            break;
          }
        }
      }
      for (int se : std::vector<int32_t>(vse[v2]))
        if (sev[se - 1] == v2) vse[v1].push_back(se);
    };
    const double* pc = T.vert_coord.data();
    match_planes(pc, nv, [&](int, int i, int j) {
      process_pair(i + 1, j + 1);
      process_pair(j + 1, i + 1);
    });
    // edge diagonals xy, xz, yz then the xyz corner (:1158-1220)
    const int dg[3][3] = {{0, 1, 2}, {0, 2, 1}, {1, 2, 0}};
    for (const auto& g : dg) {
      std::vector<int> L, R;
      for (int i = 0; i < nv; ++i) {
        if (near(pc[3 * i + g[0]], lo) && near(pc[3 * i + g[1]], lo)) L.push_back(i);
        if (near(pc[3 * i + g[0]], hi) && near(pc[3 * i + g[1]], hi)) R.push_back(i);
      }
      for (int i : L)
        for (int j : R)
          if (std::fabs(pc[3 * i + g[2]] - pc[3 * j + g[2]]) < 1e-12) {
            process_pair(i + 1, j + 1);
            process_pair(j + 1, i + 1);
          }
    }
    {
      std::vector<int> L, R;
      for (int i = 0; i < nv; ++i) {
        if (near(pc[3 * i], lo) && near(pc[3 * i + 1], lo) && near(pc[3 * i + 2], lo)) L.push_back(i);
        if (near(pc[3 * i], hi) && near(pc[3 * i + 1], hi) && near(pc[3 * i + 2], hi)) R.push_back(i);
      }
      for (int i : L)
        for (int j : R) {
          process_pair(i + 1, j + 1);
          process_pair(j + 1, i + 1);
        }
    }
    V& o = T.arr["vert_sub_face_off"];
    V& l = T.arr["vert_sub_face"];
    V& o2 = T.arr["vert_sub_elem_off"];
    V& l2 = T.arr["vert_sub_elem"];
    l.clear();
    l2.clear();
    for (int v = 1; v <= nv; ++v) {
      l.insert(l.end(), vsf[v].begin(), vsf[v].end());
      o[v] = (int32_t)l.size();
      l2.insert(l2.end(), vse[v].begin(), vse[v].end());
      o2[v] = (int32_t)l2.size();
    }
  }

  // boundary flags as build_mesh leaves them: face normals are still zero there (:726-750)
  V& vb = T.arr["vert_is_bound"];
  vb.assign(nv, 0);
  for (int v = 1; v <= nv; ++v)
    for (int q = vfo[v - 1]; q < vfo[v]; ++q)
      if (fr[vfl[q] - 1] <= 0) vb[v - 1] = 1;
  T.arr["sizes"] = {nv, ne, nf, nsf, nse, T.n_max_sub_faces_around_node};
  return 0;
}

}  // namespace subfv
