// Test infrastructure only (oracle). Restatement of the subfv mesh pipeline:
// MSH2 element->face tables, build_mesh topology, compute_geometry_mesh.
// PARITY UNPINNED (no Fortran compiler here; the reference tests hold no golden data).
#include <algorithm>
#include "oracle.h"
#include <cmath>
#include <cstdio>
#include <stdexcept>

namespace oracle {

double fnorm2(const double* a, int n) {
  double scale = 1.0, res = 0.0;
  for (int i = 0; i < n; ++i) {
    if (a[i] != 0.0) {
      double ax = std::fabs(a[i]);
      if (ax > scale) {
        double v = scale / ax;
        res = 1.0 + res * v * v;
        scale = ax;
      } else {
        double v = ax / scale;
        res += v * v;
      }
    }
  }
  return scale * std::sqrt(res);
}

// ---------------------------------------------------------------------------------
// src/mesh/mesh_reading_module.F90:1144-1320: one minimal face per element face, in
// element order, with the per-kind local vertex tables (1-based local indices).
static const int kTet[4][4] = {{1, 3, 2, 0}, {1, 2, 4, 0}, {1, 4, 3, 0}, {2, 3, 4, 0}};
static const int kHex[6][4] = {{1, 4, 3, 2}, {3, 4, 8, 7}, {7, 8, 5, 6},
                               {1, 2, 6, 5}, {1, 5, 8, 4}, {2, 3, 7, 6}};
static const int kPri[5][4] = {{1, 3, 2, 0}, {4, 5, 6, 0}, {1, 2, 5, 4}, {2, 3, 6, 5}, {1, 4, 6, 3}};
static const int kPyr[5][4] = {{1, 4, 3, 2}, {1, 2, 5, 0}, {2, 3, 5, 0}, {3, 4, 5, 0}, {1, 5, 4, 0}};

static int n_face_kind(int k) { return k == 4 ? 4 : k == 5 ? 6 : (k == 6 || k == 7) ? 5 : 0; }
static int n_vert_kind(int k) { return k == 4 ? 4 : k == 5 ? 8 : k == 6 ? 6 : k == 7 ? 5 : 0; }

void read_raw(Mesh& m, int n_vert, const double* coords, int n_elems, const int* kind,
              const int* ev_off, const int* ev, int n_bf, const int* bf_off, const int* bf_vert,
              const int* bf_tag) {
  m.n_vert = n_vert;
  m.n_elems = n_elems;
  int nf = 0;
  for (int i = 0; i < n_elems; ++i) nf += n_face_kind(kind[i]);
  m.n_faces = nf;
  m.n_boundary_faces = n_bf;
  m.vert.assign(n_vert + 1, Vert());
  m.elem.assign(n_elems + 1, Elem());
  m.minimal_face.assign(nf + 1, MinFace());
  m.boundary_face.assign(n_bf + 1, BFace());
  for (int i = 1; i <= n_vert; ++i)
    for (int d = 1; d <= 3; ++d) m.vert[i].coord[d] = coords[3 * (i - 1) + d - 1];
  for (int j = 1; j <= n_bf; ++j) {
    BFace& b = m.boundary_face[j];
    b.tag = bf_tag ? bf_tag[j - 1] : 0;
    b.n_vert = bf_off[j] - bf_off[j - 1];
    b.vert.assign(b.n_vert + 1, 0);
    for (int k = 1; k <= b.n_vert; ++k) b.vert[k] = bf_vert[bf_off[j - 1] + k - 1];
  }
  int n_faces = 1;
  for (int iloc = 1; iloc <= n_elems; ++iloc) {
    Elem& e = m.elem[iloc];
    int k = kind[iloc - 1];
    if (ev_off[iloc] - ev_off[iloc - 1] != n_vert_kind(k)) throw std::runtime_error("bad element");
    e.elem_kind = k;
    e.n_vert = n_vert_kind(k);
    e.n_faces = n_face_kind(k);
    e.vert.assign(e.n_vert + 1, 0);
    for (int j = 1; j <= e.n_vert; ++j) e.vert[j] = ev[ev_off[iloc - 1] + j - 1];
    e.face.assign(e.n_faces + 1, 0);
    const int(*tab)[4] = k == 4 ? kTet : k == 5 ? kHex : k == 6 ? kPri : kPyr;
    for (int j = 1; j <= e.n_faces; ++j) {
      MinFace& f = m.minimal_face[n_faces + j - 1];
      f.left_neigh = iloc;
      f.left_neigh_face = j;
      int nv = tab[j - 1][3] ? 4 : 3;
      f.n_vert = nv;
      f.vert.assign(nv + 1, 0);
      for (int q = 1; q <= nv; ++q) f.vert[q] = e.vert[tab[j - 1][q - 1]];
      e.face[j] = n_faces + j - 1;
    }
    n_faces += e.n_faces;
  }
}

// ---------------------------------------------------------------------------------
// mesh_connectivity_module.F90:475-509
static void build_node_elem_neigh(Mesh& m) {
  for (int i = 1; i <= m.n_vert; ++i) m.vert[i].n_elems_neigh = 0;
  for (int i = 1; i <= m.n_elems; ++i)
    for (int j = 1; j <= m.elem[i].n_vert; ++j) m.vert[m.elem[i].vert[j]].n_elems_neigh++;
  for (int i = 1; i <= m.n_vert; ++i) m.vert[i].elem_neigh.assign(m.vert[i].n_elems_neigh + 1, 0);
  for (int i = 1; i <= m.n_vert; ++i) m.vert[i].n_elems_neigh = 0;
  for (int i = 1; i <= m.n_elems; ++i)
    for (int j = 1; j <= m.elem[i].n_vert; ++j) {
      Vert& v = m.vert[m.elem[i].vert[j]];
      v.elem_neigh[v.n_elems_neigh + 1] = i;
      v.n_elems_neigh++;
    }
}

// mesh_connectivity_module.F90:851-926 (BFS by element adjacency, level by level)
static void renumber_vert_mesh(Mesh& m) {
  int nv = m.n_vert;
  std::vector<int> otn(nv + 1, -1), nto(nv + 1, -1);
  otn[1] = 1;
  nto[1] = 1;
  int iloc = 2;
  int iloc_start = iloc - 1, iloc_end = iloc - 1;
  while (iloc <= nv) {
    int iloc_before = iloc;
    for (int i = iloc_start; i <= iloc_end; ++i) {  // bounds fixed at loop entry
      int id_vert = nto[i];
      for (int j = 1; j <= m.vert[id_vert].n_elems_neigh; ++j) {
        int id_elem = m.vert[id_vert].elem_neigh[j];
        for (int k = 1; k <= m.elem[id_elem].n_vert; ++k) {
          int nb = m.elem[id_elem].vert[k];
          if (otn[nb] < 0) {
            otn[nb] = iloc;
            nto[iloc] = nb;
            iloc++;
          }
        }
      }
    }
    if (iloc == iloc_before) {
      for (int i = 1; i <= nv; ++i)
        if (otn[i] < 0) {
          otn[i] = iloc;
          nto[iloc] = i;
          iloc++;
          break;
        }
    }
    iloc_start = iloc_end + 1;
    iloc_end = iloc - 1;
  }
  std::vector<Vert> tmp = m.vert;
  for (int i = 1; i <= nv; ++i) m.vert[otn[i]] = tmp[i];
  for (int i = 1; i <= m.n_elems; ++i)
    for (int j = 1; j <= m.elem[i].n_vert; ++j) m.elem[i].vert[j] = otn[m.elem[i].vert[j]];
  for (int i = 1; i <= m.n_faces; ++i)
    for (int j = 1; j <= m.minimal_face[i].n_vert; ++j)
      m.minimal_face[i].vert[j] = otn[m.minimal_face[i].vert[j]];
  for (int i = 1; i <= m.n_boundary_faces; ++i)
    for (int j = 1; j <= m.boundary_face[i].n_vert; ++j)
      m.boundary_face[i].vert[j] = otn[m.boundary_face[i].vert[j]];
}

// Not in the reference: the vertices along a Hilbert curve instead of the BFS order, for
// checking the library's optional renumbering. J. Skilling, "Programming the Hilbert
// curve", AIP Conf. Proc. 707, 381 (2004): the grid point's coordinates are turned into
// the transposed Hilbert index (inverse undo, then Gray encode) and its bits read most
// significant first across the axes. Slabs use (x, y) with 31 bits, else (x, y, z) with
// 21 bits, on a cube of the largest extent; equal keys keep the input order.
static unsigned long long skilling_key(unsigned int x[3], int n, int b) {
  unsigned int m = 1u << (b - 1);
  for (unsigned int q = m; q > 1; q >>= 1) {
    unsigned int p = q - 1;
    for (int i = 0; i < n; ++i) {
      if (x[i] & q) {
        x[0] ^= p;
      } else {
        unsigned int t = (x[0] ^ x[i]) & p;
        x[0] ^= t;
        x[i] ^= t;
      }
    }
  }
  for (int i = 1; i < n; ++i) x[i] ^= x[i - 1];
  unsigned int t = 0;
  for (unsigned int q = m; q > 1; q >>= 1)
    if (x[n - 1] & q) t ^= q - 1;
  for (int i = 0; i < n; ++i) x[i] ^= t;
  unsigned long long key = 0;
  for (int bit = b - 1; bit >= 0; --bit)
    for (int i = 0; i < n; ++i) key = (key << 1) | ((x[i] >> bit) & 1u);
  return key;
}

static void apply_vert_order(Mesh& m, const std::vector<int>& otn) {
  std::vector<Vert> tmp = m.vert;
  for (int i = 1; i <= m.n_vert; ++i) m.vert[otn[i]] = tmp[i];
  for (int i = 1; i <= m.n_elems; ++i)
    for (int j = 1; j <= m.elem[i].n_vert; ++j) m.elem[i].vert[j] = otn[m.elem[i].vert[j]];
  for (int i = 1; i <= m.n_faces; ++i)
    for (int j = 1; j <= m.minimal_face[i].n_vert; ++j)
      m.minimal_face[i].vert[j] = otn[m.minimal_face[i].vert[j]];
  for (int i = 1; i <= m.n_boundary_faces; ++i)
    for (int j = 1; j <= m.boundary_face[i].n_vert; ++j)
      m.boundary_face[i].vert[j] = otn[m.boundary_face[i].vert[j]];
}

static void renumber_vert_hilbert(Mesh& m, bool b2d) {
  int nv = m.n_vert, n = b2d ? 2 : 3, bits = b2d ? 31 : 21;
  double lo[3], hi[3];
  for (int d = 0; d < 3; ++d) lo[d] = hi[d] = m.vert[1].coord[d + 1];
  for (int i = 2; i <= nv; ++i)
    for (int d = 0; d < 3; ++d) {
      if (m.vert[i].coord[d + 1] < lo[d]) lo[d] = m.vert[i].coord[d + 1];
      if (m.vert[i].coord[d + 1] > hi[d]) hi[d] = m.vert[i].coord[d + 1];
    }
  double ext = 0.0;
  for (int d = 0; d < n; ++d)
    if (hi[d] - lo[d] > ext) ext = hi[d] - lo[d];
  double top = (double)((1u << bits) - 1u);
  double scale = ext > 0.0 ? top / ext : 0.0;
  std::vector<std::pair<unsigned long long, int>> order(nv);
  for (int i = 1; i <= nv; ++i) {
    unsigned int x[3] = {0, 0, 0};
    for (int d = 0; d < n; ++d) {
      double q = (m.vert[i].coord[d + 1] - lo[d]) * scale;
      if (q < 0.0) q = 0.0;
      if (q > top) q = top;
      x[d] = (unsigned int)q;
    }
    order[i - 1] = std::make_pair(skilling_key(x, n, bits), i);
  }
  std::sort(order.begin(), order.end());
  std::vector<int> otn(nv + 1, -1);
  for (int k = 0; k < nv; ++k) otn[order[k].second] = k + 1;
  apply_vert_order(m, otn);
}

// mesh_connectivity_module.F90:752-849 (num_procs = 1: first touch over vertices)
static void renumber_elem_mesh(Mesh& m) {
  std::vector<int> otn(m.n_elems + 1, -1);
  int iloc = 1;
  for (int i = 1; i <= m.n_vert; ++i)
    for (int j = 1; j <= m.vert[i].n_elems_neigh; ++j) {
      int le = m.vert[i].elem_neigh[j];
      if (otn[le] <= 0) {
        otn[le] = iloc;
        iloc++;
      }
    }
  std::vector<Elem> tmp = m.elem;
  for (int i = 1; i <= m.n_elems; ++i) m.elem[otn[i]] = tmp[i];
  for (int i = 1; i <= m.n_faces; ++i) m.minimal_face[i].left_neigh = otn[m.minimal_face[i].left_neigh];
  for (int i = 1; i <= m.n_vert; ++i)
    for (int j = 1; j <= m.vert[i].n_elems_neigh; ++j)
      m.vert[i].elem_neigh[j] = otn[m.vert[i].elem_neigh[j]];
}

// mesh_connectivity_module.F90:679-724
static bool same_faces(const std::vector<int>& av, int an, const std::vector<int>& bv, int bn) {
  if (an != bn) return false;
  bool same = true;
  for (int i = 1; i <= an; ++i) {
    bool found = false;
    for (int j = 1; j <= bn; ++j)
      if (av[i] == bv[j]) found = true;
    same = found && same;
  }
  return same;
}

// mesh_connectivity_module.F90:61-211
static void build_faces(Mesh& m) {
  int n_faces = 0, id_glob_max = 0;
  auto idmin = [](const std::vector<int>& v, int n) {
    int r = v[1];
    for (int k = 2; k <= n; ++k) r = std::min(r, v[k]);
    return r;
  };
  for (int j = 1; j <= m.n_faces; ++j)
    id_glob_max = std::max(id_glob_max, idmin(m.minimal_face[j].vert, m.minimal_face[j].n_vert));
  std::vector<int> n_collision(id_glob_max + 1, 0);
  for (int j = 1; j <= m.n_faces; ++j) n_collision[idmin(m.minimal_face[j].vert, m.minimal_face[j].n_vert)]++;
  std::vector<std::vector<MinFace>> cont(id_glob_max + 1);
  for (int j = 1; j <= id_glob_max; ++j) cont[j].assign(n_collision[j] + 1, MinFace());
  for (int j = 1; j <= m.n_faces; ++j) {
    const MinFace& mf = m.minimal_face[j];
    int id = idmin(mf.vert, mf.n_vert);
    bool already = false;
    for (int k = 1; k <= n_collision[id]; ++k) {
      MinFace& c = cont[id][k];
      if (c.n_vert > 0 && same_faces(mf.vert, mf.n_vert, c.vert, c.n_vert)) {
        already = true;
        c.right_neigh = mf.left_neigh;
        c.right_neigh_face = mf.left_neigh_face;
        break;
      }
    }
    if (!already) {
      for (int k = 1; k <= n_collision[id]; ++k) {
        MinFace& c = cont[id][k];
        if (c.n_vert <= 0) {
          n_faces++;
          c.n_vert = mf.n_vert;
          c.vert = mf.vert;
          c.left_neigh = mf.left_neigh;
          c.left_neigh_face = mf.left_neigh_face;
          break;
        }
      }
    }
  }
  for (int j = 1; j <= m.n_boundary_faces; ++j) {
    const BFace& bf = m.boundary_face[j];
    int id = idmin(bf.vert, bf.n_vert);
    if (id > id_glob_max) continue;  // a boundary face with no element face
    for (int k = 1; k <= n_collision[id]; ++k) {
      MinFace& c = cont[id][k];
      if (c.n_vert > 0 && same_faces(bf.vert, bf.n_vert, c.vert, c.n_vert)) {
        if (c.right_neigh <= 0) {
          c.right_neigh = -bf.tag;
          c.right_neigh_face = 0;
        }
        break;
      }
    }
  }
  m.minimal_face.clear();
  m.n_faces = n_faces;
  m.face.assign(n_faces + 1, Face());
  n_faces = 0;
  for (int j = 1; j <= id_glob_max; ++j)
    for (int k = 1; k <= n_collision[j]; ++k) {
      MinFace& c = cont[j][k];
      if (c.n_vert > 0) {
        n_faces++;
        Face& f = m.face[n_faces];
        f.n_vert = c.n_vert;
        f.vert = c.vert;
        f.left_neigh = c.left_neigh;
        f.left_neigh_face = c.left_neigh_face;
        f.right_neigh = c.right_neigh;
        f.right_neigh_face = c.right_neigh_face;
        m.elem[f.left_neigh].face[f.left_neigh_face] = n_faces;
        if (f.right_neigh > 0) m.elem[f.right_neigh].face[f.right_neigh_face] = n_faces;
      }
    }
}

// mesh_connectivity_module.F90:299-333
static void build_node_face_connectivity(Mesh& m) {
  for (int i = 1; i <= m.n_vert; ++i) m.vert[i].n_faces_neigh = 0;
  for (int i = 1; i <= m.n_faces; ++i)
    for (int j = 1; j <= m.face[i].n_vert; ++j) m.vert[m.face[i].vert[j]].n_faces_neigh++;
  for (int i = 1; i <= m.n_vert; ++i) m.vert[i].face_neigh.assign(m.vert[i].n_faces_neigh + 1, -1);
  for (int i = 1; i <= m.n_faces; ++i)
    for (int j = 1; j <= m.face[i].n_vert; ++j) {
      Vert& v = m.vert[m.face[i].vert[j]];
      for (int k = 1; k <= v.n_faces_neigh; ++k)
        if (v.face_neigh[k] < 0) {
          v.face_neigh[k] = i;
          break;
        }
    }
}

// mesh_connectivity_module.F90:928-974
static void renumber_faces_mesh(Mesh& m) {
  std::vector<int> otn(m.n_faces + 1, -1);
  int iloc = 1;
  for (int i = 1; i <= m.n_vert; ++i)
    for (int j = 1; j <= m.vert[i].n_faces_neigh; ++j) {
      int f = m.vert[i].face_neigh[j];
      if (otn[f] < 0) otn[f] = iloc++;
    }
  std::vector<Face> tmp = m.face;
  for (int i = 1; i <= m.n_faces; ++i) m.face[otn[i]] = tmp[i];
  for (int i = 1; i <= m.n_elems; ++i)
    for (int j = 1; j <= m.elem[i].n_faces; ++j) m.elem[i].face[j] = otn[m.elem[i].face[j]];
  for (int i = 1; i <= m.n_vert; ++i)
    for (int j = 1; j <= m.vert[i].n_faces_neigh; ++j) m.vert[i].face_neigh[j] = otn[m.vert[i].face_neigh[j]];
}

// mesh_connectivity_module.F90:335-402
static void build_sub_faces(Mesh& m) {
  m.n_sub_faces = 0;
  for (int i = 1; i <= m.n_faces; ++i) {
    m.face[i].n_sub_faces = m.face[i].n_vert;
    m.face[i].sub_face.assign(m.face[i].n_sub_faces + 1, -1);
    m.n_sub_faces += m.face[i].n_vert;
  }
  m.sub_face.assign(m.n_sub_faces + 1, SubFace());
  for (int i = 1; i <= m.n_elems; ++i) {
    Elem& e = m.elem[i];
    e.n_sub_faces = 0;
    for (int j = 1; j <= e.n_faces; ++j) e.n_sub_faces += m.face[e.face[j]].n_vert;
    e.sub_face.assign(e.n_sub_faces + 1, -1);
  }
  int id_sub_face = 1;
  for (int i = 1; i <= m.n_vert; ++i)
    for (int j = 1; j <= m.vert[i].n_faces_neigh; ++j) {
      int id_face = m.vert[i].face_neigh[j];
      Face& f = m.face[id_face];
      for (int k = 1; k <= f.n_sub_faces; ++k)
        if (f.sub_face[k] < 0) {
          f.sub_face[k] = id_sub_face;
          break;
        }
      SubFace& s = m.sub_face[id_sub_face];
      s.mesh_face = id_face;
      s.mesh_vert = i;
      s.left_elem_neigh = f.left_neigh;
      s.right_elem_neigh = f.right_neigh;
      Elem& el = m.elem[f.left_neigh];
      for (int k = 1; k <= el.n_sub_faces; ++k)
        if (el.sub_face[k] < 0) {
          el.sub_face[k] = id_sub_face;
          break;
        }
      if (f.right_neigh > 0) {
        Elem& er = m.elem[f.right_neigh];
        for (int k = 1; k <= er.n_sub_faces; ++k)
          if (er.sub_face[k] < 0) {
            er.sub_face[k] = id_sub_face;
            break;
          }
      }
      id_sub_face++;
    }
}

// mesh_connectivity_module.F90:404-452
static void build_sub_elems(Mesh& m) {
  m.n_sub_elems = 0;
  for (int i = 1; i <= m.n_elems; ++i) {
    m.elem[i].n_sub_elems = m.elem[i].n_vert;
    m.elem[i].sub_elem.assign(m.elem[i].n_sub_elems + 1, 0);
    m.n_sub_elems += m.elem[i].n_sub_elems;
  }
  m.sub_elem.assign(m.n_sub_elems + 1, SubElem());
  int id_sub_elem = 1;
  for (int i = 1; i <= m.n_elems; ++i)
    for (int j = 1; j <= m.elem[i].n_vert; ++j) {
      SubElem& se = m.sub_elem[id_sub_elem];
      se.n_sub_faces = 0;
      for (int k = 1; k <= m.elem[i].n_sub_faces; ++k)
        if (m.sub_face[m.elem[i].sub_face[k]].mesh_vert == m.elem[i].vert[j]) se.n_sub_faces++;
      se.sub_face.assign(se.n_sub_faces + 1, 0);
      id_sub_elem++;
    }
  id_sub_elem = 1;
  for (int i = 1; i <= m.n_elems; ++i)
    for (int j = 1; j <= m.elem[i].n_vert; ++j) {
      int loc = 1;
      m.elem[i].sub_elem[j] = id_sub_elem;
      SubElem& se = m.sub_elem[id_sub_elem];
      for (int k = 1; k <= m.elem[i].n_sub_faces; ++k) {
        int sf = m.elem[i].sub_face[k];
        if (m.sub_face[sf].mesh_vert == m.elem[i].vert[j]) {
          se.mesh_elem = i;
          se.mesh_vert = m.sub_face[sf].mesh_vert;
          se.sub_face[loc] = sf;
          loc++;
        }
      }
      id_sub_elem++;
    }
}

// mesh_connectivity_module.F90:454-473
static void find_sub_elems_around_sub_face(Mesh& m) {
  for (int i = 1; i <= m.n_sub_elems; ++i) {
    int e = m.sub_elem[i].mesh_elem;
    for (int j = 1; j <= m.sub_elem[i].n_sub_faces; ++j) {
      SubFace& s = m.sub_face[m.sub_elem[i].sub_face[j]];
      if (s.left_elem_neigh == e) s.left_sub_elem_neigh = i;
      if (s.right_elem_neigh == e) s.right_sub_elem_neigh = i;
    }
  }
}

// mesh_connectivity_module.F90:511-556
static void build_node_sub_face_connectivity(Mesh& m) {
  for (int i = 1; i <= m.n_vert; ++i) m.vert[i].n_sub_faces_neigh = m.vert[i].n_sub_elems_neigh = 0;
  for (int i = 1; i <= m.n_sub_faces; ++i) m.vert[m.sub_face[i].mesh_vert].n_sub_faces_neigh++;
  for (int i = 1; i <= m.n_sub_elems; ++i) m.vert[m.sub_elem[i].mesh_vert].n_sub_elems_neigh++;
  for (int i = 1; i <= m.n_vert; ++i) {
    m.vert[i].sub_face_neigh.assign(m.vert[i].n_sub_faces_neigh + 1, 0);
    m.vert[i].sub_elem_neigh.assign(m.vert[i].n_sub_elems_neigh + 1, 0);
    m.vert[i].n_sub_faces_neigh = m.vert[i].n_sub_elems_neigh = 0;
  }
  for (int i = 1; i <= m.n_sub_faces; ++i) {
    Vert& v = m.vert[m.sub_face[i].mesh_vert];
    m.sub_face[i].id_loc_around_node = v.n_sub_faces_neigh + 1;
    v.sub_face_neigh[v.n_sub_faces_neigh + 1] = i;
    v.n_sub_faces_neigh++;
  }
  for (int i = 1; i <= m.n_sub_elems; ++i) {
    Vert& v = m.vert[m.sub_elem[i].mesh_vert];
    m.sub_elem[i].id_loc_around_node = v.n_sub_elems_neigh + 1;
    v.sub_elem_neigh[v.n_sub_elems_neigh + 1] = i;
    v.n_sub_elems_neigh++;
  }
}

// mesh_connectivity_module.F90:558-593
static void compute_elem_tag(Mesh& m) {
  for (int i = 1; i <= m.n_faces; ++i)
    if (m.face[i].right_neigh < 0) {
      int tag = -m.face[i].right_neigh;
      Elem& e = m.elem[m.face[i].left_neigh];
      if (e.tag < 0) e.tag = tag;
      else if (e.tag > tag) e.tag = tag;
    }
  m.n_max_sub_faces_around_node = 0;
  for (int i = 1; i <= m.n_vert; ++i)
    m.n_max_sub_faces_around_node = std::max(m.n_max_sub_faces_around_node, m.vert[i].n_sub_faces_neigh);
}

// mesh_connectivity_module.F90:595-654
static void compute_neigh_by_vert(Mesh& m) {
  for (int i = 1; i <= m.n_elems; ++i) {
    Elem& e = m.elem[i];
    std::vector<int> tmp(1, 0);
    for (int j = 1; j <= e.n_vert; ++j) {
      const Vert& v = m.vert[e.vert[j]];
      for (int k = 1; k <= v.n_elems_neigh; ++k)
        if (v.elem_neigh[k] != i) tmp.push_back(v.elem_neigh[k]);
    }
    int n = (int)tmp.size() - 1;
    e.n_neigh_by_vert = n;
    for (int j = 1; j <= n; ++j)
      for (int k = j + 1; k <= n; ++k)
        if (tmp[k] > 0 && tmp[j] == tmp[k]) {
          tmp[k] = -1;
          e.n_neigh_by_vert--;
        }
    e.neigh_by_vert.assign(1, 0);
    for (int j = 1; j <= n; ++j)
      if (tmp[j] > 0) e.neigh_by_vert.push_back(tmp[j]);
  }
}

// mesh_connectivity_module.F90:726-750
void find_if_vert_is_bound(Mesh& m, bool b2d) {
  for (int i = 1; i <= m.n_vert; ++i) {
    Vert& v = m.vert[i];
    v.is_bound = false;
    for (int j = 1; j <= v.n_faces_neigh; ++j) {
      const Face& f = m.face[v.face_neigh[j]];
      if (b2d) {
        if (f.right_neigh <= 0 && std::fabs(f.norm[3]) < 1e-12) v.is_bound = true;
      } else if (f.right_neigh <= 0) {
        v.is_bound = true;
      }
    }
  }
}

// mesh_connectivity_module.F90:976-1073
static bool near(double a, double b) { return a < b + 1e-12 && a > b - 1e-12; }
static void stitch_periodic_faces(Mesh& m) {
  const double tol = 1e-12, lo = -0.5, hi = 0.5;
  std::vector<int> L[3], R[3];
  for (int i = 1; i <= m.n_faces; ++i)
    for (int d = 0; d < 3; ++d) {
      if (near(m.face[i].coord[d + 1], lo)) L[d].push_back(i);
      if (near(m.face[i].coord[d + 1], hi)) R[d].push_back(i);
    }
  for (int d = 0; d < 3; ++d)
    if (L[d].size() != R[d].size()) throw std::runtime_error("Error periodic boundaries !");
  for (int d = 0; d < 3; ++d) {
    int a = d == 0 ? 2 : 1, b = d == 2 ? 2 : 3;
    for (int ii : L[d])
      for (int jj : R[d]) {
        double da = m.face[ii].coord[a] - m.face[jj].coord[a];
        double db = m.face[ii].coord[b] - m.face[jj].coord[b];
        if (std::sqrt(da * da + db * db) < tol) {
          m.face[ii].right_neigh = m.face[jj].left_neigh;
          m.face[jj].right_neigh = m.face[ii].left_neigh;
        }
      }
  }
  for (int i = 1; i <= m.n_sub_faces; ++i) {
    m.sub_face[i].left_elem_neigh = m.face[m.sub_face[i].mesh_face].left_neigh;
    m.sub_face[i].right_elem_neigh = m.face[m.sub_face[i].mesh_face].right_neigh;
  }
}

// mesh_connectivity_module.F90:1226-1326 (process_pair)
static bool sf_match(const Mesh& m, int a, int b) {
  const SubFace &p = m.sub_face[a], &q = m.sub_face[b];
  return (p.left_elem_neigh == q.right_elem_neigh && p.right_elem_neigh == q.left_elem_neigh) ||
         (p.left_elem_neigh == q.left_elem_neigh && p.right_elem_neigh == q.right_elem_neigh);
}
static void process_pair(Mesh& m, int v1, int v2) {
  Vert& a = m.vert[v1];
  const Vert& b = m.vert[v2];
  for (int ki = 1; ki <= a.n_sub_faces_neigh; ++ki) {
    int sfki = a.sub_face_neigh[ki];
    int re = m.sub_face[sfki].right_elem_neigh;
    if (re > 0 && m.sub_face[sfki].right_sub_elem_neigh == 0)
      for (int k = 1; k <= b.n_sub_elems_neigh; ++k) {
        int id_se = b.sub_elem_neigh[k];
        if (m.sub_elem[id_se].mesh_elem == re) {
          m.sub_face[sfki].right_sub_elem_neigh = id_se;
          break;
        }
      }
  }
  int nm = 0;
  for (int ki = 1; ki <= a.n_sub_faces_neigh; ++ki)
    for (int kii = 1; kii <= b.n_sub_faces_neigh; ++kii)
      if (sf_match(m, a.sub_face_neigh[ki], b.sub_face_neigh[kii])) nm++;
  int st = a.n_sub_faces_neigh + b.n_sub_faces_neigh - nm;
  std::vector<int> tmp(st + 1, -1);
  for (int k = 1; k <= a.n_sub_faces_neigh; ++k) tmp[k] = a.sub_face_neigh[k];
  a.sub_face_neigh = tmp;
  a.n_sub_faces_neigh = st;
  for (int ki = 1; ki <= a.n_sub_faces_neigh; ++ki) {
    if (a.sub_face_neigh[ki] < 0) {
      for (int kii = 1; kii <= b.n_sub_faces_neigh; ++kii) {
        int sfkii = b.sub_face_neigh[kii];
        bool found = false;
        for (int p = 1; p <= ki - 1; ++p) {
          int sfp = a.sub_face_neigh[p];
          if (sfp < 0) continue;
          if (sf_match(m, sfp, sfkii)) found = true;
        }
        if (!found) {
          a.sub_face_neigh[ki] = sfkii;
          break;
        }
      }
    }
  }
  nm = 0;
  for (int k = 1; k <= b.n_sub_elems_neigh; ++k)
    if (m.sub_elem[b.sub_elem_neigh[k]].mesh_vert == v2) nm++;
  std::vector<int> t2(a.n_sub_elems_neigh + nm + 1, 0);
  for (int k = 1; k <= a.n_sub_elems_neigh; ++k) t2[k] = a.sub_elem_neigh[k];
  nm = 0;
  for (int k = 1; k <= b.n_sub_elems_neigh; ++k) {
    int id_se = b.sub_elem_neigh[k];
    if (m.sub_elem[id_se].mesh_vert == v2) t2[a.n_sub_elems_neigh + (++nm)] = id_se;
  }
  a.sub_elem_neigh = t2;
  a.n_sub_elems_neigh = (int)t2.size() - 1;
}

// mesh_connectivity_module.F90:1075-1222
static void build_periodic_stencil(Mesh& m) {
  const double lo = -0.5, hi = 0.5;
  std::vector<int> L[3], R[3];
  for (int i = 1; i <= m.n_vert; ++i)
    for (int d = 0; d < 3; ++d) {
      if (near(m.vert[i].coord[d + 1], lo)) L[d].push_back(i);
      if (near(m.vert[i].coord[d + 1], hi)) R[d].push_back(i);
    }
  for (int d = 0; d < 3; ++d) {
    int a = d == 0 ? 2 : 1, b = d == 2 ? 2 : 3;
    for (int ii : L[d])
      for (int jj : R[d]) {
        double da = m.vert[ii].coord[a] - m.vert[jj].coord[a];
        double db = m.vert[ii].coord[b] - m.vert[jj].coord[b];
        if (std::sqrt(da * da + db * db) < 1e-12) {
          process_pair(m, ii, jj);
          process_pair(m, jj, ii);
        }
      }
  }
  // xy, xz, yz edge diagonals, then the xyz corner (:1158-1220)
  struct Diag { int ld, lo_axis, match_axis; };
  const Diag diags[3] = {{0, 2, 3}, {0, 3, 2}, {1, 3, 1}};
  for (const Diag& dg : diags) {
    int d = dg.ld, ax = dg.lo_axis;
    for (int ii : L[d]) {
      if (!near(m.vert[ii].coord[ax], lo)) continue;
      for (int jj : R[d]) {
        if (!near(m.vert[jj].coord[ax], hi)) continue;
        if (std::fabs(m.vert[ii].coord[dg.match_axis] - m.vert[jj].coord[dg.match_axis]) < 1e-12) {
          process_pair(m, ii, jj);
          process_pair(m, jj, ii);
        }
      }
    }
  }
  for (int ii : L[0]) {
    if (!(near(m.vert[ii].coord[2], lo) && near(m.vert[ii].coord[3], lo))) continue;
    for (int jj : R[0]) {
      if (!(near(m.vert[jj].coord[2], hi) && near(m.vert[jj].coord[3], hi))) continue;
      process_pair(m, ii, jj);
      process_pair(m, jj, ii);
    }
  }
}

// mesh_connectivity_module.F90:12-59 (single rank)
void build_mesh(Mesh& m, bool use_sub_entities, bool b2d, bool periodic, int renumber) {
  build_node_elem_neigh(m);
  if (renumber == 1)
    renumber_vert_hilbert(m, b2d);
  else
    renumber_vert_mesh(m);
  renumber_elem_mesh(m);
  build_faces(m);
  build_node_face_connectivity(m);
  renumber_faces_mesh(m);
  if (use_sub_entities) {
    build_sub_faces(m);
    build_sub_elems(m);
    find_sub_elems_around_sub_face(m);
    build_node_sub_face_connectivity(m);
  }
  compute_elem_tag(m);
  compute_neigh_by_vert(m);
  if (periodic) {
    for (int i = 1; i <= m.n_faces; ++i) {
      Face& f = m.face[i];
      for (int d = 1; d <= 3; ++d) f.coord[d] = 0.0;
      for (int j = 1; j <= f.n_vert; ++j)
        for (int d = 1; d <= 3; ++d) f.coord[d] = f.coord[d] + m.vert[f.vert[j]].coord[d];
      for (int d = 1; d <= 3; ++d) f.coord[d] = f.coord[d] / (double)f.n_vert;
    }
    stitch_periodic_faces(m);
    if (use_sub_entities) build_periodic_stencil(m);
  }
  find_if_vert_is_bound(m, b2d);
}

// ---------------------------------------------------------------------------------
// mesh_geometry_module.F90
static inline void cross(const double* a, const double* b, double* c) {
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}
static inline double dot3(const double* a, const double* b) {
  double s = 0.0;
  s = s + a[0] * b[0];
  s = s + a[1] * b[1];
  s = s + a[2] * b[2];
  return s;
}
static inline void sub3(const double* a, const double* b, double* c) {
  for (int d = 0; d < 3; ++d) c[d] = a[d] - b[d];
}

// :193-235
static void face_centroid(const Mesh& m, int i, double* out) {
  const Face& f = m.face[i];
  double cg[3] = {0, 0, 0};
  for (int j = 1; j <= f.n_vert; ++j)
    for (int d = 0; d < 3; ++d) cg[d] = cg[d] + m.vert[f.vert[j]].coord[d + 1];
  for (int d = 0; d < 3; ++d) cg[d] = cg[d] / f.n_vert;
  double c[3] = {0, 0, 0}, sum_area = 0.0;
  for (int j = 1; j <= f.n_vert; ++j) {
    int jp = 1 + (j % f.n_vert);
    const double* cv = &m.vert[f.vert[j]].coord[1];
    const double* cvp = &m.vert[f.vert[jp]].coord[1];
    double a[3], b[3], x[3];
    sub3(cv, cg, a);
    sub3(cvp, cg, b);
    cross(a, b, x);
    double area = 0.5 * fnorm2(x, 3);
    for (int d = 0; d < 3; ++d) c[d] = c[d] + area * (cv[d] + cvp[d] + cg[d]) / 3.0;
    sum_area = sum_area + area;
  }
  for (int d = 0; d < 3; ++d) out[d] = c[d] / sum_area;
}

// :75-127
static void elem_centroid(const Mesh& m, int i, double* out) {
  const Elem& e = m.elem[i];
  double ce[3] = {0, 0, 0};
  for (int j = 1; j <= e.n_vert; ++j)
    for (int d = 0; d < 3; ++d) ce[d] = ce[d] + m.vert[e.vert[j]].coord[d + 1];
  for (int d = 0; d < 3; ++d) ce[d] = ce[d] / e.n_vert;
  double c[3] = {0, 0, 0}, sum_vol = 0.0;
  for (int j = 1; j <= e.n_faces; ++j) {
    const Face& f = m.face[e.face[j]];
    const double* cf = &f.coord[1];
    for (int k = 1; k <= f.n_vert; ++k) {
      int kp = 1 + (k % f.n_vert);
      const double* cp = &m.vert[f.vert[k]].coord[1];
      const double* cpp = &m.vert[f.vert[kp]].coord[1];
      double a[3], b[3], x[3], fe[3];
      sub3(cf, ce, fe);
      if (f.left_neigh == i) {
        sub3(cp, cf, a);
        sub3(cpp, cf, b);
      } else {
        sub3(cpp, cf, a);
        sub3(cp, cf, b);
      }
      cross(a, b, x);
      double vol = dot3(x, fe) / 6.0;
      for (int d = 0; d < 3; ++d) c[d] = c[d] + vol * (cp[d] + cpp[d] + cf[d] + ce[d]) / 4.0;
      sum_vol = sum_vol + vol;
    }
  }
  for (int d = 0; d < 3; ++d) out[d] = c[d] / sum_vol;
}

// :237-271
static void subface_norm(const Mesh& m, int i, double* out) {
  const SubFace& s = m.sub_face[i];
  const Face& f = m.face[s.mesh_face];
  int jp = 0, jm = 0, idv = 0;
  for (int j = 1; j <= f.n_vert; ++j) {
    idv = f.vert[j];
    if (idv == s.mesh_vert) {
      jp = 1 + (j % f.n_vert);
      jm = 1 + ((j - 2 + f.n_vert) % f.n_vert);
      break;
    }
  }
  const double* cf = &f.coord[1];
  const double* cp = &m.vert[idv].coord[1];
  double cpm[3], cpp[3];
  for (int d = 0; d < 3; ++d) {
    cpm[d] = 0.5 * (m.vert[f.vert[jm]].coord[d + 1] + cp[d]);
    cpp[d] = 0.5 * (m.vert[f.vert[jp]].coord[d + 1] + cp[d]);
  }
  double a[3], b[3], c[3], x1[3], x2[3];
  sub3(cpm, cf, a);
  sub3(cp, cf, b);
  sub3(cpp, cf, c);
  cross(a, b, x1);
  cross(b, c, x2);
  for (int d = 0; d < 3; ++d) out[d] = 0.5 * (x1[d] + x2[d]);
}

// :129-175
static double subelem_volume(const Mesh& m, int i) {
  const SubElem& se = m.sub_elem[i];
  int id_elem = se.mesh_elem;
  const double* ce = &m.elem[id_elem].coord[1];
  double vol = 0.0;
  for (int j = 1; j <= se.n_sub_faces; ++j) {
    const SubFace& s = m.sub_face[se.sub_face[j]];
    const Face& f = m.face[s.mesh_face];
    const double* cf = &f.coord[1];
    int kp = 0, km = 0, idv = 0;
    for (int k = 1; k <= f.n_vert; ++k) {
      idv = f.vert[k];
      if (idv == s.mesh_vert) {
        kp = 1 + (k % f.n_vert);
        km = 1 + ((k - 2 + f.n_vert) % f.n_vert);
        break;
      }
    }
    const double* cp = &m.vert[idv].coord[1];
    double cpm[3], cpp[3];
    for (int d = 0; d < 3; ++d) {
      cpm[d] = 0.5 * (m.vert[f.vert[km]].coord[d + 1] + cp[d]);
      cpp[d] = 0.5 * (m.vert[f.vert[kp]].coord[d + 1] + cp[d]);
    }
    double fe[3], a[3], b[3], c[3], x1[3], x2[3];
    sub3(cf, ce, fe);
    sub3(cpm, cf, a);
    sub3(cp, cf, b);
    sub3(cpp, cf, c);
    if (f.left_neigh == id_elem) {
      cross(a, b, x1);
      cross(b, c, x2);
    } else {
      cross(c, b, x1);
      cross(b, a, x2);
    }
    vol = vol + dot3(x1, fe) / 6.0 + dot3(x2, fe) / 6.0;
  }
  return vol;
}

// :290-411 (per-element checks; logs nothing, records the verdict)
static bool check_mesh(const Mesh& m) {
  bool ok = true;
  for (int i = 1; i <= m.n_elems; ++i) {
    const Elem& e = m.elem[i];
    double vol = 0.0, nt[3] = {0, 0, 0}, ns[3] = {0, 0, 0};
    for (int j = 1; j <= e.n_faces; ++j) {
      const Face& f = m.face[e.face[j]];
      double n[3];
      for (int d = 0; d < 3; ++d) n[d] = f.left_neigh == i ? f.norm[d + 1] : -f.norm[d + 1];
      double an[3];
      for (int d = 0; d < 3; ++d) an[d] = f.area * n[d];
      vol = vol + dot3(&f.coord[1], an);
    }
    vol = vol / 3.0;
    ok = ok && (std::fabs(e.volume - vol) < 1e-14);
    for (int j = 1; j <= e.n_faces; ++j) {
      const Face& f = m.face[e.face[j]];
      for (int d = 0; d < 3; ++d)
        nt[d] = nt[d] + f.area * (f.left_neigh == i ? f.norm[d + 1] : -f.norm[d + 1]);
    }
    ok = ok && (fnorm2(nt, 3) < 1e-14);
    for (int j = 1; j <= e.n_faces; ++j) {
      const Face& f = m.face[e.face[j]];
      for (int k = 1; k <= f.n_sub_faces; ++k) {
        const SubFace& s = m.sub_face[f.sub_face[k]];
        for (int d = 0; d < 3; ++d)
          ns[d] = ns[d] + s.area * (f.left_neigh == i ? s.norm[d + 1] : -s.norm[d + 1]);
      }
    }
    ok = ok && (fnorm2(ns, 3) < 1e-14);
  }
  for (int i = 1; i <= m.n_sub_elems; ++i) ok = ok && (m.sub_elem[i].volume > 0.0);
  return ok;
}

// :16-57
void compute_geometry_mesh(Mesh& m, bool b2d) {
  for (int i = 1; i <= m.n_faces; ++i) face_centroid(m, i, &m.face[i].coord[1]);
  for (int i = 1; i <= m.n_elems; ++i) elem_centroid(m, i, &m.elem[i].coord[1]);
  for (int i = 1; i <= m.n_sub_faces; ++i) {
    SubFace& s = m.sub_face[i];
    subface_norm(m, i, &s.norm[1]);
    s.area = fnorm2(&s.norm[1], 3);
    for (int d = 1; d <= 3; ++d) s.norm[d] = s.norm[d] / s.area;
  }
  for (int i = 1; i <= m.n_faces; ++i) {
    Face& f = m.face[i];
    double n[3] = {0, 0, 0};
    for (int j = 1; j <= f.n_sub_faces; ++j) {
      double x[3];
      subface_norm(m, f.sub_face[j], x);
      for (int d = 0; d < 3; ++d) n[d] = n[d] + x[d];
    }
    f.area = fnorm2(n, 3);
    for (int d = 0; d < 3; ++d) f.norm[d + 1] = n[d] / f.area;
  }
  for (int i = 1; i <= m.n_sub_elems; ++i) m.sub_elem[i].volume = subelem_volume(m, i);
  for (int i = 1; i <= m.n_elems; ++i) {
    double v = 0.0;
    for (int j = 1; j <= m.elem[i].n_sub_elems; ++j) v = v + m.sub_elem[m.elem[i].sub_elem[j]].volume;
    m.elem[i].volume = v;
  }
  m.geometry_ok = check_mesh(m);
  find_if_vert_is_bound(m, b2d);
  for (int i = 1; i <= m.n_vert; ++i) {
    Vert& v = m.vert[i];
    v.volume = 0.0;
    for (int j = 1; j <= v.n_sub_elems_neigh; ++j) v.volume = v.volume + m.sub_elem[v.sub_elem_neigh[j]].volume;
  }
}

// ---------------------------------------------------------------------------------
std::map<std::string, std::vector<int32_t>> export_topology(const Mesh& m) {
  std::map<std::string, std::vector<int32_t>> o;
  auto csr = [&](const std::string& name, int n, auto cnt, auto item) {
    std::vector<int32_t> off(n + 1, 0), val;
    for (int i = 1; i <= n; ++i) {
      int c = cnt(i);
      for (int k = 1; k <= c; ++k) val.push_back(item(i, k));
      off[i] = (int32_t)val.size();
    }
    o[name + "_off"] = off;
    o[name] = val;
  };
  o["sizes"] = {m.n_vert, m.n_elems, m.n_faces, m.n_sub_faces, m.n_sub_elems, m.n_max_sub_faces_around_node};
  csr("elem_vert", m.n_elems, [&](int i) { return m.elem[i].n_vert; }, [&](int i, int k) { return m.elem[i].vert[k]; });
  csr("elem_face", m.n_elems, [&](int i) { return m.elem[i].n_faces; }, [&](int i, int k) { return m.elem[i].face[k]; });
  csr("elem_sub_face", m.n_elems, [&](int i) { return m.elem[i].n_sub_faces; }, [&](int i, int k) { return m.elem[i].sub_face[k]; });
  csr("elem_sub_elem", m.n_elems, [&](int i) { return m.elem[i].n_sub_elems; }, [&](int i, int k) { return m.elem[i].sub_elem[k]; });
  csr("elem_neigh_by_vert", m.n_elems, [&](int i) { return m.elem[i].n_neigh_by_vert; }, [&](int i, int k) { return m.elem[i].neigh_by_vert[k]; });
  std::vector<int32_t> ek, et;
  for (int i = 1; i <= m.n_elems; ++i) {
    ek.push_back(m.elem[i].elem_kind);
    et.push_back(m.elem[i].tag);
  }
  o["elem_kind"] = ek;
  o["elem_tag"] = et;
  csr("face_vert", m.n_faces, [&](int i) { return m.face[i].n_vert; }, [&](int i, int k) { return m.face[i].vert[k]; });
  csr("face_sub_face", m.n_faces, [&](int i) { return m.face[i].n_sub_faces; }, [&](int i, int k) { return m.face[i].sub_face[k]; });
  std::vector<int32_t> fl, fr, flf, frf;
  for (int i = 1; i <= m.n_faces; ++i) {
    fl.push_back(m.face[i].left_neigh);
    fr.push_back(m.face[i].right_neigh);
    flf.push_back(m.face[i].left_neigh_face);
    frf.push_back(m.face[i].right_neigh_face);
  }
  o["face_left"] = fl;
  o["face_right"] = fr;
  o["face_left_face"] = flf;
  o["face_right_face"] = frf;
  std::vector<int32_t> sv, sfc, sl, sr, sls, srs, sloc;
  for (int i = 1; i <= m.n_sub_faces; ++i) {
    const SubFace& s = m.sub_face[i];
    sv.push_back(s.mesh_vert);
    sfc.push_back(s.mesh_face);
    sl.push_back(s.left_elem_neigh);
    sr.push_back(s.right_elem_neigh);
    sls.push_back(s.left_sub_elem_neigh);
    srs.push_back(s.right_sub_elem_neigh);
    sloc.push_back(s.id_loc_around_node);
  }
  o["sub_face_vert"] = sv;
  o["sub_face_face"] = sfc;
  o["sub_face_left_elem"] = sl;
  o["sub_face_right_elem"] = sr;
  o["sub_face_left_sub_elem"] = sls;
  o["sub_face_right_sub_elem"] = srs;
  o["sub_face_loc"] = sloc;
  std::vector<int32_t> se_e, se_v, se_loc;
  for (int i = 1; i <= m.n_sub_elems; ++i) {
    se_e.push_back(m.sub_elem[i].mesh_elem);
    se_v.push_back(m.sub_elem[i].mesh_vert);
    se_loc.push_back(m.sub_elem[i].id_loc_around_node);
  }
  o["sub_elem_elem"] = se_e;
  o["sub_elem_vert"] = se_v;
  o["sub_elem_loc"] = se_loc;
  csr("sub_elem_sub_face", m.n_sub_elems, [&](int i) { return m.sub_elem[i].n_sub_faces; }, [&](int i, int k) { return m.sub_elem[i].sub_face[k]; });
  csr("vert_sub_face", m.n_vert, [&](int i) { return m.vert[i].n_sub_faces_neigh; }, [&](int i, int k) { return m.vert[i].sub_face_neigh[k]; });
  csr("vert_sub_elem", m.n_vert, [&](int i) { return m.vert[i].n_sub_elems_neigh; }, [&](int i, int k) { return m.vert[i].sub_elem_neigh[k]; });
  csr("vert_face", m.n_vert, [&](int i) { return m.vert[i].n_faces_neigh; }, [&](int i, int k) { return m.vert[i].face_neigh[k]; });
  csr("vert_elem", m.n_vert, [&](int i) { return m.vert[i].n_elems_neigh; }, [&](int i, int k) { return m.vert[i].elem_neigh[k]; });
  std::vector<int32_t> vb;
  for (int i = 1; i <= m.n_vert; ++i) vb.push_back(m.vert[i].is_bound ? 1 : 0);
  o["vert_is_bound"] = vb;
  return o;
}

}  // namespace oracle
