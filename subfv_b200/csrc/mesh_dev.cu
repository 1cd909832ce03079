// Device mesh upload and the geometry kernels of compute_geometry_mesh
// (src/mesh/mesh_geometry_module.F90:16-57). One thread per face / cell / vertex;
// each recomputes what it needs from the vertex coordinates in the reference's order.
#include <algorithm>
#include <array>
#include <functional>
#include <map>
#include <vector>

#include "../../include/subfv.h"
#include "common.cuh"
#include "geom_body.cuh"
#include "mesh_dev.cuh"

namespace subfv {

namespace {

template <class T>
int upload(T** dst, const std::vector<T>& h, size_t* bytes, cudaStream_t s) {
  size_t n = std::max<size_t>(h.size(), 1);
  SUBFV_CUDA(cudaMallocAsync((void**)dst, n * sizeof(T), s));
  *bytes += n * sizeof(T);
  if (!h.empty()) SUBFV_CUDA(cudaMemcpyAsync(*dst, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, s));
  return 0;
}
template <class T>
int alloc(T** dst, size_t n, size_t* bytes, cudaStream_t s) {
  n = std::max<size_t>(n, 1);
  SUBFV_CUDA(cudaMallocAsync((void**)dst, n * sizeof(T), s));
  SUBFV_CUDA(cudaMemsetAsync(*dst, 0, n * sizeof(T), s));
  *bytes += n * sizeof(T);
  return 0;
}

// Diffusion stencils of DevMesh (layout in mesh_dev.cuh). Periodic images are the
// vertices whose subface lists hold each other's subfaces (build_periodic_stencil,
// mesh_connectivity_module.F90:1075-1328); a node's images are taken in ascending order.
struct DiffStencil {
  std::vector<int> sf_off, sf, se_off, se;
  std::vector<int2> sf_se, sf_seloc;
  std::vector<int4> se_sfloc;
  int max_sf = 0, max_se = 0;
  bool complete = true;
};

int build_diffusion_stencil(int nv, const std::vector<int>& vsf_off, const std::vector<int>& vsf,
                            const std::vector<int>& vse_off, const std::vector<int>& vse,
                            const std::vector<int>& sf_face, const std::vector<int>& sf_vert,
                            const std::vector<int2>& flr, const std::vector<int>& se_elem,
                            const std::vector<int>& se_vert, const std::vector<int4>& se_sf, DiffStencil* out) {
  std::vector<int> parent(nv);
  for (int v = 0; v < nv; ++v) parent[v] = v;
  std::function<int(int)> find = [&](int x) {
    while (parent[x] != x) x = parent[x] = parent[parent[x]];
    return x;
  };
  for (int v = 0; v < nv; ++v)
    for (int p = vsf_off[v]; p < vsf_off[v + 1]; ++p) {
      const int a = find(v), b = find(sf_vert[vsf[p]]);
      if (a != b) parent[std::max(a, b)] = std::min(a, b);
    }
  std::vector<std::vector<int>> members(nv);
  for (int v = 0; v < nv; ++v) members[find(v)].push_back(v);  // ascending within a class
  // a subface's key: its cells, unordered, for an interior face (the two copies of a
  // periodic face share it); its cell, boundary and face for a boundary face
  auto key = [&](int s) {
    const int f = sf_face[s];
    const int2 lr = flr[f];
    if (lr.y >= 0) return std::array<long, 3>{std::min(lr.x, lr.y), std::max(lr.x, lr.y), -1};
    return std::array<long, 3>{lr.x, lr.y, f};
  };
  struct Cls {
    std::vector<int> sf, se;
    std::vector<int2> sf_se, sf_seloc;
    std::vector<int4> se_sfloc;
  };
  std::vector<int> cls_of(nv, -1);
  std::vector<Cls> classes;
  for (int r = 0; r < nv; ++r) {
    if (members[r].empty()) continue;
    Cls c;
    std::map<std::array<long, 3>, int> fpos;
    std::map<int, int> epos;  // cell -> position in the subcell list
    for (int v : members[r])
      for (int p = vsf_off[v]; p < vsf_off[v + 1]; ++p) {
        const int sfi = vsf[p];
        if (fpos.emplace(key(sfi), (int)c.sf.size()).second) c.sf.push_back(sfi);
      }
    for (int v : members[r])
      for (int q = vse_off[v]; q < vse_off[v + 1]; ++q) {
        const int e = vse[q];
        if (se_vert[e] != v) continue;
        if (!epos.emplace(se_elem[e], (int)c.se.size()).second) {
          set_error("subfv_mesh_create: a cell touches one periodic node twice");
          return -2;
        }
        c.se.push_back(e);
      }
    for (int sfi : c.sf) {
      const int2 lr = flr[sf_face[sfi]];
      int2 pos = make_int2(-1, -1), ids = make_int2(-1, -1);
      auto it = epos.find(lr.x);
      if (it != epos.end()) pos.x = it->second, ids.x = c.se[it->second];
      if (lr.y >= 0 && (it = epos.find(lr.y)) != epos.end()) pos.y = it->second, ids.y = c.se[it->second];
      if (pos.x < 0 || (lr.y >= 0 && pos.y < 0)) out->complete = false;
      c.sf_se.push_back(ids);
      c.sf_seloc.push_back(pos);
    }
    for (int e : c.se) {
      const int4 q4 = se_sf[e];
      const int q[4] = {q4.x, q4.y, q4.z, q4.w};
      int loc[4] = {-1, -1, -1, -1};
      for (int k = 0; k < 4; ++k)
        if (q[k] >= 0) {
          auto jt = fpos.find(key(q[k]));
          loc[k] = jt == fpos.end() ? -1 : jt->second;
          if (loc[k] < 0) out->complete = false;
        }
      c.se_sfloc.push_back(make_int4(loc[0], loc[1], loc[2], loc[3]));
    }
    for (int v : members[r]) cls_of[v] = (int)classes.size();
    classes.push_back(std::move(c));
  }
  DiffStencil& D = *out;
  D.sf_off.assign(nv + 1, 0);
  D.se_off.assign(nv + 1, 0);
  for (int v = 0; v < nv; ++v) {
    const Cls& c = classes[cls_of[v]];
    D.sf_off[v + 1] = D.sf_off[v] + (int)c.sf.size();
    D.se_off[v + 1] = D.se_off[v] + (int)c.se.size();
    D.max_sf = std::max(D.max_sf, (int)c.sf.size());
    D.max_se = std::max(D.max_se, (int)c.se.size());
    D.sf.insert(D.sf.end(), c.sf.begin(), c.sf.end());
    D.sf_se.insert(D.sf_se.end(), c.sf_se.begin(), c.sf_se.end());
    D.sf_seloc.insert(D.sf_seloc.end(), c.sf_seloc.begin(), c.sf_seloc.end());
    D.se.insert(D.se.end(), c.se.begin(), c.se.end());
    D.se_sfloc.insert(D.se_sfloc.end(), c.se_sfloc.begin(), c.se_sfloc.end());
  }
  return 0;
}

}  // namespace

int devmesh_create(const subfv_mesh_desc* d, DevMesh* m) {
  const int nv = d->n_vert, ne = d->n_elems, nf = d->n_faces, nsf = d->n_sub_faces, nse = d->n_sub_elems;
  if (nv <= 0 || ne <= 0 || nf <= 0 || nsf <= 0 || nse <= 0) {
    set_error("subfv_mesh_create: empty mesh");
    return -2;
  }
  m->nv = nv;
  m->ne = ne;
  m->nf = nf;
  m->nsf = nsf;
  m->nse = nse;
  m->b2d = d->b2d;
  SUBFV_CUDA(cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking));
  cudaStream_t s = m->stream;
  size_t* B = &m->bytes;

  std::vector<double4> x(nv);
  for (int i = 0; i < nv; ++i) x[i] = make_double4(d->vert_coord[3 * i], d->vert_coord[3 * i + 1], d->vert_coord[3 * i + 2], 0.0);
  std::vector<int8_t> isb(nv);
  for (int i = 0; i < nv; ++i) isb[i] = d->vert_is_bound ? (int8_t)(d->vert_is_bound[i] != 0) : 0;

  std::vector<int4> fvert(nf), fsf(nf);
  std::vector<int2> flr(nf);
  for (int f = 0; f < nf; ++f) {
    int b = d->face_vert_off[f], n = d->face_vert_off[f + 1] - b;
    if (n < 3 || n > 4) {
      set_error("subfv_mesh_create: faces must have 3 or 4 vertices");
      return -2;
    }
    int v[4] = {-1, -1, -1, -1}, sfi[4] = {-1, -1, -1, -1};
    for (int k = 0; k < n; ++k) {
      v[k] = d->face_vert[b + k] - 1;
      sfi[k] = d->face_sub_face[b + k] - 1;
    }
    fvert[f] = make_int4(v[0], v[1], v[2], v[3]);
    fsf[f] = make_int4(sfi[0], sfi[1], sfi[2], sfi[3]);
    int r = d->face_right[f];
    flr[f] = make_int2(d->face_left[f] - 1, r > 0 ? r - 1 : r - 1);  // wall 0 -> -1, -tag -> -tag-1
  }
  std::vector<int> sf_face(nsf), sf_vert(nsf), sf_loc(nsf);
  std::vector<int2> sf_se(nsf);
  for (int i = 0; i < nsf; ++i) {
    sf_face[i] = d->sub_face_face[i] - 1;
    sf_vert[i] = d->sub_face_vert[i] - 1;
    sf_se[i] = make_int2(d->sub_face_left_sub_elem[i] - 1, d->sub_face_right_sub_elem[i] - 1);
    sf_loc[i] = d->sub_face_loc ? d->sub_face_loc[i] - 1 : 0;
  }
  // fpos: the vertex slot, in the face's vertex order, of each of the face's subfaces
  // (face%sub_face order), 2 bits each; the first slot holding the subface's vertex (the
  // last slot when none does), as the search of compute_subface_norm finds it
  std::vector<uint8_t> fpos(nf, 0);
  for (int f = 0; f < nf; ++f) {
    const int v[4] = {fvert[f].x, fvert[f].y, fvert[f].z, fvert[f].w};
    const int sfi[4] = {fsf[f].x, fsf[f].y, fsf[f].z, fsf[f].w};
    const int n = v[3] < 0 ? 3 : 4;
    unsigned code = 0;
    for (int k = 0; k < n; ++k) {
      const int vert = sfi[k] >= 0 && sfi[k] < nsf ? sf_vert[sfi[k]] : -1;
      int j = 0;
      while (j < n - 1 && v[j] != vert) ++j;
      code |= (unsigned)j << (2 * k);
    }
    fpos[f] = (uint8_t)code;
  }
  std::vector<int> se_elem(nse), se_vert(nse), se_loc(nse);
  std::vector<int4> se_sf(nse);
  for (int i = 0; i < nse; ++i) {
    se_elem[i] = d->sub_elem_elem[i] - 1;
    se_vert[i] = d->sub_elem_vert[i] - 1;
    se_loc[i] = d->sub_elem_loc ? d->sub_elem_loc[i] - 1 : 0;
    int b = d->sub_elem_sub_face_off[i], n = d->sub_elem_sub_face_off[i + 1] - b;
    if (n > 4) {
      set_error("subfv_mesh_create: a subcell with more than four subfaces");
      return -2;
    }
    int q[4] = {-1, -1, -1, -1};
    for (int k = 0; k < n; ++k) q[k] = d->sub_elem_sub_face[b + k] - 1;
    se_sf[i] = make_int4(q[0], q[1], q[2], q[3]);
  }
  std::vector<int> ev_off(ne + 1), ev(d->elem_vert_off[ne]), ef8(8 * (size_t)ne, -1), ekind(ne);
  for (int c = 0; c <= ne; ++c) ev_off[c] = d->elem_vert_off[c];
  m->max_evc = 0;
  for (int c = 0; c < ne; ++c) m->max_evc = std::max(m->max_evc, ev_off[c + 1] - ev_off[c]);
  for (int c = 0; c < ne; ++c) {
    ekind[c] = d->elem_kind ? d->elem_kind[c] : 0;
    for (int k = ev_off[c]; k < ev_off[c + 1]; ++k) {
      ev[k] = d->elem_vert[k] - 1;
      if (d->elem_sub_elem[k] - 1 != k) {
        set_error("subfv_mesh_create: elem%sub_elem must number subcells cell by cell in vertex order");
        return -2;
      }
    }
    int b = d->elem_face_off[c], n = d->elem_face_off[c + 1] - b;
    if (n > 8) {
      set_error("subfv_mesh_create: a cell with more than eight faces");
      return -2;
    }
    for (int k = 0; k < n; ++k) ef8[8 * (size_t)c + k] = d->elem_face[b + k] - 1;
  }
  const int nvsf = d->vert_sub_face_off[nv];
  std::vector<int> vsf_off(nv + 1), vsf(nvsf), vse_off(nv + 1), vse(d->vert_sub_elem_off[nv]);
  std::vector<int> p_node(nvsf);
  bool ident = true;
  int max_vsf = 0;
  for (int v = 0; v <= nv; ++v) {
    vsf_off[v] = d->vert_sub_face_off[v];
    vse_off[v] = d->vert_sub_elem_off[v];
  }
  for (int v = 0; v < nv; ++v) {
    max_vsf = std::max(max_vsf, vsf_off[v + 1] - vsf_off[v]);
    for (int p = vsf_off[v]; p < vsf_off[v + 1]; ++p) {
      vsf[p] = d->vert_sub_face[p] - 1;
      p_node[p] = v;
      if (vsf[p] != p) ident = false;
    }
  }
  for (size_t k = 0; k < vse.size(); ++k) vse[k] = d->vert_sub_elem[k] - 1;
  int max_vse = 0;
  for (int v = 0; v < nv; ++v) max_vse = std::max(max_vse, vse_off[v + 1] - vse_off[v]);
  m->max_vse = max_vse;
  m->nvsf = nvsf;
  m->vsf_identity = ident ? 1 : 0;
  m->max_vsf = max_vsf;
  // cell CSR over node-ordered subface positions (ascending p = the reference's scatter order)
  std::vector<int> csf_off(ne + 1, 0);
  for (int p = 0; p < nvsf; ++p) {
    int f = sf_face[vsf[p]];
    csf_off[flr[f].x + 1]++;
    if (flr[f].y >= 0) csf_off[flr[f].y + 1]++;
  }
  for (int c = 0; c < ne; ++c) csf_off[c + 1] += csf_off[c];
  std::vector<int> csf(csf_off[ne]);
  {
    std::vector<int> fill(csf_off.begin(), csf_off.end() - 1);
    for (int p = 0; p < nvsf; ++p) {
      int f = sf_face[vsf[p]];
      csf[fill[flr[f].x]++] = 2 * p;
      if (flr[f].y >= 0) csf[fill[flr[f].y]++] = 2 * p + 1;
    }
  }
  m->ncsf = csf_off[ne];
  std::vector<int> vel_off(nv + 1, 0), vel;
  if (d->vert_elem_off && d->vert_elem) {
    for (int v = 0; v <= nv; ++v) vel_off[v] = d->vert_elem_off[v];
    vel.resize(vel_off[nv]);
    for (int k = 0; k < vel_off[nv]; ++k) vel[k] = d->vert_elem[k] - 1;
  }
  std::vector<int> cse_sorted(ev_off[ne]);
  for (int c = 0; c < ne; ++c) {
    int b = ev_off[c], n = ev_off[c + 1] - b;
    for (int k = 0; k < n; ++k) cse_sorted[b + k] = b + k;
    std::sort(cse_sorted.begin() + b, cse_sorted.begin() + b + n,
              [&](int a, int q) { return ev[a] < ev[q]; });
  }

  if (upload(&m->vel_off, vel_off, B, s) || upload(&m->vel, vel, B, s) || upload(&m->cse_sorted, cse_sorted, B, s))
    return -1;
  // launch orders: stable sorts by a code-path key
  std::vector<int> forder(nf), vorder(nv);
  {
    std::vector<int> key(nf);
    for (int f = 0; f < nf; ++f) key[f] = (fvert[f].w < 0 ? 0 : 2) + (flr[f].y >= 0 ? 0 : 1);
    for (int f = 0; f < nf; ++f) forder[f] = f;
    std::stable_sort(forder.begin(), forder.end(), [&](int a, int b) { return key[a] < key[b]; });
    std::vector<long> vkey(nv);
    for (int v = 0; v < nv; ++v) {
      int nb = 0;
      for (int p = vsf_off[v]; p < vsf_off[v + 1]; ++p) nb += flr[sf_face[vsf[p]]].y < 0 ? 1 : 0;
      vkey[v] = ((long)(vsf_off[v + 1] - vsf_off[v]) << 20) + ((long)(vse_off[v + 1] - vse_off[v]) << 10) + nb;
    }
    for (int v = 0; v < nv; ++v) vorder[v] = v;
    std::stable_sort(vorder.begin(), vorder.end(), [&](int a, int b) { return vkey[a] < vkey[b]; });
  }
  if (upload(&m->forder, forder, B, s) || upload(&m->vorder, vorder, B, s)) return -1;
  if (upload(&m->x, x, B, s) || alloc(&m->vp, nv, B, s) || alloc(&m->vol_v, nv, B, s) || upload(&m->is_bound, isb, B, s) ||
      upload(&m->fvert, fvert, B, s) || upload(&m->flr, flr, B, s) || upload(&m->fsf, fsf, B, s) ||
      alloc(&m->fc, nf, B, s) || alloc(&m->fn, nf, B, s) || upload(&m->sf_face, sf_face, B, s) ||
      upload(&m->sf_vert, sf_vert, B, s) || upload(&m->sf_se, sf_se, B, s) || upload(&m->sf_loc, sf_loc, B, s) ||
      alloc(&m->sfn, nsf, B, s) || alloc(&m->sfa, nsf, B, s) || upload(&m->se_elem, se_elem, B, s) || upload(&m->se_vert, se_vert, B, s) ||
      upload(&m->se_loc, se_loc, B, s) || upload(&m->se_sf, se_sf, B, s) || alloc(&m->vol_se, nse, B, s) ||
      upload(&m->ev_off, ev_off, B, s) || upload(&m->ev, ev, B, s) || upload(&m->ef8, ef8, B, s) ||
      upload(&m->ekind, ekind, B, s) || alloc(&m->cc, ne, B, s) || alloc(&m->vol, ne, B, s) ||
      upload(&m->vsf_off, vsf_off, B, s) || upload(&m->vsf, vsf, B, s) || upload(&m->p_node, p_node, B, s) ||
      upload(&m->vse_off, vse_off, B, s) || upload(&m->vse, vse, B, s) || upload(&m->csf_off, csf_off, B, s) ||
      upload(&m->csf, csf, B, s) || alloc(&m->status, 4, B, s) || upload(&m->fpos, fpos, B, s))
    return -1;
  SUBFV_CUDA(cudaStreamSynchronize(s));
  return 0;
}

namespace {
template <class T>
int fetch(std::vector<T>& h, const T* d, size_t n, cudaStream_t s) {
  h.resize(n);
  if (n) SUBFV_CUDA(cudaMemcpyAsync(h.data(), d, n * sizeof(T), cudaMemcpyDeviceToHost, s));
  return 0;
}
}  // namespace

// The diffusion stencil is only read by the Navier-Stokes diffusion terms: it is built the
// first time a state asks for them, from the node lists already on the device (a mesh
// that never runs diffusion holds none of its arrays).
int ensure_diffusion_stencil(DevMesh* m) {
  if (m->dstencil_built) return 0;
  cudaStream_t s = m->stream;
  std::vector<int> vsf_off, vsf, vse_off, vse, sf_face, sf_vert, se_elem, se_vert;
  std::vector<int2> flr;
  std::vector<int4> se_sf;
  if (fetch(vsf_off, m->vsf_off, (size_t)m->nv + 1, s) || fetch(vse_off, m->vse_off, (size_t)m->nv + 1, s) ||
      fetch(sf_face, m->sf_face, (size_t)m->nsf, s) || fetch(sf_vert, m->sf_vert, (size_t)m->nsf, s) ||
      fetch(flr, m->flr, (size_t)m->nf, s) || fetch(se_elem, m->se_elem, (size_t)m->nse, s) ||
      fetch(se_vert, m->se_vert, (size_t)m->nse, s) || fetch(se_sf, m->se_sf, (size_t)m->nse, s))
    return -1;
  SUBFV_CUDA(cudaStreamSynchronize(s));
  if (fetch(vsf, m->vsf, (size_t)vsf_off[m->nv], s) || fetch(vse, m->vse, (size_t)vse_off[m->nv], s)) return -1;
  SUBFV_CUDA(cudaStreamSynchronize(s));
  DiffStencil D;
  if (int rc = build_diffusion_stencil(m->nv, vsf_off, vsf, vse_off, vse, sf_face, sf_vert, flr, se_elem, se_vert,
                                       se_sf, &D))
    return rc;
  size_t* B = &m->bytes;
  if (upload(&m->dsf_off, D.sf_off, B, s) || upload(&m->dsf, D.sf, B, s) || upload(&m->dsf_se, D.sf_se, B, s) ||
      upload(&m->dsf_seloc, D.sf_seloc, B, s) || upload(&m->dse_off, D.se_off, B, s) ||
      upload(&m->dse, D.se, B, s) || upload(&m->dse_sfloc, D.se_sfloc, B, s))
    return -1;
  SUBFV_CUDA(cudaStreamSynchronize(s));  // the host vectors go out of scope
  m->max_dsf = D.max_sf;
  m->max_dse = D.max_se;
  m->dstencil_ok = D.complete ? 1 : 0;
  m->dstencil_built = 1;
  return 0;
}

void devmesh_free(DevMesh* m) {
  void* ptrs[] = {m->x, m->vp, m->vol_v, m->is_bound, m->fvert, m->flr, m->fsf, m->fc, m->fn,
                  m->sf_face, m->sf_vert, m->sf_se, m->sf_loc, m->sfn, m->sfa, m->se_elem, m->se_vert, m->se_loc,
                  m->se_sf, m->vol_se, m->ev_off, m->ev, m->ef8, m->ekind, m->cc, m->vol, m->vsf_off,
                  m->vsf, m->p_node, m->vse_off, m->vse, m->csf_off, m->csf, m->status,
                  m->vel_off, m->vel, m->cse_sorted, m->frec, m->centry, m->fS, m->fpos, m->gface, m->gsub, m->forder, m->vorder,
                  m->dsf_off, m->dsf, m->dsf_se, m->dsf_seloc, m->dse_off, m->dse, m->dse_sfloc,
                  m->dcache, m->dcache_off, m->npinv};
  diffusion_cache_forget(m);
  // stream-ordered frees: they wait for the mesh stream's work but not for other
  // streams (a caller that used the mesh elsewhere orders that work first)
  for (void* p : ptrs)
    if (p) {
      if (m->stream) cudaFreeAsync(p, m->stream);
      else cudaFree(p);
    }
  if (m->stream) cudaStreamDestroy(m->stream);
  *m = DevMesh();
}

// ---------------------------------------------------------------------------------
// Geometry kernels

namespace {
using namespace geo;

// ---- full geometry: one thread per face, then one per cell (every array written)

// compute_elem_centroid, compute_subelem_volume, compute_elem_volume, check_mesh
// (:59-175, :290-396) from the stored face geometry; any cell, periodic faces included.
__global__ void k_cell_geometry(DevMesh m) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= m.ne) return;
  int vb = m.ev_off[c], nvc = m.ev_off[c + 1] - vb;
  V3 ce = {0.0, 0.0, 0.0};
  for (int k = 0; k < nvc; ++k) {
    V3 p = ld3(m.x, m.ev[vb + k]);
    ce = {ce.x + p.x, ce.y + p.y, ce.z + p.z};
  }
  ce = {ce.x / nvc, ce.y / nvc, ce.z / nvc};
  int faces[8];
  int nfc = 0;
  for (int k = 0; k < 8; ++k) {
    int f = m.ef8[8 * c + k];
    if (f < 0) break;
    faces[nfc++] = f;
  }
  V3 cen = {0.0, 0.0, 0.0};
  double sum_vol = 0.0;
  for (int j = 0; j < nfc; ++j) {
    int f = faces[j];
    int4 fv = m.fvert[f];
    int vid[4] = {fv.x, fv.y, fv.z, fv.w};
    int n = fv.w < 0 ? 3 : 4;
    bool left = m.flr[f].x == c;
    V3 cf = ld3(m.fc, f);
    V3 fe = sub(cf, ce);
    for (int k = 0; k < n; ++k) {
      V3 cp = ld3(m.x, vid[k]), cpp = ld3(m.x, vid[(k + 1) % n]);
      V3 x = left ? cross(sub(cp, cf), sub(cpp, cf)) : cross(sub(cpp, cf), sub(cp, cf));
      double vol = dot(x, fe) / 6.0;
      cen.x = cen.x + vol * (cp.x + cpp.x + cf.x + ce.x) / 4.0;
      cen.y = cen.y + vol * (cp.y + cpp.y + cf.y + ce.y) / 4.0;
      cen.z = cen.z + vol * (cp.z + cpp.z + cf.z + ce.z) / 4.0;
      sum_vol = sum_vol + vol;
    }
  }
  cen = {cen.x / sum_vol, cen.y / sum_vol, cen.z / sum_vol};
  m.cc[c] = make_double4(cen.x, cen.y, cen.z, 0.0);
  bool ok = true;
  double vcell = 0.0;
  for (int s = vb; s < vb + nvc; ++s) {
    int4 q4 = m.se_sf[s];
    int q[4] = {q4.x, q4.y, q4.z, q4.w};
    double vol = 0.0;
    for (int j = 0; j < 4 && q[j] >= 0; ++j) {
      int sf = q[j];
      int f = m.sf_face[sf], vert = m.sf_vert[sf];
      int4 fv = m.fvert[f];
      int vid[4] = {fv.x, fv.y, fv.z, fv.w};
      int n = fv.w < 0 ? 3 : 4;
      int k = 0;
      while (k < n - 1 && vid[k] != vert) ++k;
      V3 cp = ld3(m.x, vid[k]);
      V3 cpm = half_sum(ld3(m.x, vid[(k - 1 + n) % n]), cp);
      V3 cpp = half_sum(ld3(m.x, vid[(k + 1) % n]), cp);
      V3 cf = ld3(m.fc, f);
      V3 fe = sub(cf, cen);
      V3 a = sub(cpm, cf), b = sub(cp, cf), cc3 = sub(cpp, cf);
      V3 x1, x2;
      if (m.flr[f].x == c) {
        x1 = cross(a, b);
        x2 = cross(b, cc3);
      } else {
        x1 = cross(cc3, b);
        x2 = cross(b, a);
      }
      vol = vol + dot(x1, fe) / 6.0 + dot(x2, fe) / 6.0;
    }
    m.vol_se[s] = vol;
    ok = ok && (vol > 0.0);
    vcell = vcell + vol;
  }
  m.vol[c] = vcell;
  // check_mesh_elem_volume / _closed / _subface_closed
  double vdiv = 0.0;
  V3 nt = {0.0, 0.0, 0.0}, ns = {0.0, 0.0, 0.0};
  for (int j = 0; j < nfc; ++j) {
    int f = faces[j];
    double4 fn = m.fn[f];
    double sg = m.flr[f].x == c ? 1.0 : -1.0;
    V3 nn = {sg * fn.x, sg * fn.y, sg * fn.z};
    V3 an = {fn.w * nn.x, fn.w * nn.y, fn.w * nn.z};
    vdiv = vdiv + dot(ld3(m.fc, f), an);
    nt = {nt.x + an.x, nt.y + an.y, nt.z + an.z};
  }
  vdiv = vdiv / 3.0;
  for (int j = 0; j < nfc; ++j) {
    int f = faces[j];
    double sg = m.flr[f].x == c ? 1.0 : -1.0;
    int4 fs = m.fsf[f];
    int sfi[4] = {fs.x, fs.y, fs.z, fs.w};
    for (int k = 0; k < 4 && sfi[k] >= 0; ++k) {
      double4 sn = m.sfn[sfi[k]];
      ns = {ns.x + sn.w * (sg * sn.x), ns.y + sn.w * (sg * sn.y), ns.z + sn.w * (sg * sn.z)};
    }
  }
  ok = ok && (fabs(vcell - vdiv) < 1e-14);
  ok = ok && (fnorm2_3(nt.x, nt.y, nt.z) < 1e-14);
  ok = ok && (fnorm2_3(ns.x, ns.y, ns.z) < 1e-14);
  if (!ok) atomicOr(m.status, kErrMeshCheck);

}

template <int FULL>
__global__ void __launch_bounds__(128) k_face_geom(DevMesh m, const LagScalars* sc) {
  if (sc && sc->skip) return;
  geo::face_geom_body<FULL>(m, face_at(m, blockIdx.x * blockDim.x + threadIdx.x));
}

__global__ void __launch_bounds__(geo::kGeoBlock) k_geom_step(DevMesh m, double* sol6, const double* rhs6,
                                                              const LagScalars* sc) {
  if (sc && sc->skip) return;
  geo::geom_step_body(m, sol6, rhs6, sol6 ? sc->dt : 0.0, blockIdx.x * geo::kGeoBlock + threadIdx.x);
}

__global__ void k_build_geom_codes(DevMesh m) { geo::build_geom_codes(m, blockIdx.x * blockDim.x + threadIdx.x); }

__global__ void k_lag_update(DevMesh m, double* sol6, const double* rhs6, const LagScalars* sc) {
  if (sc->skip) return;
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < m.ne) geo::state_update(m, sol6, rhs6, sc->dt, c);
}

// compute_vert_volume (:273-288)
__global__ void k_vert_volume(DevMesh m) {
  int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= m.nv) return;
  double s = 0.0;
  for (int q = m.vse_off[v]; q < m.vse_off[v + 1]; ++q) s = s + m.vol_se[m.vse[q]];
  m.vol_v[v] = s;
}

// find_if_vert_is_bound (mesh_connectivity_module.F90:726-750) over the vertex's own
// subfaces (one per face touching it)
__global__ void k_vert_is_bound(DevMesh m) {
  int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= m.nv) return;
  int8_t b = 0;
  for (int p = m.vsf_off[v]; p < m.vsf_off[v + 1]; ++p) {
    int sf = m.vsf[p];
    if (m.sf_vert[sf] != v) continue;
    int f = m.sf_face[sf];
    if (m.flr[f].y >= 0) continue;
    if (!m.b2d || fabs(m.fn[f].z) < 1e-12) b = 1;
  }
  m.is_bound[v] = b;
}

}  // namespace

void launch_geometry(const DevMesh& m, int full, double* sol6, const double* rhs6, const LagScalars* sc) {
  if (full) {
    k_face_geom<1><<<grid_for(m.nf, 128), 128, 0, m.stream>>>(m, nullptr);
    k_cell_geometry<<<grid_for(m.ne, 128), 128, 0, m.stream>>>(m);
  } else {
    launch_face_geometry_step(m, sc);
    launch_cell_geometry_step(m, sol6, rhs6, sc);
  }
}
void launch_face_geometry_step(const DevMesh& m, const LagScalars* sc) {
  k_face_geom<0><<<grid_for(m.nf, 128), 128, 0, m.stream>>>(m, sc);
}
void launch_cell_geometry_step(const DevMesh& m, double* sol6, const double* rhs6, const LagScalars* sc) {
  k_geom_step<<<grid_for(m.ne, geo::kGeoBlock), geo::kGeoBlock, 0, m.stream>>>(m, sol6, rhs6, sc);
}
void launch_lag_update(const DevMesh& m, double* sol6, const double* rhs6, const LagScalars* sc) {
  k_lag_update<<<grid_for(m.ne, 256), 256, 0, m.stream>>>(m, sol6, rhs6, sc);
}
void launch_build_geom_codes(const DevMesh& m) {
  k_build_geom_codes<<<grid_for(m.ne, 128), 128, 0, m.stream>>>(m);
}
void launch_vert_volume(const DevMesh& m) { k_vert_volume<<<grid_for(m.nv, 256), 256, 0, m.stream>>>(m); }
void launch_vert_is_bound(const DevMesh& m) { k_vert_is_bound<<<grid_for(m.nv, 256), 256, 0, m.stream>>>(m); }

}  // namespace subfv
