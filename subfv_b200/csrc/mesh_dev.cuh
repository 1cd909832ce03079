// Device-resident mesh: the reference's mesh_type (src/mesh/mesh_module.F90:17-89)
// flattened into 0-based structure-of-arrays and fixed-width records so that
// per-entity kernels load whole records with vector loads.
//
// Layout in HBM (all 0-based):
//   vertices   x[nv] double4 (x, y, z, -), vp[nv] double4, vol_v[nv]
//   faces      fvert[nf] int4 (vertex ids, -1 pad), flr[nf] int2 (left cell, right cell
//              or -(tag+1) for a boundary), fsf[nf] int4 (subface ids in the face's order),
//              fc[nf] double4 (centroid), fn[nf] double4 (unit normal, area)
//   subfaces   sf_face, sf_vert [nsf] int, sf_se[nsf] int2 (left/right subcell, -1 none),
//              sfn[nsf] double4 (unit normal, area), sfa[nsf] (area alone)
//   subcells   se_elem, se_vert [nse], se_sf[nse] int4 (subfaces, -1 pad), vol_se[nse]
//   cells      ev_off[ne+1] (cell subcells are ev_off[c]..ev_off[c+1]-1, one per vertex),
//              ev[], ef8[ne] (faces, -1 pad to 8), cc[ne] double4 (centroid), vol[ne]
//   node CSR   vsf_off[nv+1], vsf[] (subface ids), vse_off[nv+1], vse[] (subcell ids)
//   cell CSR   csf_off[ne+1], csf[] = 2*p + side over the node-ordered subface
//              positions p that touch the cell, ascending (the order in which the
//              reference's node loop scatters into that cell).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

#include "common.cuh"

namespace subfv {

struct DevMesh {
  int nv = 0, ne = 0, nf = 0, nsf = 0, nse = 0, nvsf = 0, ncsf = 0;
  int b2d = 1;
  int vsf_identity = 0;  // vsf[p] == p for every p (no periodic extension)
  int max_vsf = 0, max_vse = 0;  // the most subfaces / subcells around one vertex
  int max_evc = 0;               // the most vertices of one cell
  // vertices
  double4* x = nullptr;
  double4* vp = nullptr;
  double* vol_v = nullptr;
  int8_t* is_bound = nullptr;
  // faces
  int4* fvert = nullptr;
  int2* flr = nullptr;
  int4* fsf = nullptr;
  double4* fc = nullptr;
  double4* fn = nullptr;
  // subfaces
  int* sf_face = nullptr;
  int* sf_vert = nullptr;
  int2* sf_se = nullptr;
  int* sf_loc = nullptr;
  double4* sfn = nullptr;
  double* sfa = nullptr;
  // Lagrangian face records (6 doubles per face, allocated on first Lagrangian use):
  // wave speeds and normal velocities of the face's two sides for the current state
  double* frec = nullptr;
  // per cell-CSR entry: subface, face, owning node | side << 30, subcell (Lagrangian
  // cell kernel; built on first Lagrangian use)
  int4* centry = nullptr;
  // per face: sum of area * unit normal over its subfaces (Lagrangian step's mesh check)
  double4* fS = nullptr;
  // Static local topology for the geometry kernels (the topology never changes, so the
  // per-step kernels need no id searches; layouts in geom_body.cuh). fpos: per face,
  // built at creation; gface (8 per cell, face slot order of ef8) and gsub (per subcell):
  // built on first Lagrangian use.
  uint8_t* fpos = nullptr;
  uint16_t* gface = nullptr;
  uint32_t* gsub = nullptr;
  // Launch orders (built at creation): the faces grouped by vertex count and interior /
  // boundary, the vertices by subface count, subcell count and boundary subfaces, each
  // group in numbering order. The long per-entity kernels (face geometry, the explicit
  // Euler node kernel and nodal gradient) map thread t to forder[t] / vorder[t], so the
  // threads of a warp follow the same code path; no result depends on the order. The short
  // gather-bound kernels keep the numbering order, which coalesces better.
  int* forder = nullptr;
  int* vorder = nullptr;
  // Diffusion stencils (built at creation). A vertex's diffusion system runs over the
  // subfaces dsf[dsf_off[v]..] and subcells dse[dse_off[v]..]; rows and columns are the
  // positions in these lists. Without periodic faces they are the vertex's own lists
  // (positions = the reference's id_loc_around_node). At a periodic node every image
  // vertex gets the same stencil: the union over the images of their subfaces (the two
  // copies of a periodic face merged, keyed by their cells) and their own subcells.
  // dsf_se: a stencil subface's left / right subcells (-1 none), dsf_seloc their
  // positions in the subcell list; dse_sfloc: a stencil subcell's subfaces' positions in
  // the subface list (-1 pad).
  int* dsf_off = nullptr;
  int* dsf = nullptr;
  int2* dsf_se = nullptr;
  int2* dsf_seloc = nullptr;
  int* dse_off = nullptr;
  int* dse = nullptr;
  int4* dse_sfloc = nullptr;
  int max_dsf = 0, max_dse = 0;
  int dstencil_ok = 1;     // every stencil subface's subcells and subcell's subfaces found
  int dstencil_built = 0;  // the d* arrays exist (ensure_diffusion_stencil)
  // With a constant viscosity the diffusion systems of a vertex depend on the mesh and
  // the diffusion constants only: their inverse and products, computed once, are kept
  // here (per vertex at dcache_off[v] doubles), for the constants in dcache_key (a host
  // object; ns_diffusion.cu). Null when not built.
  double* dcache = nullptr;
  long long* dcache_off = nullptr;
  void* dcache_key = nullptr;
  // Geometry changes the cache must see: geom_epoch counts host calls that move the
  // vertices or recompute the geometry; moving is set once a Lagrangian state or batch
  // owns the mesh (it then moves every step, and the cache is not used).
  unsigned long long geom_epoch = 0;
  int moving = 0;
  // The pseudo-inverse of each vertex's nodal-gradient matrix (9 doubles per vertex, row
  // major), valid while npinv_epoch == geom_epoch (ensure_nodal_pinv in ns.cuh).
  double* npinv = nullptr;
  unsigned long long npinv_epoch = 0;
  // set when a Lagrangian step refreshed only the arrays the next step reads (face
  // normals and areas, subface areas, volumes); the rest is recomputed on demand
  int geom_partial = 0;
  // subcells
  int* se_elem = nullptr;
  int* se_vert = nullptr;
  int* se_loc = nullptr;
  int4* se_sf = nullptr;
  double* vol_se = nullptr;
  // cells
  int* ev_off = nullptr;
  int* ev = nullptr;
  int* ef8 = nullptr;
  int* ekind = nullptr;
  double4* cc = nullptr;
  double* vol = nullptr;
  // node and cell CSR
  int* vsf_off = nullptr;
  int* vsf = nullptr;
  int* p_node = nullptr;  // vertex owning node-ordered position p
  int* vse_off = nullptr;
  int* vse = nullptr;
  int* csf_off = nullptr;
  int* csf = nullptr;
  // vertex -> cell lists (vert%elem_neigh), and each cell's subcells in ascending
  // vertex order (the order the reference's node loop scatters into the cell)
  int* vel_off = nullptr;
  int* vel = nullptr;
  int* cse_sorted = nullptr;
  // status word (StatusBits) and the stream the mesh's work runs on
  unsigned* status = nullptr;
  cudaStream_t stream = nullptr;
  size_t bytes = 0;
};

// the face / vertex a per-entity kernel's thread t works on (t past the end stays past it)
__device__ inline int face_at(const DevMesh& m, int t) { return t < m.nf ? m.forder[t] : t; }
__device__ inline int vert_at(const DevMesh& m, int t) { return t < m.nv ? m.vorder[t] : t; }

int devmesh_create(const struct subfv_mesh_desc* d, DevMesh* m);
void devmesh_free(DevMesh* m);
// Builds the Navier-Stokes diffusion stencil (dsf*, dse*, max_dsf, max_dse, dstencil_ok)
// on first use; later calls return at once.
int ensure_diffusion_stencil(DevMesh* m);
// releases the host side of the diffusion cache (the device arrays go with the mesh's)
void diffusion_cache_forget(DevMesh* m);

// Geometry kernels (mesh_geometry_module.F90:16-57), launched on m.stream.
// sc (optional): a step whose skip flag is set leaves everything untouched; with sol6
// the cell kernel also applies sol += dt*rhs using sc->dt.
// full: every geometric array; otherwise the Lagrangian step's subset (with sol6, the
// update sol += dt*rhs fused in)
void launch_geometry(const DevMesh& m, int full, double* sol6 = nullptr, const double* rhs6 = nullptr,
                     const LagScalars* sc = nullptr);
// the two halves of launch_geometry(m, 0, ...): the face kernel, then the cell kernel
void launch_face_geometry_step(const DevMesh& m, const LagScalars* sc);
void launch_cell_geometry_step(const DevMesh& m, double* sol6, const double* rhs6, const LagScalars* sc);
// sol += dt*rhs alone (the update launch_geometry otherwise fuses in)
void launch_lag_update(const DevMesh& m, double* sol6, const double* rhs6, const LagScalars* sc);
void launch_vert_volume(const DevMesh& m);
// the static local-topology codes of the Lagrangian geometry kernel (gface, gsub must be
// allocated: 8 per cell, one per subcell)
void launch_build_geom_codes(const DevMesh& m);
void launch_vert_is_bound(const DevMesh& m);

}  // namespace subfv
