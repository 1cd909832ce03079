// Host-side mesh topology: the subfv build_mesh pipeline re-designed as linear-time
// passes (counting sorts and per-vertex grouping) that reproduce the reference's
// numbering exactly: BFS vertex order, first-touch cell order, faces grouped by their
// smallest vertex id, first-touch face order, subfaces numbered vertex by vertex.
// Reference: src/mesh/mesh_connectivity_module.F90:12-59 and the element face tables
// of src/mesh/mesh_reading_module.F90:1144-1320.
#pragma once
#include <cstdint>
#include <map>
#include <string>
#include <vector>

namespace subfv {

struct RawMeshView {
  int n_vert;
  const double* coords;  // [3*n_vert], file order
  int n_elems;
  const int32_t* elem_kind;      // gmsh kinds 4 (tet), 5 (hex), 6 (prism), 7 (pyramid)
  const int32_t* elem_vert_off;  // [n_elems+1]
  const int32_t* elem_vert;      // 1-based vertex ids
  int n_bfaces;
  const int32_t* bface_off;   // [n_bfaces+1] or null
  const int32_t* bface_vert;  // 1-based
  const int32_t* bface_tag;   // boundary-condition index (0 = none / wall)
  int b2d;
  int periodic;
  int renumber = 0;  // 0: the reference's BFS vertex order; 1: along a Hilbert curve
};

// All ids are 1-based like the reference's; face_right: >0 cell, 0 wall, <0 -tag.
struct Topology {
  int n_vert = 0, n_elems = 0, n_faces = 0, n_sub_faces = 0, n_sub_elems = 0;
  int n_max_sub_faces_around_node = 0;
  std::vector<double> vert_coord;  // renumbered, [3*n_vert]
  std::map<std::string, std::vector<int32_t>> arr;
  const std::vector<int32_t>& a(const char* n) const { return arr.at(n); }
};

// Returns 0 on success, a positive code on malformed input.
int build_topology(const RawMeshView& in, Topology& out, std::string* err);

// Position of each vertex along a Hilbert curve: new id (1-based) of input vertex i at
// otn[i], input id of new vertex k at nto[k] (both 1-based, entry 0 unused). Slabs
// (b2d) follow the 2-D curve of (x, y), so a column's vertices share a key; 3-D meshes
// the 3-D curve of (x, y, z); both on a cube around the mesh, ties by input id.
void hilbert_vertex_order(int n_vert, const double* coords, int b2d, std::vector<int32_t>& otn,
                          std::vector<int32_t>& nto);

}  // namespace subfv
