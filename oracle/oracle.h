// Test infrastructure only: the oracle that the CUDA path is checked against.
//
// A serial CPU restatement, in C++, of the subfv (vdelmas/subfv) Fortran routines on
// the subface finite-volume hot path. Every routine cites the Fortran file:line it
// follows; loops, branch structure and floating-point evaluation order follow the
// Fortran source (left-to-right, no FMA contraction: built with -ffp-contract=off).
//
// PARITY UNPINNED: the reference is Fortran 2008 + MPI + LAPACK and no Fortran
// compiler exists in this environment, and the reference's own tests hold no golden
// vectors (they only run the solver and plot). The LAPACK-replacing pieces are
// cross-checked against scipy's LAPACK in the CPU tests.
//
// Nothing outside tests/, the smoke check and the bench's CPU-baseline leg may link
// or call this library.
#pragma once
#include <cstdint>
#include <vector>
#include <string>
#include <map>

namespace oracle {

// Mirrors mesh_module.F90 types (src/mesh/mesh_module.F90:17-89). Arrays are 1-based
// (index 0 unused) so the restatement reads like the Fortran.
struct Vert {
  bool is_bound = false;
  int n_sub_faces_neigh = 0, n_sub_elems_neigh = 0, n_elems_neigh = 0, n_faces_neigh = 0;
  std::vector<int> sub_face_neigh, sub_elem_neigh, elem_neigh, face_neigh;  // 1-based
  double coord[4] = {0, 0, 0, 0};                                            // [1..3]
  double volume = 0;
};
struct Face {
  int n_vert = -1, n_sub_faces = -1;
  int left_neigh = 0, left_neigh_face = 0, right_neigh = 0, right_neigh_face = 0;
  std::vector<int> sub_face, vert;
  double area = 0;
  double coord[4] = {0, 0, 0, 0}, norm[4] = {0, 0, 0, 0};
};
struct MinFace {
  int n_vert = -1;
  int left_neigh = 0, left_neigh_face = 0, right_neigh = 0, right_neigh_face = 0;
  std::vector<int> vert;
};
struct BFace {
  int n_vert = -1;
  std::vector<int> vert;
  int tag = 0;
};
struct SubFace {
  int mesh_vert = 0, mesh_face = 0, id_loc_around_node = 0;
  int left_elem_neigh = 0, right_elem_neigh = 0, left_sub_elem_neigh = 0, right_sub_elem_neigh = 0;
  double area = 0;
  double norm[4] = {0, 0, 0, 0};
};
struct Elem {
  int n_vert = 0, n_faces = 0, n_sub_faces = 0, n_sub_elems = 0, elem_kind = 0, tag = -1;
  int n_neigh_by_vert = 0;
  std::vector<int> vert, face, sub_face, sub_elem, neigh_by_vert;
  double volume = 0;
  double coord[4] = {0, 0, 0, 0};
};
struct SubElem {
  int id_loc_around_node = 0, mesh_vert = 0, mesh_elem = 0, n_sub_faces = 0;
  std::vector<int> sub_face;
  double volume = 0;
};
struct Mesh {
  int n_vert = 0, n_elems = 0, n_faces = 0, n_sub_faces = 0, n_boundary_faces = 0, n_sub_elems = 0;
  int n_max_sub_faces_around_node = 0;
  std::vector<Vert> vert;
  std::vector<Elem> elem;
  std::vector<Face> face;
  std::vector<SubFace> sub_face;
  std::vector<BFace> boundary_face;
  std::vector<SubElem> sub_elem;
  std::vector<MinFace> minimal_face;
  bool geometry_ok = true;
};

// gfortran's inline NORM2: scaled sum of squares (scale starts at 1).
double fnorm2(const double* a, int n);

// mesh_reading_module.F90:1144-1320 per-kind face tables and minimal-face fill.
void read_raw(Mesh& m, int n_vert, const double* coords, int n_elems, const int* kind,
              const int* ev_off, const int* ev, int n_bf, const int* bf_off, const int* bf_vert,
              const int* bf_tag);
// mesh_connectivity_module.F90:12-59 (num_procs = 1).
// renumber 0: the reference's BFS vertex order; 1: vertices along a Hilbert curve
void build_mesh(Mesh& m, bool use_sub_entities, bool b2d, bool periodic, int renumber = 0);
// mesh_geometry_module.F90:16-57.
void compute_geometry_mesh(Mesh& m, bool b2d);
void find_if_vert_is_bound(Mesh& m, bool b2d);

// Named flattened arrays (the C-ABI mesh descriptor layout; ids 1-based as in Fortran).
std::map<std::string, std::vector<int32_t>> export_topology(const Mesh& m);

}  // namespace oracle
