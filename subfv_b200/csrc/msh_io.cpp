// Mesh and solution files on the host: the gmsh MSH2 / MSH4 (ASCII) readers of
// src/mesh/mesh_reading_module.F90:154-1324 (one process), the VTU solution writers of
// src/ns/ns_io_module.F90:403-884 (its cell fields) and
// src/lagrange/lagrange_io_module.F90:26-289, and the VTU restart reader of
// src/ns/ns_io_module.F90:1333-1382.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/subfv.h"

namespace subfv {
void set_error(const std::string& msg);
}
using subfv::set_error;

struct subfv_msh {
  std::vector<double> coords;
  std::vector<int32_t> elem_kind, elem_vert_off{0}, elem_vert, bface_off{0}, bface_vert, bface_tag;
};

namespace {

// vertices per gmsh element type (types 1-31)
const int kNVertKind[31] = {2, 3, 4, 4, 8, 6, 5, 3, 6, 9, 10, 27, 18, 14, 1, 8,
                            20, 15, 13, 9, 10, 12, 15, 15, 21, 4, 5, 6, 20, 35, 56};
int n_vert_kind(int k) { return k >= 1 && k <= 31 ? kNVertKind[k - 1] : -1; }
bool is_volume(int k) { return k >= 4 && k <= 7; }
bool is_bface(int k) { return k == 2 || k == 3; }

struct Lines {
  std::ifstream f;
  std::string line;
  bool next() { return static_cast<bool>(std::getline(f, line)); }
  // advance to the line that starts with tag; false at end of file
  bool seek(const char* tag, const char* stop = nullptr) {
    const size_t n = std::strlen(tag);
    while (next()) {
      if (line.compare(0, n, tag) == 0) return true;
      if (stop && line.compare(0, std::strlen(stop), stop) == 0) return false;
    }
    return false;
  }
};

std::vector<std::string> tokens(const std::string& s) {
  std::vector<std::string> t;
  std::istringstream is(s);
  std::string w;
  while (is >> w) t.push_back(w);
  return t;
}
std::string unquote(const std::string& s) {
  std::string r = s;
  r.erase(std::remove(r.begin(), r.end(), '"'), r.end());
  return r;
}

// $PhysicalNames: bc_tag(j) = the physical tag named bc_names[j] (-1 if absent)
bool read_physical_names(Lines& L, int n_bc, const char* const* bc_names, std::vector<long>& bc_tag) {
  bc_tag.assign(n_bc, -1);
  if (n_bc == 0) return true;
  if (!L.seek("$PhysicalNames", "$Nodes")) {
    set_error("subfv_msh_read: no physical names inside the mesh");
    return false;
  }
  L.next();
  const long n = std::stol(tokens(L.line).at(0));
  for (long i = 0; i < n; ++i) {
    L.next();
    std::istringstream is(L.line);
    long dim = 0, tag = 0;
    is >> dim >> tag;
    std::string rest;
    std::getline(is, rest);
    std::string name = unquote(rest);
    name.erase(0, name.find_first_not_of(" \t"));
    name.erase(name.find_last_not_of(" \t\r") + 1);
    for (int j = 0; j < n_bc; ++j)
      if (name == bc_names[j]) bc_tag[j] = tag;
  }
  return true;
}

int tag_of(const std::vector<long>& bc_tag, long phys) {  // the last bc whose tag matches (0: none)
  int t = 0;
  for (size_t j = 0; j < bc_tag.size(); ++j)
    if (bc_tag[j] == phys) t = (int)j + 1;
  return t;
}

// read_mesh_msh_2 (:989-1324): node ids are the lines' order; the first element tag is
// the physical one
int read_msh2(const char* path, int n_bc, const char* const* bc_names, subfv_msh* M) {
  Lines L;
  L.f.open(path);
  std::vector<long> bc_tag;
  if (!read_physical_names(L, n_bc, bc_names, bc_tag)) return -2;
  L.f.clear();
  L.f.seekg(0);
  if (!L.seek("$Nodes")) {
    set_error("subfv_msh_read: no $Nodes section");
    return -2;
  }
  L.next();
  const long nv = std::stol(tokens(L.line).at(0));
  M->coords.resize(3 * nv);
  for (long i = 0; i < nv; ++i) {
    if (!L.next()) return set_error("subfv_msh_read: truncated $Nodes"), -2;
    auto t = tokens(L.line);
    if (t.size() < 4) return set_error("subfv_msh_read: bad node line"), -2;
    for (int d = 0; d < 3; ++d) M->coords[3 * i + d] = std::stod(t[1 + d]);
  }
  if (!L.seek("$Elements")) return set_error("subfv_msh_read: no $Elements section"), -2;
  L.next();
  const long ne = std::stol(tokens(L.line).at(0));
  for (long i = 0; i < ne; ++i) {
    if (!L.next()) return set_error("subfv_msh_read: truncated $Elements"), -2;
    auto t = tokens(L.line);
    if (t.size() < 3) return set_error("subfv_msh_read: bad element line"), -2;
    const int kind = std::stoi(t[1]), ntag = std::stoi(t[2]), nvk = n_vert_kind(kind);
    if (nvk < 0 || (long)t.size() < 3 + ntag + nvk) return set_error("subfv_msh_read: bad element line"), -2;
    std::vector<int32_t> v(nvk);
    for (int k = 0; k < nvk; ++k) {
      const long id = std::stol(t[3 + ntag + k]);
      if (id < 1 || id > nv) return set_error("subfv_msh_read: element refers to an unknown node"), -2;
      v[k] = (int32_t)id;
    }
    if (is_bface(kind)) {
      const long phys = ntag > 0 ? std::stol(t[3]) : 0;
      M->bface_tag.push_back(tag_of(bc_tag, phys));
      M->bface_vert.insert(M->bface_vert.end(), v.begin(), v.end());
      M->bface_off.push_back((int32_t)M->bface_vert.size());
    } else if (is_volume(kind)) {
      M->elem_kind.push_back(kind);
      M->elem_vert.insert(M->elem_vert.end(), v.begin(), v.end());
      M->elem_vert_off.push_back((int32_t)M->elem_vert.size());
    }
  }
  return 0;
}

// read_mesh_msh_4 (:207-987), one partition: surfaces' physical tags from $Entities,
// boundary faces from 2-D blocks, volumes from 3-D blocks; the vertices are the nodes the
// volumes use, numbered in their order of appearance in $Nodes
int read_msh4(const char* path, int n_bc, const char* const* bc_names, subfv_msh* M) {
  Lines L;
  L.f.open(path);
  std::vector<long> bc_tag;
  if (!read_physical_names(L, n_bc, bc_names, bc_tag)) return -2;
  L.f.clear();
  L.f.seekg(0);
  if (!L.seek("$Entities")) return set_error("subfv_msh_read: no $Entities section"), -2;
  L.next();
  auto h = tokens(L.line);
  if (h.size() < 4) return set_error("subfv_msh_read: bad $Entities header"), -2;
  const long np = std::stol(h[0]), nc = std::stol(h[1]), ns = std::stol(h[2]);
  for (long i = 0; i < np + nc; ++i) L.next();
  std::vector<std::pair<long, long>> surf_phys;  // (surface tag, physical tag used)
  for (long i = 0; i < ns; ++i) {
    L.next();
    auto t = tokens(L.line);
    if (t.size() < 8) return set_error("subfv_msh_read: bad surface entity"), -2;
    const long tag = std::stol(t[0]), nphys = std::stol(t[7]);
    long phys = 0;  // the first of the surface's physical tags that names a bc
    for (long k = 0; k < nphys && 8 + k < (long)t.size() && phys == 0; ++k) {
      const long p = std::stol(t[8 + k]);
      for (long b : bc_tag)
        if (b == p) {
          phys = p;
          break;
        }
    }
    surf_phys.emplace_back(tag, phys);
  }
  if (!L.seek("$Elements")) return set_error("subfv_msh_read: no $Elements section"), -2;
  L.next();
  const long nblocks = std::stol(tokens(L.line).at(0));
  std::vector<long> ev_glob, bv_glob;
  for (long b = 0; b < nblocks; ++b) {
    L.next();
    auto t = tokens(L.line);
    if (t.size() < 4) return set_error("subfv_msh_read: bad element block"), -2;
    const int dim = std::stoi(t[0]), kind = std::stoi(t[2]);
    const long etag = std::stol(t[1]), n = std::stol(t[3]);
    const int nvk = n_vert_kind(kind);
    long phys = -1;
    if (dim == 2 && is_bface(kind)) {
      for (auto& sp : surf_phys)
        if (sp.first == etag) phys = sp.second;
      if (phys < 0) return set_error("subfv_msh_read: entity physical tag not found"), -2;
    }
    for (long i = 0; i < n; ++i) {
      L.next();
      if ((dim == 2 && is_bface(kind)) || (dim == 3 && is_volume(kind))) {
        auto e = tokens(L.line);
        if ((long)e.size() < 1 + nvk) return set_error("subfv_msh_read: bad element line"), -2;
        if (dim == 2) {
          M->bface_tag.push_back(tag_of(bc_tag, phys));
          for (int k = 0; k < nvk; ++k) bv_glob.push_back(std::stol(e[1 + k]));
          M->bface_off.push_back((int32_t)bv_glob.size());
        } else {
          M->elem_kind.push_back(kind);
          for (int k = 0; k < nvk; ++k) ev_glob.push_back(std::stol(e[1 + k]));
          M->elem_vert_off.push_back((int32_t)ev_glob.size());
        }
      }
    }
  }
  std::vector<long> used(ev_glob);
  std::sort(used.begin(), used.end());
  used.erase(std::unique(used.begin(), used.end()), used.end());
  L.f.clear();
  L.f.seekg(0);
  if (!L.seek("$Nodes")) return set_error("subfv_msh_read: no $Nodes section"), -2;
  L.next();
  const long nnb = std::stol(tokens(L.line).at(0));
  std::vector<std::pair<long, int32_t>> id;  // (node tag, local id), local ids from 1
  M->coords.clear();
  for (long b = 0; b < nnb; ++b) {
    L.next();
    auto t = tokens(L.line);
    if (t.size() < 4) return set_error("subfv_msh_read: bad node block"), -2;
    const long n = std::stol(t[3]);
    std::vector<char> keep(n);
    for (long i = 0; i < n; ++i) {
      L.next();
      const long tag = std::stol(tokens(L.line).at(0));
      keep[i] = std::binary_search(used.begin(), used.end(), tag);
      if (keep[i]) id.emplace_back(tag, (int32_t)(id.size() + 1));
    }
    for (long i = 0; i < n; ++i) {
      L.next();
      if (!keep[i]) continue;
      auto c = tokens(L.line);
      if (c.size() < 3) return set_error("subfv_msh_read: bad node coordinates"), -2;
      for (int d = 0; d < 3; ++d) M->coords.push_back(std::stod(c[d]));
    }
  }
  std::sort(id.begin(), id.end());
  auto local = [&](long tag) -> int32_t {
    auto it = std::lower_bound(id.begin(), id.end(), std::make_pair(tag, (int32_t)0));
    return it != id.end() && it->first == tag ? it->second : -1;
  };
  for (long g : ev_glob) {
    const int32_t l = local(g);
    if (l < 0) return set_error("subfv_msh_read: element refers to an unknown node"), -2;
    M->elem_vert.push_back(l);
  }
  for (long g : bv_glob) {
    const int32_t l = local(g);
    if (l < 0) return set_error("subfv_msh_read: boundary face refers to a node no volume uses"), -2;
    M->bface_vert.push_back(l);
  }
  return 0;
}

void put(std::FILE* f, double x) { std::fprintf(f, " %.17g", x); }

// gfortran's NORM2 (scaled sum of squares)
double norm2(const double* a, int n) {
  double scale = 1.0, res = 0.0;
  for (int i = 0; i < n; ++i)
    if (a[i] != 0.0) {
      const double ax = std::fabs(a[i]);
      if (ax > scale) {
        const double q = scale / ax;
        res = 1.0 + res * q * q;
        scale = ax;
      } else {
        const double q = ax / scale;
        res += q * q;
      }
    }
  return scale * std::sqrt(res);
}

std::vector<int32_t> topo_array(const subfv_topology* t, const char* name) {
  const int64_t n = subfv_topology_array_len(t, name);
  std::vector<int32_t> v(n > 0 ? n : 0);
  if (n > 0) subfv_topology_array_get(t, name, v.data());
  return v;
}

}  // namespace

// The VTU's mesh part shared by the Euler and Lagrangian writers: header, points,
// polyhedral cells with their faces (the reference writes cell type 42); leaves the file
// open before the point data. Returns the number of cells (0 on error).
static int64_t write_vtu_mesh(std::FILE* f, const subfv_topology* t, std::vector<int32_t>& etag, int64_t& nv) {
  const auto ev_off = topo_array(t, "elem_vert_off"), ev = topo_array(t, "elem_vert");
  const auto ef_off = topo_array(t, "elem_face_off"), ef = topo_array(t, "elem_face");
  const auto fv_off = topo_array(t, "face_vert_off"), fv = topo_array(t, "face_vert");
  etag = topo_array(t, "elem_tag");
  const int64_t ne = (int64_t)ev_off.size() - 1;
  nv = subfv_topology_array_len(t, "vert_is_bound");
  if (ne < 1 || nv < 1) return 0;
  std::vector<double> x(3 * nv);
  subfv_topology_coords(t, x.data());
  double dmin = 1e100, dmax = -1e100;
  for (double c : x) dmin = std::min(dmin, c), dmax = std::max(dmax, c);
  std::fprintf(f, " <VTKFile type='UnstructuredGrid' version='1.0' byte_order='LittleEndian' header_type='UInt64'>\n");
  std::fprintf(f, " <UnstructuredGrid>\n <Piece NumberOfPoints='%lld' NumberOfCells='%lld'>\n", (long long)nv,
               (long long)ne);
  std::fprintf(f, " <Points>\n <DataArray type='Float64' Name='Points' NumberOfComponents='3' format='ascii' "
                  "RangeMin='%.17g' RangeMax='%.17g'>\n", dmin, dmax);
  for (int64_t i = 0; i < nv; ++i) {
    for (int d = 0; d < 3; ++d) put(f, x[3 * i + d]);
    std::fputc('\n', f);
  }
  std::fprintf(f, " </DataArray>\n </Points>\n <Cells>\n");
  std::fprintf(f, " <DataArray type='Int64' Name='connectivity' format='ascii' RangeMin='0' RangeMax='%lld'>\n",
               (long long)(nv - 1));
  for (int64_t c = 0; c < ne; ++c) {
    for (int q = ev_off[c]; q < ev_off[c + 1]; ++q) std::fprintf(f, " %d", ev[q] - 1);
    std::fputc('\n', f);
  }
  std::fprintf(f, " </DataArray>\n <DataArray type='Int64' Name='offsets' format='ascii' RangeMin='0' "
                  "RangeMax='%d'>\n", ev_off[ne]);
  for (int64_t c = 0; c < ne; ++c) std::fprintf(f, " %d\n", ev_off[c + 1]);
  std::fprintf(f, " </DataArray>\n <DataArray type='UInt8' Name='types' format='ascii' RangeMin='42' "
                  "RangeMax='42'>\n");
  for (int64_t c = 0; c < ne; ++c) std::fprintf(f, " 42\n");  // polyhedra, faces below
  std::fprintf(f, " </DataArray>\n <DataArray type='Int64' Name='faces' format='ascii' RangeMin='0' "
                  "RangeMax='%lld'>\n", (long long)(nv - 1));
  std::vector<int64_t> foff(ne);
  int64_t s = 0;
  for (int64_t c = 0; c < ne; ++c) {
    const int nfc = ef_off[c + 1] - ef_off[c];
    std::fprintf(f, " %d\n", nfc);
    s += 1;
    for (int q = ef_off[c]; q < ef_off[c + 1]; ++q) {
      const int fc = ef[q] - 1;
      std::fprintf(f, " %d", fv_off[fc + 1] - fv_off[fc]);
      for (int k = fv_off[fc]; k < fv_off[fc + 1]; ++k) std::fprintf(f, " %d", fv[k] - 1);
      std::fputc('\n', f);
      s += 1 + fv_off[fc + 1] - fv_off[fc];
    }
    foff[c] = s;
  }
  std::fprintf(f, " </DataArray>\n <DataArray type='Int64' Name='faceoffsets' format='ascii' RangeMin='0' "
                  "RangeMax='%lld'>\n", (long long)s);
  for (int64_t c = 0; c < ne; ++c) std::fprintf(f, " %lld\n", (long long)foff[c]);
  std::fprintf(f, " </DataArray>\n </Cells>\n");
  return ne;
}

struct VtuFields {  // writes one DataArray per call, one line per entity
  std::FILE* f;
  template <class Fn>
  void operator()(const char* type, const char* name, int nc, int64_t n, Fn&& fn) {
    std::fprintf(f, " <DataArray type='%s' Name='%s' format='ascii' NumberOfComponents='%d'>\n", type, name, nc);
    for (int64_t i = 0; i < n; ++i) {
      fn(i);
      std::fputc('\n', f);
    }
    std::fprintf(f, " </DataArray>\n");
  }
};

extern "C" {

int subfv_msh_read(const char* path, int n_bc, const char* const* bc_names, subfv_msh** out) {
  if (!path || !out || n_bc < 0 || (n_bc > 0 && !bc_names)) {
    set_error("subfv_msh_read: bad argument");
    return -2;
  }
  std::ifstream f(path);
  if (!f) {
    set_error(std::string("subfv_msh_read: cannot open ") + path);
    return -2;
  }
  std::string line;
  double version = 0.0;
  while (std::getline(f, line))
    if (line.compare(0, 11, "$MeshFormat") == 0) {
      std::getline(f, line);
      auto t = tokens(line);
      version = t.empty() ? 0.0 : std::stod(t[0]);
      if (t.size() > 1 && t[1] != "0") {
        set_error("subfv_msh_read: binary MSH files are not read (ASCII only)");
        return -2;
      }
      break;
    }
  auto* M = new subfv_msh();
  int rc;
  try {
    if (std::floor(version) == 4) rc = read_msh4(path, n_bc, bc_names, M);
    else if (std::floor(version) == 2) rc = read_msh2(path, n_bc, bc_names, M);
    else {
      set_error("subfv_msh_read: MSH version 2 or 4 expected");
      rc = -2;
    }
  } catch (const std::exception& e) {
    set_error(std::string("subfv_msh_read: malformed file (") + e.what() + ")");
    rc = -2;
  }
  if (rc == 0 && (M->elem_kind.empty() || M->coords.empty())) {
    set_error("subfv_msh_read: no 3-D elements in the mesh");
    rc = -2;
  }
  if (rc) {
    delete M;
    return rc;
  }
  *out = M;
  return 0;
}

int subfv_msh_sizes(const subfv_msh* m, int64_t* sizes) {
  if (!m || !sizes) return -2;
  sizes[0] = (int64_t)(m->coords.size() / 3);
  sizes[1] = (int64_t)m->elem_kind.size();
  sizes[2] = (int64_t)m->elem_vert.size();
  sizes[3] = (int64_t)m->bface_tag.size();
  sizes[4] = (int64_t)m->bface_vert.size();
  return 0;
}

int subfv_msh_get(const subfv_msh* m, double* coords, int32_t* elem_kind, int32_t* elem_vert_off,
                  int32_t* elem_vert, int32_t* bface_off, int32_t* bface_vert, int32_t* bface_tag) {
  if (!m) return -2;
  auto cp = [](auto* dst, const auto& src) {
    if (dst && !src.empty()) std::memcpy(dst, src.data(), src.size() * sizeof(src[0]));
  };
  cp(coords, m->coords);
  cp(elem_kind, m->elem_kind);
  cp(elem_vert_off, m->elem_vert_off);
  cp(elem_vert, m->elem_vert);
  cp(bface_off, m->bface_off);
  cp(bface_vert, m->bface_vert);
  cp(bface_tag, m->bface_tag);
  return 0;
}

void subfv_msh_destroy(subfv_msh* m) { delete m; }

int subfv_write_sol_vtu(const char* path, const subfv_topology* t, const double* sol, const double* delta,
                        const double* vp, const double* elem_coord, double Cv_p, double mu) {
  if (!path || !t || !sol || !(Cv_p > 0.0)) {
    set_error("subfv_write_sol_vtu: bad argument");
    return -2;
  }
  const double G = 1.4;  // ns_global_data_module.F90:9
  std::FILE* f = std::fopen(path, "w");
  if (!f) {
    set_error(std::string("subfv_write_sol_vtu: cannot open ") + path);
    return -2;
  }
  std::vector<int32_t> etag;
  int64_t nv = 0;
  const int64_t ne = write_vtu_mesh(f, t, etag, nv);
  if (ne == 0) {
    std::fclose(f);
    set_error("subfv_write_sol_vtu: empty topology");
    return -2;
  }
  VtuFields fw{f};
  if (vp) {
    std::fprintf(f, " <PointData>\n");
    fw("Float64", "Nodal_Velocity", 3, nv, [&](int64_t i) {
      for (int d = 0; d < 3; ++d) put(f, vp[3 * i + d]);
    });
    std::fprintf(f, " </PointData>\n");
  }
  std::fprintf(f, " <CellData>\n");
  auto field = [&](const char* type, const char* name, int nc, auto&& fn) {
    std::fprintf(f, " <DataArray type='%s' Name='%s' format='ascii' NumberOfComponents='%d'>\n", type, name, nc);
    for (int64_t c = 0; c < ne; ++c) {
      fn(c);
      std::fputc('\n', f);
    }
    std::fprintf(f, " </DataArray>\n");
  };
  auto u = [&](int64_t c) { return sol + 5 * c; };
  auto pressure = [&](int64_t c) {
    const double* q = u(c);
    const double w[3] = {q[1] / q[0], q[2] / q[0], q[3] / q[0]};
    return (G - 1) * (q[4] - 0.5 * q[0] * (w[0] * w[0] + w[1] * w[1] + w[2] * w[2]));
  };
  if (elem_coord)
    field("Float64", "Centroid", 3, [&](int64_t c) {
      for (int d = 0; d < 3; ++d) put(f, elem_coord[3 * c + d]);
    });
  field("Int32", "Tag", 1, [&](int64_t c) { std::fprintf(f, " %d", etag.empty() ? -1 : etag[c]); });
  field("Int32", "MPI_Color", 1, [&](int64_t) { std::fprintf(f, " 0"); });
  field("Float64", "Density", 1, [&](int64_t c) { put(f, u(c)[0]); });
  field("Float64", "Momentum", 3, [&](int64_t c) {
    for (int d = 1; d < 4; ++d) put(f, u(c)[d]);
  });
  field("Float64", "Energy", 1, [&](int64_t c) { put(f, u(c)[4] / u(c)[0]); });
  field("Float64", "Velocity", 3, [&](int64_t c) {
    for (int d = 1; d < 4; ++d) put(f, u(c)[d] / u(c)[0]);
  });
  field("Float64", "Pressure", 1, [&](int64_t c) { put(f, pressure(c)); });
  field("Float64", "Internal_energy", 1, [&](int64_t c) {
    const double* q = u(c);
    const double w[3] = {q[1] / q[0], q[2] / q[0], q[3] / q[0]};
    const double n = norm2(w, 3);
    put(f, q[4] / q[0] - 0.5 * (n * n));
  });
  field("Float64", "H", 1, [&](int64_t c) { put(f, u(c)[4] / u(c)[0] + pressure(c) / u(c)[0]); });
  field("Float64", "Mach", 1, [&](int64_t c) {
    const double* q = u(c);
    const double w[3] = {q[1] / q[0], q[2] / q[0], q[3] / q[0]};
    put(f, norm2(w, 3) / std::sqrt(G * pressure(c) / q[0]));
  });
  field("Float64", "Temperature", 1, [&](int64_t c) {
    const double* q = u(c);
    const double tau = 1.0 / q[0];
    put(f, (q[4] * tau - 0.5 * (q[1] * q[1] + q[2] * q[2] + q[3] * q[3]) * (tau * tau)) / Cv_p);
  });
  if (mu >= 0.0) field("Float64", "mu", 1, [&](int64_t) { put(f, mu); });
  if (delta) field("Float64", "Residual", 1, [&](int64_t c) { put(f, norm2(delta + 5 * c, 5)); });
  std::fprintf(f, " </CellData>\n </Piece>\n </UnstructuredGrid>\n </VTKFile>\n");
  const bool ok = std::ferror(f) == 0;
  std::fclose(f);
  if (!ok) {
    set_error("subfv_write_sol_vtu: write failed");
    return -1;
  }
  return 0;
}

int subfv_write_sol_vtu_lag(const char* path, const subfv_topology* t, const double* sol, const double* vp,
                            const double* pp, const double* elem_coord) {
  if (!path || !t || !sol || !vp) {
    set_error("subfv_write_sol_vtu_lag: bad argument");
    return -2;
  }
  const double G = 1.4;  // the Lagrangian module's gamma
  std::FILE* f = std::fopen(path, "w");
  if (!f) {
    set_error(std::string("subfv_write_sol_vtu_lag: cannot open ") + path);
    return -2;
  }
  std::vector<int32_t> etag;
  int64_t nv = 0;
  const int64_t ne = write_vtu_mesh(f, t, etag, nv);
  if (ne == 0) {
    std::fclose(f);
    set_error("subfv_write_sol_vtu_lag: empty topology");
    return -2;
  }
  VtuFields fw{f};
  auto u = [&](int64_t c) { return sol + 5 * c; };
  auto pressure = [&](int64_t c) {  // lagrange_module.F90:429-436
    const double* q = u(c);
    const double n = norm2(q + 1, 3);
    return (G - 1.0) / q[0] * (q[4] - 0.5 * (n * n));
  };
  std::fprintf(f, " <PointData>\n");
  fw("Float64", "Vp", 3, nv, [&](int64_t i) {
    for (int d = 0; d < 3; ++d) put(f, vp[3 * i + d]);
  });
  if (pp) fw("Float64", "Pp", 1, nv, [&](int64_t i) { put(f, pp[i]); });
  std::fprintf(f, " </PointData>\n <CellData>\n");
  if (elem_coord) {
    fw("Float64", "Centroid", 3, ne, [&](int64_t c) {
      for (int d = 0; d < 3; ++d) put(f, elem_coord[3 * c + d]);
    });
    fw("Float64", "Rxy", 1, ne, [&](int64_t c) { put(f, norm2(elem_coord + 3 * c, 2)); });
    fw("Float64", "R", 1, ne, [&](int64_t c) { put(f, norm2(elem_coord + 3 * c, 3)); });
  }
  fw("Int32", "Tag", 1, ne, [&](int64_t c) { std::fprintf(f, " %d", etag.empty() ? -1 : etag[c]); });
  fw("Int32", "MPI_Color", 1, ne, [&](int64_t) { std::fprintf(f, " 0"); });
  fw("Float64", "Density", 1, ne, [&](int64_t c) { put(f, 1.0 / u(c)[0]); });
  fw("Float64", "Velocity", 3, ne, [&](int64_t c) {
    for (int d = 1; d < 4; ++d) put(f, u(c)[d]);
  });
  fw("Float64", "Pressure", 1, ne, [&](int64_t c) { put(f, pressure(c)); });
  fw("Float64", "Internal_energy", 1, ne, [&](int64_t c) { put(f, pressure(c) * u(c)[0] / (G - 1.0)); });
  std::fprintf(f, " </CellData>\n </Piece>\n </UnstructuredGrid>\n </VTKFile>\n");
  const bool ok = std::ferror(f) == 0;
  std::fclose(f);
  if (!ok) {
    set_error("subfv_write_sol_vtu_lag: write failed");
    return -1;
  }
  return 0;
}

int subfv_restart_from_vtu(const char* path, int64_t n_elems, double* sol) {
  if (!path || n_elems < 1 || !sol) {
    set_error("subfv_restart_from_vtu: bad argument");
    return -2;
  }
  Lines L;
  L.f.open(path);
  if (!L.f) {
    set_error(std::string("subfv_restart_from_vtu: cannot open ") + path);
    return -2;
  }
  auto find = [&](const char* name) {
    const std::string key = std::string("Name='") + name + "'";
    while (L.next())
      if (L.line.find("<DataArray") != std::string::npos && L.line.find(key) != std::string::npos) return true;
    return false;
  };
  auto values = [&](int nc, int first) {
    for (int64_t c = 0; c < n_elems; ++c) {
      if (!L.next()) return false;
      auto t = tokens(L.line);
      if ((int)t.size() < nc) return false;
      for (int k = 0; k < nc; ++k) sol[5 * c + first + k] = std::stod(t[k]);
    }
    return true;
  };
  try {  // ns_io_module.F90:1355-1381: density, momentum, then energy per unit mass times density
    if (!find("Density") || !values(1, 0) || !find("Momentum") || !values(3, 1) || !find("Energy") ||
        !values(1, 4)) {
      set_error("subfv_restart_from_vtu: Density, Momentum or Energy missing or short");
      return -2;
    }
  } catch (const std::exception&) {
    set_error("subfv_restart_from_vtu: malformed value");
    return -2;
  }
  for (int64_t c = 0; c < n_elems; ++c) sol[5 * c + 4] = sol[5 * c + 4] * sol[5 * c];
  return 0;
}

}  // extern "C"
