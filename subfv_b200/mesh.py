"""Host mirror of the reference's mesh pipeline: build_mesh (topology, on the host in
C++) and compute_geometry_mesh (on the GPU).

Reference: src/mesh/mesh_connectivity_module.F90:12-59 (build_mesh),
src/mesh/mesh_geometry_module.F90:16-57 (compute_geometry_mesh).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check, f64, i32, pd, pi
from .meshgen import RawMesh

SUBFV_ERR_MESH_CHECK = 1
SUBFV_ERR_NONFINITE = 2
SUBFV_ERR_NEG_DENSITY = 4
SUBFV_ERR_BAD_OMEGA = 8
SUBFV_ERR_GMRES = 16


RENUMBER = {"bfs": 0, "hilbert": 1}


class Topology:
    """build_mesh output, arrays fetched by mesh_type name. renumber "bfs" is the
    reference's numbering; "hilbert" orders the vertices along a Hilbert curve (cells,
    faces and subfaces then follow the reference's rules over that order)."""

    def __init__(self, raw: RawMesh, renumber: str = "bfs"):
        lib = _lib.load()
        if renumber not in RENUMBER:
            raise ValueError(f"renumber must be one of {sorted(RENUMBER)}")
        self.renumber = renumber
        self.raw = raw
        h = C.c_void_p()
        coords = f64(raw.coords.reshape(-1))
        kind, off, ev = i32(raw.elem_kind), i32(raw.elem_vert_off), i32(raw.elem_vert)
        bo, bv, bt = i32(raw.bface_off), i32(raw.bface_vert), i32(raw.bface_tag)
        nbf = int(bo.size - 1)
        check(lib.subfv_topology_build_ex(raw.n_vert, pd(coords), raw.n_elems, pi(kind), pi(off), pi(ev), nbf,
                                          pi(bo), pi(bv), pi(bt), int(raw.b2d), int(raw.periodic),
                                          RENUMBER[renumber], C.byref(h)),
              "subfv_topology_build_ex")
        self._h = h
        s = self.array("sizes")
        self.n_vert, self.n_elems, self.n_faces, self.n_sub_faces, self.n_sub_elems, self.n_max_sub_faces_around_node = map(int, s)

    def array(self, name: str) -> np.ndarray:
        lib = _lib.load()
        n = lib.subfv_topology_array_len(self._h, name.encode())
        if n < 0:
            raise KeyError(name)
        out = np.empty(int(n), np.int32)
        check(lib.subfv_topology_array_get(self._h, name.encode(), pi(out)), "subfv_topology_array_get")
        return out

    def coords(self) -> np.ndarray:
        out = np.empty(3 * self.n_vert, np.float64)
        check(_lib.load().subfv_topology_coords(self._h, pd(out)), "subfv_topology_coords")
        return out.reshape(-1, 3)

    def close(self):
        if getattr(self, "_h", None):
            _lib.load().subfv_topology_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Mesh:
    """A device-resident mesh (topology + geometry) on the current CUDA device."""

    def __init__(self, topo: Topology, b2d: bool = True, geometry: bool = True):
        lib = _lib.load()
        self.topo = topo
        self.b2d = bool(b2d)
        h = C.c_void_p()
        check(lib.subfv_mesh_create_from_topology(topo._h, int(b2d), C.byref(h)), "subfv_mesh_create")
        self._h = h
        self.n_vert, self.n_elems = topo.n_vert, topo.n_elems
        self.n_faces, self.n_sub_faces, self.n_sub_elems = topo.n_faces, topo.n_sub_faces, topo.n_sub_elems
        self.geometry_status = self.compute_geometry_mesh() if geometry else 0

    @classmethod
    def from_raw(cls, raw: RawMesh, geometry: bool = True, renumber: str = "bfs") -> "Mesh":
        return cls(Topology(raw, renumber), b2d=raw.b2d, geometry=geometry)

    def compute_geometry_mesh(self) -> int:
        """Returns SUBFV_ERR_MESH_CHECK where the reference error-stops on check_mesh."""
        return check(_lib.load().subfv_compute_geometry_mesh(self._h), "subfv_compute_geometry_mesh")

    _SHAPES = {"face_coord": ("n_faces", 3), "face_norm": ("n_faces", 3), "face_area": ("n_faces", 0),
               "sub_face_norm": ("n_sub_faces", 3), "sub_face_area": ("n_sub_faces", 0),
               "elem_coord": ("n_elems", 3), "elem_volume": ("n_elems", 0),
               "sub_elem_volume": ("n_sub_elems", 0), "vert_volume": ("n_vert", 0), "vert_is_bound": ("n_vert", 0)}

    def geometry(self, name: str) -> np.ndarray:
        cnt, comp = self._SHAPES[name]
        n = getattr(self, cnt)
        out = np.empty(n * max(comp, 1), np.float64)
        check(_lib.load().subfv_mesh_get_geometry(self._h, name.encode(), pd(out)), "subfv_mesh_get_geometry")
        return out.reshape(n, comp) if comp else out

    def coords(self) -> np.ndarray:
        out = np.empty(3 * self.n_vert, np.float64)
        check(_lib.load().subfv_mesh_get_coords(self._h, pd(out)), "subfv_mesh_get_coords")
        return out.reshape(-1, 3)

    def set_coords(self, c: np.ndarray):
        c = f64(np.asarray(c).reshape(-1))
        check(_lib.load().subfv_mesh_set_coords(self._h, pd(c)), "subfv_mesh_set_coords")

    @property
    def device_bytes(self) -> int:
        return int(_lib.load().subfv_mesh_device_bytes(self._h))

    def close(self):
        if getattr(self, "_h", None):
            _lib.load().subfv_mesh_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
