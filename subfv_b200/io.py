"""Mesh and solution files: gmsh MSH 2 / 4 (ASCII) in, VTU solutions out and back in
(read_mesh_msh, mesh_reading_module.F90:154-1324; write_sol_vtu and
restart_from_vtu_file, ns_io_module.F90:403-884, 1333-1382), through the host code of
the native library."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check, f64, pd
from .meshgen import RawMesh


def read_msh(path: str, bc_names=(), b2d: bool = True, periodic: bool = False) -> RawMesh:
    """The mesh of an MSH file; boundary faces carry the 1-based index of the bc_names
    entry that names their physical group (0: none), the reference's boundary tags."""
    lib = _lib.load()
    names = (C.c_char_p * max(1, len(bc_names)))(*[n.encode() for n in bc_names])
    h = C.c_void_p()
    check(lib.subfv_msh_read(str(path).encode(), len(bc_names), names, C.byref(h)), "subfv_msh_read")
    try:
        s = (C.c_int64 * 5)()
        check(lib.subfv_msh_sizes(h, s), "subfv_msh_sizes")
        nv, ne, nev, nbf, nbv = (int(x) for x in s)
        coords = np.empty((nv, 3))
        kind = np.empty(ne, np.int32)
        off = np.empty(ne + 1, np.int32)
        ev = np.empty(nev, np.int32)
        boff = np.empty(nbf + 1, np.int32)
        bv = np.empty(nbv, np.int32)
        bt = np.empty(nbf, np.int32)
        pi = lambda a: a.ctypes.data_as(C.POINTER(C.c_int32))
        check(lib.subfv_msh_get(h, pd(coords), pi(kind), pi(off), pi(ev), pi(boff), pi(bv), pi(bt)), "subfv_msh_get")
    finally:
        lib.subfv_msh_destroy(h)
    return RawMesh(coords, kind, off, ev, boff, bv, bt, b2d=b2d, periodic=periodic)


def write_sol_vtu(path: str, topology, sol, delta=None, vp=None, elem_coord=None, Cv_p: float = 720.19471,
                  mu: float = -1.0) -> None:
    """The reference's solution file for cell states sol (n, 5); topology is the mesh's
    subfv_b200.mesh.Topology."""
    arrs = [None if a is None else f64(a) for a in (sol, delta, vp, elem_coord)]
    ptr = [None if a is None else pd(a) for a in arrs]
    check(_lib.load().subfv_write_sol_vtu(str(path).encode(), topology._h, *ptr, float(Cv_p), float(mu)),
          "subfv_write_sol_vtu")


def write_sol_vtu_lag(path: str, topology, sol, vp, pp=None, elem_coord=None) -> None:
    """The Lagrangian solver's solution file for states sol (n, 5) = (tau, u, v, w, E),
    nodal velocities vp (n_vert, 3) and optional nodal pressures pp."""
    arrs = [None if a is None else f64(a) for a in (sol, vp, pp, elem_coord)]
    ptr = [None if a is None else pd(a) for a in arrs]
    check(_lib.load().subfv_write_sol_vtu_lag(str(path).encode(), topology._h, *ptr), "subfv_write_sol_vtu_lag")


def restart_from_vtu(path: str, n_elems: int) -> np.ndarray:
    """Cell states (n_elems, 5) from a solution VTU (Density, Momentum, Energy per unit mass)."""
    sol = np.empty((n_elems, 5))
    check(_lib.load().subfv_restart_from_vtu(str(path).encode(), int(n_elems), pd(sol)), "subfv_restart_from_vtu")
    return sol
