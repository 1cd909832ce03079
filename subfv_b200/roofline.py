"""Algorithmic (compulsory) bytes of the Lagrangian step kernels.

Each term is one array the kernel must read or write once, at its device record
size, for the mesh it runs on; re-reads through L2 or L1 are not counted. Units: bytes
per launch (one launch processes the whole mesh once). The per-cell figure is the sum
divided by the number of cells.
"""
from __future__ import annotations

from dataclasses import dataclass


@dataclass
class MeshSizes:
    nv: int
    ne: int
    nf: int
    nsf: int
    nse: int
    ncsf: int  # cell -> subface gather entries (2 per interior subface, 1 per boundary)


def lag_kernel_bytes(s: MeshSizes) -> dict:
    nv, ne, nf, nsf, nse, ncsf = s.nv, s.ne, s.nf, s.nsf, s.nse, s.ncsf
    b = {}
    # k_lag_node: node CSR offsets, subface->face, face L/R, face normal record,
    # subface record (area), cell state records, vp write, vertex volume (vse list, vol_se, write)
    b["node"] = (4 * (nv + 1) + 4 * nsf + 8 * nf + 32 * nf + 32 * nsf + 48 * ne + 32 * nv
                 + 4 * (nv + 1) + 4 * nse + 8 * nse + 8 * nv)
    # k_lag_cell: cell CSR, subface->face/vertex, face L/R and normal, subface area,
    # subcell ids, subcell volumes, vp, cell states, rhs write
    b["cell"] = (4 * (ne + 1) + 4 * ncsf + 8 * nsf + 8 * nf + 32 * nf + 32 * nsf + 8 * nsf
                 + 8 * nse + 32 * nv + 48 * ne + 48 * ne)
    b["finalize"] = 64
    b["move"] = 32 * nv * 3  # x read+write, vp read
    # k_face_geometry: face vertex ids, vertex records, face subface ids, subface vertex,
    # writes: face centroid, face normal, subface records
    b["face_geom"] = 16 * nf + 32 * nv + 16 * nf + 4 * nsf + 32 * nf + 32 * nf + 32 * nsf
    # k_cell_geometry: cell vertex ids + offsets, cell faces, vertex records, face records
    # (vertex ids, L/R, centroid, normal, subface ids), subcell subfaces, subface face/vertex,
    # subface records, writes: centroid, volume, subcell volumes; update: sol and rhs read, sol write
    b["cell_geom"] = (4 * (ne + 1) + 4 * nse + 32 * ne + 32 * nv + 16 * nf + 8 * nf + 32 * nf + 32 * nf
                      + 16 * nf + 16 * nse + 8 * nsf + 32 * nsf + 32 * ne + 8 * ne + 8 * nse
                      + 48 * ne * 3)
    return b


def step_bytes(s: MeshSizes) -> int:
    return sum(lag_kernel_bytes(s).values())
