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
    # k_lag_face: face L/R, face normal record, the cell records (each once), face record write
    b["face"] = 8 * nf + 32 * nf + 64 * ne + 48 * nf
    # k_lag_node: node CSR offsets, subface->face, face normal, subface area, face record, vp write
    b["node"] = 4 * (nv + 1) + 4 * nsf + 32 * nf + 8 * nsf + 48 * nf + 32 * nv
    # k_lag_cell: cell CSR, subface->face/vertex, face normal, subface area, face record, vp,
    # subface->subcells, subcell volumes, cell records, rhs write
    b["cell"] = (4 * (ne + 1) + 4 * ncsf + 8 * nsf + 32 * nf + 8 * nsf + 48 * nf + 32 * nv
                 + 8 * nsf + 8 * nse + 64 * ne + 48 * ne)
    b["finalize"] = 64
    b["move"] = 32 * nv * 3  # x read+write, vp read
    # k_geom<0>: cell vertex lists, vertex records, cell faces, face vertex ids, L/R, face
    # subface ids, subcell subface ids, subface->face/vertex; writes: face normal records,
    # subface areas, subcell and cell volumes; update: cell records read+write, rhs read
    b["geom"] = (4 * (ne + 1) + 4 * nse + 32 * nv + 32 * ne + 16 * nf + 8 * nf + 16 * nf + 16 * nse
                 + 8 * nsf + 32 * nf + 8 * nsf + 8 * nse + 8 * ne + 64 * ne * 2 + 48 * ne)
    return b


def step_bytes(s: MeshSizes) -> int:
    return sum(lag_kernel_bytes(s).values())
