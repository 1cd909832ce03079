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
    # k_face_geom<0>: vertex records, face vertex and subface ids, the subfaces' vertex
    # slots; writes: face centroids, normal records and subface sums, subface areas
    b["face_geom"] = 32 * nv + 16 * nf + 16 * nf + nf + 32 * nf + 32 * nf + 32 * nf + 8 * nsf
    # k_geom_step: cell vertex lists, vertex records, cell faces and their static codes,
    # the face centroids, normal records and subface sums, the subcells' codes; writes:
    # subcell and cell volumes; update: cell records read + write, rhs read
    b["cell_geom"] = (4 * (ne + 1) + 4 * nse + 32 * nv + 32 * ne + 16 * ne + 96 * nf + 4 * nse
                      + 8 * nse + 8 * ne + 64 * ne * 2 + 48 * ne)
    return b


def step_bytes(s: MeshSizes) -> int:
    return sum(lag_kernel_bytes(s).values())


def algorithmic_bytes(path: str, *, ne: int = 0, nv: int = 0, nsf: int = 0, nse: int = 0, stages: int = 1,
                      m: int = 0, bs: int = 5, nnzb: int = 0, w: int = 8, krylov: int = 30,
                      precond: str = "diag", sizes: MeshSizes | None = None) -> int:
    """Compulsory HBM bytes of one unit of work on a path (each array touched once):

    - "lagrange_step": one Lagrangian step, the sum of lag_kernel_bytes(sizes);
    - "ns_stage": one explicit Euler stage, state read and write (2 x 40 B), volume (8),
      subface normal + area (32) and left/right cell ids (8), node CSR offsets (4) and
      the corner -> cell map (4): 80 C + 8 C + 32 SF + 8 SF + 4 (V + 1) + 4 SE;
    - "ns_update": `stages` stages plus the re-read of U^n (40 C) in the two-stage scheme;
    - "spmv": nnzb (bs^2 w + 4) + (m + 1) 4 + 2 m bs 8 (values of w bytes);
    - "gmres_cycle": one restart cycle of GMRES(krylov): krylov SpMVs and preconditioner
      applications (block Jacobi: the packed LU, bs^2 8 per row, and two vectors), the
      modified Gram-Schmidt projections (column j: j projections of 3 vectors, fused
      axpy + next dot) and the normalisations (2 vectors).
    """
    if path == "lagrange_step":
        return step_bytes(sizes)
    if path == "ns_stage":
        return 80 * ne + 8 * ne + 32 * nsf + 8 * nsf + 4 * (nv + 1) + 4 * nse
    if path == "ns_update":
        b = stages * algorithmic_bytes("ns_stage", ne=ne, nv=nv, nsf=nsf, nse=nse)
        return b + (40 * ne if stages == 2 else 0)
    if path == "spmv":
        return nnzb * (bs * bs * w + 4) + (m + 1) * 4 + 2 * m * bs * 8
    if path == "gmres_cycle":
        n = m * bs
        vec = 8 * n
        pc = (bs * bs * 8 * m + 2 * vec) if precond == "diag" else 0
        spmv = algorithmic_bytes("spmv", m=m, bs=bs, nnzb=nnzb, w=w)
        mgs = sum(3 * j * vec + 2 * vec for j in range(1, krylov + 1))
        return krylov * (spmv + pc) + mgs
    raise ValueError(f"unknown path {path}")
