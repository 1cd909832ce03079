"""Host mirror of the reference's sparse_bcsr_linear_module
(src/linear_algebra/sparse_bcsr_linear_module.F90): bcsr_matrix_type, bcsr_matmul,
bcsr_diag, bcsr_gmres_diag, bcsr_gmres, bcsr_parallel_lusgs, bcsr_gmres_parallel_lusgs;
all compute on the GPU through the C-ABI.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import check, f64, i32, pd, pi


@dataclass
class BcsrMatrix:
    """bcsr_matrix_type (:6-11): m block rows, blc_size, row(m+1)/col(nnz) 1-based,
    v(blc_size, blc_size, nnz) column-major blocks (numpy (nnz, bs, bs) with v[j].T the
    Fortran block)."""

    m: int
    blc_size: int
    row: np.ndarray
    col: np.ndarray
    v: np.ndarray  # (nnz, bs, bs): v[j, c, r] = Fortran v(r+1, c+1, j+1)

    @property
    def nnz(self):
        return int(self.col.size)

    def flat_values(self) -> np.ndarray:
        return np.ascontiguousarray(self.v.reshape(-1), np.float64)


class DeviceBcsr:
    """A BCSR matrix resident on the GPU."""

    def __init__(self, A: BcsrMatrix):
        self.A = A
        self.n = A.m * A.blc_size
        self._row, self._col = i32(A.row), i32(A.col)
        v = A.flat_values()
        h = C.c_void_p()
        check(_lib.load().subfv_bcsr_create(A.m, A.blc_size, pi(self._row), pi(self._col), pd(v), C.byref(h)),
              "subfv_bcsr_create")
        self._h = h

    def set_values(self, v):
        v = f64(np.asarray(v).reshape(-1))
        check(_lib.load().subfv_bcsr_set_values(self._h, pd(v)), "subfv_bcsr_set_values")

    def matmul(self, x) -> np.ndarray:
        x = f64(x)
        y = np.empty(self.n)
        check(_lib.load().subfv_bcsr_matmul(self._h, pd(x), pd(y)), "subfv_bcsr_matmul")
        return y

    def diag(self, b) -> np.ndarray:
        b = f64(b)
        x = np.empty(self.n)
        check(_lib.load().subfv_bcsr_diag(self._h, pd(x), pd(b)), "subfv_bcsr_diag")
        return x

    def set_colors(self, n_color_sets: int, color):
        """Colour (1..n_color_sets) of each block row for the parallel LU-SGS."""
        self._color = i32(color)
        check(_lib.load().subfv_bcsr_set_colors(self._h, int(n_color_sets), pi(self._color)), "subfv_bcsr_set_colors")

    def parallel_lusgs(self, b) -> np.ndarray:
        """bcsr_parallel_lusgs (:1438-1502): x = (U+D)^-1 D (L+D)^-1 b by colour sets."""
        b = f64(b)
        x = np.empty(self.n)
        check(_lib.load().subfv_bcsr_parallel_lusgs(self._h, pd(x), pd(b)), "subfv_bcsr_parallel_lusgs")
        return x

    def gmres_lusgs(self, b, tol, m=30):
        """bcsr_gmres_parallel_lusgs (:885-993); returns (x, conv, restarts, rho)."""
        b = f64(b)
        x = np.empty(self.n)
        conv, it, rho = C.c_int(), C.c_int(), C.c_double()
        check(_lib.load().subfv_bcsr_gmres_ex(self._h, pd(x), pd(b), float(tol), int(m), 2, C.byref(conv),
                                              C.byref(it), C.byref(rho), None), "subfv_bcsr_gmres_parallel_lusgs")
        return x, bool(conv.value), it.value, rho.value

    def pcgm(self, b, tol, x0=None):
        """bcsr_pcgm (:1110-1169) from x0 (zeros if None); returns (x, iterations, status
        bits, sqrt(r.M^-1 r)). Status SUBFV_ERR_GMRES: not converged (the reference stops)."""
        b = f64(b)
        x = np.zeros(self.n) if x0 is None else np.array(x0, np.float64)
        it, res = C.c_int(), C.c_double()
        st = _lib.load().subfv_bcsr_pcgm(self._h, pd(x), pd(b), float(tol), C.byref(it), C.byref(res))
        if st < 0:
            check(st, "subfv_bcsr_pcgm")
        return x, it.value, st, res.value

    def gmres(self, b, tol, m=30, precond=True, want_h=False):
        """bcsr_gmres_diag (precond) / bcsr_gmres; returns (x, conv, restarts, rho[, H_first])."""
        b = f64(b)
        x = np.empty(self.n)
        conv, it, rho = C.c_int(), C.c_int(), C.c_double()
        H = np.zeros((m, m + 1)) if want_h else None  # Fortran H(m+1, m) column-major
        check(_lib.load().subfv_bcsr_gmres_ex(self._h, pd(x), pd(b), float(tol), int(m), int(precond),
                                              C.byref(conv), C.byref(it), C.byref(rho),
                                              pd(H) if want_h else None), "subfv_bcsr_gmres")
        out = (x, bool(conv.value), it.value, rho.value)
        return out + (H,) if want_h else out

    def gmres_refine(self, b, rel_tol=1e-8, m=30):
        """FP64 iterative refinement around FP32-matrix block-Jacobi GMRES(m)."""
        b = f64(b)
        x = np.empty(self.n)
        conv, outer, rho = C.c_int(), C.c_int(), C.c_double()
        check(_lib.load().subfv_bcsr_gmres_refine(self._h, pd(x), pd(b), float(rel_tol), int(m), C.byref(conv),
                                                  C.byref(outer), C.byref(rho)), "subfv_bcsr_gmres_refine")
        return x, bool(conv.value), outer.value, rho.value

    def profile_spmv(self, n_iter=20, fp32=False) -> float:
        ms = C.c_double()
        check(_lib.load().subfv_bcsr_profile_spmv(self._h, int(n_iter), int(fp32), C.byref(ms)), "profile_spmv")
        return ms.value

    def close(self):
        if getattr(self, "_h", None):
            _lib.load().subfv_bcsr_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def bcsr_matmul(A: DeviceBcsr, x):
    """y = bcsr_matmul(A, x) (:13-29)."""
    return A.matmul(x)


def bcsr_gmres_diag(A: DeviceBcsr, b, tol, m):
    """bcsr_gmres_diag(A, x, b, tol, m, conv, ...) (:1592-1691); returns (x, conv)."""
    x, conv, _, _ = A.gmres(b, tol, m, precond=True)
    return x, conv


def grid_matrix(nx, ny, nz, bs=5, stencil=27, seed=0, diag_shift=None, periodic=False):
    """A seeded BCSR matrix on an nx*ny*nz grid of block rows with the 7- or 27-point
    neighbour pattern, block-diagonally dominant so block-Jacobi GMRES converges."""
    rng = np.random.default_rng(seed)
    m = nx * ny * nz
    offs = [(i, j, k) for k in (-1, 0, 1) for j in (-1, 0, 1) for i in (-1, 0, 1)
            if stencil == 27 or abs(i) + abs(j) + abs(k) <= 1]
    rows = [[] for _ in range(m)]
    for kk in range(nz):
        for jj in range(ny):
            for ii in range(nx):
                r = (kk * ny + jj) * nx + ii
                for (di, dj, dk) in offs:
                    a, b_, c = ii + di, jj + dj, kk + dk
                    if periodic:
                        a, b_, c = a % nx, b_ % ny, c % nz
                    elif not (0 <= a < nx and 0 <= b_ < ny and 0 <= c < nz):
                        continue
                    rows[r].append((c * ny + b_) * nx + a)
    row = np.zeros(m + 1, np.int32)
    cols = []
    for r in range(m):
        cs = sorted(set(rows[r]))
        cols.extend(cs)
        row[r + 1] = row[r] + len(cs)
    col = np.array(cols, np.int32)
    nnz = col.size
    v = rng.uniform(-1.0, 1.0, (nnz, bs, bs)) / len(offs)
    shift = diag_shift if diag_shift is not None else 2.0
    rr = np.repeat(np.arange(m), np.diff(row))
    dmask = col == rr
    v[dmask] += shift * np.eye(bs)[None]
    return BcsrMatrix(m, bs, row + 1, col + 1, v)


def greedy_colors(A: BcsrMatrix) -> tuple[int, np.ndarray]:
    """A colouring of the block rows for the parallel LU-SGS (the reference takes it from
    its caller): rows in order, each the smallest colour (1-based) not used by a coupled
    row of lower index. Returns (n_color_sets, color)."""
    row, col = np.asarray(A.row) - 1, np.asarray(A.col) - 1
    color = np.zeros(A.m, np.int32)
    for i in range(A.m):
        used = {int(color[c]) for c in col[row[i]:row[i + 1]] if c < i}
        k = 1
        while k in used:
            k += 1
        color[i] = k
    return int(color.max()), color
