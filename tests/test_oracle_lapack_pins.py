"""Pins for the oracle's LAPACK stand-ins against scipy's LAPACK (the reference calls
dgesvd for pseudo_inverse_inplace_lapack and dgetrf/dgetrs for lu_solve_inplace_lapack,
src/linear_algebra/linear_solver_module.F90:643-715)."""
import ctypes as C

import numpy as np
import scipy.linalg as sla
from scipy.linalg import lapack

P = C.POINTER(C.c_double)


def test_pinv3_matches_dgesvd_pinv(oracle_lib):
    rng = np.random.default_rng(0)
    for i in range(1000):
        a = rng.normal(size=(3, 3)) * 10 ** rng.uniform(-3, 3)
        if i % 3 == 0:
            a[:, 2] = 0.5 * a[:, 0] + a[:, 1]  # rank 2, as at slab vertices
        u, s, vt, info = lapack.dgesvd(a)
        assert info == 0
        tol = 3 * 1e-12 * s.max()
        sp = np.where(s > tol, 1.0 / s, 0.0)
        ref = vt.T @ (np.diag(sp) @ u.T)
        a9 = a.reshape(-1).copy()
        oracle_lib.or_pinv3(a9.ctypes.data_as(P))
        assert np.abs(a9.reshape(3, 3) - ref).max() <= 1e-9 * np.abs(ref).max(), i


def test_lu3_matches_dgetrf_dgetrs(oracle_lib):
    rng = np.random.default_rng(1)
    for i in range(1000):
        a = rng.normal(size=(3, 3))
        if i % 2:
            a = a @ a.T + 0.1 * np.eye(3)
        b = rng.normal(size=3)
        lu, piv, info = lapack.dgetrf(a)
        ref, info2 = lapack.dgetrs(lu, piv, b)
        x = np.zeros(3)
        m9 = a.reshape(-1).copy()
        oracle_lib.or_lu3(m9.ctypes.data_as(P), x.ctypes.data_as(P), b.ctypes.data_as(P))
        np.testing.assert_allclose(x, ref, rtol=1e-12, atol=1e-14 * np.abs(ref).max())
        np.testing.assert_allclose(x, sla.solve(a, b), rtol=1e-10)


def test_inverse_matches_dgetrf_dgetri(oracle_lib):
    """inv_lapack (linear_solver_module.F90:629-641) restated for the diffusion systems:
    against scipy's dgetrf + dgetri at the sizes a vertex produces (3 nsfn up to 48)."""
    rng = np.random.default_rng(2)
    for i, n in enumerate([1, 2, 5, 8, 12, 24, 36, 48] * 25):
        a = rng.normal(size=(n, n))
        if i % 2:
            a = a @ a.T + 0.05 * n * np.eye(n)  # SPD, like the nodal diffusion matrices
        lu, piv, info = lapack.dgetrf(a)
        ref, info2 = lapack.dgetri(lu, piv)
        assert info == info2 == 0
        m = np.asfortranarray(a).reshape(-1, order="F").copy()
        oracle_lib.or_lapack_inverse(n, m.ctypes.data_as(P))
        got = m.reshape(n, n, order="F")
        assert np.abs(got - ref).max() <= 1e-10 * np.abs(ref).max(), (i, n)


def test_solve5_matches_dgesv(oracle_lib):
    """The 5x5 pivoting solve of add_timedisc_and_solve (dgetrf + dgetrs) against dgesv."""
    rng = np.random.default_rng(3)
    for i in range(1000):
        a = rng.normal(size=(5, 5)) + (3.0 * np.eye(5) if i % 2 else 0.0)
        b = rng.normal(size=5)
        lu, piv, x_ref, info = lapack.dgesv(a, b)
        assert info == 0
        m = a.reshape(-1, order="F").copy()
        x = b.copy()
        oracle_lib.or_lapack_solve(5, m.ctypes.data_as(P), x.ctypes.data_as(P))
        assert np.abs(x - x_ref).max() <= 1e-11 * max(1.0, np.abs(x_ref).max()), i
