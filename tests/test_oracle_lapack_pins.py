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
