"""Pins for the oracle's small dense pieces (the reference calls LAPACK or its own
helpers here): checked against numpy/scipy LAPACK on random cases."""
import ctypes as C

import numpy as np
import pytest


def _pd(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def test_inverse_3_by_3_matches_lapack(oracle_lib):
    rng = np.random.default_rng(0)
    for _ in range(200):
        a = rng.normal(size=(3, 3))
        m = a @ a.T + 0.1 * np.eye(3)  # the nodal matrices are SPD
        m = np.ascontiguousarray(m)
        inv = np.zeros(9)
        oracle_lib.or_inverse_3_by_3(_pd(m.reshape(-1)), _pd(inv))
        ref = np.linalg.inv(m)
        np.testing.assert_allclose(inv.reshape(3, 3), ref, rtol=1e-11, atol=1e-12 * np.abs(ref).max())


def test_fnorm2_is_the_scaled_norm(oracle_lib):
    rng = np.random.default_rng(1)
    for scale in (1e-300, 1e-8, 1.0, 1e8, 1e300):
        a = np.ascontiguousarray(rng.normal(size=3) * scale)
        got = oracle_lib.or_fnorm2(_pd(a), 3)
        ref = scale * np.linalg.norm(a / scale)  # unscaled numpy would overflow at 1e300
        assert got == pytest.approx(ref, rel=4e-16 * 4)
    z = np.zeros(3)
    assert oracle_lib.or_fnorm2(_pd(z), 3) == 0.0
