"""CPU checks of the oracle's three_wave and modified_three_wave restatements
(ns_euler_rs_module.F90:9-152): consistency (equal states give the physical flux
F(U).n), conservation (lr(:,2) = -lr(:,1)), the modified form equal to the plain one
when the tangential velocities agree, and both equal to two_wave's bounds (sl, sr)."""
import ctypes as C

import numpy as np
import pytest

G = 1.4


def _flux(lib, scheme, wl, wr, n):
    pd = C.POINTER(C.c_double)
    wl, wr, n = (np.ascontiguousarray(a, dtype=np.float64) for a in (wl, wr, n))
    lr, s = np.zeros(10), np.zeros(2)
    lib.or_ns_flux(scheme, wl.ctypes.data_as(pd), wr.ctypes.data_as(pd), n.ctypes.data_as(pd),
                   lr.ctypes.data_as(pd), s.ctypes.data_as(pd))
    return lr[:5], lr[5:], s


def _phys(w, n):
    rho, u, p = w[0], w[1:4], w[4]
    vn = u @ n
    E = p / (G - 1) + 0.5 * rho * u @ u
    return np.array([rho * vn, *(rho * vn * u + p * n), (E + p) * vn])


def _states(rng):
    n = rng.normal(size=3)
    n /= np.linalg.norm(n)
    wl = np.array([rng.uniform(0.2, 5), *rng.uniform(-1, 1, 3), rng.uniform(0.1, 10)])
    wr = np.array([rng.uniform(0.2, 5), *rng.uniform(-1, 1, 3), rng.uniform(0.1, 10)])
    return wl, wr, n


@pytest.mark.parametrize("scheme", [3, 5])
def test_consistency_and_conservation(oracle_lib, scheme):
    rng = np.random.default_rng(3)
    for _ in range(50):
        wl, wr, n = _states(rng)
        f0, f1, _ = _flux(oracle_lib, scheme, wl, wl, n)
        np.testing.assert_allclose(f0, _phys(wl, n), rtol=1e-12, atol=1e-12)
        f0, f1, _ = _flux(oracle_lib, scheme, wl, wr, n)
        np.testing.assert_array_equal(f1, -f0)
        assert np.all(np.isfinite(f0))


def test_modified_equals_plain_without_tangential_jump(oracle_lib):
    rng = np.random.default_rng(4)
    for _ in range(50):
        wl, wr, n = _states(rng)
        vt = wl[1:4] - (wl[1:4] @ n) * n
        wr[1:4] = vt + (wr[1:4] @ n) * n  # same tangential velocity on both sides
        f3, _, s3 = _flux(oracle_lib, 3, wl, wr, n)
        f5, _, s5 = _flux(oracle_lib, 5, wl, wr, n)
        np.testing.assert_allclose(f5, f3, rtol=1e-11, atol=1e-11)
        np.testing.assert_array_equal(s3, s5)
        _, _, s2 = _flux(oracle_lib, 4, wl, wr, n)
        np.testing.assert_array_equal(s3, s2)
