"""Host-side initial states of init_sol (src/ns/ns_euler_module.F90:12-140): the potential
flows agree with the oracle's boundary-state restatement of the same exact solutions, the
isentropic vortex is isentropic (p = rho^gamma) and swirls about the origin, and the
piecewise states fall on the reference's sides."""
import ctypes as C

import numpy as np
import pytest


def _centroids(n=200, seed=0, lo=-3.0, hi=3.0):
    rng = np.random.default_rng(seed)
    x = rng.uniform(lo, hi, (n, 3))
    r = np.linalg.norm(x[:, :2], axis=1)
    return x[r > 0.6]


@pytest.mark.parametrize("three_d", [False, True])
def test_potential_flow_matches_oracle(oracle_lib, three_d):
    from subfv_b200.ns_init import init_potential_flow, primit_to_conserv
    x = _centroids()
    if three_d:
        x = x[np.linalg.norm(x, axis=1) > 0.6]
    sol = init_potential_flow(x, three_d)
    pd = C.POINTER(C.c_double)
    for i in range(len(x)):
        xi = np.ascontiguousarray(x[i])
        w = np.zeros(5)
        oracle_lib.or_potential_flow(xi.ctypes.data_as(pd), int(three_d), w.ctypes.data_as(pd))
        np.testing.assert_allclose(sol[i], primit_to_conserv(w)[0], rtol=1e-13, atol=1e-18)


def test_isentropic_vortex():
    from subfv_b200.ns_init import GAMMA, init_isentropic_vortex
    x = _centroids(seed=1)
    u = init_isentropic_vortex(x)
    rho = u[:, 0]
    vel = u[:, 1:4] / rho[:, None]
    p = (GAMMA - 1) * (u[:, 4] - 0.5 * rho * (vel ** 2).sum(1))
    np.testing.assert_allclose(p, rho ** GAMMA, rtol=1e-12)
    np.testing.assert_allclose((vel[:, :2] * x[:, :2]).sum(1), 0.0, atol=1e-14)  # purely azimuthal
    assert np.all(rho < 1.0)


def test_piecewise_states():
    from subfv_b200.ns_init import init_double_mach, init_kelvin_helmholtz, init_riemann_1d, init_uniform
    x = _centroids(seed=2, lo=-0.5, hi=1.0)
    s = init_riemann_1d(x, 0.3, [1, 0, 0, 0, 1], [0.125, 0, 0, 0, 0.1])
    assert np.all((s[:, 0] == 1.0) == (x[:, 0] < 0.3))
    dm, tmax = init_double_mach(x)
    assert tmax == 0.2 and np.all((dm[:, 0] == 1.4) == (x[:, 1] < 1.732 * (x[:, 0] - 0.1667)))
    kh, tk = init_kelvin_helmholtz(x)
    assert tk == pytest.approx(80.0) and np.all(np.abs(kh[:, 0] - 1.4) <= 1e-2 + 1e-15)
    u = init_uniform(4, [1.0, 0.1, 0.2, 0.3, 2.0])
    assert u.shape == (4, 5) and np.all(u == u[0])


def test_sedov_energy_in_the_central_cell():
    from subfv_b200.ns_init import init_sedov
    x = np.array([[0.3, 0.1, 0.0], [0.05, -0.02, 0.4], [-0.05, 0.02, 0.0], [1.0, 1.0, 1.0]])
    vol = np.array([0.1, 0.2, 0.3, 0.4])
    s = init_sedov(x, vol, boundary_2d=True)
    assert s[1, 4] == pytest.approx(0.984042 / 0.2)  # first of the two cells at the smallest radius
    assert np.all(s[[0, 2, 3], 4] == 1e-16 / (1.4 - 1.0)) and np.all(s[:, 0] == 1.0)
    s3 = init_sedov(x, vol, boundary_2d=False)
    assert s3[2, 4] == pytest.approx(0.851072 / 0.3)
