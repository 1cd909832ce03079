"""The oracle's boundary states of compute_right_state (src/ns/ns_euler_recon_module.F90:
331-409) that have no golden vectors: the potential flows of ns_euler_exact_sol_module.F90:
105-170 are checked against their closed-form properties (no penetration on the body of
radius 0.5, the uniform stream's radial velocity on the outer circle of radius 5.5 in 2-D,
Bernoulli's pressure), and the time-dependent double-Mach boundary and the other kinds
through the oracle's time loop on a slab with tagged sides."""
import ctypes as C

import numpy as np
import pytest

R0, R1, RHOINF, PINF, G = 0.5, 5.5, 1.4, 1.0, 1.4


def _pf(x, three_d):
    from oracle.oracle import load
    x = np.ascontiguousarray(x, np.float64)
    w = np.zeros(5)
    pd = C.POINTER(C.c_double)
    load().or_potential_flow(x.ctypes.data_as(pd), int(three_d), w.ctypes.data_as(pd))
    return w


def _vinf(three_d):
    mach = 1e-4 if three_d else float(np.float32(1e-4))
    return mach * np.sqrt(G * PINF / RHOINF)


@pytest.mark.parametrize("theta", np.linspace(-3.0, 3.0, 7))
def test_potential_flow_2d_boundaries(oracle_lib, theta):
    vinf = _vinf(False)
    for r, vr_expect in ((R0, 0.0), (R1, vinf * np.cos(theta))):
        x = np.array([r * np.cos(theta), r * np.sin(theta), 0.3])
        w = _pf(x, False)
        vr = w[1] * np.cos(theta) + w[2] * np.sin(theta)
        assert vr == pytest.approx(vr_expect, abs=1e-14 * vinf)
        assert w[0] == RHOINF and w[3] == 0.0
        assert w[4] == pytest.approx(PINF + 0.5 * RHOINF * (vinf ** 2 - w[1] ** 2 - w[2] ** 2), rel=1e-15)


def test_potential_flow_2d_mach_is_single_precision(oracle_lib):
    """The 2-D routine's Mach literal has default (single) kind: at theta = 0 on the outer
    circle the velocity is the float nearest 1e-4 times the sound speed, not 1e-4's."""
    w = _pf(np.array([R1, 0.0, 0.0]), False)
    assert w[1] == pytest.approx(_vinf(False), rel=1e-14)
    assert abs(w[1] - _vinf(True)) > 1e-14 * _vinf(True)


def test_potential_flow_3d_no_penetration_and_far_field(oracle_lib):
    rng = np.random.default_rng(7)
    vinf = _vinf(True)
    for _ in range(6):
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        w = _pf(R0 * d, True)
        assert np.dot(w[1:4], d) == pytest.approx(0.0, abs=1e-14 * vinf)
        far = _pf(1e4 * d, True)
        np.testing.assert_allclose(far[1:4], [vinf, 0.0, 0.0], atol=1e-9 * vinf)
        assert w[4] == pytest.approx(PINF + 0.5 * RHOINF * (vinf ** 2 - np.sum(w[1:4] ** 2)), rel=1e-15)


def _tagged_slab():
    from subfv_b200 import meshgen
    raw = meshgen.hex_slab(8, 6, jitter=0.1, seed=3)
    return meshgen.tag_slab_sides(raw, 8, 6, {"xlo": 1, "xhi": 2, "ylo": 3, "yhi": 4})


def _state(m):
    rng = np.random.default_rng(5)
    n = m.n_elems
    w = np.column_stack([rng.uniform(1.3, 1.5, n), rng.uniform(-0.1, 0.1, (n, 2)), np.zeros(n),
                         rng.uniform(0.9, 1.1, n)])
    return np.ascontiguousarray(np.column_stack([w[:, 0], w[:, 1:4] * w[:, :1],
                                                 w[:, 4] / 0.4 + 0.5 * w[:, 0] * (w[:, 1:4] ** 2).sum(1)]))


def _cfg(kinds, vals):
    return dict(scheme=1, second_order=1, method=4, bc_style=2, b2d=1, exclude_bound_vert=0, local_time_step=0,
                cfl=0.3, tmax=1e30, n_bc=len(kinds), bc_type=np.array(kinds, np.int32),
                bc_val=np.array(vals, np.float64))


VALS = [[1.4, 0.2, 0.0, 0.0, 1.0], [1.4, 0.2, 0.0, 0.0, 1.0], [1.0, 0.05, 0.0, 0.0, 1.0], [1.0, 0.0, 0.0, 0.0, 1.0]]


def test_oracle_time_dependent_double_mach(oracle_lib):
    """Kind 6 reads the time of the step: the same state run from two start times differs,
    while a mesh without that kind gives identical results from either start."""
    from oracle.oracle import OracleMesh
    o = OracleMesh(_tagged_slab())
    sol = _state(o)
    out = {}
    for kinds in ((5, 6, 2, 6), (5, 7, 2, 7)):
        for t0 in (0.0, 0.02):
            s = sol.copy()
            st, it, t, _, _, _ = o.ns_run(_cfg(kinds, VALS), s, 3, t0=t0)
            assert st == 0 and it == 4 and np.isfinite(s).all()
            out[kinds, t0] = s
    assert not np.array_equal(out[(5, 6, 2, 6), 0.0], out[(5, 6, 2, 6), 0.02])
    np.testing.assert_array_equal(out[(5, 7, 2, 7), 0.0], out[(5, 7, 2, 7), 0.02])


def test_oracle_adherence_wall_at_rest_matches_slip_wall_mass(oracle_lib):
    """An adherence wall at rest reflects the whole velocity; like the slip wall it lets no
    mass through, so total mass over a closed slab is conserved to round-off."""
    from oracle.oracle import OracleMesh
    o = OracleMesh(_tagged_slab())
    sol = _state(o)
    s = sol.copy()
    zero = [[1.0, 0.0, 0.0, 0.0, 1.0]] * 4
    st, it, _, _, _, _ = o.ns_run(_cfg((2, 2, 2, 2), zero), s, 5)
    assert st == 0
    vol = o.geom("elem_volume")
    m0, m1 = float(np.sum(sol[:, 0] * vol)), float(np.sum(s[:, 0] * vol))
    assert abs(m1 - m0) <= 1e-13 * m0
