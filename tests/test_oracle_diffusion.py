"""The oracle's restatement of the Navier-Stokes diffusion terms (activate_diffusion:
src/ns/ns_vectorial_diffusion_module.F90 for momentum and viscous work,
src/ns/ns_diffusion_module.F90 for heat, assembled point-implicitly into mat_diag and
solved per cell by add_timedisc_and_solve, src/ns/ns_euler_module.F90:521-609) has no
golden vectors; these tests check its physics: a fluid at rest at uniform temperature
stays at rest (Neumann walls, and Dirichlet walls at the fluid's velocity and
temperature), a moving Dirichlet wall drags the fluid along it, heat flows from a hot
Dirichlet wall into the fluid, and diffusion changes the result of the inviscid run."""
import numpy as np
import pytest

NX, NY = 8, 6


def _mesh():
    from oracle.oracle import OracleMesh
    from subfv_b200 import meshgen
    raw = meshgen.tag_slab_sides(meshgen.hex_slab(NX, NY, jitter=0.1, seed=3), NX, NY,
                                 {"xlo": 1, "xhi": 2, "ylo": 3, "yhi": 4})
    return OracleMesh(raw)


def _cons(w):
    return np.ascontiguousarray(np.column_stack([w[:, 0], w[:, 1:4] * w[:, :1],
                                                 w[:, 4] / 0.4 + 0.5 * w[:, 0] * (w[:, 1:4] ** 2).sum(1)]))


def _cfg(**kw):
    d = dict(scheme=1, second_order=1, method=4, bc_style=2, b2d=1, exclude_bound_vert=0, local_time_step=0,
             cfl=0.3, tmax=1e30, n_bc=4, bc_type=np.ones(4, np.int32), bc_val=np.zeros((4, 5)),
             activate_diffusion=1, diff_dc=[0.05, 1.716e-5, 273.15, 2.5])
    d.update(kw)
    return d


CV = 2.5


@pytest.mark.parametrize("walls", ["neumann", "dirichlet"])
def test_rest_state_is_preserved(oracle_lib, walls):
    o = _mesh()
    sol = _cons(np.tile([1.2, 0.0, 0.0, 0.0, 1.0], (o.n_elems, 1)))
    T = sol[0, 4] / sol[0, 0] / CV
    kw = {}
    if walls == "dirichlet":
        kw = dict(bc_type_V=np.full(4, 2, np.int32), bc_val_V=np.zeros((4, 3)),
                  bc_type_T=np.full(4, 2, np.int32), bc_val_T=np.full(4, T))
    s = sol.copy()
    st, it, _, _, _, _ = o.ns_run(_cfg(**kw), s, 4)
    assert st == 0 and it == 5
    np.testing.assert_allclose(s, sol, rtol=0, atol=1e-14)


def test_moving_wall_drags_fluid(oracle_lib):
    o = _mesh()
    sol = _cons(np.tile([1.2, 0.0, 0.0, 0.0, 1.0], (o.n_elems, 1)))
    kw = dict(bc_type_V=np.array([1, 1, 2, 2], np.int32), bc_val_V=np.array([[0, 0, 0]] * 3 + [[0.1, 0, 0]], float))
    s = sol.copy()
    st, _, _, _, _, _ = o.ns_run(_cfg(**kw), s, 20)
    assert st == 0
    y = o.geom("elem_coord")[:, 1]
    top, bottom = s[y > 0.3, 1].mean(), s[y < -0.3, 1].mean()
    assert top > 10 * abs(bottom) and top > 1e-3


def test_hot_wall_heats_fluid(oracle_lib):
    o = _mesh()
    sol = _cons(np.tile([1.2, 0.0, 0.0, 0.0, 1.0], (o.n_elems, 1)))
    T = sol[0, 4] / sol[0, 0] / CV
    kw = dict(bc_type_T=np.array([2, 1, 1, 1], np.int32), bc_val_T=np.array([1.5 * T, 0, 0, 0]))
    s = sol.copy()
    st, _, _, _, _, _ = o.ns_run(_cfg(**kw), s, 10)
    assert st == 0
    vol = o.geom("elem_volume")
    assert np.sum(s[:, 4] * vol) > np.sum(sol[:, 4] * vol) * (1 + 1e-6)
    x = o.geom("elem_coord")[:, 0]
    assert s[x < -0.3, 4].mean() > s[x > 0.3, 4].mean()


def test_diffusion_changes_the_inviscid_result(oracle_lib):
    o = _mesh()
    rng = np.random.default_rng(2)
    w = np.column_stack([rng.uniform(1.1, 1.3, o.n_elems), rng.uniform(-0.1, 0.1, (o.n_elems, 2)),
                         np.zeros(o.n_elems), rng.uniform(0.9, 1.1, o.n_elems)])
    sol = _cons(w)
    a, b, c = sol.copy(), sol.copy(), sol.copy()
    assert o.ns_run(_cfg(), a, 3)[0] == 0
    assert o.ns_run(_cfg(activate_diffusion=0), b, 3)[0] == 0
    assert o.ns_run(_cfg(use_sutherland=1, diff_dc=[0.05, 0.05, 0.4, CV]), c, 3)[0] == 0
    assert np.isfinite(a).all() and np.isfinite(c).all()
    assert np.abs(a - b).max() > 1e-4 and np.abs(c - a).max() > 1e-6


def test_linear_temperature_is_steady_on_an_orthogonal_slab(oracle_lib):
    """Fluid at rest at uniform pressure with a temperature linear in x between two
    Dirichlet walls at the matching temperatures (adiabatic elsewhere): the heat flux is
    uniform, so nothing changes — to round-off on an orthogonal slab, where the sub-cell
    flux reconstruction is exact for linear fields."""
    from oracle.oracle import OracleMesh
    from subfv_b200 import meshgen
    raw = meshgen.tag_slab_sides(meshgen.hex_slab(NX, NY, jitter=0.0, seed=3), NX, NY,
                                 {"xlo": 1, "xhi": 2, "ylo": 3, "yhi": 4})
    o = OracleMesh(raw)
    x = o.geom("elem_coord")[:, 0]
    T = 0.4 + 0.1 * (x + 0.5)
    e = CV * T
    rho = 1.0 / (0.4 * e)
    sol = np.ascontiguousarray(np.column_stack([rho, np.zeros((o.n_elems, 3)), rho * e]))
    s = sol.copy()
    kw = dict(bc_type_T=np.array([2, 2, 1, 1], np.int32), bc_val_T=np.array([0.4, 0.5, 0, 0]))
    st, _, _, _, _, _ = o.ns_run(_cfg(**kw), s, 4)
    assert st == 0
    np.testing.assert_allclose(s, sol, rtol=0, atol=1e-14)
    # the same field with a colder right wall does change
    s2 = sol.copy()
    kw["bc_val_T"] = np.array([0.4, 0.45, 0, 0])
    assert o.ns_run(_cfg(**kw), s2, 4)[0] == 0
    assert np.abs(s2 - sol).max() > 1e-6


def _periodic_pair(n):
    from oracle.oracle import OracleMesh
    from subfv_b200 import meshgen
    return OracleMesh(meshgen.hex_box(n, jitter=0.0, seed=0, periodic=True))


def _prim_to_cons(w):
    return np.ascontiguousarray(np.column_stack([w[:, 0], w[:, 1:4] * w[:, :1],
                                                 w[:, 4] / 0.4 + 0.5 * w[:, 0] * (w[:, 1:4] ** 2).sum(1)]))


def _viscous_term(o, sol, mu):
    """The full diffusion term of each cell, rhs_visc - mat_diag U (the reference's
    point-implicit split: add_timedisc_and_solve solves (mat_diag + s I) U_new = rhs + s U)."""
    from subfv_b200.ns import NsConfig
    base = dict(scheme=4, second_order=False, method=0, bc_style=2, boundary_2d=False, cfl=0.5)
    _, r_d, _, diag = o.ns_rhs_diag(NsConfig(**base, activate_diffusion=True, mu_p=mu).oracle_dict(), sol)
    _, r_e, _, _, _ = o.ns_rhs(NsConfig(**base).oracle_dict(), sol)
    return (r_d - r_e) - np.einsum('nij,nj->ni', diag.transpose(0, 2, 1), sol)


def test_periodic_box_diffusion_is_consistent(oracle_lib):
    """Diffusion on a periodic box (each periodic node's system over the union of its
    images' subfaces and subcells): a uniform flow has no viscous or heat term, and the
    x-momentum term of a shear wave u = A sin(2 pi y) converges to mu u'' at second order."""
    mu, A = 1e-2, 0.01
    errs = []
    for n in (8, 16):
        o = _periodic_pair(n)
        cc, vol = o.geom("elem_coord"), o.geom("elem_volume")
        ones = np.ones(len(cc))
        uni = _prim_to_cons(np.column_stack([ones, 0.3 * ones, 0.1 * ones, -0.2 * ones, ones]))
        assert np.abs(_viscous_term(o, uni, mu)).max() <= 1e-13 * mu * 0.3
        ux = A * np.sin(2 * np.pi * cc[:, 1])
        shear = _prim_to_cons(np.column_stack([ones, ux, 0 * ux, 0 * ux, ones]))
        visc = _viscous_term(o, shear, mu)
        exact = -mu * (2 * np.pi) ** 2 * ux * vol
        errs.append(np.abs(visc[:, 1] - exact).max() / np.abs(exact).max())
    print("shear-wave viscous term, max relative error at 8^3 and 16^3:", errs)
    assert errs[1] < 0.02 and errs[0] / errs[1] > 3.5
