"""The procedures ns_main's loop calls, one entry each (the drop-in a shim binds so
src/ns/ns_main.F90:83-107 stays as it is): compute_euler_flux, compute_cell_grad_from_
nodal_grad, flux_limiting and add_timedisc_and_solve, through the C-ABI with host
arrays, bit for bit against the oracle's restatement of the same procedures; then the
reference's time loop written with these four calls only, against the oracle's ns_run."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _meshes():
    from subfv_b200 import meshgen
    return {
        "hex_slab": meshgen.hex_slab(12, 10, jitter=0.1, seed=31),
        "prism_slab": meshgen.prism_slab(10, 9, -0.5, 0.5, -0.5, 0.5, -0.5, 0.5, jitter=0.05, seed=32),
    }


def _pair(name):
    from oracle.oracle import OracleMesh
    from subfv_b200.mesh import Mesh
    raw = _meshes()[name]
    return Mesh.from_raw(raw), OracleMesh(raw)


def _state(m, seed):
    from subfv_b200.ns import init_gresho
    sol = init_gresho(m, 0.1)
    rng = np.random.default_rng(seed)
    sol[:, 0] *= 1.0 + 0.02 * rng.uniform(-1, 1, m.n_elems)
    sol[:, 1:3] += 0.05 * rng.uniform(-1, 1, (m.n_elems, 2))
    return np.ascontiguousarray(sol)


@pytest.mark.parametrize("name", ["hex_slab", "prism_slab"])
@pytest.mark.parametrize("scheme", [1, 4])
def test_compute_euler_flux_bit_exact(native, oracle_lib, cuda_ok, name, scheme):
    from subfv_b200.ns import NsConfig, compute_euler_flux
    m, o = _pair(name)
    cfg = NsConfig(scheme=scheme, method=4, bc_style=2, cfl=0.4)
    sol = _state(m, 3)
    grad, _ = o.cell_grads(cfg.oracle_dict(), sol)
    for so in (False, True):
        rhs, sl, vp = np.zeros((m.n_elems, 5)), np.zeros(m.n_elems), np.zeros((m.n_vert, 3))
        st = compute_euler_flux(m, cfg, sol, rhs, grad, sl, so, vp)
        st_o, rhs_o, sl_o, vp_o = o.euler_flux(cfg.oracle_dict(), sol, grad, so)
        assert st == st_o == 0
        np.testing.assert_array_equal(rhs, rhs_o)
        np.testing.assert_array_equal(sl, sl_o)
        if scheme == 1:
            np.testing.assert_array_equal(vp, vp_o)


@pytest.mark.parametrize("name", ["hex_slab", "prism_slab"])
@pytest.mark.parametrize("method", [0, 2, 3, 4, 5, 6])
def test_compute_cell_grad_from_nodal_grad_bit_exact(native, oracle_lib, cuda_ok, name, method):
    from subfv_b200.ns import NsConfig, compute_cell_grad_from_nodal_grad
    m, o = _pair(name)
    cfg = NsConfig(method=method, cfl=0.4)
    sol = _state(m, 4)
    grad, ngrad = np.empty((m.n_elems, 5, 3)), np.empty((m.n_vert, 5, 3))
    assert compute_cell_grad_from_nodal_grad(m, sol, grad, ngrad, method, cfg) == 0
    grad_o, ngrad_o = o.cell_grads(cfg.oracle_dict(), sol)
    np.testing.assert_array_equal(ngrad, ngrad_o)
    np.testing.assert_array_equal(grad, grad_o)
    if method == 0:
        assert not grad.any()


@pytest.mark.parametrize("name", ["hex_slab", "prism_slab"])
def test_flux_limiting_bit_exact(native, oracle_lib, cuda_ok, name):
    from subfv_b200.ns import NsConfig, flux_limiting
    m, o = _pair(name)
    cfg = NsConfig(cfl=0.4)
    sol = _state(m, 5)
    grad, _ = o.cell_grads(cfg.oracle_dict(), sol)
    _, rhs, sl, _ = o.euler_flux(cfg.oracle_dict(), sol, None, False)
    _, rhs_o2, _, _ = o.euler_flux(cfg.oracle_dict(), sol, grad, True)
    # a second-order residual pushed towards negative density in a few cells, so the
    # positivity limiter acts there
    rhs_o2[::7, 0] -= 50.0 * np.abs(rhs_o2[::7, 0]) + 1.0
    got = rhs.copy()
    assert flux_limiting(m, sol, got, rhs_o2, sl, 0.4) == 0
    expected = o.flux_limiting(sol, rhs, rhs_o2, sl, 0.4)
    np.testing.assert_array_equal(got, expected)
    assert not np.array_equal(got, rhs_o2)  # the limiter acted


@pytest.mark.parametrize("name", ["hex_slab", "prism_slab"])
@pytest.mark.parametrize("with_diag", [False, True])
@pytest.mark.parametrize("a1", [2.0, 1.0])
def test_add_timedisc_and_solve_bit_exact(native, oracle_lib, cuda_ok, name, with_diag, a1):
    from subfv_b200.ns import NsConfig, add_timedisc_and_solve
    m, o = _pair(name)
    cfg = NsConfig(cfl=0.4, tmax=1.0)
    sol = _state(m, 6)
    _, rhs, sl, _ = o.euler_flux(cfg.oracle_dict(), sol, None, False)
    diag = None
    if with_diag:  # blocks like the diffusion terms leave: small, not symmetric
        rng = np.random.default_rng(7)
        diag = np.ascontiguousarray(rng.uniform(-1.0, 1.0, (m.n_elems, 5, 5)) * 1e-2)
    args = dict(sol=sol.copy(), rhs=rhs.copy(), diag=None if diag is None else diag.copy(), sum_lambda=sl.copy())
    ora = {k: (None if v is None else v.copy()) for k, v in args.items()}
    delta = np.zeros((m.n_elems, 5))
    st, res, rv, dt = add_timedisc_and_solve(m, args["sol"], args["rhs"], args["diag"], args["sum_lambda"], delta,
                                             1, 0, a1, 1.0, 0.4, 0.25, tmax=1.0)
    st_o, delta_o, res_o, rv_o, dt_o = o.add_timedisc(cfg.oracle_dict(), ora["sol"], ora["rhs"], ora["diag"],
                                                      ora["sum_lambda"], a1, 1.0, 0.25)
    assert st == st_o == 0
    assert dt == dt_o and res == res_o
    np.testing.assert_array_equal(rv, rv_o)
    for k in ("sol", "rhs", "diag", "sum_lambda"):
        if args[k] is not None:
            np.testing.assert_array_equal(args[k], ora[k], err_msg=k)
    np.testing.assert_array_equal(delta, delta_o)
    assert not args["sum_lambda"].any()


def test_add_timedisc_and_solve_clips_to_tmax(native, oracle_lib, cuda_ok):
    from subfv_b200.ns import NsConfig, add_timedisc_and_solve
    m, o = _pair("hex_slab")
    sol = _state(m, 8)
    _, rhs, sl, _ = o.euler_flux(NsConfig(cfl=0.4).oracle_dict(), sol, None, False)
    t, tmax = 0.5, 0.5 + 1e-7
    s1, delta = sol.copy(), np.zeros((m.n_elems, 5))
    st, _, _, dt = add_timedisc_and_solve(m, s1, rhs.copy(), None, sl.copy(), delta, 1, 0, 1.0, 1.0, 0.4, t, tmax)
    assert st == 0 and dt == pytest.approx(tmax - t + 1e-12, rel=1e-12)


@pytest.mark.parametrize("cfg_kw", [dict(scheme=1, second_order=True, method=4, bc_style=2),
                                    dict(scheme=4, second_order=False, method=0, bc_style=2)])
def test_ns_main_loop_from_procedures_bit_exact(native, oracle_lib, cuda_ok, cfg_kw):
    """ns_main.F90:83-107 written with the four entries (and compute_rhs_ns of
    :130-179 from the first three), against the oracle's time loop."""
    from subfv_b200.ns import (NsConfig, add_timedisc_and_solve, compute_cell_grad_from_nodal_grad,
                               compute_euler_flux, flux_limiting, init_gresho)
    m, o = _pair("hex_slab")
    cfg = NsConfig(**cfg_kw, cfl=0.4)
    n_e, n_v = m.n_elems, m.n_vert

    def compute_rhs_ns(sol):
        rhs, sl, vp = np.zeros((n_e, 5)), np.zeros(n_e), np.zeros((n_v, 3))
        grad = np.zeros((n_e, 5, 3))
        compute_euler_flux(m, cfg, sol, rhs, grad, sl, False, vp)
        if cfg.second_order:
            ngrad = np.zeros((n_v, 5, 3))
            compute_cell_grad_from_nodal_grad(m, sol, grad, ngrad, cfg.method, cfg)
            rhs_o2, sl_o2 = np.zeros((n_e, 5)), np.zeros(n_e)
            compute_euler_flux(m, cfg, sol, rhs_o2, grad, sl_o2, True, vp)
            flux_limiting(m, sol, rhs, rhs_o2, sl, cfg.cfl)
        return rhs, sl

    sol0 = init_gresho(m, 0.1)
    sol = sol0.copy()
    t, iters = 0.0, 4
    delta = np.zeros((n_e, 5))
    for _ in range(iters):
        rhs, sl = compute_rhs_ns(sol)
        if cfg.second_order:
            soln = sol.copy()
            st, res, rv, dt = add_timedisc_and_solve(m, sol, rhs, None, sl, delta, 1, 0, 2.0, 1.0, cfg.cfl, t)
            rhs, sl = compute_rhs_ns(sol)
            st, res, rv, dt = add_timedisc_and_solve(m, soln, rhs, None, sl, delta, 1, 0, 1.0, 1.0, cfg.cfl, t)
            sol = soln
        else:
            st, res, rv, dt = add_timedisc_and_solve(m, sol, rhs, None, sl, delta, 1, 0, 1.0, 1.0, cfg.cfl, t)
        assert st == 0
        t = t + dt
    sol_o = sol0.copy()
    st_o, it, t_o, res_o, rv_o, _ = o.ns_run(cfg.oracle_dict(), sol_o, iters - 1)
    assert st_o == 0 and it == iters and t == t_o and res == res_o
    np.testing.assert_array_equal(rv, rv_o)
    np.testing.assert_array_equal(sol, sol_o)
