"""Backward-Euler step (new code; the reference has no Jacobian assembly): the GPU
Jacobian is bit-identical to the oracle's restatement of the same formulas, and one
implicit step agrees with the oracle's assemble + bcsr_gmres_diag + update to GMRES
round-off."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _meshes():
    from subfv_b200 import meshgen
    return {
        "box_walls": meshgen.hex_box(5, jitter=0.05, seed=41, periodic=False),
        "box_periodic": meshgen.hex_box(6, periodic=True),
    }


def _cfg():
    from subfv_b200.ns import NsConfig
    return NsConfig(scheme=4, second_order=False, method=0, bc_style=2, boundary_2d=False, cfl=0.5)


@pytest.mark.parametrize("name", list(_meshes()))
def test_be_jacobian_bit_exact(native, oracle_lib, cuda_ok, name):
    from oracle.oracle import OracleMesh
    from subfv_b200.mesh import Mesh
    from subfv_b200.ns import NsState, init_fourier_flow
    raw = _meshes()[name]
    m, o = Mesh.from_raw(raw), OracleMesh(raw)
    sol = init_fourier_flow(m, seed=3)
    s = NsState(m, _cfg(), sol)
    row, col, v = s.be_jacobian(0.013)
    ro, co, vo = o.be_jacobian(_cfg().oracle_dict(), sol, 0.013)
    np.testing.assert_array_equal(row, ro)
    np.testing.assert_array_equal(col, co)
    np.testing.assert_array_equal(v, vo)


@pytest.mark.parametrize("refine", [False, True])
def test_implicit_step_matches_oracle(native, oracle_lib, cuda_ok, refine):
    from oracle.oracle import OracleBcsr, OracleMesh
    from subfv_b200.bcsr import BcsrMatrix
    from subfv_b200.mesh import Mesh
    from subfv_b200.ns import NsState, init_fourier_flow
    raw = _meshes()["box_periodic"]
    m, o = Mesh.from_raw(raw), OracleMesh(raw)
    sol = init_fourier_flow(m, seed=4)
    cfl = 10.0
    s = NsState(m, _cfg(), sol)
    st, stats = s.implicit_step(cfl_implicit=cfl, krylov=30, rel_tol=1e-8, refine_fp32=refine)
    assert st == 0 and stats["conv"] == 1
    # oracle: the same residual, dt, matrix, solve and update
    _, rhs_o, sl_o, _, _ = o.ns_rhs(_cfg().oracle_dict(), sol)
    vol = o.geom("elem_volume")
    dt = cfl * min(1e10, float(np.min(vol / sl_o)))
    assert stats["dt"] == dt
    row, col, v = o.be_jacobian(_cfg().oracle_dict(), sol, dt)
    A = OracleBcsr(BcsrMatrix(o.n_elems, 5, row, col, v))
    b = rhs_o.reshape(-1)
    x, conv, it, rho, _ = A.gmres(b, 1e-8 * np.linalg.norm(b), 30, precond=True)
    assert conv
    new_o = sol + x.reshape(-1, 5)
    got = s.sol()
    scale = np.abs(x).max()
    assert np.abs(got - new_o).max() <= (1e-5 if refine else 1e-8) * scale
    # the step solved the linear system it claims to
    assert stats["res_norm"] < 1e-8 * stats["b_norm"] * (1.0001 if not refine else 1.0)


def test_implicit_steps_conserve_mass_periodic(native, cuda_ok):
    from subfv_b200 import meshgen
    from subfv_b200.mesh import Mesh
    from subfv_b200.ns import NsState, init_fourier_flow
    m = Mesh.from_raw(meshgen.hex_box(8, periodic=True))
    sol = init_fourier_flow(m, seed=5)
    vol = m.geometry("elem_volume")
    s = NsState(m, _cfg(), sol)
    for _ in range(3):
        st, stats = s.implicit_step(cfl_implicit=20.0)
        assert st == 0 and stats["conv"] == 1
    out = s.sol()
    for k in (0, 4):
        t0, t1 = float(np.sum(sol[:, k] * vol)), float(np.sum(out[:, k] * vol))
        # exact up to the linear solve's residual (the Jacobian rows sum to the flux balance)
        assert abs(t1 - t0) <= 1e-7 * abs(t0), (k, t1 - t0)


def test_implicit_step_lusgs_matches_oracle(native, oracle_lib, cuda_ok):
    """The implicit step preconditioned by the coloured LU-SGS (cells coloured greedily
    in order): same update as the oracle's assemble + bcsr_gmres_parallel_lusgs with
    that colouring, to GMRES round-off; fewer restarts than block Jacobi."""
    from oracle.oracle import OracleBcsr, OracleMesh
    from subfv_b200.bcsr import BcsrMatrix, greedy_colors
    from subfv_b200.mesh import Mesh
    from subfv_b200.ns import NsState, init_fourier_flow
    raw = _meshes()["box_walls"]
    m, o = Mesh.from_raw(raw), OracleMesh(raw)
    sol = init_fourier_flow(m, seed=6)
    cfl = 10.0
    s = NsState(m, _cfg(), sol)
    st, stats = s.implicit_step(cfl_implicit=cfl, krylov=30, rel_tol=1e-8, precond=2)
    assert st == 0 and stats["conv"] == 1
    _, rhs_o, sl_o, _, _ = o.ns_rhs(_cfg().oracle_dict(), sol)
    dt = cfl * min(1e10, float(np.min(o.geom("elem_volume") / sl_o)))
    assert stats["dt"] == dt
    row, col, v = o.be_jacobian(_cfg().oracle_dict(), sol, dt)
    Am = BcsrMatrix(o.n_elems, 5, row, col, v)
    ncs, color = greedy_colors(Am)
    b = rhs_o.reshape(-1)
    x, conv, it, rho = OracleBcsr(Am).gmres_lusgs(b, 1e-8 * np.linalg.norm(b), 30, ncs, color)
    assert conv and it == stats["restarts"]
    np.testing.assert_allclose(s.sol(), sol + x.reshape(-1, 5), rtol=0, atol=1e-8 * np.abs(x).max())
    s2 = NsState(m, _cfg(), sol)
    _, stats_bj = s2.implicit_step(cfl_implicit=cfl, krylov=30, rel_tol=1e-8, precond=1)
    assert stats["restarts"] <= stats_bj["restarts"]


def _diff_cfg():
    from subfv_b200.ns import NsConfig
    return NsConfig(scheme=4, second_order=False, method=0, bc_style=2, boundary_2d=False, cfl=0.5,
                    activate_diffusion=True, mu_p=2e-3, Cv_p=2.5, prandtl=0.72)


def test_be_jacobian_with_diffusion_bit_exact(native, oracle_lib, cuda_ok):
    """With diffusion the assembled matrix is the frozen-speed Euler Jacobian plus the
    reference's point-implicit diffusion blocks on the diagonal, on a periodic box."""
    from oracle.oracle import OracleMesh
    from subfv_b200.mesh import Mesh
    from subfv_b200.ns import NsState, init_fourier_flow
    raw = _meshes()["box_periodic"]
    m, o = Mesh.from_raw(raw), OracleMesh(raw)
    sol = init_fourier_flow(m, seed=3)
    s = NsState(m, _diff_cfg(), sol)
    row, col, v = s.be_jacobian(0.013)
    ro, co, vo = o.be_jacobian(_diff_cfg().oracle_dict(), sol, 0.013)
    _, _, _, diag = o.ns_rhs_diag(_diff_cfg().oracle_dict(), sol)
    for c in range(o.n_elems):
        j = ro[c] - 1 + int(np.searchsorted(co[ro[c] - 1:ro[c + 1] - 1], c + 1))
        vo[j] = vo[j] + diag[c]
    np.testing.assert_array_equal(row, ro)
    np.testing.assert_array_equal(col, co)
    np.testing.assert_array_equal(v, vo)


def test_implicit_step_with_diffusion_matches_oracle(native, oracle_lib, cuda_ok):
    """One backward-Euler step with viscous and heat terms on a periodic box equals the
    oracle's matrix and right-hand side (rhs - mat_diag U) solved by bcsr_gmres_diag, to
    GMRES round-off."""
    from oracle.oracle import OracleBcsr, OracleMesh
    from subfv_b200.bcsr import BcsrMatrix
    from subfv_b200.mesh import Mesh
    from subfv_b200.ns import NsState, init_fourier_flow
    raw = _meshes()["box_periodic"]
    m, o = Mesh.from_raw(raw), OracleMesh(raw)
    cfg = _diff_cfg()
    sol = init_fourier_flow(m, seed=4)
    cfl = 10.0
    s = NsState(m, cfg, sol)
    st, stats = s.implicit_step(cfl_implicit=cfl, krylov=30, rel_tol=1e-8)
    assert st == 0 and stats["conv"] == 1
    _, rhs_o, sl_o, diag = o.ns_rhs_diag(cfg.oracle_dict(), sol)
    dt = cfl * min(1e10, float(np.min(o.geom("elem_volume") / sl_o)))
    assert stats["dt"] == dt
    row, col, v = o.be_jacobian(cfg.oracle_dict(), sol, dt)
    for c in range(o.n_elems):
        j = row[c] - 1 + int(np.searchsorted(col[row[c] - 1:row[c + 1] - 1], c + 1))
        v[j] = v[j] + diag[c]
    b = (rhs_o - np.einsum('nij,nj->ni', diag.transpose(0, 2, 1), sol)).reshape(-1)
    x, conv, it, _, _ = OracleBcsr(BcsrMatrix(o.n_elems, 5, row, col, v)).gmres(b, 1e-8 * np.linalg.norm(b), 30,
                                                                                precond=True)
    assert conv
    assert np.abs(s.sol() - (sol + x.reshape(-1, 5))).max() <= 1e-8 * np.abs(x).max()
