"""Explicit Euler (subfvns) on the GPU against the oracle restatement of
src/ns/ns_euler_*.F90 and src/ns/ns_main.F90. Plain FP64 is bit-identical for the
state, residual, wave-speed sums, nodal velocities and cell gradients; the residual
norms res/res_vect are summed in a different (tree) order and compared at 1e-13."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _meshes():
    from subfv_b200 import meshgen
    return {
        "hex_slab": meshgen.hex_slab(12, 10, jitter=0.1, seed=31),
        "prism_slab": meshgen.prism_slab(10, 9, -0.5, 0.5, -0.5, 0.5, -0.5, 0.5, jitter=0.05, seed=32),
    }


CFGS = {
    "mp_o2_bc2": dict(scheme=1, second_order=True, method=4, bc_style=2),
    "mp_o1_bc2": dict(scheme=1, second_order=False, method=4, bc_style=2),
    "mp_o1_bc1": dict(scheme=1, second_order=False, method=4, bc_style=1),
    "mp_o1_bc0": dict(scheme=1, second_order=False, method=4, bc_style=0),
    "tw_o2": dict(scheme=4, second_order=True, method=4, bc_style=2),
    "3w_o1": dict(scheme=3, second_order=False, method=4, bc_style=2),
    "3w_o2": dict(scheme=3, second_order=True, method=4, bc_style=2),
    "m3w_o1": dict(scheme=5, second_order=False, method=4, bc_style=2),
    "m3w_o2": dict(scheme=5, second_order=True, method=4, bc_style=2),
    "iso_o1_bc2": dict(scheme=2, second_order=False, method=4, bc_style=2),
    "iso_o2_bc2": dict(scheme=2, second_order=True, method=4, bc_style=2),
    "iso_o1_bc0": dict(scheme=2, second_order=False, method=4, bc_style=0),
    "mpp_o1_bc2": dict(scheme=6, second_order=False, method=4, bc_style=2),
    "mpp_o2_bc1": dict(scheme=6, second_order=True, method=4, bc_style=1),
    "mpph_o1_bc1": dict(scheme=8, second_order=False, method=4, bc_style=1),
    "mpph_o2_bc2": dict(scheme=8, second_order=True, method=4, bc_style=2),
    "mp_o2_m2": dict(scheme=1, second_order=True, method=2, bc_style=2),
    "mp_o2_m3": dict(scheme=1, second_order=True, method=3, bc_style=2),
    "mp_o2_m5": dict(scheme=1, second_order=True, method=5, bc_style=2),
    "tw_o2_m6": dict(scheme=4, second_order=True, method=6, bc_style=2),
}


def _pair(raw):
    from oracle.oracle import OracleMesh
    from subfv_b200.mesh import Mesh
    return Mesh.from_raw(raw), OracleMesh(raw)


def _perturbed_gresho(m, seed):
    from subfv_b200.ns import init_gresho
    sol = init_gresho(m, 0.1)
    rng = np.random.default_rng(seed)
    sol[:, 0] *= 1.0 + 0.02 * rng.uniform(-1, 1, m.n_elems)
    sol[:, 1:3] += 0.05 * rng.uniform(-1, 1, (m.n_elems, 2))
    return np.ascontiguousarray(sol)


@pytest.mark.parametrize("mesh_name", ["hex_slab", "prism_slab"])
@pytest.mark.parametrize("cfg_name", list(CFGS))
def test_compute_rhs_ns_bit_exact(native, oracle_lib, cuda_ok, mesh_name, cfg_name):
    from subfv_b200.ns import NsConfig, compute_rhs_ns
    m, o = _pair(_meshes()[mesh_name])
    cfg = NsConfig(**CFGS[cfg_name], boundary_2d=True, cfl=0.4)
    sol = _perturbed_gresho(m, 5)
    st, rhs, sl, vp, grad = compute_rhs_ns(m, cfg, sol)
    st_o, rhs_o, sl_o, vp_o, grad_o = o.ns_rhs(cfg.oracle_dict(), sol)
    assert st == st_o == 0
    np.testing.assert_array_equal(sl, sl_o)
    np.testing.assert_array_equal(rhs, rhs_o)
    if cfg.scheme in (1, 2):
        np.testing.assert_array_equal(vp, vp_o)
    # oracle grad rows are [d*5 + var]; product (5, 3) per cell is grad(d, var) at [var, d]
    np.testing.assert_array_equal(grad.transpose(0, 2, 1).reshape(-1, 15), grad_o)


@pytest.mark.parametrize("method", [2, 3, 4, 5, 6])
def test_grouped_gradients_bitwise(native, cuda_ok, method):
    """The cell gradient with a group of 8 lanes per cell (each vertex's terms on its own
    lane, the sums in vertex order by shuffles, the min / max folds per lane and then over
    the lanes in vertex order) and the nodal gradient with a group of 8 or 16 lanes per
    vertex (a subface per lane, sums in subface order) give the thread kernels' states bit
    for bit: FP64 and the FP32 level, hexahedral and prism slabs and a periodic hexahedral
    box. set_node_kernel(0) selects a thread per vertex and per cell, 1 the lane groups."""
    from subfv_b200 import meshgen
    from subfv_b200.mesh import Mesh
    from subfv_b200.ns import NsConfig, NsState, init_fourier_flow
    cases = [(Mesh.from_raw(raw), True) for raw in _meshes().values()]
    cases.append((Mesh.from_raw(meshgen.hex_box(5, jitter=0.05, seed=3, periodic=True)), False))
    for m, b2d in cases:
        sol = _perturbed_gresho(m, 9) if b2d else init_fourier_flow(m, seed=4)
        for prec in (0, 2):
            cfg = NsConfig(scheme=1, second_order=True, method=method, bc_style=2, boundary_2d=b2d, cfl=0.4,
                           precision=prec, tmax=1e30)
            out = []
            for lanes in (0, 1):
                s = NsState(m, cfg, sol)
                s.set_node_kernel(lanes)
                out.append((s.advance(6), s.sol()))
                s.close()
            assert out[0][0] == out[1][0] and out[0][0][0] == 0
            np.testing.assert_array_equal(out[0][1], out[1][1])


@pytest.mark.parametrize("lanes", [0, 1])
def test_state_follows_geometry_changes(native, oracle_lib, cuda_ok, lanes):
    """A state that keeps running after its mesh's vertices move (subfv_mesh_set_coords,
    then subfv_compute_geometry_mesh) drops its captured step loop and refills the mesh's
    geometry caches (the nodal-gradient pseudo-inverses): its states are the oracle's, run
    eight steps on the first geometry and eight on the moved one. Both node layouts."""
    from dataclasses import replace as dc_replace
    from oracle.oracle import OracleMesh
    from subfv_b200.ns import NsConfig, NsState, init_gresho
    raw = _meshes()["hex_slab"]
    m, o = _pair(raw)
    cfg = NsConfig(**CFGS["mp_o2_m5"], boundary_2d=True, cfl=0.4)
    sol = _perturbed_gresho(m, 3)
    s = NsState(m, cfg, sol)
    s.set_node_kernel(lanes)
    st, n, t = s.advance(8)  # one captured graph of eight steps
    assert st == 0 and n == 8
    c = raw.coords.copy()
    lo, hi = c.min(0), c.max(0)
    inner = (c[:, 0] > lo[0] + 1e-9) & (c[:, 0] < hi[0] - 1e-9) & (c[:, 1] > lo[1] + 1e-9) & (c[:, 1] < hi[1] - 1e-9)
    rng = np.random.default_rng(12)
    shift = rng.uniform(-0.02, 0.02, (len(c), 2)) / 12
    _, col = np.unique(np.round(c[:, :2], 9), axis=0, return_inverse=True)  # one shift per column
    c[inner, :2] += shift[col.ravel()][inner]
    o2 = OracleMesh(dc_replace(raw, coords=c))
    m.set_coords(o2.geom("vert_coord"))
    assert m.compute_geometry_mesh() == 0
    st, n, t = s.advance(8)
    assert st == 0 and n == 16
    sol_o = sol.copy()
    st_o, it, t_o, _, _, _ = o.ns_run(cfg.oracle_dict(), sol_o, 7)
    assert st_o == 0 and it == 8
    st_o, it, t_o, _, _, _ = o2.ns_run(cfg.oracle_dict(), sol_o, 7, t0=t_o)
    assert st_o == 0 and it == 8
    assert t == t_o
    np.testing.assert_array_equal(s.sol(), sol_o)
    s.close()


def test_gresho_init_matches_oracle(native, oracle_lib, cuda_ok):
    from subfv_b200.ns import init_gresho
    m, o = _pair(_meshes()["hex_slab"])
    np.testing.assert_array_equal(init_gresho(m, 0.1), o.ns_gresho(0.1))


@pytest.mark.parametrize("cfg_name", ["mp_o2_bc2", "tw_o2", "mp_o1_bc1", "3w_o2", "m3w_o2", "iso_o2_bc2", "mpp_o2_bc1",
                                      "mpph_o2_bc2", "mp_o2_m3", "tw_o2_m6"])
def test_ns_time_loop_bit_exact(native, oracle_lib, cuda_ok, cfg_name):
    from subfv_b200.ns import NsConfig, NsState, init_gresho
    m, o = _pair(_meshes()["hex_slab"])
    cfg = NsConfig(**CFGS[cfg_name], boundary_2d=True, cfl=0.4)
    sol = init_gresho(m, 0.1)
    steps = 12
    s = NsState(m, cfg, sol)
    st, n, t = s.advance(steps)
    assert st == 0 and n == steps
    sol_o = sol.copy()
    st_o, it, t_o, res_o, rv_o, vp_o = o.ns_run(cfg.oracle_dict(), sol_o, steps - 1)
    assert st_o == 0 and it == steps
    assert t == t_o
    np.testing.assert_array_equal(s.sol(), sol_o)
    res, rv, _ = s.residuals()
    assert res == pytest.approx(res_o, rel=1e-13)
    np.testing.assert_allclose(rv, rv_o, rtol=1e-13)


def test_ns_conservation_walls(native, cuda_ok):
    """Closed slip walls: total mass and energy are conserved to round-off."""
    from subfv_b200 import meshgen
    from subfv_b200.mesh import Mesh
    from subfv_b200.ns import NsConfig, NsState, init_gresho
    m = Mesh.from_raw(meshgen.hex_slab(32, 32, jitter=0.1, seed=33))
    vol = m.geometry("elem_volume")
    sol = init_gresho(m, 0.1)
    s = NsState(m, NsConfig(cfl=0.4), sol)
    st, n, _ = s.advance(40)
    assert st == 0
    out = s.sol()
    for k in (0, 4):
        tot0, tot1 = float(np.sum(sol[:, k] * vol)), float(np.sum(out[:, k] * vol))
        assert abs(tot1 - tot0) <= 1e-13 * abs(tot0) * n, (k, tot1 - tot0)


def test_ns_mixed_precision_close(native, cuda_ok):
    """Gresho, 20 iterations: precision 1 (FP32 wave-speed bounds) within 1e-6 of plain
    FP64 per field in L1 and Linf; precision 2 (also FP32 reconstruction, limiters and
    flux, the pressure-jump term FP64) reported. Both conserve mass and energy to
    round-off on the closed slab."""
    from meshes import field_errors
    from subfv_b200 import meshgen
    from subfv_b200.mesh import Mesh
    from subfv_b200.ns import NsConfig, NsState, init_gresho
    raw = meshgen.hex_slab(32, 32, jitter=0.1, seed=34)
    out = {}
    for prec in (0, 1, 2):
        m = Mesh.from_raw(raw)
        vol = m.geometry("elem_volume")
        sol = init_gresho(m, 0.1)
        s = NsState(m, NsConfig(cfl=0.4, precision=prec), sol)
        st, n, _ = s.advance(20)
        assert st == 0
        out[prec] = s.sol()
        for k in (0, 4):
            t0, t1 = float(np.sum(sol[:, k] * vol)), float(np.sum(out[prec][:, k] * vol))
            assert abs(t1 - t0) <= 2 * 8 * n * np.finfo(float).eps * float(np.sum(np.abs(sol[:, k]) * vol)), \
                (prec, k, t1 - t0)
    for prec in (1, 2):
        l1, linf = field_errors(out[0], out[prec])
        print(f"precision {prec} vs plain FP64: L1", l1.tolist(), "Linf", linf.tolist())
        if prec == 1:
            assert l1.max() <= 1e-6 and linf.max() <= 1e-6, (l1, linf)


def test_ns_3d_box_walls_bit_exact(native, oracle_lib, cuda_ok):
    from subfv_b200 import meshgen
    from subfv_b200.ns import NsConfig, NsState
    m, o = _pair(meshgen.hex_box(5, jitter=0.05, seed=35, periodic=False))
    rng = np.random.default_rng(36)
    w = np.column_stack([rng.uniform(0.8, 1.2, m.n_elems), rng.uniform(-0.2, 0.2, (m.n_elems, 3)),
                         rng.uniform(0.8, 1.2, m.n_elems)])
    sol = np.column_stack([w[:, 0], w[:, 1:4] * w[:, :1], w[:, 4] / 0.4 + 0.5 * w[:, 0] * (w[:, 1:4] ** 2).sum(1)])
    sol = np.ascontiguousarray(sol)
    cfg = NsConfig(scheme=1, second_order=True, method=4, bc_style=2, boundary_2d=False, cfl=0.3)
    s = NsState(m, cfg, sol)
    st, n, t = s.advance(5)
    sol_o = sol.copy()
    st_o, it, t_o, _, _, _ = o.ns_run(cfg.oracle_dict(), sol_o, 4)
    assert st == st_o == 0 and t == t_o
    np.testing.assert_array_equal(s.sol(), sol_o)


def test_prepare_leaves_state_and_results_unchanged(native, cuda_ok):
    """Capturing the step graph ahead (prepare) neither moves the state nor changes the run."""
    from subfv_b200 import meshgen
    from subfv_b200.lagrange import LagrangeState
    from subfv_b200.mesh import Mesh
    from subfv_b200.ns import NsConfig, NsState, init_gresho
    raw = meshgen.hex_slab(12, 10, jitter=0.1, seed=31)
    outs = []
    for prep in (False, True):
        m = Mesh.from_raw(raw)
        s = NsState(m, NsConfig(cfl=0.4), init_gresho(m, 0.1))
        if prep:
            s.prepare()
            assert s.sync()[1] == 0
        outs.append((s.advance(19), s.sol()))
        s.close()
    assert outs[0][0] == outs[1][0]
    np.testing.assert_array_equal(outs[0][1], outs[1][1])
    lag = []
    for prep in (False, True):
        m = Mesh.from_raw(raw)
        sol = init_gresho(m, 0.1)
        st = LagrangeState(m, sol, m.geometry("elem_volume") / sol[:, 0], cfl=0.5, t_max=1.0)
        if prep:
            st.prepare()
        lag.append((st.advance(21), st.sol()))
    assert lag[0][0] == lag[1][0]
    np.testing.assert_array_equal(lag[0][1], lag[1][1])
