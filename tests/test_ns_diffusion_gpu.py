"""Navier-Stokes diffusion (activate_diffusion) on the GPU against the oracle restatement
of src/ns/ns_vectorial_diffusion_module.F90 (momentum, viscous work) and
src/ns/ns_diffusion_module.F90 (heat), with the point-implicit 5x5 solve of
add_timedisc_and_solve (src/ns/ns_euler_module.F90:521-609). With a constant viscosity
the residual, the diffusion blocks of mat_diag and the time loop are bit-identical to the
oracle, on slabs, a closed box and a periodic box; Sutherland's law evaluates pow, whose last bits differ between CUDA and the host C
library, so it is compared at 1e-12 of the scale. Unsupported uses are rejected."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NX, NY = 8, 6
TAGS = {"xlo": 1, "xhi": 2, "ylo": 3, "yhi": 4}


def _raws():
    from subfv_b200 import meshgen
    return {
        "hex": meshgen.tag_slab_sides(meshgen.hex_slab(NX, NY, jitter=0.1, seed=3), NX, NY, TAGS),
        "prism": meshgen.tag_slab_sides(
            meshgen.prism_slab(NX, NY, -0.5, 0.5, -0.5, 0.5, -0.5, 0.5, jitter=0.05, seed=4), NX, NY, TAGS),
        "box": meshgen.hex_box(4, jitter=0.05, seed=5, periodic=False),
        # periodic nodes: every image's system over the union of the images' subfaces and
        # subcells (no counterpart in the reference, whose extended lists collide)
        "box_periodic": meshgen.hex_box(4, jitter=0.05, seed=6, periodic=True),
    }


def _pair(raw):
    from oracle.oracle import OracleMesh
    from subfv_b200.mesh import Mesh
    return Mesh.from_raw(raw), OracleMesh(raw)


def _state(n, seed=5):
    rng = np.random.default_rng(seed)
    w = np.column_stack([rng.uniform(1.1, 1.3, n), rng.uniform(-0.1, 0.1, (n, 3)), rng.uniform(0.9, 1.1, n)])
    return np.ascontiguousarray(np.column_stack([w[:, 0], w[:, 1:4] * w[:, :1],
                                                 w[:, 4] / 0.4 + 0.5 * w[:, 0] * (w[:, 1:4] ** 2).sum(1)]))


DIFF = {
    "neumann": dict(),
    "dirichlet": dict(bc_type_V=[1, 2, 2, 2], bc_val_V=[[0, 0, 0], [0, 0, 0], [0, 0, 0], [0.1, 0, 0]],
                      bc_type_T=[2, 0, 1, 2], bc_val_T=[0.5, 0, 0, 0.35]),
}


def _cfg(mesh_name, diff_name, **kw):
    from subfv_b200.ns import NsConfig
    box = mesh_name.startswith("box")
    base = dict(scheme=1, second_order=True, method=4, bc_style=2, boundary_2d=not box, cfl=0.3,
                activate_diffusion=True, mu_p=0.02, Cv_p=2.5)
    if not box:
        base.update(bc_type=[1, 1, 1, 1], bc_val=[[0] * 5] * 4, **DIFF[diff_name])
    base.update(kw)
    return NsConfig(**base)


@pytest.mark.parametrize("mesh_name", ["hex", "prism", "box", "box_periodic"])
@pytest.mark.parametrize("diff_name", ["neumann", "dirichlet"])
@pytest.mark.parametrize("scheme,order", [(1, True), (4, False)])
def test_rhs_and_diag_bit_exact(native, oracle_lib, cuda_ok, mesh_name, diff_name, scheme, order):
    from subfv_b200.ns import compute_rhs_ns_diag
    if mesh_name.startswith("box") and diff_name == "dirichlet":
        pytest.skip("the box has only the default (Neumann) walls")
    m, o = _pair(_raws()[mesh_name])
    cfg = _cfg(mesh_name, diff_name, scheme=scheme, second_order=order)
    sol = _state(m.n_elems)
    st, rhs, sl, diag = compute_rhs_ns_diag(m, cfg, sol)
    st_o, rhs_o, sl_o, diag_o = o.ns_rhs_diag(cfg.oracle_dict(), sol)
    assert st == st_o == 0
    assert np.abs(diag_o).max() > 0.0
    np.testing.assert_array_equal(sl, sl_o)
    np.testing.assert_array_equal(diag, diag_o)
    np.testing.assert_array_equal(rhs, rhs_o)


@pytest.mark.parametrize("mesh_name,diff_name", [("hex", "dirichlet"), ("prism", "neumann"), ("box", "neumann"),
                                                  ("box_periodic", "neumann")])
def test_time_loop_bit_exact(native, oracle_lib, cuda_ok, mesh_name, diff_name):
    from subfv_b200.ns import NsState
    m, o = _pair(_raws()[mesh_name])
    cfg = _cfg(mesh_name, diff_name)
    sol = _state(m.n_elems, seed=9)
    s = NsState(m, cfg, sol)
    st, n, t = s.advance(6)
    sol_o = sol.copy()
    st_o, it, t_o, res_o, rv_o, _ = o.ns_run(cfg.oracle_dict(), sol_o, 5)
    assert st == st_o == 0 and n == it == 6 and t == t_o
    np.testing.assert_array_equal(s.sol(), sol_o)
    res, rv, _ = s.residuals()
    assert res == pytest.approx(res_o, rel=1e-13)
    np.testing.assert_allclose(rv, rv_o, rtol=1e-13)
    s.close()


def test_sutherland_close(native, oracle_lib, cuda_ok):
    from subfv_b200.ns import compute_rhs_ns_diag
    m, o = _pair(_raws()["hex"])
    cfg = _cfg("hex", "dirichlet", use_sutherland=True, mu0=0.02, T0=0.4)
    sol = _state(m.n_elems)
    st, rhs, sl, diag = compute_rhs_ns_diag(m, cfg, sol)
    st_o, rhs_o, sl_o, diag_o = o.ns_rhs_diag(cfg.oracle_dict(), sol)
    assert st == st_o == 0
    np.testing.assert_array_equal(sl, sl_o)
    for k in range(5):
        assert np.abs(rhs[:, k] - rhs_o[:, k]).max() <= 1e-12 * np.abs(rhs_o).max(), k
    assert np.abs(diag - diag_o).max() <= 1e-12 * np.abs(diag_o).max()


def test_unsupported_uses_rejected(native, cuda_ok):
    from subfv_b200 import meshgen
    from subfv_b200.mesh import Mesh
    from subfv_b200.ns import NsBatch, NsState
    with pytest.raises(Exception):
        NsBatch(_cfg("hex", "neumann"), capacity=2, budget_bytes=1 << 30)
    m = Mesh.from_raw(_raws()["hex"])
    with pytest.raises(Exception):
        NsState(m, _cfg("hex", "neumann", bc_type_V=[3, 0, 0, 0]), _state(m.n_elems))
    with pytest.raises(Exception):
        NsState(m, _cfg("hex", "neumann", prandtl=-1.0), _state(m.n_elems))


def test_states_of_different_meshes_coexist(native, oracle_lib, cuda_ok):
    """A state on a mesh with larger vertex systems keeps running after one on a smaller
    mesh is created (the kernel's shared-memory allowance only grows)."""
    from subfv_b200.ns import NsState
    raws = _raws()
    mb, ob = _pair(raws["box"])
    ms = _pair(raws["hex"])[0]
    cfg = _cfg("box", "neumann")
    sol = _state(mb.n_elems, seed=4)
    big = NsState(mb, cfg, sol)
    small = NsState(ms, _cfg("hex", "neumann"), _state(ms.n_elems))
    assert small.advance(2)[0] == 0
    st, n, _ = big.advance(3)
    sol_o = sol.copy()
    st_o, it, _, _, _, _ = ob.ns_run(cfg.oracle_dict(), sol_o, 2)
    assert st == st_o == 0 and n == it
    np.testing.assert_array_equal(big.sol(), sol_o)
    big.close()
    small.close()


def test_stencil_built_on_first_diffusion_state(native, oracle_lib, cuda_ok):
    """A mesh holds no diffusion stencil until a state with the diffusion terms asks for
    it (a second-order inviscid state adds only the nodal-gradient pseudo-inverses, 72
    bytes per vertex); a second such state reuses it, and the residual is the oracle's
    either way."""
    from subfv_b200.ns import NsState, compute_rhs_ns_diag
    raw = _raws()["box_periodic"]
    m, o = _pair(raw)
    before = m.device_bytes
    NsState(m, _cfg("box_periodic", "neumann", activate_diffusion=False), _state(m.n_elems)).close()
    assert m.device_bytes == before + 72 * m.n_vert  # no diffusion arrays
    cfg = _cfg("box_periodic", "neumann")
    sol = _state(m.n_elems)
    st, rhs, sl, diag = compute_rhs_ns_diag(m, cfg, sol)
    grown = m.device_bytes
    assert grown > before
    st2, rhs2, _, diag2 = compute_rhs_ns_diag(m, cfg, sol)
    assert m.device_bytes == grown
    np.testing.assert_array_equal(rhs, rhs2)
    np.testing.assert_array_equal(diag, diag2)
    st_o, rhs_o, sl_o, diag_o = o.ns_rhs_diag(cfg.oracle_dict(), sol)
    assert st == st_o == 0
    np.testing.assert_array_equal(rhs, rhs_o)


def test_cached_and_recomputed_paths_agree(native, oracle_lib, cuda_ok):
    """With a constant viscosity the first diffusion state on a mesh stores each vertex's
    state-independent arrays (the systems' inverses and products) and later evaluations
    use them; a state with other constants on the same mesh recomputes them every time.
    Both are the oracle's bit for bit, on a periodic box and on a slab with Dirichlet walls."""
    from subfv_b200.ns import compute_rhs_ns_diag
    for mesh_name, diff_name in (("box_periodic", "neumann"), ("hex", "dirichlet")):
        m, o = _pair(_raws()[mesh_name])
        sol = _state(m.n_elems)
        sizes = []
        for mu in (0.02, 0.05, 0.02):  # builds the cache, recomputes, reads the cache
            cfg = _cfg(mesh_name, diff_name, mu_p=mu)
            st, rhs, sl, diag = compute_rhs_ns_diag(m, cfg, sol)
            st_o, rhs_o, sl_o, diag_o = o.ns_rhs_diag(cfg.oracle_dict(), sol)
            assert st == st_o == 0
            np.testing.assert_array_equal(rhs, rhs_o, err_msg=f"{mesh_name} mu {mu}")
            np.testing.assert_array_equal(diag, diag_o, err_msg=f"{mesh_name} mu {mu}")
            sizes.append(m.device_bytes)
        assert sizes[0] == sizes[1] == sizes[2]  # one cache, built once


def test_cache_follows_geometry_changes(native, oracle_lib, cuda_ok):
    """The cached diffusion arrays belong to one geometry: after the vertices move
    (subfv_mesh_set_coords, then subfv_compute_geometry_mesh) a new state refills them,
    and its residual is the oracle's on the moved mesh."""
    from dataclasses import replace as dc_replace
    from oracle.oracle import OracleMesh
    from subfv_b200.ns import compute_rhs_ns_diag
    raw = _raws()["hex"]
    m, o = _pair(raw)
    cfg = _cfg("hex", "dirichlet")
    sol = _state(m.n_elems)
    st, rhs, _, diag = compute_rhs_ns_diag(m, cfg, sol)
    st_o, rhs_o, _, diag_o = o.ns_rhs_diag(cfg.oracle_dict(), sol)
    np.testing.assert_array_equal(rhs, rhs_o)
    # move the interior vertices a little (the walls and the two z layers stay flat)
    c = raw.coords.copy()
    lo, hi = c.min(0), c.max(0)
    inner = (c[:, 0] > lo[0] + 1e-9) & (c[:, 0] < hi[0] - 1e-9) & (c[:, 1] > lo[1] + 1e-9) & (c[:, 1] < hi[1] - 1e-9)
    rng = np.random.default_rng(11)
    shift = rng.uniform(-0.02, 0.02, (len(c), 2)) / NX
    key = np.round(c[:, :2], 9)
    _, col = np.unique(key, axis=0, return_inverse=True)  # the same shift on both layers of a column
    c[inner, :2] += shift[col.ravel()][inner]
    raw2 = dc_replace(raw, coords=c)
    o2 = OracleMesh(raw2)
    m.set_coords(o2.geom("vert_coord"))
    assert m.compute_geometry_mesh() == 0
    st2, rhs2, _, diag2 = compute_rhs_ns_diag(m, cfg, sol)
    st2_o, rhs2_o, _, diag2_o = o2.ns_rhs_diag(cfg.oracle_dict(), sol)
    assert st2 == st2_o == 0
    assert not np.array_equal(rhs2_o, rhs_o)
    np.testing.assert_array_equal(rhs2, rhs2_o)
    np.testing.assert_array_equal(diag2, diag2_o)


def test_running_state_follows_geometry_changes(native, oracle_lib, cuda_ok):
    """A viscous state that keeps running after its mesh's vertices move drops its
    captured step loop and refills the cached diffusion arrays and nodal-gradient
    pseudo-inverses: eight steps on the first geometry and eight on the moved one equal
    the oracle's, bit for bit."""
    from dataclasses import replace as dc_replace
    from oracle.oracle import OracleMesh
    from subfv_b200.ns import NsState
    raw = _raws()["hex"]
    m, o = _pair(raw)
    cfg = _cfg("hex", "dirichlet")
    sol = _state(m.n_elems)
    s = NsState(m, cfg, sol)
    st, n, _ = s.advance(8)  # one captured graph of eight steps
    assert st == 0 and n == 8
    c = raw.coords.copy()
    lo, hi = c.min(0), c.max(0)
    inner = (c[:, 0] > lo[0] + 1e-9) & (c[:, 0] < hi[0] - 1e-9) & (c[:, 1] > lo[1] + 1e-9) & (c[:, 1] < hi[1] - 1e-9)
    rng = np.random.default_rng(13)
    shift = rng.uniform(-0.02, 0.02, (len(c), 2)) / NX
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
