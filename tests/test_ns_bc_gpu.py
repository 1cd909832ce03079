"""Boundary kinds of compute_right_state (src/ns/ns_euler_recon_module.F90:331-409) on the
GPU against the oracle, on slabs whose four sides carry tags: the adherence wall, the
pondered inflow (imposed where the given stream enters, copied where it leaves), the
double-Mach inflow/outflow (which reads the step's time) and bottom, are bit-identical in
the residual, the time loop, the batched engine and the backward-Euler Jacobian. The
potential flows evaluate atan2/cos/sin, whose last bits differ between CUDA's and the host
C library, so their residual is compared at 1e-12 of its scale in FP64 (1e-4 with the FP32
reconstruction and fluxes of precision 2). Unknown kinds are
rejected like the reference's select case, which stops on them."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NX, NY = 10, 8
TAGS = {"xlo": 1, "xhi": 2, "ylo": 3, "yhi": 4}
VALS = [[1.4, 0.2, 0.0, 0.0, 1.0], [1.4, 0.2, 0.0, 0.0, 1.0], [1.0, 0.05, 0.0, 0.0, 1.0], [1.0, 0.0, 0.0, 0.0, 1.0]]
KINDS = {
    "pond_pond_adh_dmach": (5, 5, 2, 6),
    "pond_dmach_adh_bottom": (5, 6, 2, 7),
    "free_out_bottom_dmach": (3, 4, 7, 6),
}


def _raws():
    from subfv_b200 import meshgen
    return {
        "hex": meshgen.tag_slab_sides(meshgen.hex_slab(NX, NY, jitter=0.1, seed=3), NX, NY, TAGS),
        "prism": meshgen.tag_slab_sides(
            meshgen.prism_slab(NX, NY, -0.5, 0.5, -0.5, 0.5, -0.5, 0.5, jitter=0.05, seed=4), NX, NY, TAGS),
    }


def _pair(raw):
    from oracle.oracle import OracleMesh
    from subfv_b200.mesh import Mesh
    return Mesh.from_raw(raw), OracleMesh(raw)


def _state(n, seed=5):
    rng = np.random.default_rng(seed)
    w = np.column_stack([rng.uniform(1.3, 1.5, n), rng.uniform(-0.1, 0.1, (n, 2)), np.zeros(n),
                         rng.uniform(0.9, 1.1, n)])
    return np.ascontiguousarray(np.column_stack([w[:, 0], w[:, 1:4] * w[:, :1],
                                                 w[:, 4] / 0.4 + 0.5 * w[:, 0] * (w[:, 1:4] ** 2).sum(1)]))


def _cfg(kinds, **kw):
    from subfv_b200.ns import NsConfig
    base = dict(scheme=1, second_order=True, method=4, bc_style=2, boundary_2d=True, cfl=0.3)
    base.update(kw)
    return NsConfig(**base, bc_type=list(kinds), bc_val=[list(v) for v in VALS[:len(kinds)]])


@pytest.mark.parametrize("mesh_name", ["hex", "prism"])
@pytest.mark.parametrize("kinds_name", list(KINDS))
@pytest.mark.parametrize("scheme,order", [(1, True), (4, False), (3, True)])
def test_rhs_boundary_kinds_bit_exact(native, oracle_lib, cuda_ok, mesh_name, kinds_name, scheme, order):
    from subfv_b200.ns import compute_rhs_ns
    m, o = _pair(_raws()[mesh_name])
    cfg = _cfg(KINDS[kinds_name], scheme=scheme, second_order=order)
    sol = _state(m.n_elems)
    st, rhs, sl, vp, grad = compute_rhs_ns(m, cfg, sol)
    st_o, rhs_o, sl_o, vp_o, grad_o = o.ns_rhs(cfg.oracle_dict(), sol)
    assert st == st_o == 0
    np.testing.assert_array_equal(sl, sl_o)
    np.testing.assert_array_equal(rhs, rhs_o)


@pytest.mark.parametrize("kinds_name", ["pond_pond_adh_dmach", "pond_dmach_adh_bottom"])
@pytest.mark.parametrize("t0", [0.0, 0.02])
def test_time_loop_boundary_kinds_bit_exact(native, oracle_lib, cuda_ok, kinds_name, t0):
    """The double-Mach kind reads the time of the step: both stages of a step see its
    start time, advanced after the step, on the device as in the oracle."""
    from subfv_b200.ns import NsState
    m, o = _pair(_raws()["hex"])
    cfg = _cfg(KINDS[kinds_name])
    sol = _state(m.n_elems)
    sol_o = sol.copy()
    st_o, it, t_o, _, _, _ = o.ns_run(cfg.oracle_dict(), sol_o, 7, t0=t0)
    for lanes in (0, 1):  # thread-per-vertex and lane-group node kernels
        s = NsState(m, cfg, sol, t0=t0)
        s.set_node_kernel(lanes)
        st, n, t = s.advance(8)
        assert st == st_o == 0 and n == it == 8 and t == t_o
        np.testing.assert_array_equal(s.sol(), sol_o)
        s.close()


def test_batch_boundary_kinds_equal_solo(native, cuda_ok):
    """Each batched problem reads its own time (two start times in one batch)."""
    from subfv_b200.mesh import Mesh
    from subfv_b200.ns import NsBatch, NsState
    raws = _raws()
    cfg = _cfg(KINDS["pond_dmach_adh_bottom"])
    probs = [(Mesh.from_raw(raws["hex"]), 0.0), (Mesh.from_raw(raws["prism"]), 0.02), (Mesh.from_raw(raws["hex"]), 0.02)]
    sols = [_state(m.n_elems, seed=7 + i) for i, (m, _) in enumerate(probs)]
    b = NsBatch(cfg, capacity=4, budget_bytes=1 << 32)
    slots = [b.add(m, s, 1e30, t0=t0) for (m, t0), s in zip(probs, sols)]
    assert None not in slots
    b.advance(6)
    b.sync()
    for ((m, t0), s0), k in zip(zip(probs, sols), slots):
        s = NsState(m, cfg, s0, t0=t0)
        st, n, t = s.advance(6)
        assert st == 0
        bt, bsteps, _, bst = b.info(k)
        assert bst == 0 and bsteps == n and bt == t
        np.testing.assert_array_equal(b.sol(k, m.n_elems), s.sol())
        s.close()
    b.close()


@pytest.mark.parametrize("kinds_name", list(KINDS))
def test_be_jacobian_boundary_kinds_bit_exact(native, oracle_lib, cuda_ok, kinds_name):
    from subfv_b200.ns import NsState
    m, o = _pair(_raws()["hex"])
    cfg = _cfg(KINDS[kinds_name], scheme=4, second_order=False, method=0)
    sol = _state(m.n_elems)
    s = NsState(m, cfg, sol)
    row, col, v = s.be_jacobian(0.011)
    ro, co, vo = o.be_jacobian(cfg.oracle_dict(), sol, 0.011)
    np.testing.assert_array_equal(row, ro)
    np.testing.assert_array_equal(col, co)
    np.testing.assert_array_equal(v, vo)
    s.close()


@pytest.mark.parametrize("kinds", [(8, 8, 8, 8), (9, 9, 9, 9), (8, 9, 1, 4)])
@pytest.mark.parametrize("precision", [0, 2])
def test_rhs_potential_flow_kinds_close(native, oracle_lib, cuda_ok, kinds, precision):
    from subfv_b200.ns import compute_rhs_ns
    m, o = _pair(_raws()["hex"])
    cfg = _cfg(kinds, precision=precision)
    sol = _state(m.n_elems)
    st, rhs, sl, _, _ = compute_rhs_ns(m, cfg, sol)
    st_o, rhs_o, sl_o, _, _ = o.ns_rhs(cfg.oracle_dict(), sol)
    assert st == st_o == 0
    tol = 1e-12 if precision == 0 else 1e-4
    np.testing.assert_allclose(sl, sl_o, rtol=tol)
    for k in range(5):
        scale = np.abs(rhs_o[:, k]).max() + np.abs(rhs_o[:, 1:3]).max()
        assert np.abs(rhs[:, k] - rhs_o[:, k]).max() <= tol * scale, k


@pytest.mark.parametrize("bad", [0, 10, -1])
def test_unknown_boundary_kind_rejected(native, cuda_ok, bad):
    from subfv_b200.mesh import Mesh
    from subfv_b200.ns import NsState
    m = Mesh.from_raw(_raws()["hex"])
    with pytest.raises(Exception):
        NsState(m, _cfg((1, bad, 1, 1)), _state(m.n_elems))
