"""The kernels on meshes numbered along a Hilbert curve (subfv_topology_build_ex,
renumber 1): the same arithmetic as on the breadth-first numbering, so the Lagrangian
time loop and the Navier-Stokes residual and loop are bit-identical to the oracle built
with the same numbering, and the conserved totals agree with the breadth-first mesh's to
round-off (only the order of the sums differs)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _pair(raw, renumber):
    from oracle.oracle import OracleMesh
    from subfv_b200.mesh import Mesh
    return Mesh.from_raw(raw, renumber=renumber), OracleMesh(raw, renumber=renumber)


def _sedov_run(m, steps):
    from subfv_b200 import meshgen
    from subfv_b200.lagrange import LagrangeState, init_sol_sedov
    t = m.topo
    mask = meshgen.sedov_origin_mask(t.array("elem_vert_off"), t.array("elem_vert"), t.coords())
    sol = init_sol_sedov(m, e_total=0.244816, mask=mask)
    mass = m.geometry("elem_volume") / sol[:, 0]
    s = LagrangeState(m, sol, mass, cfl=0.5, t_max=1.0)
    st, n, t_end = s.run(max_steps=steps)
    assert st == 0 and n == steps
    return sol, mass, s, t_end


def test_lagrange_sedov_on_hilbert_mesh_bit_exact(native, oracle_lib, cuda_ok):
    from subfv_b200 import meshgen
    raw = meshgen.prism_slab(24, 24, 0.0, 1.2, 0.0, 1.2, 0.0, 1.0, jitter=0.05, seed=2)
    m, o = _pair(raw, "hilbert")
    steps = 40
    sol0, mass, s, t = _sedov_run(m, steps)
    sol_o = sol0.copy()
    n_o, t_o, dt_o, vp_o = o.lag_run(sol_o, mass, 0.5, 1.0, steps)
    assert n_o == steps and t == t_o and s.last_dt() == dt_o
    np.testing.assert_array_equal(s.sol(), sol_o)
    np.testing.assert_array_equal(m.coords(), o.geom("vert_coord"))
    # the same physics as the breadth-first mesh: energy totals to round-off
    mb = _pair(raw, "bfs")[0]
    solb, massb, sb, tb = _sedov_run(mb, steps)
    eh = float((s.sol()[:, 4] * mass).sum())
    eb = float((sb.sol()[:, 4] * massb).sum())
    assert abs(eh - eb) <= 1e-12 * abs(eb)
    assert abs(t - tb) <= 1e-9 * tb


@pytest.mark.parametrize("box", [False, True])
def test_ns_residual_and_loop_on_hilbert_mesh_bit_exact(native, oracle_lib, cuda_ok, box):
    from subfv_b200 import meshgen
    from subfv_b200.ns import NsConfig, NsState, compute_rhs_ns, init_fourier_flow, init_gresho
    if box:
        raw = meshgen.hex_box(6, jitter=0.05, seed=3, periodic=True)
        cfg = NsConfig(scheme=4, second_order=True, method=4, bc_style=2, boundary_2d=False, cfl=0.4)
    else:
        raw = meshgen.hex_slab(16, 12, jitter=0.1, seed=4)
        cfg = NsConfig(cfl=0.4)
    m, o = _pair(raw, "hilbert")
    sol = init_fourier_flow(m, seed=2) if box else init_gresho(m, 0.1)
    st, rhs, sl, vp, grad = compute_rhs_ns(m, cfg, sol)
    st_o, rhs_o, sl_o, vp_o, grad_o = o.ns_rhs(cfg.oracle_dict(), sol)
    assert st == st_o == 0
    np.testing.assert_array_equal(rhs, rhs_o)
    np.testing.assert_array_equal(sl, sl_o)
    s = NsState(m, cfg, sol)
    st, n, t = s.advance(6)
    sol_o = sol.copy()
    st_o, it, t_o, _, _, _ = o.ns_run(cfg.oracle_dict(), sol_o, 5)
    assert st == st_o == 0 and n == it == 6 and t == t_o
    np.testing.assert_array_equal(s.sol(), sol_o)
    s.close()
