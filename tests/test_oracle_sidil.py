"""CPU checks of the oracle's scheme "sidil" (lagrange_module.F90:149-223, 538-809): a
gas at rest with uniform pressure gives zero nodal velocities and a residual that is
round-off (closed walls, the face pressures cancel around every cell)."""
import numpy as np


def test_sidil_rest_state(oracle_lib):
    from oracle.oracle import OracleMesh
    from subfv_b200 import meshgen
    o = OracleMesh(meshgen.prism_slab(6, 5, jitter=0.05, seed=8))
    n = o.n_elems
    tau, p = 0.8, 1.7
    sol = np.zeros((n, 5))
    sol[:, 0] = tau
    sol[:, 4] = p * tau / 0.4
    vol = o.geom("elem_volume")
    mass = vol / tau
    for method in (0, 1, 3):
        st, vp, rhs = o.lag_rhs_sidil(sol, mass, method)
        assert st == 0
        assert np.abs(vp).max() == 0.0
        assert np.abs(rhs).max() < 1e-11 * p * np.abs(1.0 / mass).max()
