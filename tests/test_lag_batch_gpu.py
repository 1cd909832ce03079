"""Batched Lagrangian hydro: Sedov problems of uneven size, CFL number and end time
advanced together in shared launches end, each, with the result of the same problem run
alone through LagrangeState (state, time, step count and moved mesh, bit for bit),
whatever the grid, the order of admission or the other problems in the batch."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _cases():
    """(raw mesh, cfl, t_max) of uneven size: prism and hex slabs."""
    from subfv_b200 import meshgen
    return [
        (meshgen.prism_slab(12, 12, 0.0, 1.2, 0.0, 1.2, 0.0, 0.1, jitter=0.05, seed=3), 0.5, 0.3),
        (meshgen.prism_slab(20, 16, 0.0, 1.2, 0.0, 1.2, 0.0, 0.1, jitter=0.05, seed=4), 0.4, 1.0),
        (meshgen.hex_slab(9, 11, 0.0, 1.2, 0.0, 1.2, 0.0, 0.1, jitter=0.05, seed=5), 0.5, 0.05),
        (meshgen.prism_slab(5, 7, 0.0, 1.2, 0.0, 1.2, 0.0, 0.1, jitter=0.0, seed=0), 0.3, 0.2),
    ]


def _problem(raw):
    from subfv_b200 import meshgen
    from subfv_b200.lagrange import init_sol_sedov
    from subfv_b200.mesh import Mesh
    m = Mesh.from_raw(raw)
    t = m.topo
    mask = meshgen.sedov_origin_mask(t.array("elem_vert_off"), t.array("elem_vert"), t.coords())
    sol = init_sol_sedov(m, e_total=0.244816, mask=mask)
    return m, sol


def _solo(raw, cfl, t_max, n_steps, precision):
    from subfv_b200.lagrange import LagrangeState
    m, sol = _problem(raw)
    s = LagrangeState(m, sol, cfl=cfl, t_max=t_max, precision=precision)
    st, steps, t = s.advance(n_steps)
    from subfv_b200 import _lib
    from subfv_b200._lib import pd
    out = np.empty((m.n_elems, 5))
    _lib.check(_lib.load().subfv_lag_get_sol(s._h, pd(out)), "subfv_lag_get_sol")
    return st, steps, t, out, m.coords()


@pytest.mark.parametrize("precision", [0, 1])
def test_lag_batch_equals_solo(native, cuda_ok, precision):
    from subfv_b200.lagrange import LagBatch
    cases = _cases()
    n_steps = 29
    b = LagBatch(capacity=8, budget_bytes=1 << 34, precision=precision)
    probs = []
    for raw, cfl, t_max in cases:
        m, sol = _problem(raw)
        probs.append((m, b.add(m, sol, t_max, cfl=cfl)))
    b.advance(16)
    b.advance(n_steps - 16)
    b.sync()
    for (raw, cfl, t_max), (m, k) in zip(cases, probs):
        st, steps, t, ref, xref = _solo(raw, cfl, t_max, n_steps, precision)
        bt, bsteps, bdone, bst = b.info(k)
        assert bst == st == 0
        assert bsteps == steps and bt == t
        assert bdone == (t >= t_max)
        np.testing.assert_array_equal(b.sol(k, m.n_elems), ref)
        np.testing.assert_array_equal(m.coords(), xref)
    b.close()


def test_lag_batch_join_leave_and_grid(native, cuda_ok):
    from subfv_b200.lagrange import LagBatch
    cases = _cases()
    b = LagBatch(capacity=2, budget_bytes=1 << 34)
    b.set_grid(5)
    pending = list(range(len(cases)))
    live, steps_of, results = {}, {}, {}
    chunks = [7, 3, 12, 5, 9, 4]
    ci = 0
    while pending or live:
        while pending:
            i = pending[0]
            raw, cfl, t_max = cases[i]
            m, sol = _problem(raw)
            k = b.add(m, sol, t_max, cfl=cfl)
            if k is None:
                break
            pending.pop(0)
            live[k] = (i, m)
            steps_of[i] = 0
        n = chunks[ci % len(chunks)]
        ci += 1
        b.advance(n)
        for i, _ in live.values():
            steps_of[i] += n
        b.sync()
        k = min(live)
        i, m = live.pop(k)
        results[i] = (b.info(k), b.sol(k, m.n_elems), m.coords())
        b.remove(k)
    for i, ((t, steps, done, st), got, x) in results.items():
        raw, cfl, t_max = cases[i]
        st0, steps0, t0, ref, xref = _solo(raw, cfl, t_max, steps_of[i], 0)
        assert st == st0 == 0 and steps == steps0 and t == t0
        np.testing.assert_array_equal(got, ref)
        np.testing.assert_array_equal(x, xref)
    b.close()


def test_empty_lag_batch_advances_and_then_admits(native, cuda_ok):
    """An empty Lagrangian batch advances without error; a problem admitted afterwards
    ends with its solo state, and the batch can be emptied and advanced again."""
    from subfv_b200.lagrange import LagBatch
    raw, cfl, t_max = _cases()[0]
    b = LagBatch(capacity=2, budget_bytes=1 << 34)
    b.advance(4)
    b.sync()
    m, sol = _problem(raw)
    k = b.add(m, sol, t_max, cfl=cfl)
    assert k is not None
    b.advance(11)
    b.sync()
    t, steps, done, st = b.info(k)
    got, x = b.sol(k, m.n_elems), m.coords()
    b.remove(k)
    b.advance(3)
    b.sync()
    st0, steps0, t0, ref, x0 = _solo(raw, cfl, t_max, 11, 0)
    assert st == st0 == 0 and steps == steps0 and t == t0
    np.testing.assert_array_equal(got, ref)
    np.testing.assert_array_equal(x, x0)
    b.close()
