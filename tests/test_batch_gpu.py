"""Batched explicit Euler: problems of uneven size advanced together in shared launches
give, each, the result of the same problem run alone (bit for bit), whatever the launch
shape, the order of admission, or the other problems in the batch; problems join and
leave while others run; admission respects the HBM budget."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _problems():
    """(raw mesh, init kind, seed, tmax) of uneven size and end time."""
    from subfv_b200 import meshgen
    return [
        (meshgen.hex_slab(12, 10, jitter=0.1, seed=31), "gresho", 1, 0.02),
        (meshgen.prism_slab(10, 9, -0.5, 0.5, -0.5, 0.5, -0.5, 0.5, jitter=0.05, seed=32), "gresho", 2, 0.05),
        (meshgen.hex_slab(33, 17, jitter=0.1, seed=33), "gresho", 3, 1e30),
        (meshgen.strip(300), "tube", 4, None),
        (meshgen.strip(41), "tube", 5, None),
        (meshgen.hex_slab(3, 2, jitter=0.0, seed=0), "gresho", 6, 0.01),
    ]


def _init(m, kind, seed):
    from subfv_b200 import shocktube
    from subfv_b200.ns import init_gresho
    if kind == "tube":
        tube = shocktube.sample(1, seed=seed, n_min=10, n_max=20)[0]
        return shocktube.initial_state(m, tube), tube.t_end
    sol = init_gresho(m, 0.1)
    rng = np.random.default_rng(seed)
    sol[:, 0] *= 1.0 + 0.02 * rng.uniform(-1, 1, m.n_elems)
    sol[:, 1:3] += 0.05 * rng.uniform(-1, 1, (m.n_elems, 2))
    return np.ascontiguousarray(sol), None


def _setup():
    from subfv_b200.mesh import Mesh
    out = []
    for raw, kind, seed, tmax in _problems():
        m = Mesh.from_raw(raw)
        sol, t_end = _init(m, kind, seed)
        out.append((m, sol, tmax if tmax is not None else t_end))
    return out


def _solo(m, cfg, sol, tmax, n_steps):
    from dataclasses import replace
    from subfv_b200.ns import NsState
    s = NsState(m, replace(cfg, tmax=tmax), sol)
    st, steps, t = s.advance(n_steps)
    return st, steps, t, s.sol()


CFGS = {
    "mp_o2": dict(scheme=1, second_order=True, method=4, bc_style=2, precision=0),
    "mp_o1_fp32": dict(scheme=1, second_order=False, method=4, bc_style=2, precision=1),
    "tw_o2_fp32": dict(scheme=4, second_order=True, method=4, bc_style=2, precision=1),
    "m3w_o2": dict(scheme=5, second_order=True, method=4, bc_style=2, precision=0),
    "iso_o1_fp32": dict(scheme=2, second_order=False, method=4, bc_style=2, precision=1),
    "mpph_o2": dict(scheme=8, second_order=True, method=4, bc_style=1, precision=0),
}


@pytest.mark.parametrize("cfg_name", list(CFGS))
def test_batch_equals_solo(native, cuda_ok, cfg_name):
    from subfv_b200.ns import NsBatch, NsConfig
    cfg = NsConfig(**CFGS[cfg_name], boundary_2d=True, cfl=0.4)
    probs = _setup()
    n_steps = 37
    b = NsBatch(cfg, capacity=16, budget_bytes=1 << 34)
    slots = [b.add(m, sol, tmax) for m, sol, tmax in probs]
    assert None not in slots
    b.advance(16)
    b.advance(n_steps - 16)
    b.sync()
    for (m, sol, tmax), k in zip(probs, slots):
        st, steps, t, ref = _solo(m, cfg, sol, tmax, n_steps)
        bt, bsteps, bdone, bst = b.info(k)
        assert bst == st == 0
        assert bsteps == steps and bt == t, (k, bsteps, steps, bt, t)
        assert bdone == (t >= tmax)
        np.testing.assert_array_equal(b.sol(k, m.n_elems), ref)
    b.close()


@pytest.mark.parametrize("shape", [(64, 1, 1), (256, 7, 3), (128, 10000, 10000)])
def test_batch_launch_shape_invariant(native, cuda_ok, shape):
    from subfv_b200.ns import NsBatch, NsConfig
    cfg = NsConfig(**CFGS["mp_o2"], boundary_2d=True, cfl=0.4)
    probs = _setup()
    res = []
    for sh in [(128, 148 * 8, 148 * 8), shape]:
        b = NsBatch(cfg, capacity=8, budget_bytes=1 << 34)
        b.set_launch(*sh)
        slots = [b.add(m, sol, tmax) for m, sol, tmax in probs]
        b.advance(11)
        b.sync()
        res.append([b.sol(k, m.n_elems) for (m, _, _), k in zip(probs, slots)])
        b.close()
    for a, c in zip(*res):
        np.testing.assert_array_equal(a, c)


def test_batch_join_and_leave(native, cuda_ok):
    """Problems admitted at different points of the run, and slots reused after removal,
    each end with their solo result (same number of steps from their own start)."""
    from subfv_b200.ns import NsBatch, NsConfig
    cfg = NsConfig(**CFGS["mp_o2"], boundary_2d=True, cfl=0.4)
    probs = _setup()
    b = NsBatch(cfg, capacity=3, budget_bytes=1 << 34)
    steps_of = {}   # problem index -> steps it was advanced in the batch
    live = {}       # slot -> problem index
    pending = list(range(len(probs)))
    chunk = [5, 9, 8, 3, 12, 7, 4, 6, 10, 2]
    ci = 0
    results = {}
    while pending or live:
        while pending:
            i = pending[0]
            m, sol, tmax = probs[i]
            k = b.add(m, sol, tmax)
            if k is None:
                break
            pending.pop(0)
            live[k] = i
            steps_of[i] = 0
        n = chunk[ci % len(chunk)]
        ci += 1
        b.advance(n)
        for i in live.values():
            steps_of[i] += n
        b.sync()
        # retire the oldest problem every round (done or not), keeping its state
        k = min(live, key=lambda s: (probs[live[s]][0].n_elems, s))
        i = live.pop(k)
        results[i] = (b.info(k), b.sol(k, probs[i][0].n_elems))
        b.remove(k)
    assert sorted(results) == list(range(len(probs)))
    for i, ((t, steps, done, st), got) in results.items():
        m, sol, tmax = probs[i]
        st0, steps0, t0, ref = _solo(m, cfg, sol, tmax, steps_of[i])
        assert st == st0 == 0 and steps == steps0 and t == t0
        np.testing.assert_array_equal(got, ref)
    b.close()


def test_batch_budget_and_ownership(native, cuda_ok):
    from subfv_b200 import meshgen
    from subfv_b200.mesh import Mesh
    from subfv_b200.ns import NsBatch, NsConfig, init_gresho
    cfg = NsConfig(**CFGS["mp_o1_fp32"], boundary_2d=True, cfl=0.4)
    m1 = Mesh.from_raw(meshgen.hex_slab(20, 20, jitter=0.1, seed=7))
    probe = NsBatch(cfg, capacity=1, budget_bytes=1 << 30)
    need = probe.state_bytes(m1) + m1.device_bytes
    probe.close()
    b = NsBatch(cfg, capacity=4, budget_bytes=int(1.5 * need))
    sol = init_gresho(m1, 0.1)
    k1 = b.add(m1, sol, 0.01)
    assert k1 is not None
    assert b.free_bytes() == int(1.5 * need) - need
    m2 = Mesh.from_raw(meshgen.hex_slab(20, 20, jitter=0.1, seed=8))
    assert b.add(m2, init_gresho(m2, 0.1), 0.01) is None  # over budget: not admitted
    b.advance(200)
    b.sync()
    t, steps, done, st = b.info(k1)
    assert done and t >= 0.01 and st == 0
    b.remove(k1)
    b.advance(1)  # the table rewrite releases the slot
    b.sync()
    assert b.size() == (0, 0)
    k2 = b.add(m2, init_gresho(m2, 0.1), 0.01, take_mesh=True)
    assert k2 is not None and m2._h is None
    b.advance(3)
    b.sync()
    assert b.info(k2)[1] == 3
    b.remove(k2)
    b.close()


NODE_CFGS = dict(CFGS, mp_o1_fp32flux=dict(scheme=1, second_order=False, method=4, bc_style=2, precision=2))


@pytest.mark.parametrize("cfg_name", list(NODE_CFGS))
def test_node_group_kernel_bitwise(native, cuda_ok, cfg_name):
    """The lane-per-subface node kernel (a group of 8/16/32 lanes per vertex, per-vertex
    sums in shared memory) gives the thread-per-vertex kernel's results bit for bit, solo
    and batched, on 2-D slabs and strips (up to 8 subfaces per vertex), prism slabs (16)
    and a periodic 3-D box (12), in groups of 8, 16 and 32 lanes."""
    from dataclasses import replace
    from subfv_b200 import meshgen
    from subfv_b200.mesh import Mesh
    from subfv_b200.ns import NsBatch, NsConfig, NsState, init_fourier_flow
    cfg = NsConfig(**NODE_CFGS[cfg_name], boundary_2d=True, cfl=0.4)
    probs = _setup()
    box = Mesh.from_raw(meshgen.hex_box(5, jitter=0.05, seed=3, periodic=True))
    box_sol = init_fourier_flow(box, seed=4)
    for m, sol, tmax in probs[:3]:
        out = []
        for lanes in (0, 1, 32):
            s = NsState(m, replace(cfg, tmax=tmax), sol)
            s.set_node_kernel(lanes)
            out.append((s.advance(9), s.sol()))
            s.close()
        for o in out[1:]:
            assert out[0][0] == o[0]
            np.testing.assert_array_equal(out[0][1], o[1])
    cfg3 = replace(cfg, boundary_2d=False, tmax=1e30)
    out = []
    for lanes in (0, 1):
        s = NsState(box, cfg3, box_sol)
        s.set_node_kernel(lanes)
        out.append((s.advance(5), s.sol()))
        s.close()
    assert out[0][0] == out[1][0]
    np.testing.assert_array_equal(out[0][1], out[1][1])
    res = []
    for lanes, shape in ((0, (128, 148 * 8, 148 * 8)), (1, (128, 148 * 8, 148 * 8)), (1, (64, 5, 3)),
                         (32, (256, 300, 7))):
        b = NsBatch(cfg, capacity=8, budget_bytes=1 << 34)
        b.set_launch(*shape)
        b.set_node_kernel(lanes)
        slots = [b.add(m, sol, tmax) for m, sol, tmax in probs]
        b.advance(13)
        b.sync()
        res.append([b.sol(k, m.n_elems) for (m, _, _), k in zip(probs, slots)])
        b.close()
    for other in res[1:]:
        for a, c in zip(res[0], other):
            np.testing.assert_array_equal(a, c)


def test_empty_batch_advances_and_then_admits(native, cuda_ok):
    """An empty batch (none admitted yet, or all removed) advances without error and
    without touching anything; a problem admitted afterwards still gets its solo result."""
    from subfv_b200.ns import NsBatch, NsConfig
    cfg = NsConfig(**CFGS["mp_o1_fp32"], boundary_2d=True, cfl=0.4)
    m, sol, tmax = _setup()[0]
    b = NsBatch(cfg, capacity=2, budget_bytes=1 << 34)
    b.advance(7)
    b.sync()
    k = b.add(m, sol, tmax)
    assert k is not None
    b.advance(9)
    b.sync()
    t, steps, done, st = b.info(k)
    got = b.sol(k, m.n_elems)
    b.remove(k)
    b.advance(5)  # empty again
    b.sync()
    st0, steps0, t0, ref = _solo(m, cfg, sol, tmax, 9)
    assert st == st0 == 0 and steps == steps0 == 9 and t == t0
    np.testing.assert_array_equal(got, ref)
    b.close()
