"""The optional space-filling-curve numbering (subfv_topology_build_ex, renumber 1):
vertices along a Hilbert curve, cells, faces and subfaces then numbered by the
reference's rules over that order. Checked on the CPU against the oracle's own
restatement of the same curve (bit-exact topology), against the curve's defining
property on a regular grid, and for locality against the breadth-first order."""
import numpy as np
import pytest

from meshes import topology_cases
from test_topology import ARRAYS


@pytest.mark.parametrize("case", list(topology_cases()))
def test_hilbert_topology_bit_exact(native, oracle_lib, case):
    from oracle.oracle import OracleMesh
    from subfv_b200.mesh import Topology
    raw = topology_cases()[case]
    t, o = Topology(raw, "hilbert"), OracleMesh(raw, renumber="hilbert")
    for name in ARRAYS:
        a, b = t.array(name), o.topo(name)
        assert a.shape == b.shape and np.array_equal(a, b), name
    assert np.array_equal(t.coords(), o.geom("vert_coord"))


def test_hilbert_order_is_a_hilbert_walk(native):
    """On a regular 2^k x 2^k slab (a column of two vertices per grid point) every step
    of a Hilbert walk goes to a grid neighbour: consecutive columns are one spacing apart
    and a column's two vertices are consecutive."""
    from subfv_b200 import meshgen
    from subfv_b200.mesh import Topology
    n = 15  # 16 x 16 vertex columns
    t = Topology(meshgen.hex_slab(n, n, jitter=0.0, seed=1), "hilbert")
    c = t.coords()
    assert c.shape[0] == 2 * (n + 1) ** 2
    xy = c[:, :2]
    assert np.allclose(xy[0::2], xy[1::2])  # top and bottom of a column together
    cols = xy[0::2]
    steps = np.abs(np.diff(cols, axis=0)).sum(1)
    h = 1.0 / n
    assert np.allclose(steps, h), np.unique(np.round(steps / h, 6))
    grid = np.round((cols - cols.min(0)) / h).astype(int)
    assert len({tuple(p) for p in grid}) == (n + 1) ** 2


def test_hilbert_is_a_permutation_with_better_locality(native):
    from subfv_b200 import meshgen
    from subfv_b200.mesh import Topology
    raw = meshgen.prism_slab(40, 40, 0.0, 1.2, 0.0, 1.2, 0.0, 0.1, jitter=0.05, seed=3)
    tb, th = Topology(raw, "bfs"), Topology(raw, "hilbert")
    cb, ch = tb.coords(), th.coords()
    key = lambda c: np.lexsort(c.T[::-1])
    assert np.array_equal(cb[key(cb)], ch[key(ch)])  # the same vertices
    for t in (tb, th):  # every cell keeps its vertex set
        assert t.n_elems == raw.n_elems

    def span(t):
        ev = t.array("elem_vert").reshape(-1, 6)
        return float(np.median(ev.max(1) - ev.min(1)))
    # most cells' vertices sit within a few records of each other along the curve, while
    # the breadth-first front puts a cell's bottom and top rows a front's width apart
    assert span(th) * 4 < span(tb), (span(th), span(tb))


def test_renumber_mode_checked(native):
    import ctypes as C
    from subfv_b200 import _lib, meshgen
    from subfv_b200.mesh import Topology
    with pytest.raises(ValueError):
        Topology(meshgen.hex_slab(2, 2), "morton")
    raw = meshgen.hex_slab(2, 2)
    lib = _lib.load()
    h = C.c_void_p()
    i32 = lambda a: np.ascontiguousarray(a, np.int32)
    bo, bv, bt = i32(raw.bface_off), i32(raw.bface_vert), i32(raw.bface_tag)
    k, o, v = i32(raw.elem_kind), i32(raw.elem_vert_off), i32(raw.elem_vert)
    c = np.ascontiguousarray(raw.coords.reshape(-1), np.float64)
    P = lambda a, t: a.ctypes.data_as(C.POINTER(t))
    rc = lib.subfv_topology_build_ex(raw.n_vert, P(c, C.c_double), raw.n_elems, P(k, C.c_int32), P(o, C.c_int32),
                                     P(v, C.c_int32), int(bo.size - 1), P(bo, C.c_int32), P(bv, C.c_int32),
                                     P(bt, C.c_int32), 1, 0, 7, C.byref(h))
    assert rc < 0 and b"renumber" in lib.subfv_last_error()
