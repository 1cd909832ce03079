"""build_mesh numbering: the product's linear-time builder against the oracle's
line-by-line restatement (src/mesh/mesh_connectivity_module.F90:12-59). Bit-exact."""
import numpy as np
import pytest

from meshes import topology_cases

ARRAYS = ["sizes", "elem_kind", "elem_tag", "elem_vert_off", "elem_vert", "elem_face_off", "elem_face",
          "elem_sub_face_off", "elem_sub_face", "elem_sub_elem", "elem_neigh_by_vert_off", "elem_neigh_by_vert",
          "face_vert_off", "face_vert", "face_sub_face", "face_left", "face_right", "face_left_face",
          "face_right_face", "sub_face_vert", "sub_face_face", "sub_face_left_elem", "sub_face_right_elem",
          "sub_face_left_sub_elem", "sub_face_right_sub_elem", "sub_face_loc", "sub_elem_elem", "sub_elem_vert",
          "sub_elem_loc", "sub_elem_sub_face_off", "sub_elem_sub_face", "vert_sub_face_off", "vert_sub_face",
          "vert_sub_elem_off", "vert_sub_elem", "vert_face_off", "vert_face", "vert_elem_off", "vert_elem",
          "vert_is_bound"]


@pytest.mark.parametrize("case", list(topology_cases()))
def test_topology_bit_exact(native, oracle_lib, case):
    from oracle.oracle import OracleMesh
    from subfv_b200.mesh import Topology
    raw = topology_cases()[case]
    t, o = Topology(raw), OracleMesh(raw)
    for name in ARRAYS:
        a, b = t.array(name), o.topo(name)
        assert a.shape == b.shape and np.array_equal(a, b), name
    assert np.array_equal(t.coords(), o.geom("vert_coord"))


def test_periodic_stitching_closes_all_faces(native):
    from subfv_b200 import meshgen
    from subfv_b200.mesh import Topology
    t = Topology(meshgen.hex_box(4, periodic=True))
    assert (t.array("face_right") > 0).all()
    # stencil extension: corner vertices see the subfaces of their 7 periodic images
    off = t.array("vert_sub_face_off")
    assert (np.diff(off) >= 12).all()


def test_disconnected_and_shuffled_input(native, oracle_lib):
    """Two components and a shuffled element order exercise the BFS restart and the
    first-touch renumbering."""
    from oracle.oracle import OracleMesh
    from subfv_b200 import meshgen
    from subfv_b200.meshgen import RawMesh
    from subfv_b200.mesh import Topology
    a = meshgen.hex_slab(3, 3, jitter=0.1, seed=5)
    b = meshgen.prism_slab(3, 2, x0=2.0, x1=3.0, jitter=0.1, seed=6)
    coords = np.concatenate([b.coords, a.coords])
    ev_a = a.elem_vert.reshape(-1, 8) + b.n_vert
    ev_b = b.elem_vert.reshape(-1, 6)
    rng = np.random.default_rng(7)
    elems = [("h", e) for e in ev_a] + [("p", e) for e in ev_b]
    order = rng.permutation(len(elems))
    kinds, flat, off = [], [], [0]
    for i in order:
        k, e = elems[i]
        kinds.append(5 if k == "h" else 6)
        flat.extend(e.tolist())
        off.append(len(flat))
    raw = RawMesh(coords, np.array(kinds, np.int32), np.array(off, np.int32), np.array(flat, np.int32))
    t, o = Topology(raw), OracleMesh(raw)
    for name in ARRAYS:
        assert np.array_equal(t.array(name), o.topo(name)), name


def test_bad_input_rejected(native):
    from subfv_b200._lib import SubfvError
    from subfv_b200.meshgen import RawMesh
    from subfv_b200.mesh import Topology
    raw = RawMesh(np.zeros((4, 3)), np.array([5], np.int32), np.array([0, 4], np.int32),
                  np.array([1, 2, 3, 4], np.int32))
    with pytest.raises(SubfvError):
        Topology(raw)
