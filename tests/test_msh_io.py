"""Mesh and solution files through the native host code: gmsh ASCII MSH 2 and 4 read as
read_mesh_msh does (src/mesh/mesh_reading_module.F90:154-1324), the VTU solution file of
write_sol_vtu (src/ns/ns_io_module.F90:403-884) and its restart reader (:1333-1382).
The MSH files are written here from generated meshes, in gmsh's published layouts; the
reader must give back the same mesh, with the boundary faces tagged by the position of
their physical group's name in bc_names."""
import xml.etree.ElementTree as ET

import numpy as np
import pytest

NX, NY = 5, 4
SIDES = {"xlo": 11, "xhi": 12, "ylo": 13, "yhi": 14}  # physical tags in the file


def _mesh(kind="hex"):
    from subfv_b200 import meshgen
    raw = meshgen.hex_slab(NX, NY, jitter=0.1, seed=3) if kind == "hex" else meshgen.prism_slab(
        NX, NY, -0.5, 0.5, -0.5, 0.5, -0.5, 0.5, jitter=0.05, seed=4)
    return meshgen.tag_slab_sides(raw, NX, NY, SIDES)  # bface_tag holds the physical tag


def _bfaces(raw):
    return [(raw.bface_vert[raw.bface_off[i]:raw.bface_off[i + 1]], int(raw.bface_tag[i]))
            for i in range(raw.bface_off.size - 1)]


def _elems(raw):
    return [(int(raw.elem_kind[i]), raw.elem_vert[raw.elem_vert_off[i]:raw.elem_vert_off[i + 1]])
            for i in range(raw.n_elems)]


def _write_msh2(path, raw):
    names = {v: k for k, v in SIDES.items()}
    with open(path, "w") as f:
        f.write("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$PhysicalNames\n%d\n" % (len(names) + 1))
        for tag, name in names.items():
            f.write('2 %d "%s"\n' % (tag, name))
        f.write('3 99 "fluid"\n$EndPhysicalNames\n$Nodes\n%d\n' % raw.n_vert)
        for i, c in enumerate(raw.coords):
            f.write("%d %.17g %.17g %.17g\n" % (i + 1, *c))
        f.write("$EndNodes\n$Elements\n")
        lines = []
        for v, tag in _bfaces(raw):
            lines.append((3, [tag, 1], v))
        for kind, v in _elems(raw):
            lines.append((kind, [99, 2], v))
        f.write("%d\n" % len(lines))
        for i, (kind, tags, v) in enumerate(lines):
            f.write("%d %d %d %s %s\n" % (i + 1, kind, len(tags), " ".join(map(str, tags)), " ".join(map(str, v))))
        f.write("$EndElements\n")


def _write_msh4(path, raw, node_tag):
    """MSH 4.1 with node tags node_tag[i] for vertex i, one surface entity per side
    (surface 4 carries a second physical group first), two node blocks and an extra node
    no volume uses."""
    names = {v: k for k, v in SIDES.items()}
    with open(path, "w") as f:
        f.write("$MeshFormat\n4.1 0 8\n$EndMeshFormat\n$PhysicalNames\n%d\n" % (len(names) + 2))
        for tag, name in names.items():
            f.write('2 %d "%s"\n' % (tag, name))
        f.write('2 50 "other"\n3 99 "fluid"\n$EndPhysicalNames\n')
        f.write("$Entities\n1 0 4 1\n1 0 0 0 0\n")
        for s, tag in enumerate(SIDES.values()):
            phys = [50, tag] if s == 3 else [tag]
            f.write("%d -1 -1 -1 1 1 1 %d %s 0\n" % (s + 1, len(phys), " ".join(map(str, phys))))
        f.write("1 -1 -1 -1 1 1 1 1 99 4 1 2 3 4\n$EndEntities\n")
        n = raw.n_vert
        half = n // 2
        blocks = [(list(range(half)), 3), (list(range(half, n)), 3)]
        f.write("$Nodes\n3 %d 1 %d\n" % (n + 1, max(node_tag) + 5))
        f.write("0 1 0 1\n%d\n0.25 0.25 9\n" % (max(node_tag) + 5))
        for ids, dim in blocks:
            f.write("%d 1 0 %d\n" % (dim, len(ids)))
            for i in ids:
                f.write("%d\n" % node_tag[i])
            for i in ids:
                f.write("%.17g %.17g %.17g\n" % tuple(raw.coords[i]))
        f.write("$EndNodes\n")
        by_side = {}
        for v, tag in _bfaces(raw):
            by_side.setdefault(tag, []).append(v)
        kinds = {}
        for kind, v in _elems(raw):
            kinds.setdefault(kind, []).append(v)
        blocks = [(2, s + 1, 3, by_side[tag]) for s, tag in enumerate(SIDES.values())]
        blocks += [(3, 1, kind, vs) for kind, vs in kinds.items()]
        blocks.insert(0, (1, 1, 1, [[1, 2]]))  # a line element, skipped
        ne = sum(len(b[3]) for b in blocks)
        f.write("$Elements\n%d %d 1 %d\n" % (len(blocks), ne, ne))
        k = 1
        for dim, etag, kind, vs in blocks:
            f.write("%d %d %d %d\n" % (dim, etag, kind, len(vs)))
            for v in vs:
                vv = v if dim == 1 else [node_tag[x - 1] for x in v]
                f.write("%d %s\n" % (k, " ".join(map(str, vv))))
                k += 1
        f.write("$EndElements\n")


BC_NAMES = ["yhi", "xlo", "ylo", "xhi"]  # the reference's bc_name order, not the file's


def _expected_tags(raw):
    inv = {v: k for k, v in SIDES.items()}
    return np.array([BC_NAMES.index(inv[t]) + 1 for t in raw.bface_tag], np.int32)


@pytest.mark.parametrize("kind", ["hex", "prism"])
def test_msh2_round_trip(native, tmp_path, kind):
    from subfv_b200.io import read_msh
    raw = _mesh(kind)
    p = tmp_path / "m2.msh"
    _write_msh2(p, raw)
    got = read_msh(p, BC_NAMES)
    np.testing.assert_array_equal(got.coords, raw.coords)
    for a in ("elem_kind", "elem_vert_off", "elem_vert", "bface_off", "bface_vert"):
        np.testing.assert_array_equal(getattr(got, a), getattr(raw, a), a)
    np.testing.assert_array_equal(got.bface_tag, _expected_tags(raw))
    assert (read_msh(p).bface_tag == 0).all()  # no bc names: every face untagged


@pytest.mark.parametrize("kind", ["hex", "prism"])
def test_msh4_round_trip_renumbers_nodes(native, tmp_path, kind):
    from subfv_b200.io import read_msh
    raw = _mesh(kind)
    rng = np.random.default_rng(1)
    node_tag = list(rng.permutation(np.arange(10, 10 + 3 * raw.n_vert))[:raw.n_vert])
    p = tmp_path / "m4.msh"
    _write_msh4(p, raw, node_tag)
    got = read_msh(p, BC_NAMES)
    # the reader numbers the used nodes in their order in $Nodes, which is the original order
    np.testing.assert_array_equal(got.coords, raw.coords)
    for a in ("elem_kind", "elem_vert_off", "bface_off"):
        np.testing.assert_array_equal(getattr(got, a), getattr(raw, a), a)
    # volumes come grouped by element type; for one type the order is the file's
    np.testing.assert_array_equal(got.elem_vert, raw.elem_vert)
    np.testing.assert_array_equal(np.sort(got.bface_vert), np.sort(raw.bface_vert))
    # faces come side by side; each keeps the tag of its side's name
    tags = {tuple(sorted(v)): t for v, t in zip([got.bface_vert[got.bface_off[i]:got.bface_off[i + 1]]
                                                 for i in range(got.bface_off.size - 1)], got.bface_tag)}
    exp = _expected_tags(raw)
    for (v, _), t in zip(_bfaces(raw), exp):
        assert tags[tuple(sorted(v))] == t


def test_msh_mesh_builds_same_topology(native, tmp_path):
    from subfv_b200.io import read_msh
    from subfv_b200.mesh import Topology
    raw = _mesh("prism")
    p = tmp_path / "m2.msh"
    _write_msh2(p, raw)
    got = read_msh(p, BC_NAMES)
    raw.bface_tag = _expected_tags(raw)
    a, b = Topology(raw), Topology(got)
    for name in ("face_vert", "face_left", "face_right", "sub_face_loc", "elem_tag"):
        np.testing.assert_array_equal(a.array(name), b.array(name), name)
    assert (b.array("face_right") < 0).any()
    a.close()
    b.close()


def test_msh_errors(native, tmp_path):
    from subfv_b200._lib import SubfvError
    from subfv_b200.io import read_msh
    with pytest.raises(SubfvError):
        read_msh(tmp_path / "missing.msh")
    p = tmp_path / "bin.msh"
    p.write_text("$MeshFormat\n4.1 1 8\n$EndMeshFormat\n")
    with pytest.raises(SubfvError):
        read_msh(p)
    q = tmp_path / "nonames.msh"
    raw = _mesh("hex")
    _write_msh2(q, raw)
    text = q.read_text()
    start, end = text.index("$PhysicalNames"), text.index("$EndPhysicalNames") + len("$EndPhysicalNames\n")
    q.write_text(text[:start] + text[end:])
    with pytest.raises(SubfvError):
        read_msh(q, ["xlo"])
    assert read_msh(q).n_elems == raw.n_elems


def test_vtu_write_and_restart(native, tmp_path):
    from subfv_b200.io import restart_from_vtu, write_sol_vtu
    from subfv_b200.mesh import Topology
    raw = _mesh("hex")
    topo = Topology(raw)
    rng = np.random.default_rng(2)
    n = raw.n_elems
    w = np.column_stack([rng.uniform(0.5, 2, n), rng.uniform(-1, 1, (n, 3)), rng.uniform(0.5, 2, n)])
    sol = np.column_stack([w[:, 0], w[:, 1:4] * w[:, :1], w[:, 4] / 0.4 + 0.5 * w[:, 0] * (w[:, 1:4] ** 2).sum(1)])
    delta = rng.normal(size=(n, 5))
    vp = rng.normal(size=(raw.n_vert, 3))
    p = tmp_path / "sol.vtu"
    write_sol_vtu(p, topo, sol, delta=delta, vp=vp, Cv_p=2.5, mu=0.01)
    root = ET.parse(p).getroot()
    piece = root.find("UnstructuredGrid/Piece")
    assert int(piece.get("NumberOfCells")) == n and int(piece.get("NumberOfPoints")) == raw.n_vert
    arrays = {a.get("Name"): a for a in root.iter("DataArray")}
    for name in ("Points", "connectivity", "offsets", "types", "faces", "faceoffsets", "Nodal_Velocity", "Density",
                 "Momentum", "Energy", "Velocity", "Pressure", "Internal_energy", "H", "Mach", "Temperature", "mu",
                 "Residual", "Tag"):
        assert name in arrays, name
    vals = lambda name: np.array(arrays[name].text.split(), float)
    np.testing.assert_allclose(vals("Pressure"), w[:, 4], rtol=1e-13)
    np.testing.assert_allclose(vals("Velocity").reshape(-1, 3), w[:, 1:4], rtol=1e-13, atol=1e-15)
    np.testing.assert_allclose(vals("Temperature"), w[:, 4] / w[:, 0] / 0.4 / 2.5, rtol=1e-13)
    np.testing.assert_allclose(vals("Residual"), np.linalg.norm(delta, axis=1), rtol=1e-14)
    np.testing.assert_array_equal(vals("types"), 42)
    np.testing.assert_array_equal(vals("offsets"), raw.elem_vert_off[1:])
    back = restart_from_vtu(p, n)
    np.testing.assert_array_equal(back[:, :4], sol[:, :4])
    np.testing.assert_allclose(back[:, 4], sol[:, 4], rtol=4e-16)
    topo.close()


@pytest.mark.gpu
def test_msh_mesh_runs_on_gpu_like_oracle(native, oracle_lib, cuda_ok, tmp_path):
    """A mesh read from an MSH file, with freestream / outflow / adherence-wall tags by
    name, gives the oracle's residual bit for bit on the GPU."""
    from oracle.oracle import OracleMesh
    from subfv_b200.io import read_msh
    from subfv_b200.mesh import Mesh
    from subfv_b200.ns import NsConfig, compute_rhs_ns
    raw = _mesh("prism")
    p = tmp_path / "m4.msh"
    _write_msh4(p, raw, list(range(1, raw.n_vert + 1)))
    got = read_msh(p, BC_NAMES)
    m, o = Mesh.from_raw(got), OracleMesh(got)
    # BC_NAMES order: yhi, xlo, ylo, xhi
    cfg = NsConfig(scheme=1, second_order=True, method=4, bc_style=2, boundary_2d=True, cfl=0.3,
                   bc_type=[4, 3, 2, 4], bc_val=[[0] * 5, [1.2, 0.1, 0, 0, 1.0], [1.0, 0.05, 0, 0, 1.0], [0] * 5])
    rng = np.random.default_rng(3)
    n = m.n_elems
    w = np.column_stack([rng.uniform(1.1, 1.3, n), rng.uniform(-0.1, 0.1, (n, 2)), np.zeros(n),
                         rng.uniform(0.9, 1.1, n)])
    sol = np.ascontiguousarray(np.column_stack([w[:, 0], w[:, 1:4] * w[:, :1],
                                                w[:, 4] / 0.4 + 0.5 * w[:, 0] * (w[:, 1:4] ** 2).sum(1)]))
    st, rhs, sl, _, _ = compute_rhs_ns(m, cfg, sol)
    st_o, rhs_o, sl_o, _, _ = o.ns_rhs(cfg.oracle_dict(), sol)
    assert st == st_o == 0
    np.testing.assert_array_equal(rhs, rhs_o)
    np.testing.assert_array_equal(sl, sl_o)


def test_lagrangian_vtu(native, tmp_path):
    """write_sol_vtu_lag's fields from a Lagrangian state (tau, u, v, w, E)."""
    from subfv_b200.io import write_sol_vtu_lag
    from subfv_b200.mesh import Topology
    raw = _mesh("prism")
    topo = Topology(raw)
    rng = np.random.default_rng(4)
    n = raw.n_elems
    tau = rng.uniform(0.5, 2, n)
    u = rng.uniform(-1, 1, (n, 3))
    p = rng.uniform(0.5, 2, n)
    E = p * tau / 0.4 + 0.5 * (u ** 2).sum(1)
    sol = np.column_stack([tau, u, E])
    vp = rng.normal(size=(raw.n_vert, 3))
    cc = rng.normal(size=(n, 3))
    path = tmp_path / "lag.vtu"
    write_sol_vtu_lag(path, topo, sol, vp, pp=np.ones(raw.n_vert), elem_coord=cc)
    root = ET.parse(path).getroot()
    arrays = {a.get("Name"): np.array(a.text.split(), float) for a in root.iter("DataArray")}
    np.testing.assert_allclose(arrays["Density"], 1 / tau, rtol=1e-15)
    np.testing.assert_allclose(arrays["Pressure"], p, rtol=1e-13)
    np.testing.assert_allclose(arrays["Internal_energy"], p * tau / 0.4, rtol=1e-13)
    np.testing.assert_allclose(arrays["Rxy"], np.hypot(cc[:, 0], cc[:, 1]), rtol=1e-14)
    np.testing.assert_allclose(arrays["Vp"].reshape(-1, 3), vp, rtol=1e-15)
    assert arrays["Pp"].size == raw.n_vert and arrays["Tag"].size == n
    topo.close()


def test_msh_mesh_runs_in_the_oracle(native, oracle_lib, tmp_path):
    """A named-boundary MSH mesh drives the oracle's explicit loop: freestream entering
    through one side leaves through the supersonic-outflow side."""
    from oracle.oracle import OracleMesh
    from subfv_b200.io import read_msh
    raw = _mesh("hex")
    p = tmp_path / "m2.msh"
    _write_msh2(p, raw)
    got = read_msh(p, ["xlo", "xhi", "ylo", "yhi"])
    o = OracleMesh(got)
    n = o.n_elems
    w = np.tile([1.0, 0.0, 0.0, 0.0, 1.0], (n, 1))
    sol = np.ascontiguousarray(np.column_stack([w[:, 0], w[:, 1:4] * w[:, :1], w[:, 4] / 0.4]))
    inflow = [1.2, 0.5, 0.0, 0.0, 1.3]
    cfg = dict(scheme=1, second_order=1, method=4, bc_style=2, b2d=1, exclude_bound_vert=0, local_time_step=0,
               cfl=0.3, tmax=1e30, n_bc=4, bc_type=np.array([3, 4, 1, 1], np.int32),
               bc_val=np.array([inflow, [0] * 5, [0] * 5, [0] * 5], float))
    st, it, t, _, _, _ = o.ns_run(cfg, sol, 29)
    assert st == 0 and it == 30 and np.isfinite(sol).all()
    x = o.geom("elem_coord")[:, 0]
    left = sol[x < x.min() + 0.2]
    assert left[:, 0].mean() > 1.05 and left[:, 1].mean() > 0.1  # the inflow has come in
