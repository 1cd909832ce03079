"""The reference's coordinate maps applied before build_mesh: cylinder_mapping
(src/mesh/mesh_geometry_module.F90:413-518) keeps the body's radius and stretches the
outer boundary by its angle polynomial; rescale_mesh scales every coordinate."""
import numpy as np

R2 = 1.3851721918740656


def _raw(points):
    from subfv_b200.meshgen import KIND_TET, RawMesh
    pts = np.asarray(points, np.float64)
    return RawMesh(pts, np.full(1, KIND_TET, np.int32), np.array([0, 4], np.int32), np.array([1, 2, 3, 4], np.int32))


def test_cylinder_map_2d():
    from subfv_b200.meshgen import map_cylinder
    th = np.array([0.0, 0.4, 1.0, 1.5])
    body = np.column_stack([-np.cos(th), np.sin(th), [0.1, 0.2, 0.3, 0.4]])
    out = map_cylinder(_raw(body), 2).coords
    np.testing.assert_allclose(out, body, atol=1e-15)  # r = 1 stays on the body
    outer = np.column_stack([-R2 * np.cos(th), R2 * np.sin(th), np.zeros(4)])
    got = map_cylinder(_raw(outer), 2).coords
    want_r = (R2 + 0.22082080765324227 * th ** 2 + 0.07247276314520341 * th ** 4
              - 0.01622444200319442 * th ** 6 + 0.00780545523147566 * th ** 8)
    np.testing.assert_allclose(np.hypot(got[:, 0], got[:, 1]), want_r, rtol=1e-14)
    np.testing.assert_allclose(np.arctan2(got[:, 1], -got[:, 0]), th, atol=1e-14)
    half = map_cylinder(_raw(0.5 * outer), 21).coords
    np.testing.assert_allclose(half, 0.5 * got, rtol=1e-14, atol=1e-16)


def test_cylinder_map_3d_and_rescale():
    from subfv_b200.meshgen import map_cylinder, rescale_mesh
    rng = np.random.default_rng(0)
    d = rng.normal(size=(4, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    np.testing.assert_allclose(map_cylinder(_raw(d), 3).coords, d, atol=1e-15)
    raw = _raw(2.0 * d)
    np.testing.assert_array_equal(rescale_mesh(raw, 0.25).coords, 0.5 * d)
