"""Seeded synthetic meshes in the reference's native frames.

The reference is 3-D only: a "2-D" case is a one-cell-thick extruded slab whose
z-faces are walls (src/mesh/mesh_reading_module.F90:1144-1146; test/gresho_quad/
gresho_quad.geo extrudes one layer of thickness 1). Elements use the gmsh vertex
order the reference's MSH2 reader expects: hexahedron (kind 5) = bottom quad
counter-clockwise seen from +z then the top quad; prism (kind 6) = bottom triangle
counter-clockwise then the top triangle (mesh_reading_module.F90:1192-1278).

Interior vertices are jittered in x and y identically on both z-layers; boundary
vertices stay on the box so walls remain planar.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

KIND_TET, KIND_HEX, KIND_PRISM, KIND_PYRAMID = 4, 5, 6, 7
N_VERT_KIND = {KIND_TET: 4, KIND_HEX: 8, KIND_PRISM: 6, KIND_PYRAMID: 5}


@dataclass
class RawMesh:
    """A mesh as the reference reads it from MSH2: vertices and volume elements in
    file order, vertex ids 1-based; optional tagged boundary faces."""

    coords: np.ndarray  # (n_vert, 3) float64
    elem_kind: np.ndarray  # (n_elems,) int32
    elem_vert_off: np.ndarray  # (n_elems+1,) int32
    elem_vert: np.ndarray  # int32, 1-based vertex ids
    bface_off: np.ndarray = field(default_factory=lambda: np.zeros(1, np.int32))
    bface_vert: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    bface_tag: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    b2d: bool = True
    periodic: bool = False

    @property
    def n_vert(self) -> int:
        return int(self.coords.shape[0])

    @property
    def n_elems(self) -> int:
        return int(self.elem_kind.shape[0])


def _grid_xy(nx, ny, x0, x1, y0, y1, jitter, rng):
    xs = np.linspace(x0, x1, nx + 1)
    ys = np.linspace(y0, y1, ny + 1)
    X, Y = np.meshgrid(xs, ys, indexing="xy")  # (ny+1, nx+1), row j, column i
    if jitter > 0.0:
        hx = (x1 - x0) / nx
        hy = (y1 - y0) / ny
        dx = rng.uniform(-jitter * hx, jitter * hx, size=X.shape)
        dy = rng.uniform(-jitter * hy, jitter * hy, size=Y.shape)
        interior = np.zeros(X.shape, bool)
        interior[1:-1, 1:-1] = True
        X = np.where(interior, X + dx, X)
        Y = np.where(interior, Y + dy, Y)
    return X.ravel(), Y.ravel()


def _slab_coords(X, Y, z0, z1):
    n = X.size
    c = np.empty((2 * n, 3), np.float64)
    c[:n, 0] = X
    c[:n, 1] = Y
    c[:n, 2] = z0
    c[n:, 0] = X
    c[n:, 1] = Y
    c[n:, 2] = z1
    return c


def hex_slab(nx, ny, x0=-0.5, x1=0.5, y0=-0.5, y1=0.5, z0=-0.5, z1=0.5, jitter=0.0, seed=0):
    """nx*ny hexahedra, one layer thick (a quad mesh in the reference's 2-D mode)."""
    rng = np.random.default_rng(seed)
    X, Y = _grid_xy(nx, ny, x0, x1, y0, y1, jitter, rng)
    coords = _slab_coords(X, Y, z0, z1)
    nl = (nx + 1) * (ny + 1)
    j, i = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    a = (j * (nx + 1) + i).ravel()
    b, c, d = a + 1, a + nx + 2, a + nx + 1
    ev = np.stack([a, b, c, d, a + nl, b + nl, c + nl, d + nl], axis=1) + 1
    n = ev.shape[0]
    return RawMesh(coords, np.full(n, KIND_HEX, np.int32), (np.arange(n + 1) * 8).astype(np.int32),
                   ev.astype(np.int32).ravel(), b2d=True)


def _norm2(a):
    """gfortran's NORM2 (scaled sum of squares) over the last axis."""
    a = np.abs(np.asarray(a, np.float64))
    scale = np.ones(a.shape[:-1])
    res = np.zeros(a.shape[:-1])
    for i in range(a.shape[-1]):
        x = a[..., i]
        nz = x != 0.0
        big = nz & (x > scale)
        q = np.where(big, scale / np.where(big, x, 1.0), 0.0)
        res = np.where(big, 1.0 + res * q * q, res)
        scale = np.where(big, x, scale)
        small = nz & ~big
        q2 = np.where(small, x / scale, 0.0)
        res = np.where(small, res + q2 * q2, res)
    return scale * np.sqrt(res)


def map_cylinder(raw: RawMesh, dimen: int) -> RawMesh:
    """A copy with the vertices moved by cylinder_mapping (mesh_geometry_module.F90:413-518),
    the radial stretching the reference applies to its half-cylinder meshes before
    build_mesh (dimen 2: unit cylinder about z, 21: radius 0.5, 3: unit sphere)."""
    c = np.asarray(raw.coords, np.float64)
    x, y = c[:, 0], c[:, 1]
    if dimen == 2 or dimen == 21:
        s = 2.0 if dimen == 21 else 1.0
        r = _norm2(np.column_stack([s * x, s * y]))
        th = np.arctan2(s * y, -s * x)
    elif dimen == 3:
        r = _norm2(c)
        th = np.arctan2(_norm2(c[:, 1:]), -x)
    else:
        raise ValueError("dimen must be 2, 21 or 3")
    r1, r2 = 1.0, 1.3851721918740656
    t2 = th * th
    t4 = t2 * t2
    new_r2 = (r2 + 0.22082080765324227 * t2 + 0.07247276314520341 * t4 - 0.01622444200319442 * (t4 * t2)
              + 0.00780545523147566 * (t4 * t4))
    new_r = (r - r1) * (new_r2 - r1) / (r2 - r1) + r1
    out = c.copy()
    if dimen == 3:
        out = c + (new_r - r)[:, None] * c
    else:
        out[:, 0] = -new_r * np.cos(th) / s
        out[:, 1] = new_r * np.sin(th) / s
    return RawMesh(out, raw.elem_kind, raw.elem_vert_off, raw.elem_vert, raw.bface_off, raw.bface_vert,
                   raw.bface_tag, b2d=raw.b2d, periodic=raw.periodic)


def rescale_mesh(raw: RawMesh, sf: float) -> RawMesh:
    """A copy with every coordinate scaled by sf (mesh_reading_module.F90:1366-1377)."""
    return RawMesh(sf * np.asarray(raw.coords, np.float64), raw.elem_kind, raw.elem_vert_off, raw.elem_vert,
                   raw.bface_off, raw.bface_vert, raw.bface_tag, b2d=raw.b2d, periodic=raw.periodic)


def tag_slab_sides(raw: RawMesh, nx: int, ny: int, tags: dict) -> RawMesh:
    """A copy of a hex_slab / prism_slab mesh of nx*ny columns with its side boundaries
    tagged (the MSH2 boundary elements the reference reads): tags maps "xlo", "xhi",
    "ylo", "yhi" to a physical tag (1-based; a side left out stays a default wall)."""
    nl = (nx + 1) * (ny + 1)
    vid = lambda i, j: j * (nx + 1) + i
    edges = {"ylo": [(vid(i, 0), vid(i + 1, 0)) for i in range(nx)],
             "yhi": [(vid(i, ny), vid(i + 1, ny)) for i in range(nx)],
             "xlo": [(vid(0, j), vid(0, j + 1)) for j in range(ny)],
             "xhi": [(vid(nx, j), vid(nx, j + 1)) for j in range(ny)]}
    fv, ft = [], []
    for side, tag in tags.items():
        for p, q in edges[side]:
            fv.append([p + 1, q + 1, q + nl + 1, p + nl + 1])
            ft.append(int(tag))
    off = (np.arange(len(fv) + 1) * 4).astype(np.int32)
    return RawMesh(raw.coords, raw.elem_kind, raw.elem_vert_off, raw.elem_vert, off,
                   np.asarray(fv, np.int32).reshape(-1), np.asarray(ft, np.int32), b2d=raw.b2d,
                   periodic=raw.periodic)


def prism_slab(nx, ny, x0=0.0, x1=1.2, y0=0.0, y1=1.2, z0=0.0, z1=1.0, jitter=0.0, seed=0):
    """Each square split into two triangles along alternating diagonals, extruded
    one layer: 2*nx*ny prisms (a triangle mesh in the reference's 2-D mode)."""
    rng = np.random.default_rng(seed)
    X, Y = _grid_xy(nx, ny, x0, x1, y0, y1, jitter, rng)
    coords = _slab_coords(X, Y, z0, z1)
    nl = (nx + 1) * (ny + 1)
    j, i = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    a = (j * (nx + 1) + i).ravel()
    b, c, d = a + 1, a + nx + 2, a + nx + 1
    alt = ((i + j) % 2 == 0).ravel()
    # diagonal a-c when alt, else b-d; both triangles counter-clockwise
    t1 = np.where(alt[:, None], np.stack([a, b, c], 1), np.stack([a, b, d], 1))
    t2 = np.where(alt[:, None], np.stack([a, c, d], 1), np.stack([b, c, d], 1))
    tri = np.stack([t1, t2], axis=1).reshape(-1, 3)
    ev = np.concatenate([tri, tri + nl], axis=1) + 1
    n = ev.shape[0]
    return RawMesh(coords, np.full(n, KIND_PRISM, np.int32), (np.arange(n + 1) * 6).astype(np.int32),
                   ev.astype(np.int32).ravel(), b2d=True)


def hex_box(n, lo=-0.5, hi=0.5, jitter=0.0, seed=0, periodic=True):
    """n^3 hexahedra on [lo,hi]^3; interior vertices jittered in x, y and z."""
    rng = np.random.default_rng(seed)
    xs = np.linspace(lo, hi, n + 1)
    Z, Y, X = np.meshgrid(xs, xs, xs, indexing="ij")
    if jitter > 0.0:
        h = (hi - lo) / n
        interior = np.zeros(X.shape, bool)
        interior[1:-1, 1:-1, 1:-1] = True
        for A in (X, Y, Z):
            A[interior] += rng.uniform(-jitter * h, jitter * h, size=int(interior.sum()))
    coords = np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1).astype(np.float64)
    k, j, i = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    s = n + 1
    a = (k * s * s + j * s + i).ravel()
    b, c, d = a + 1, a + s + 1, a + s
    ev = np.stack([a, b, c, d, a + s * s, b + s * s, c + s * s, d + s * s], 1) + 1
    m = ev.shape[0]
    return RawMesh(coords, np.full(m, KIND_HEX, np.int32), (np.arange(m + 1) * 8).astype(np.int32),
                   ev.astype(np.int32).ravel(), b2d=False, periodic=periodic)


def strip(n, jitter=0.0, seed=0):
    """An N x 4 quad strip on [0,1] x [0,4/N], one layer thick (shock-tube case)."""
    h = 1.0 / n
    return hex_slab(n, 4, 0.0, 1.0, 0.0, 4.0 * h, 0.0, h, jitter=jitter, seed=seed)


def sedov_origin_mask(elem_vert_off, elem_vert, coords) -> np.ndarray:
    """1 for cells having a vertex on the z-axis through the origin (x = y = 0).
    Works on any numbering: pass the arrays of the mesh the mask is meant for."""
    coords = np.asarray(coords).reshape(-1, 3)
    on_axis = (np.abs(coords[:, 0]) < 1e-14) & (np.abs(coords[:, 1]) < 1e-14)
    ev = np.asarray(elem_vert).reshape(-1) - 1
    off = np.asarray(elem_vert_off)
    hit = on_axis[ev].astype(np.int32)
    cell = np.repeat(np.arange(off.size - 1), np.diff(off))
    mask = np.zeros(off.size - 1, np.int32)
    np.maximum.at(mask, cell, hit)
    return mask
