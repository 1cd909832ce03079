"""The backward-Euler Jacobian (new code: the reference has no Jacobian assembly) is the
exact derivative of the first-order two-wave residual with the wave speeds sl, sr held
at their current values. Checked here on the CPU restatement against central finite
differences of that frozen-speed flux, assembled independently in numpy."""
import numpy as np
import pytest

G = 1.4


def _p2c(w):
    return np.array([w[0], w[1] * w[0], w[2] * w[0], w[3] * w[0],
                     w[4] / (G - 1) + 0.5 * w[0] * (w[1] ** 2 + w[2] ** 2 + w[3] ** 2)])


def _c2p(u):
    v = u[1:4] / u[0]
    return np.array([u[0], *v, (G - 1) * (u[4] - 0.5 * u[0] * (v @ v))])


def _phys(u, n):
    w = _c2p(u)
    vn = w[1:4] @ n
    return np.array([vn * u[0], *(vn * u[1:4] + w[4] * n), (u[4] + w[4]) * vn])


def _speeds(ul, ur, n):
    wl, wr = _c2p(ul), _c2p(ur)
    vnl, vnr = wl[1:4] @ n, wr[1:4] @ n
    al, ar = np.sqrt(G * wl[4] / wl[0]), np.sqrt(G * wr[4] / wr[0])
    lam_l = max(al * wl[0], np.sqrt(wl[0] * max(0.0, wr[4] - wl[4])), -wl[0] * (vnr - vnl))
    lam_r = max(ar * wr[0], np.sqrt(wr[0] * max(0.0, wl[4] - wr[4])), -wr[0] * (vnr - vnl))
    return vnl - lam_l / wl[0], vnr + lam_r / wr[0]


def _flux(ul, ur, n, sl, sr):
    fl, fr = _phys(ul, n), _phys(ur, n)
    us = (sr * ur - sl * ul - (fr - fl)) / (sr - sl)
    return 0.5 * (fl + fr) - 0.5 * (abs(sl) * (us - ul) + abs(sr) * (ur - us))


def _mirror(u, n):
    r = u.copy()
    r[1:4] = u[1:4] - 2.0 * (u[1:4] @ n) * n
    return r


@pytest.mark.parametrize("periodic", [False, True])
def test_be_jacobian_is_the_frozen_speed_derivative(oracle_lib, periodic):
    from oracle.oracle import OracleMesh
    from subfv_b200 import meshgen
    raw = meshgen.hex_box(3, jitter=0.0 if periodic else 0.05, seed=2, periodic=periodic)
    o = OracleMesh(raw)
    ne = o.n_elems
    rng = np.random.default_rng(0)
    w = np.column_stack([rng.uniform(0.8, 1.2, ne), rng.uniform(-0.2, 0.2, (ne, 3)), rng.uniform(0.8, 1.2, ne)])
    sol = np.ascontiguousarray(np.array([_p2c(x) for x in w]))
    cfg = dict(scheme=4, second_order=0, method=0, bc_style=2, b2d=0, exclude_bound_vert=0, local_time_step=0,
               cfl=0.5, tmax=1e30)
    dt = 0.37
    row, col, v = o.be_jacobian(cfg, sol, dt)
    J = np.zeros((5 * ne, 5 * ne))
    for i in range(ne):
        for q in range(row[i] - 1, row[i + 1] - 1):
            c = col[q] - 1
            J[5 * i:5 * i + 5, 5 * c:5 * c + 5] = v[q].T
    # independent assembly: A = V/dt I - d rhs/dU, rhs_L -= A F, rhs_R += A F
    ref = np.kron(np.diag(o.geom("elem_volume") / dt), np.eye(5))
    sff = o.topo("sub_face_face")
    fl, fr = o.topo("face_left"), o.topo("face_right")
    # compute_rhs_around_vert credits the right cell only through its subcell at the
    # subface's own vertex; a periodically stitched face's right subcell sits at the
    # image vertex, so that cell gets the flux from its own twin face instead
    sfv, rse, sev = o.topo("sub_face_vert"), o.topo("sub_face_right_sub_elem"), o.topo("sub_elem_vert")
    nrm, area = o.geom("sub_face_norm"), o.geom("sub_face_area")
    for s in range(o.n_sub_faces):
        f = sff[s] - 1
        L, R = fl[f] - 1, fr[f] - 1
        n = nrm[s]
        ul = sol[L]
        ur = sol[R] if R >= 0 else _mirror(ul, n)
        sl, sr = _speeds(ul, ur, n)
        for side, base in ((0, ul), (1, ur)):
            for k in range(5):
                h = 1e-6 * max(1.0, abs(base[k]))
                up, um = base.copy(), base.copy()
                up[k] += h
                um[k] -= h
                if side == 0:
                    gp = (up, _mirror(up, n) if R < 0 else ur)
                    gm = (um, _mirror(um, n) if R < 0 else ur)
                else:
                    gp, gm = (ul, up), (ul, um)
                dF = (_flux(*gp, n, sl, sr) - _flux(*gm, n, sl, sr)) / (2 * h)
                col_of = L if side == 0 else R
                if side == 1 and R < 0:
                    continue  # the ghost state is not an unknown
                ref[5 * L:5 * L + 5, 5 * col_of + k] += area[s] * dF
                if R >= 0 and rse[s] > 0 and sev[rse[s] - 1] == sfv[s]:
                    ref[5 * R:5 * R + 5, 5 * col_of + k] -= area[s] * dF
    assert np.abs(J - ref).max() <= 1e-6 * np.abs(ref).max()


POST = np.array([8.0, 7.145, -4.125, 0.0, 116.5])


def _ghost(ul, n, kind, bv, fx):
    """compute_right_state (ns_euler_recon_module.F90:331-409) for the kinds whose ghost
    depends on the inner state: 1 wall, 2 adherence wall, 4 outflow, 5 pondered inflow,
    7 double-Mach bottom."""
    if kind == 1 or (kind == 7 and not fx[0] < 0.1667):
        return _mirror(ul, n)
    if kind == 7:
        return _p2c(POST)
    if kind == 4:
        return ul.copy()
    if kind == 5:
        g = _p2c(bv)
        return ul.copy() if g[1:4] @ n > 0 else g
    r = ul.copy()  # adherence
    r[1:4] = 2.0 * ul[0] * bv[1:4] - ul[1:4]
    r[4] = ul[4] - 0.5 * ul[0] * np.sum((ul[1:4] / ul[0]) ** 2) + 0.5 * ul[0] * np.sum((r[1:4] / r[0]) ** 2)
    return r


@pytest.mark.parametrize("kinds", [(2, 5, 7, 4), (5, 2, 4, 7)])
def test_be_jacobian_boundary_kinds_are_the_frozen_speed_derivative(oracle_lib, kinds):
    """The ghost state's chain rule dU_R/dU_L for the boundary kinds that depend on the
    inner state, on a slab whose sides carry tags, against finite differences."""
    from oracle.oracle import OracleMesh
    from subfv_b200 import meshgen
    nx, ny = 6, 5
    raw = meshgen.tag_slab_sides(meshgen.hex_slab(nx, ny, jitter=0.1, seed=4), nx, ny,
                                 {"xlo": 1, "xhi": 2, "ylo": 3, "yhi": 4})
    o = OracleMesh(raw)
    ne = o.n_elems
    rng = np.random.default_rng(1)
    w = np.column_stack([rng.uniform(0.8, 1.2, ne), rng.uniform(-0.2, 0.2, (ne, 2)), np.zeros(ne),
                         rng.uniform(0.8, 1.2, ne)])
    sol = np.ascontiguousarray(np.array([_p2c(x) for x in w]))
    # tag 1 leaves the domain through xlo (the pondered inflow copies the inner state
    # there), tag 2 enters through xhi (the imposed state)
    vals = np.array([[1.0, -0.05, 0.02, 0, 1.0], [1.1, -0.1, 0, 0, 0.9], [1.0, 0.1, 0, 0, 1.0], [1.0, 0, 0, 0, 1]])
    cfg = dict(scheme=4, second_order=0, method=0, bc_style=2, b2d=1, exclude_bound_vert=0, local_time_step=0,
               cfl=0.5, tmax=1e30, n_bc=4, bc_type=np.array(kinds, np.int32), bc_val=vals)
    dt = 0.29
    row, col, v = o.be_jacobian(cfg, sol, dt)
    J = np.zeros((5 * ne, 5 * ne))
    for i in range(ne):
        for q in range(row[i] - 1, row[i + 1] - 1):
            J[5 * i:5 * i + 5, 5 * (col[q] - 1):5 * (col[q] - 1) + 5] = v[q].T
    ref = np.kron(np.diag(o.geom("elem_volume") / dt), np.eye(5))
    sff = o.topo("sub_face_face")
    fl, fr = o.topo("face_left"), o.topo("face_right")
    nrm, area, fxs = o.geom("sub_face_norm"), o.geom("sub_face_area"), o.geom("face_coord")
    for s in range(o.n_sub_faces):
        f = sff[s] - 1
        L, R = fl[f] - 1, fr[f] - 1
        n = nrm[s]
        ul = sol[L]
        if R >= 0:
            ghost = None
        else:
            tag = -fr[f]  # face_right holds -tag (0: the default wall)
            kind = 1 if tag == 0 else kinds[tag - 1]
            bv = vals[tag - 1] if tag > 0 else None
            ghost = lambda u, n=n, kind=kind, bv=bv, fx=fxs[f]: _ghost(u, n, kind, bv, fx)
        ur = sol[R] if R >= 0 else ghost(ul)
        sl, sr = _speeds(ul, ur, n)
        for side, base in ((0, ul), (1, ur)):
            if side == 1 and R < 0:
                continue
            for k in range(5):
                h = 1e-6 * max(1.0, abs(base[k]))
                up, um = base.copy(), base.copy()
                up[k] += h
                um[k] -= h
                if side == 0:
                    gp = (up, ghost(up) if R < 0 else ur)
                    gm = (um, ghost(um) if R < 0 else ur)
                else:
                    gp, gm = (ul, up), (ul, um)
                dF = (_flux(*gp, n, sl, sr) - _flux(*gm, n, sl, sr)) / (2 * h)
                ref[5 * L:5 * L + 5, 5 * (L if side == 0 else R) + k] += area[s] * dF
                if R >= 0:
                    ref[5 * R:5 * R + 5, 5 * (L if side == 0 else R) + k] -= area[s] * dF
    assert np.abs(J - ref).max() <= 1e-6 * np.abs(ref).max()
