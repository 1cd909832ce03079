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
