"""Initial states of the explicit Euler / Navier-Stokes driver (init_sol,
src/ns/ns_euler_module.F90:12-140, with the exact solutions of
src/ns/ns_euler_exact_sol_module.F90), evaluated on the host at the cell centroids
(mesh geometry "elem_coord") and returned as conservative states (n, 5). The Gresho
vortex is subfv_b200.ns.init_gresho; a restart is subfv_b200.io.restart_from_vtu."""
from __future__ import annotations

import math

import numpy as np

GAMMA = 1.4


def primit_to_conserv(w: np.ndarray) -> np.ndarray:
    """(rho, u, v, w, p) -> (rho, rho u, rho v, rho w, E), row by row."""
    w = np.atleast_2d(np.asarray(w, np.float64))
    out = np.empty_like(w)
    out[:, 0] = w[:, 0]
    out[:, 1:4] = w[:, 1:4] * w[:, :1]
    out[:, 4] = w[:, 4] / (GAMMA - 1) + 0.5 * w[:, 0] * (w[:, 1] * w[:, 1] + w[:, 2] * w[:, 2] + w[:, 3] * w[:, 3])
    return out


def init_uniform(n_elems: int, w) -> np.ndarray:
    """init_uniform: every cell at the primitive state sol_uniform."""
    return np.ascontiguousarray(np.repeat(primit_to_conserv(w), n_elems, axis=0))


def init_riemann_1d(elem_coord: np.ndarray, x0: float, w_left, w_right) -> np.ndarray:
    """init_1drp: w_left where the centroid's x < x1drp, w_right elsewhere."""
    left = np.asarray(elem_coord)[:, 0] < x0
    return np.ascontiguousarray(np.where(left[:, None], primit_to_conserv(w_left), primit_to_conserv(w_right)))


def init_isentropic_vortex(elem_coord: np.ndarray, t: float = 0.0) -> np.ndarray:
    """init_isentropic_vortex: sol_isentropic_vortex (beta 5, centred at the origin, at rest)."""
    x = np.asarray(elem_coord, np.float64)
    beta, pi = 5.0, math.pi
    r = x[:, 0] ** 2 + x[:, 1] ** 2
    rho = (1.0 - ((GAMMA - 1) * beta ** 2) / (8.0 * GAMMA * pi ** 2) * np.exp(1.0 - r)) ** (1.0 / (GAMMA - 1.0))
    u = -x[:, 1] * beta / (2.0 * pi) * np.exp(0.5 * (1.0 - r))
    v = x[:, 0] * beta / (2.0 * pi) * np.exp(0.5 * (1.0 - r))
    w = np.column_stack([rho, u, v, np.zeros_like(rho), rho ** GAMMA])
    return np.ascontiguousarray(primit_to_conserv(w))


def init_potential_flow(elem_coord: np.ndarray, three_d: bool = False) -> np.ndarray:
    """init_potential_flow_2d / _3d: sol_potential_flow_2d / _3d at the centroids (the 2-D
    routine's Mach number is its single-precision literal 1e-4)."""
    x = np.asarray(elem_coord, np.float64)
    r0, r1, rhoinf, pinf = 0.5, 5.5, 1.4, 1.0
    mach = 1e-4 if three_d else float(np.float32(1e-4))
    vinf = mach * math.sqrt(GAMMA * pinf / rhoinf)
    if not three_d:
        r = np.sqrt(x[:, 0] ** 2 + x[:, 1] ** 2)
        th = np.arctan2(x[:, 1], x[:, 0])
        c = r1 ** 2 / (r1 ** 2 - r0 ** 2)
        vr = c * (1.0 - (r0 / r) ** 2) * np.cos(th)
        vt = -c * (1.0 + (r0 / r) ** 2) * np.sin(th)
        ux = vinf * (np.cos(th) * vr - np.sin(th) * vt)
        uy = vinf * (np.sin(th) * vr + np.cos(th) * vt)
        uz = np.zeros_like(r)
    else:
        r = np.sqrt((x ** 2).sum(1))
        f = r0 ** 3 / (2.0 * r ** 5)
        ux = vinf * (1.0 + f * (r ** 2 - 3.0 * x[:, 0] ** 2))
        uy = -3.0 * vinf * f * x[:, 0] * x[:, 1]
        uz = -3.0 * vinf * f * x[:, 0] * x[:, 2]
    p = pinf + 0.5 * rhoinf * (vinf ** 2 - (ux ** 2 + uy ** 2 + uz ** 2))
    w = np.column_stack([np.full_like(ux, rhoinf), ux, uy, uz, p])
    return np.ascontiguousarray(primit_to_conserv(w))


def kelvin_helmholtz(y: np.ndarray) -> np.ndarray:
    """The smoothed double shear layer profile of ns_euler_exact_sol_module.F90:172-193."""
    y = np.asarray(y, np.float64)
    wk = 1.0 / 16.0
    v = np.ones_like(y)
    a = (y > -0.25 - wk / 2) & (y < -0.25 + wk / 2)
    b = (y > -0.25 + wk / 2) & (y < 0.25 - wk / 2)
    c = (y > 0.25 - wk / 2) & (y < 0.25 + wk / 2)
    v = np.where(a, -np.sin(math.pi * (y + 0.25) / wk), v)
    v = np.where(b, -1.0, v)
    v = np.where(c, np.sin(math.pi * (y - 0.25) / wk), v)
    return v


def init_kelvin_helmholtz(elem_coord: np.ndarray):
    """init_kelvin: the low-Mach double shear layer (M = 1e-2); returns (sol, tmax = 0.8 / M)."""
    x = np.asarray(elem_coord, np.float64)
    m = 1e-2
    h = kelvin_helmholtz(x[:, 1])
    w = np.column_stack([GAMMA + m * h, m * h, 0.1 * m * np.sin(2.0 * math.pi * x[:, 0]), np.zeros_like(h),
                         np.ones_like(h)])
    return np.ascontiguousarray(primit_to_conserv(w)), 0.8 / m


def init_double_mach(elem_coord: np.ndarray):
    """init_double_mach: the Mach 10 shock along y = 1.732 (x - 0.1667); returns (sol, tmax = 0.2)."""
    x = np.asarray(elem_coord, np.float64)
    pre = primit_to_conserv([1.4, 0.0, 0.0, 0.0, 1.0])
    post = primit_to_conserv([8.0, 7.145, -4.125, 0.0, 116.5])
    below = x[:, 1] < 1.732 * (x[:, 0] - 0.1667)
    return np.ascontiguousarray(np.where(below[:, None], pre, post)), 0.2


def _norm2_rows(a: np.ndarray) -> np.ndarray:
    """gfortran's NORM2 row by row (scaled sum of squares)."""
    from .meshgen import _norm2
    return _norm2(a)


def init_sedov(elem_coord: np.ndarray, elem_volume: np.ndarray, boundary_2d: bool = True) -> np.ndarray:
    """init_sedov (ns_euler_module.F90:64-112): rho = 1 at rest with E = 1e-16 / (gamma - 1),
    and the blast energy (0.984042 in 2-D, 0.851072 in 3-D) over the volume of the first
    cell of smallest centroid radius (in the x-y plane for boundary_2d)."""
    x = np.asarray(elem_coord, np.float64)
    r = _norm2_rows(x[:, :2] if boundary_2d else x)
    imin = int(np.argmin(r))  # the first index of the smallest radius, as the strict < scan keeps
    sol = np.zeros((x.shape[0], 5))
    sol[:, 0] = 1.0
    sol[:, 4] = 1e-16 / (GAMMA - 1.0)
    sol[imin, 4] = (0.984042 if boundary_2d else 0.851072) / float(elem_volume[imin])
    return np.ascontiguousarray(sol)
