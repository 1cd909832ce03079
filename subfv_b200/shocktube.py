"""Batched shock tubes: many independent Riemann problems on N x 4 quad strips.

Each problem is a strip [0,1] x [0,4/N] (one cell layer, walls all round) with a left and
a right constant state separated at x = 0.5, run to t_end = 0.25 / (the largest initial
wave speed |u| + a of the two states), so no wave reaches the end walls. Sizes and states
are drawn from a seeded generator: N uniform in [n_min, n_max], rho log-uniform in
[0.1, 10], p log-uniform in [0.01, 1000], u uniform in [-2, 2].
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import meshgen
from .mesh import Mesh

GAMMA = 1.4


@dataclass
class ShockTube:
    n: int
    left: tuple   # primitive (rho, u, p)
    right: tuple
    t_end: float
    x0: float = 0.5

    @property
    def n_cells(self) -> int:
        return 4 * self.n


def max_wave_speed(rho, u, p, gamma=GAMMA) -> float:
    return abs(u) + float(np.sqrt(gamma * p / rho))


def sample(n_problems: int, seed: int = 0, n_min: int = 200, n_max: int = 20000) -> list[ShockTube]:
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n_problems):
        n = int(rng.integers(n_min, n_max + 1))
        st = []
        for _side in range(2):
            rho = float(np.exp(rng.uniform(np.log(0.1), np.log(10.0))))
            p = float(np.exp(rng.uniform(np.log(0.01), np.log(1000.0))))
            u = float(rng.uniform(-2.0, 2.0))
            st.append((rho, u, p))
        smax = max(max_wave_speed(*st[0]), max_wave_speed(*st[1]))
        out.append(ShockTube(n, st[0], st[1], 0.25 / smax))
    return out


def raw_mesh(tube: ShockTube) -> meshgen.RawMesh:
    return meshgen.strip(tube.n)


def initial_state(mesh: Mesh, tube: ShockTube, gamma=GAMMA) -> np.ndarray:
    """Conservative (rho, rho u, rho v, rho w, E) per cell, by cell centroid side."""
    x = mesh.geometry("elem_coord")[:, 0]
    left = x < tube.x0
    rho = np.where(left, tube.left[0], tube.right[0])
    u = np.where(left, tube.left[1], tube.right[1])
    p = np.where(left, tube.left[2], tube.right[2])
    sol = np.zeros((mesh.n_elems, 5))
    sol[:, 0] = rho
    sol[:, 1] = rho * u
    sol[:, 4] = p / (gamma - 1) + 0.5 * rho * u * u
    return sol
