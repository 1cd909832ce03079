"""Seeded test meshes shared by the CPU and GPU tests (small enough for the oracle)."""
from subfv_b200 import meshgen


def lagrange_cases():
    return {
        "prism_jit": meshgen.prism_slab(12, 10, jitter=0.05, seed=11),
        "hex_jit": meshgen.hex_slab(9, 8, x0=0.0, x1=1.2, y0=0.0, y1=1.2, z0=0.0, z1=1.0, jitter=0.1, seed=12),
        "prism_reg": meshgen.prism_slab(8, 8),
    }


def topology_cases():
    return {
        "hex_slab": meshgen.hex_slab(7, 5, jitter=0.1, seed=1),
        "prism_slab": meshgen.prism_slab(9, 6, jitter=0.05, seed=2),
        "hex_box": meshgen.hex_box(5, jitter=0.05, seed=3, periodic=False),
        "hex_box_periodic": meshgen.hex_box(4, periodic=True),
        "strip": meshgen.strip(40),
    }


def field_errors(a, b):
    """Per-field relative errors of b against a, states (n, 5): L1 = sum |b - a| / sum |a|,
    Linf = max |b - a| / max |a|. The three momentum (or velocity) components share the
    scale of the largest one, so a component that is zero up to round-off (the transverse
    momentum of a slab) is measured against the flow's momentum, not against itself."""
    import numpy as np
    l1s, lis = np.abs(a).sum(0), np.abs(a).max(0)
    l1s[1:4], lis[1:4] = l1s[1:4].max(), lis[1:4].max()
    d = np.abs(b - a)
    return d.sum(0) / np.maximum(l1s, 1e-300), d.max(0) / np.maximum(lis, 1e-300)
