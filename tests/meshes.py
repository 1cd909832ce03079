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
