"""The Lagrangian step's cell kernel tests check_mesh's closure norms (norm2 < 1e-14,
src/mesh/mesh_geometry_module.F90:374-411) as a sum of squares below a constant
(subfv_b200/csrc/geom_body.cuh, kClosedSumSq). The constant must be the smallest double
whose correctly rounded square root reaches 1e-14, so that both forms agree on every
input; Python's math.sqrt is correctly rounded, as CUDA's is."""
import math
import pathlib
import re

import numpy as np

HEADER = pathlib.Path(__file__).resolve().parents[1] / "subfv_b200" / "csrc" / "geom_body.cuh"


def _constant():
    m = re.search(r"kClosedSumSq\s*=\s*(0x[0-9a-fA-F.p+-]+);", HEADER.read_text())
    assert m, "kClosedSumSq not found"
    return float.fromhex(m.group(1))


def test_constant_is_the_threshold_of_the_rounded_square_root():
    x0 = _constant()
    assert math.sqrt(x0) >= 1e-14
    assert math.sqrt(math.nextafter(x0, 0.0)) < 1e-14


def test_both_forms_agree_near_and_away_from_the_threshold():
    x0 = _constant()
    rng = np.random.default_rng(5)
    near = x0 * (1.0 + rng.uniform(-1e-12, 1e-12, 200000))
    wide = rng.uniform(0.0, 4e-28, 200000)
    steps = [x0]
    for _ in range(50):
        steps.append(math.nextafter(steps[-1], math.inf))
    down = [x0]
    for _ in range(50):
        down.append(math.nextafter(down[-1], 0.0))
    for s in list(near) + list(wide) + steps + down:
        assert (math.sqrt(s) < 1e-14) == (s < x0), s
