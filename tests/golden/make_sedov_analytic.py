"""Writes sedov_2d_analytic_rho.txt from the reference's analytic Sedov profile.

Source: test/sedov_tri/analytic_sedov_2D.dat of vdelmas/subfv (1,200 rows: index,
radius, density, then further fields), the exact cylindrical Sedov solution that the
reference's sedov_tri case (test/sedov_tri/input.template: subfvns, init_sedov,
boundary_2d, tmax = 1) plots its density against (test/sedov_tri/plot_sedov.gnu, columns
2 and 3). Every second row's radius and density are kept (dr = 0.002), which resolves the
profile far below the meshes the tests use. Run in a checkout that has the reference at
the path given as the first argument.
"""
import sys
from pathlib import Path

import numpy as np

src = Path(sys.argv[1] if len(sys.argv) > 1 else "/root/reference") / "test/sedov_tri/analytic_sedov_2D.dat"
d = np.loadtxt(src)
keep = d[::2, 1:3]
out = Path(__file__).resolve().parent / "sedov_2d_analytic_rho.txt"
np.savetxt(out, keep, fmt="%.6e", header="radius density (every second row of test/sedov_tri/analytic_sedov_2D.dat, "
                                        "the cylindrical Sedov solution at t = 1 for E = 0.984042 per unit depth)")
print(out, keep.shape)
