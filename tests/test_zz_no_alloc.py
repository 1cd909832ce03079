"""subfv_compute_dt_noalloc: the CFL reduction for callers that cannot allocate device
memory when they call (their device memory is reserved at start-up, or owned by the
host application's allocator). They pass device buffers they already own; the entry
point uses only a static device array as scratch.

Checked through the C-ABI against subfv_compute_dt (which stages host arrays in buffers
it allocates itself): equal results on two calls in a row, with different states, so a
stale scratch array would show. This file is collected last so that, if it fails, a run
stopping at the first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _state(n, seed):
    rng = np.random.default_rng(seed)
    tau = rng.uniform(0.5, 2.0, n)
    u = rng.uniform(-0.3, 0.3, (n, 3))
    u[:, 2] = 0.0
    p = rng.uniform(0.2, 3.0, n)
    e = p / (0.4 / tau) + 0.5 * (u ** 2).sum(1)
    return np.ascontiguousarray(np.column_stack([tau, u, e]))


def test_compute_dt_noalloc_matches_allocating_entry_point(native, cuda_ok):
    import torch

    from subfv_b200 import lagrange as L
    from subfv_b200 import meshgen
    from subfv_b200.mesh import Mesh

    torch.cuda.init()
    mesh = Mesh.from_raw(meshgen.prism_slab(40, 30, jitter=0.05, seed=21))
    lib = native
    for call, seed in enumerate((1, 2)):
        sol = _state(mesh.n_elems, seed)
        vp = np.ascontiguousarray(np.random.default_rng(seed + 10).uniform(-0.5, 0.5, (mesh.n_vert, 3)))
        vp[:, 2] = 0.0
        cfl = 0.8 if call == 0 else 0.37
        expected = L.compute_dt(mesh, sol, 0.0, cfl, vp)
        d_sol = torch.from_numpy(sol).cuda()
        d_vp = torch.from_numpy(vp).cuda()
        d_dt = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        rc = lib.subfv_compute_dt_noalloc(mesh._h, C.c_void_p(d_sol.data_ptr()), C.c_void_p(d_vp.data_ptr()),
                                          C.c_double(cfl), C.c_void_p(d_dt.data_ptr()))
        assert rc == 0, rc
        got = float(d_dt.cpu().item())
        assert got == expected, (call, got, expected)  # same arithmetic: bit-identical
        assert 0.0 < got < 1e6


def test_compute_dt_noalloc_rejects_null(native, cuda_ok):
    from subfv_b200 import meshgen
    from subfv_b200.mesh import Mesh
    mesh = Mesh.from_raw(meshgen.hex_slab(4, 4))
    rc = native.subfv_compute_dt_noalloc(mesh._h, None, None, C.c_double(0.5), None)
    assert rc < 0
