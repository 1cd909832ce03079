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


def _both(lib, mesh, sol, vp, cfl):
    """subfv_compute_dt (host buffers, allocating) and subfv_compute_dt_noalloc (device
    buffers, static scratch) on the same input: (rc, dt) of each."""
    import torch
    ref = C.c_double()
    pd = C.POINTER(C.c_double)
    rc_ref = lib.subfv_compute_dt(mesh._h, sol.ctypes.data_as(pd), C.c_double(cfl), vp.ctypes.data_as(pd),
                                  C.byref(ref))
    d_sol = torch.from_numpy(sol).cuda()
    d_vp = torch.from_numpy(vp).cuda()
    d_dt = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()  # the inputs must be complete before the call
    rc = lib.subfv_compute_dt_noalloc(mesh._h, C.c_void_p(d_sol.data_ptr()), C.c_void_p(d_vp.data_ptr()),
                                      C.c_double(cfl), C.c_void_p(d_dt.data_ptr()))
    return rc_ref, ref.value, rc, float(d_dt.cpu().item())


def _vp(n, seed):
    vp = np.ascontiguousarray(np.random.default_rng(seed + 10).uniform(-0.5, 0.5, (n, 3)))
    vp[:, 2] = 0.0
    return vp


@pytest.mark.parametrize("kind", ["prism", "prism_many_blocks", "periodic_box"])
def test_compute_dt_noalloc_matches_allocating_entry_point(native, cuda_ok, kind):
    import torch

    from subfv_b200 import meshgen
    from subfv_b200.mesh import Mesh

    torch.cuda.init()
    raw = {"prism": lambda: meshgen.prism_slab(40, 30, jitter=0.05, seed=21),
           # 80,000 cells: 313 blocks of partial minima
           "prism_many_blocks": lambda: meshgen.prism_slab(200, 200, jitter=0.05, seed=22),
           # periodic faces: node lists are periodic extensions (vsf is not the identity)
           "periodic_box": lambda: meshgen.hex_box(6, jitter=0.05, seed=23, periodic=True)}[kind]()
    mesh = Mesh.from_raw(raw)
    for call, seed in enumerate((1, 2)):
        sol = _state(mesh.n_elems, seed)
        vp = _vp(mesh.n_vert, seed)
        cfl = 0.8 if call == 0 else 0.37
        rc_ref, expected, rc, got = _both(native, mesh, sol, vp, cfl)
        assert rc_ref == 0 and rc == 0, (rc_ref, rc)
        assert got == expected, (call, got, expected)  # same arithmetic: bit-identical
        assert 0.0 < got < 1e6


def test_compute_dt_noalloc_reports_negative_pressure_like_allocating_entry_point(native, cuda_ok):
    """A cell of negative pressure makes the sound speed NaN: both entry points return
    the non-finite status bit instead of a plausible time step."""
    import torch

    from subfv_b200 import meshgen
    from subfv_b200.mesh import Mesh

    torch.cuda.init()
    mesh = Mesh.from_raw(meshgen.prism_slab(20, 20, jitter=0.05, seed=24))
    sol = _state(mesh.n_elems, 5)
    sol[17, 4] = 0.5 * (sol[17, 1:4] ** 2).sum() - 1.0  # internal energy < 0, so p < 0
    vp = _vp(mesh.n_vert, 5)
    rc_ref, _, rc, _ = _both(native, mesh, sol, vp, 0.5)
    assert rc_ref & 2 and rc & 2, (rc_ref, rc)  # SUBFV_ERR_NONFINITE
    # the status is cleared by the next call on a sound state
    sol = _state(mesh.n_elems, 6)
    rc_ref, expected, rc, got = _both(native, mesh, sol, vp, 0.5)
    assert rc_ref == 0 and rc == 0 and got == expected


def test_compute_dt_noalloc_rejects_null(native, cuda_ok):
    from subfv_b200 import meshgen
    from subfv_b200.mesh import Mesh
    mesh = Mesh.from_raw(meshgen.hex_slab(4, 4))
    rc = native.subfv_compute_dt_noalloc(mesh._h, None, None, C.c_double(0.5), None)
    assert rc < 0
