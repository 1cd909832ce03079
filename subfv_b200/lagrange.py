"""Host mirror of the reference's lagrange_module (subfvlagrange, scheme "classic").

Same names, argument meaning and error behaviour as
src/lagrange/lagrange_module.F90: compute_rhs_lagrange (:14-147), compute_dt
(:240-283), move_mesh (:772-784), init_sol (:285-427) and the time loop of
src/lagrange/lagrange_main.F90:81-127. Arrays use the reference's layouts:
sol and rhs are (5, n_elems) Fortran arrays, i.e. numpy (n_elems, 5); vp is (3, n_vert),
i.e. numpy (n_vert, 3). The compute runs on the GPU through the C-ABI; there is no CPU
path.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check, f64, pd
from .mesh import Mesh, SUBFV_ERR_MESH_CHECK

GAMMA = 7.0 / 5.0
PLAIN_FP64, MIXED = 0, 1


class MeshCheckError(RuntimeError):
    """check_mesh failed: the reference prints "MESH GEOMETRY IS NOT OK" and stops."""


def compute_rhs_lagrange(mesh: Mesh, sol, vp, dt, rhs, n_bc=0, bc_type=None, bc_val=None, b2d=True, mass=None):
    """lagrange_module.F90:14-147. Fills vp (n_vert, 3) and rhs (n_elems, 5) in place."""
    sol = f64(sol)
    mass = f64(mass)
    assert vp.dtype == np.float64 and vp.flags["C_CONTIGUOUS"] and vp.shape == (mesh.n_vert, 3)
    assert rhs.dtype == np.float64 and rhs.flags["C_CONTIGUOUS"] and rhs.shape == (mesh.n_elems, 5)
    return check(_lib.load().subfv_compute_rhs_lagrange(mesh._h, pd(sol), pd(vp), pd(rhs), int(b2d), pd(mass)),
                 "subfv_compute_rhs_lagrange")


def compute_rhs_lagrange_sidil(mesh: Mesh, sol, vp, dt, rhs, n_bc=0, bc_type=None, bc_val=None, b2d=True,
                               mass=None, method=0, b2d_h=0.0):
    """lagrange_module.F90:149-223 (scheme "sidil"). Fills vp (n_vert, 3) and rhs
    (n_elems, 5) in place; returns the status bits (4: a negative nodal pressure)."""
    sol = f64(sol)
    mass = f64(mass)
    assert vp.dtype == np.float64 and vp.flags["C_CONTIGUOUS"] and vp.shape == (mesh.n_vert, 3)
    assert rhs.dtype == np.float64 and rhs.flags["C_CONTIGUOUS"] and rhs.shape == (mesh.n_elems, 5)
    return check(_lib.load().subfv_compute_rhs_lagrange_sidil(mesh._h, pd(sol), pd(vp), pd(rhs), int(b2d), pd(mass),
                                                              int(method)), "subfv_compute_rhs_lagrange_sidil")


def compute_dt(mesh: Mesh, sol, dt, cfl, vp, me=0, num_procs=1) -> float:
    """lagrange_module.F90:240-283; returns the new dt (the reference's intent(inout))."""
    sol, vp = f64(sol), f64(vp)
    out = C.c_double()
    check(_lib.load().subfv_compute_dt(mesh._h, pd(sol), float(cfl), pd(vp), C.byref(out)), "subfv_compute_dt")
    return out.value


def move_mesh(mesh: Mesh, vp, dt):
    """lagrange_module.F90:772-784 (on the device copy of the vertex coordinates)."""
    vp = f64(vp)
    check(_lib.load().subfv_move_mesh(mesh._h, pd(vp), float(dt)), "subfv_move_mesh")


def compute_geometry_mesh(mesh: Mesh):
    st = mesh.compute_geometry_mesh()
    if st & SUBFV_ERR_MESH_CHECK:
        raise MeshCheckError("MESH GEOMETRY IS NOT OK")
    return st


def init_sol_sedov(mesh: Mesh, e_total=0.983909, r_sedov=0.06, mask=None) -> np.ndarray:
    """init_sol with init = 1 (lagrange_module.F90:318-356): rho = 1, u = 0, the energy
    e_total spread over the selected cells, 1e-8/(gamma-1) elsewhere. The reference
    selects cells whose centroid lies within r_sedov of the z-axis; `mask` overrides the
    selection (the benchmark deposits 0.244816 in the cells touching the origin)."""
    vol = mesh.geometry("elem_volume")
    if mask is None:
        cc = mesh.geometry("elem_coord")
        sel = np.sqrt(cc[:, 0] ** 2 + cc[:, 1] ** 2) < r_sedov
    else:
        sel = np.asarray(mask).astype(bool)
    tot_vol = 0.0
    for v in vol[sel]:  # sequential sum, as the reference's loop
        tot_vol = tot_vol + float(v)
    if tot_vol < 1e-10:
        raise ValueError(f"[-] r_sedov too small, tot_vol_init: {tot_vol}")
    sol = np.zeros((mesh.n_elems, 5))
    sol[:, 0] = 1.0
    sol[:, 4] = np.where(sel, e_total / tot_vol, 1e-8 / (GAMMA - 1.0))
    return sol


class LagrangeState:
    """The device-resident time loop of lagrange_main.F90:89-127. The state (sol, mass,
    coordinates, geometry) stays in HBM; `advance` replays graph-captured steps."""

    def __init__(self, mesh: Mesh, sol, mass=None, cfl=0.8, t0=0.0, t_max=1.0, precision=PLAIN_FP64):
        self.mesh = mesh
        sol = f64(sol)
        if mass is None:  # lagrange_main.F90:81-85: mass = volume / tau
            mass = mesh.geometry("elem_volume") / sol[:, 0]
        mass = f64(mass)
        self.mass = mass
        h = C.c_void_p()
        check(_lib.load().subfv_lag_state_create(mesh._h, pd(sol), pd(mass), float(cfl), float(t0), float(t_max),
                                                int(precision), C.byref(h)), "subfv_lag_state_create")
        self._h = h

    def set_scheme(self, scheme: int, method: int = 0):
        """0: "classic" (default); 1: "sidil" with method_length `method` (0..4)."""
        check(_lib.load().subfv_lag_state_set_scheme(self._h, int(scheme), int(method)), "subfv_lag_state_set_scheme")

    def advance(self, n_steps: int):
        steps, t = C.c_int(), C.c_double()
        st = check(_lib.load().subfv_lag_advance(self._h, int(n_steps), C.byref(steps), C.byref(t)),
                   "subfv_lag_advance")
        return st, steps.value, t.value

    def advance_async(self, n_steps: int):
        check(_lib.load().subfv_lag_advance_async(self._h, int(n_steps)), "subfv_lag_advance_async")

    def prepare(self):
        """Capture the replayed step graph now (set-up; the state does not move)."""
        check(_lib.load().subfv_lag_prepare(self._h), "subfv_lag_prepare")

    def sync(self):
        steps, t = C.c_int(), C.c_double()
        st = check(_lib.load().subfv_lag_sync(self._h, C.byref(steps), C.byref(t)), "subfv_lag_sync")
        return st, steps.value, t.value

    def run(self, max_steps: int = 10**9, chunk: int = 256):
        """Steps until t >= t_max (or max_steps); raises on a mesh-check failure.
        Returns (status bits, steps taken, t)."""
        st, steps, t = self.sync()
        start = steps
        while steps - start < max_steps:
            n = min(chunk, max_steps - (steps - start))
            st, new_steps, t = self.advance(n)
            if st & SUBFV_ERR_MESH_CHECK:
                raise MeshCheckError("MESH GEOMETRY IS NOT OK")
            if new_steps < steps + n:  # the loop reached t_max
                steps = new_steps
                break
            steps = new_steps
        return st, steps, t

    def sol(self) -> np.ndarray:
        out = np.empty((self.mesh.n_elems, 5))
        check(_lib.load().subfv_lag_get_sol(self._h, pd(out)), "subfv_lag_get_sol")
        return out

    def set_sol(self, sol):
        sol = f64(sol)
        check(_lib.load().subfv_lag_set_sol(self._h, pd(sol)), "subfv_lag_set_sol")

    def vp(self) -> np.ndarray:
        out = np.empty((self.mesh.n_vert, 3))
        check(_lib.load().subfv_lag_get_vp(self._h, pd(out)), "subfv_lag_get_vp")
        return out

    def last_dt(self) -> float:
        out = C.c_double()
        check(_lib.load().subfv_lag_last_dt(self._h, C.byref(out)), "subfv_lag_last_dt")
        return out.value

    def mesh_stream(self) -> int:
        """cudaStream_t (as an int) every kernel of this state runs on."""
        return int(_lib.load().subfv_mesh_stream(self.mesh._h))

    def profile_steps(self, n: int):
        """Per-kernel device milliseconds summed over n eager steps (face wave speeds,
        node, cell, finalize, move, face geometry, cell geometry + update)."""
        out = np.zeros(7)
        check(_lib.load().subfv_lag_profile_steps(self._h, int(n), pd(out)), "subfv_lag_profile_steps")
        return out

    def step_host(self, sol: np.ndarray) -> int:
        """One step through host buffers (upload, step, download), in place."""
        assert sol.dtype == np.float64 and sol.flags["C_CONTIGUOUS"]
        return check(_lib.load().subfv_lag_step_host(self._h, pd(sol)), "subfv_lag_step_host")

    def close(self):
        if getattr(self, "_h", None):
            _lib.load().subfv_lag_state_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


SUBFV_BATCH_FULL = -3


class LagBatch:
    """Many independent Lagrangian problems advanced together in shared launches (no
    counterpart in the reference, which runs one mesh per process). Each problem owns
    its mesh, which its steps move; each result is bit-identical to the same problem
    run alone through LagrangeState."""

    def __init__(self, capacity: int, budget_bytes: int, precision: int = PLAIN_FP64):
        h = C.c_void_p()
        check(_lib.load().subfv_lag_batch_create(int(precision), int(capacity), int(budget_bytes), C.byref(h)),
              "subfv_lag_batch_create")
        self._h = h
        self._meshes = {}

    def state_bytes(self, mesh: Mesh) -> int:
        return int(_lib.load().subfv_lag_batch_state_bytes(self._h, mesh._h))

    def free_bytes(self) -> int:
        return int(_lib.load().subfv_lag_batch_free_bytes(self._h))

    def size(self):
        n, used = C.c_int(), C.c_int64()
        check(_lib.load().subfv_lag_batch_size(self._h, C.byref(n), C.byref(used)), "subfv_lag_batch_size")
        return n.value, used.value

    def add(self, mesh: Mesh, sol, t_max: float, cfl: float = 0.8, mass=None, t0: float = 0.0,
            take_mesh: bool = False):
        """Admit a problem; returns its slot, or None when the batch is full."""
        sol = f64(sol)
        if mass is None:  # lagrange_main.F90:81-85: mass = volume / tau
            mass = mesh.geometry("elem_volume") / sol[:, 0]
        mass = f64(mass)
        slot = C.c_int(-1)
        rc = _lib.load().subfv_lag_batch_add(self._h, mesh._h, int(take_mesh), pd(sol), pd(mass), float(cfl),
                                             float(t0), float(t_max), C.byref(slot))
        if rc == SUBFV_BATCH_FULL:
            return None
        check(rc, "subfv_lag_batch_add")
        if take_mesh:
            mesh._h = None
        else:
            self._meshes[slot.value] = mesh
        return slot.value

    def remove(self, slot: int):
        check(_lib.load().subfv_lag_batch_remove(self._h, int(slot)), "subfv_lag_batch_remove")
        self._meshes.pop(slot, None)

    def advance(self, n_steps: int):
        check(_lib.load().subfv_lag_batch_advance(self._h, int(n_steps)), "subfv_lag_batch_advance")

    def time_steps(self, n_steps: int) -> float:
        ms = C.c_double()
        check(_lib.load().subfv_lag_batch_time_steps(self._h, int(n_steps), C.byref(ms)), "subfv_lag_batch_time_steps")
        return ms.value

    def poll(self, wait: bool = True) -> bool:
        return check(_lib.load().subfv_lag_batch_poll(self._h, int(wait)), "subfv_lag_batch_poll") == 0

    def sync(self):
        check(_lib.load().subfv_lag_batch_sync(self._h), "subfv_lag_batch_sync")

    def info(self, slot: int):
        """(t, steps, done, status bits) from the latest snapshot taken."""
        t, steps, done, st = C.c_double(), C.c_int64(), C.c_int(), C.c_uint()
        check(_lib.load().subfv_lag_batch_slot_info(self._h, int(slot), C.byref(t), C.byref(steps), C.byref(done),
                                                    C.byref(st)), "subfv_lag_batch_slot_info")
        return t.value, steps.value, bool(done.value), st.value

    def sol(self, slot: int, n_elems: int) -> np.ndarray:
        out = np.empty((n_elems, 5))
        check(_lib.load().subfv_lag_batch_get_sol(self._h, int(slot), pd(out)), "subfv_lag_batch_get_sol")
        return out

    def set_grid(self, grid: int):
        check(_lib.load().subfv_lag_batch_set_grid(self._h, int(grid)), "subfv_lag_batch_set_grid")

    def close(self):
        if getattr(self, "_h", None):
            _lib.load().subfv_lag_batch_destroy(self._h)
            self._h = None
            self._meshes.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
