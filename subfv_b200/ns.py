"""Host mirror of the reference's explicit Euler path (subfvns).

compute_rhs_ns mirrors the contained procedure of src/ns/ns_main.F90:130-179 (no
diffusion); NsState runs the time loop of ns_main.F90:83-107 device-resident, first
order or the two-stage scheme, with the multi-point nodal solver
(src/ns/ns_euler_rs_module.F90:200-422) or the two-wave flux (:154-198). Conservative
state sol(5, n_elems) = (rho, rho u, rho v, rho w, E), numpy (n_elems, 5).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import check, f64, pd
from .mesh import Mesh

SCHEME_MULTI_POINT, SCHEME_MULTI_POINT_ISO, SCHEME_THREE_WAVE, SCHEME_TWO_WAVE, SCHEME_MODIFIED_THREE_WAVE = 1, 2, 3, 4, 5
SCHEME_MULTI_POINT_PRESSURE, SCHEME_MULTI_POINT_PRESSURE_PH = 6, 8
# (the scheme ids of ns_global_data_module.F90:67-71)
# the Euler boundary kinds of ns_global_data_module.F90:53-61 (bc_type per tag; bc_val
# the primitive state a kind reads: freestream, pondered inflow, the adherence wall's velocity)
BC_WALL, BC_ADHERENCE_WALL, BC_FREESTREAM, BC_OUTFLOW_SUPERSONIC, BC_INFLOW_POND = 1, 2, 3, 4, 5
BC_INOUT_DOUBLE_MACH, BC_DOUBLE_MACH_BOTTOM, BC_POTENTIAL_FLOW_2D, BC_POTENTIAL_FLOW_3D = 6, 7, 8, 9


class NsCfgC(C.Structure):
    _fields_ = [("scheme", C.c_int32), ("second_order", C.c_int32), ("method", C.c_int32),
                ("bc_style", C.c_int32), ("boundary_2d", C.c_int32), ("exclude_bound_vert", C.c_int32),
                ("local_time_step", C.c_int32), ("n_bc", C.c_int32), ("bc_type", C.c_int32 * 16),
                ("bc_val", (C.c_double * 5) * 16), ("cfl", C.c_double), ("tmax", C.c_double),
                ("precision", C.c_int32), ("activate_diffusion", C.c_int32), ("use_sutherland", C.c_int32),
                ("mu_p", C.c_double), ("mu0", C.c_double), ("T0", C.c_double), ("Cv_p", C.c_double),
                ("bc_type_V", C.c_int32 * 16), ("bc_val_V", (C.c_double * 3) * 16), ("bc_type_T", C.c_int32 * 16),
                ("bc_val_T", C.c_double * 16), ("prandtl", C.c_double)]

# bc_type_V / bc_type_T per tag (ns_global_data_module.F90:49-52; 0 is the namelist's "")
BC_DIFF_NEUMANN, BC_DIFF_DIRICHLET = 1, 2


class ImplicitStats(C.Structure):
    _fields_ = [("dt", C.c_double), ("b_norm", C.c_double), ("res_norm", C.c_double), ("conv", C.c_int32),
                ("restarts", C.c_int32), ("outer", C.c_int32), ("ms_assemble", C.c_double),
                ("ms_solve", C.c_double), ("ms_update", C.c_double), ("nnz_blocks", C.c_int64)]


@dataclass
class NsConfig:
    """The namelist keys of ns_global_data_module.F90:177-213 that the residual path reads."""

    scheme: int = SCHEME_MULTI_POINT
    second_order: bool = True
    method: int = 4
    bc_style: int = 2
    boundary_2d: bool = True
    exclude_bound_vert: bool = False
    local_time_step: bool = False
    cfl: float = 0.4
    tmax: float = 1e30
    bc_type: list = field(default_factory=list)  # per tag
    bc_val: list = field(default_factory=list)   # per tag, primitive (rho, u, v, w, p)
    precision: int = 0  # 0 plain FP64, 1 FP32 wave-speed bounds, 2 also FP32 flux / reconstruction / limiters
    # diffusion (activate_diffusion; the namelist's defaults)
    activate_diffusion: bool = False
    use_sutherland: bool = False
    mu_p: float = 1.329e-5
    mu0: float = 1.716e-5
    T0: float = 273.15
    Cv_p: float = 720.19471
    prandtl: float = 0.71  # the reference's parameter (ns_global_data_module.F90:10)
    bc_type_V: list = field(default_factory=list)  # per tag
    bc_val_V: list = field(default_factory=list)   # per tag (u, v, w)
    bc_type_T: list = field(default_factory=list)  # per tag
    bc_val_T: list = field(default_factory=list)   # per tag (temperature)

    def to_c(self) -> NsCfgC:
        c = NsCfgC()
        c.scheme, c.second_order, c.method = self.scheme, int(self.second_order), self.method
        c.bc_style, c.boundary_2d = self.bc_style, int(self.boundary_2d)
        c.exclude_bound_vert, c.local_time_step = int(self.exclude_bound_vert), int(self.local_time_step)
        c.n_bc = len(self.bc_type)
        for i, t in enumerate(self.bc_type):
            c.bc_type[i] = t
            for k in range(5):
                c.bc_val[i][k] = float(self.bc_val[i][k]) if i < len(self.bc_val) else 0.0
        c.cfl, c.tmax, c.precision = float(self.cfl), float(self.tmax), int(self.precision)
        c.activate_diffusion, c.use_sutherland = int(self.activate_diffusion), int(self.use_sutherland)
        c.mu_p, c.mu0, c.T0, c.Cv_p = float(self.mu_p), float(self.mu0), float(self.T0), float(self.Cv_p)
        c.prandtl = float(self.prandtl)
        for i in range(16):
            c.bc_type_V[i] = int(self.bc_type_V[i]) if i < len(self.bc_type_V) else 0
            c.bc_type_T[i] = int(self.bc_type_T[i]) if i < len(self.bc_type_T) else 0
            c.bc_val_T[i] = float(self.bc_val_T[i]) if i < len(self.bc_val_T) else 0.0
            for k in range(3):
                c.bc_val_V[i][k] = float(self.bc_val_V[i][k]) if i < len(self.bc_val_V) else 0.0
        return c

    def oracle_dict(self) -> dict:
        d = dict(scheme=self.scheme, second_order=int(self.second_order), method=self.method,
                 bc_style=self.bc_style, b2d=int(self.boundary_2d), exclude_bound_vert=int(self.exclude_bound_vert),
                 local_time_step=int(self.local_time_step), cfl=self.cfl, tmax=self.tmax, n_bc=len(self.bc_type))
        if self.bc_type:
            d["bc_type"] = np.array(self.bc_type, np.int32)
            d["bc_val"] = np.array(self.bc_val, np.float64)
        if self.activate_diffusion:
            nb = max(1, len(self.bc_type))
            pad = lambda a, shape: np.concatenate([np.asarray(a, np.float64).reshape((-1,) + shape[1:]),
                                                   np.zeros((shape[0] - len(a),) + shape[1:])])
            d.update(activate_diffusion=1, use_sutherland=int(self.use_sutherland),
                     diff_dc=[self.mu_p, self.mu0, self.T0, self.Cv_p, self.prandtl],
                     bc_type_V=pad(self.bc_type_V, (nb,)).astype(np.int32),
                     bc_val_V=pad(self.bc_val_V, (nb, 3)), bc_type_T=pad(self.bc_type_T, (nb,)).astype(np.int32),
                     bc_val_T=pad(self.bc_val_T, (nb,)))
        return d


def init_gresho(mesh: Mesh, mach: float) -> np.ndarray:
    """init_sol with init_gresho (ns_euler_module.F90:49-53) at Mach `mach`."""
    sol = np.empty((mesh.n_elems, 5))
    check(_lib.load().subfv_ns_init_gresho(mesh._h, float(mach), pd(sol)), "subfv_ns_init_gresho")
    return sol


GRESHO_MACHS = (1.0e-1, 1.0e-2, 1.0e-3, 1.0e-4)


def gresho_convergence(mesh: Mesh, cfg: "NsConfig", machs=GRESHO_MACHS, tmax: float = 1e-2, cfl: float = 0.9,
                       n_max_iter: int = 100000, chunk: int = 256):
    """The loop of subfvgreshoconv (src/ns/ns_gresho_convergence_main.F90:42-127): for
    each Mach number, the Gresho vortex of sol_gresho_mach at the cell centroids, run
    with the configuration's scheme (global time step, CFL `cfl`) until t reaches `tmax`
    (or `n_max_iter` iterations), then the density fluctuation
    L2_rho = sqrt(sum_c V_c (rho_c - 1)^2). The iterations run on the device-resident
    loop (NsState). Returns the rows of the reference's convergence.dat: a list of
    (mach, L2_rho, t_final, n_iter, status)."""
    from dataclasses import replace
    c = replace(cfg, cfl=float(cfl), tmax=float(tmax), local_time_step=False)
    vol = mesh.geometry("elem_volume")
    rows = []
    for mach in machs:
        sol0 = init_gresho(mesh, float(mach))
        s = NsState(mesh, c, sol0)
        n, t, st = 0, 0.0, 0
        while n < n_max_iter:
            st, n_now, t = s.advance(min(chunk, n_max_iter - n))
            if st or n_now == n:
                break
            n = n_now
        sol = s.sol()
        s.close()
        l2 = float(np.sqrt(np.sum(vol * (sol[:, 0] - 1.0) ** 2)))
        rows.append((float(mach), l2, float(t), int(n), int(st)))
    return rows


def init_fourier_flow(mesh: Mesh, mach=0.3, n_modes=8, amp=0.05, seed=0, gamma=1.4) -> np.ndarray:
    """Uniform flow along x at Mach `mach` (rho = 1, |u| = 1) plus `n_modes` seeded
    divergence-free Fourier modes of velocity with relative amplitude `amp`, periodic on
    the unit box; conservative variables at the cell centroids."""
    rng = np.random.default_rng(seed)
    x = mesh.geometry("elem_coord")
    u = np.zeros_like(x)
    u[:, 0] = 1.0
    for _ in range(n_modes):
        k = rng.integers(-3, 4, size=3)
        while not k.any():
            k = rng.integers(-3, 4, size=3)
        a = rng.normal(size=3)
        a -= (a @ k) / (k @ k) * k  # transverse: divergence free
        a *= amp / np.linalg.norm(a)
        phase = rng.uniform(0, 2 * np.pi)
        u += np.sin(2 * np.pi * (x @ k) + phase)[:, None] * a[None, :]
    rho = np.ones(len(x))
    p = rho / (gamma * mach ** 2)  # sound speed 1/mach
    E = p / (gamma - 1) + 0.5 * rho * (u ** 2).sum(1)
    return np.ascontiguousarray(np.column_stack([rho, rho[:, None] * u, E]))


def compute_rhs_ns(mesh: Mesh, cfg: NsConfig, sol):
    """One residual evaluation; returns (status, rhs, sum_lambda, vp, cell_grad (n, 5, 3))."""
    sol = f64(sol)
    rhs = np.empty((mesh.n_elems, 5))
    sl = np.empty(mesh.n_elems)
    vp = np.empty((mesh.n_vert, 3))
    grad = np.empty((mesh.n_elems, 5, 3))  # Fortran grad(3, 5, n)
    c = cfg.to_c()
    st = check(_lib.load().subfv_compute_rhs_ns(mesh._h, C.byref(c), pd(sol), pd(rhs), pd(sl), pd(vp), pd(grad)),
               "subfv_compute_rhs_ns")
    return st, rhs, sl, vp, grad


def compute_rhs_ns_diag(mesh: Mesh, cfg: NsConfig, sol):
    """compute_rhs_ns with the diffusion blocks: (status, rhs, sum_lambda, mat_diag (n, 5, 5)),
    mat_diag[c].T the reference's mat_diag(:, :, c)."""
    sol = f64(sol)
    rhs = np.empty((mesh.n_elems, 5))
    sl = np.empty(mesh.n_elems)
    diag = np.empty((mesh.n_elems, 5, 5))
    c = cfg.to_c()
    st = check(_lib.load().subfv_compute_rhs_ns_ex(mesh._h, C.byref(c), pd(sol), pd(rhs), pd(sl), None, None,
                                                    pd(diag)), "subfv_compute_rhs_ns_ex")
    return st, rhs, sl, diag


def compute_euler_flux(mesh: Mesh, cfg: NsConfig, sol, rhs, grad, sum_lambda, second_order: bool, vp=None,
                       h_p=None, mat_h_p=None):
    """compute_euler_flux (ns_euler_module.F90:151-339): fills rhs (n_elems, 5),
    sum_lambda (n_elems) and vp (n_vert, 3) in place; grad (n_elems, 5, 3), the
    reference's grad(3, 5, n), is read when second_order. h_p and mat_h_p belong to the
    ZB schemes and are ignored. Returns the status bits."""
    sol = f64(sol)
    g = f64(grad) if second_order else None
    for a, shape in ((rhs, (mesh.n_elems, 5)), (sum_lambda, (mesh.n_elems,))):
        assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"] and a.shape == shape
    if vp is not None:
        assert vp.dtype == np.float64 and vp.flags["C_CONTIGUOUS"] and vp.shape == (mesh.n_vert, 3)
    c = cfg.to_c()
    return check(_lib.load().subfv_compute_euler_flux(mesh._h, C.byref(c), pd(sol), pd(rhs), pd(g) if g is not None
                                                      else None, pd(sum_lambda), int(bool(second_order)),
                                                      pd(vp) if vp is not None else None),
                 "subfv_compute_euler_flux")


def compute_cell_grad_from_nodal_grad(mesh: Mesh, sol, grad, all_nodal_grad, method: int, cfg: NsConfig | None = None):
    """compute_cell_grad_from_nodal_grad (ns_euler_recon_module.F90:8-59): fills grad
    (n_elems, 5, 3) and all_nodal_grad (n_vert, 5, 3), the reference's (3, 5, n), in
    place. cfg supplies the boundary kinds the limiters read (method overrides its
    method)."""
    from dataclasses import replace
    cfg = replace(cfg or NsConfig(), method=int(method))
    sol = f64(sol)
    assert grad.dtype == np.float64 and grad.flags["C_CONTIGUOUS"] and grad.shape == (mesh.n_elems, 5, 3)
    assert all_nodal_grad.dtype == np.float64 and all_nodal_grad.flags["C_CONTIGUOUS"] and \
        all_nodal_grad.shape == (mesh.n_vert, 5, 3)
    c = cfg.to_c()
    return check(_lib.load().subfv_compute_cell_grad_from_nodal_grad(mesh._h, C.byref(c), pd(sol), pd(grad),
                                                                     pd(all_nodal_grad)),
                 "subfv_compute_cell_grad_from_nodal_grad")


def flux_limiting(mesh: Mesh, sol, rhs, rhs_o2, sum_lambda, cfl: float):
    """flux_limiting (ns_euler_recon_module.F90:560-601): rhs (n_elems, 5) in place."""
    sol, rhs_o2, sum_lambda = f64(sol), f64(rhs_o2), f64(sum_lambda)
    assert rhs.dtype == np.float64 and rhs.flags["C_CONTIGUOUS"] and rhs.shape == (mesh.n_elems, 5)
    return check(_lib.load().subfv_flux_limiting(mesh._h, pd(sol), pd(rhs), pd(rhs_o2), pd(sum_lambda), float(cfl)),
                 "subfv_flux_limiting")


def add_timedisc_and_solve(mesh: Mesh, sol, rhs, diag, sum_lambda, delta_sol, num_procs, me, a1, a2, cfl, t,
                           tmax=1e30):
    """add_timedisc_and_solve (ns_euler_module.F90:521-609), one process, global time
    step. sol, rhs, diag (n_elems, 5, 5) with diag[c].T the reference's diag(:, :, c), or
    None for zero blocks), sum_lambda and delta_sol are updated in place; returns
    (status bits, res, res_vect (5,), dt). Status SUBFV_ERR_BAD_OMEGA (8) leaves sol as it
    was, where the reference stops."""
    assert num_procs == 1, "one process: the MPI decomposition is not used"
    for a, shape in ((sol, (mesh.n_elems, 5)), (rhs, (mesh.n_elems, 5)), (delta_sol, (mesh.n_elems, 5)),
                     (sum_lambda, (mesh.n_elems,))):
        assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"] and a.shape == shape
    if diag is not None:
        assert diag.dtype == np.float64 and diag.flags["C_CONTIGUOUS"] and diag.shape == (mesh.n_elems, 5, 5)
    res, dt = C.c_double(), C.c_double()
    rv = np.zeros(5)
    st = check(_lib.load().subfv_add_timedisc_and_solve(mesh._h, pd(sol), pd(rhs), pd(diag) if diag is not None
                                                        else None, pd(sum_lambda), pd(delta_sol), C.byref(res),
                                                        pd(rv), float(a1), float(a2), float(cfl), float(t),
                                                        float(tmax), C.byref(dt)),
               "subfv_add_timedisc_and_solve")
    return st, res.value, rv, dt.value


class NsState:
    """Device-resident time loop of ns_main.F90:83-107 (graph-replayed iterations)."""

    def __init__(self, mesh: Mesh, cfg: NsConfig, sol, t0: float = 0.0):
        self.mesh, self.cfg = mesh, cfg
        sol = f64(sol)
        self._c = cfg.to_c()
        h = C.c_void_p()
        check(_lib.load().subfv_ns_state_create(mesh._h, C.byref(self._c), pd(sol), float(t0), C.byref(h)),
              "subfv_ns_state_create")
        self._h = h

    def advance(self, n_steps: int):
        steps, t = C.c_int(), C.c_double()
        st = check(_lib.load().subfv_ns_advance(self._h, int(n_steps), C.byref(steps), C.byref(t)), "subfv_ns_advance")
        return st, steps.value, t.value

    def advance_async(self, n_steps: int):
        check(_lib.load().subfv_ns_advance_async(self._h, int(n_steps)), "subfv_ns_advance_async")

    def prepare(self):
        """Capture the replayed step graph now (set-up; the state does not move)."""
        check(_lib.load().subfv_ns_prepare(self._h), "subfv_ns_prepare")

    def sync(self):
        steps, t = C.c_int(), C.c_double()
        st = check(_lib.load().subfv_ns_sync(self._h, C.byref(steps), C.byref(t)), "subfv_ns_sync")
        return st, steps.value, t.value

    def sol(self) -> np.ndarray:
        out = np.empty((self.mesh.n_elems, 5))
        check(_lib.load().subfv_ns_get_sol(self._h, pd(out)), "subfv_ns_get_sol")
        return out

    def set_node_kernel(self, lanes: int):
        """0: one thread per vertex; 1: a group of lanes per vertex (8/16/32 as the mesh
        needs); 8, 16, 32: a group of at least that many lanes. A group layout also runs
        the cell gradient with 8 lanes per cell (cells of up to 8 vertices). Same results
        in all."""
        check(_lib.load().subfv_ns_state_set_node_kernel(self._h, int(lanes)), "subfv_ns_state_set_node_kernel")

    def residuals(self):
        res, dt = C.c_double(), C.c_double()
        rv = np.zeros(5)
        check(_lib.load().subfv_ns_residuals(self._h, C.byref(res), pd(rv), C.byref(dt)), "subfv_ns_residuals")
        return res.value, rv, dt.value

    def implicit_step(self, cfl_implicit=10.0, krylov=30, rel_tol=1e-8, refine_fp32=False, precond=1):
        """One backward-Euler step (first-order two-wave residual, exact frozen-speed
        Jacobian, GMRES preconditioned by block Jacobi (precond 1) or the coloured LU-SGS
        (2)); returns (status bits, stats dict)."""
        st = ImplicitStats()
        rc = check(_lib.load().subfv_ns_implicit_step_ex(self._h, float(cfl_implicit), int(krylov), float(rel_tol),
                                                         int(refine_fp32), int(precond), C.byref(st)),
                   "subfv_ns_implicit_step")
        return rc, {k: getattr(st, k) for k, _ in ImplicitStats._fields_}

    def be_jacobian(self, dt):
        """(row, col, v (nnz, 5, 5)) of V/dt I - d rhs/dU at the current state."""
        ne = self.mesh.n_elems
        cap = 64 * ne
        row = np.zeros(ne + 1, np.int32)
        col = np.zeros(cap, np.int32)
        v = np.zeros(25 * cap)
        nnz = check(_lib.load().subfv_ns_be_jacobian(self._h, float(dt), row.ctypes.data_as(_lib.PI32),
                                                     col.ctypes.data_as(_lib.PI32), pd(v), cap), "be_jacobian")
        return row, col[:nnz].copy(), v[:25 * nnz].reshape(nnz, 5, 5).copy()

    def close(self):
        if getattr(self, "_h", None):
            _lib.load().subfv_ns_state_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


SUBFV_BATCH_FULL = -3


class NsBatch:
    """Many independent explicit Euler problems advanced together in shared launches
    (no counterpart in the reference, which runs one mesh per process). Each problem's
    result is bit-identical to the same problem run alone through NsState."""

    def __init__(self, cfg: NsConfig, capacity: int, budget_bytes: int):
        self.cfg = cfg
        self._c = cfg.to_c()
        h = C.c_void_p()
        check(_lib.load().subfv_ns_batch_create(C.byref(self._c), int(capacity), int(budget_bytes), C.byref(h)),
              "subfv_ns_batch_create")
        self._h = h
        self._meshes = {}  # slot -> Mesh kept alive while the batch uses it

    def state_bytes(self, mesh: Mesh) -> int:
        """Device bytes of the state this batch allocates for a problem on `mesh`."""
        return int(_lib.load().subfv_ns_batch_state_bytes(self._h, mesh._h))

    def time_steps(self, n_steps: int) -> float:
        """Advance every problem n_steps; device milliseconds (CUDA events)."""
        ms = C.c_double()
        check(_lib.load().subfv_ns_batch_time_steps(self._h, int(n_steps), C.byref(ms)), "subfv_ns_batch_time_steps")
        return ms.value

    def free_bytes(self) -> int:
        return int(_lib.load().subfv_ns_batch_free_bytes(self._h))

    def size(self):
        n, used = C.c_int(), C.c_int64()
        check(_lib.load().subfv_ns_batch_size(self._h, C.byref(n), C.byref(used)), "subfv_ns_batch_size")
        return n.value, used.value

    def add(self, mesh: Mesh, sol, tmax: float, t0: float = 0.0, take_mesh: bool = False):
        """Admit a problem; returns its slot, or None when the batch is full (retry later).
        take_mesh hands the device mesh over: the batch frees it when the slot is removed."""
        sol = f64(sol)
        slot = C.c_int(-1)
        rc = _lib.load().subfv_ns_batch_add(self._h, mesh._h, int(take_mesh), pd(sol), float(t0), float(tmax),
                                            C.byref(slot))
        if rc == SUBFV_BATCH_FULL:
            return None
        check(rc, "subfv_ns_batch_add")
        if take_mesh:
            mesh._h = None  # owned by the batch now
        else:
            self._meshes[slot.value] = mesh
        return slot.value

    def remove(self, slot: int):
        check(_lib.load().subfv_ns_batch_remove(self._h, int(slot)), "subfv_ns_batch_remove")
        self._meshes.pop(slot, None)

    def advance(self, n_steps: int):
        check(_lib.load().subfv_ns_batch_advance(self._h, int(n_steps)), "subfv_ns_batch_advance")

    def poll(self, wait: bool = True) -> bool:
        """Take the oldest outstanding snapshot; False if not complete yet (wait=False)."""
        return check(_lib.load().subfv_ns_batch_poll(self._h, int(wait)), "subfv_ns_batch_poll") == 0

    def sync(self):
        check(_lib.load().subfv_ns_batch_sync(self._h), "subfv_ns_batch_sync")

    def info(self, slot: int):
        """(t, steps, done, status bits) from the latest snapshot taken."""
        t, steps, done, st = C.c_double(), C.c_int64(), C.c_int(), C.c_uint()
        check(_lib.load().subfv_ns_batch_slot_info(self._h, int(slot), C.byref(t), C.byref(steps), C.byref(done),
                                                   C.byref(st)), "subfv_ns_batch_slot_info")
        return t.value, steps.value, bool(done.value), st.value

    def sol(self, slot: int, n_elems: int) -> np.ndarray:
        out = np.empty((n_elems, 5))
        check(_lib.load().subfv_ns_batch_get_sol(self._h, int(slot), pd(out)), "subfv_ns_batch_get_sol")
        return out

    def set_launch(self, block_v: int, grid_v: int, grid_c: int):
        check(_lib.load().subfv_ns_batch_set_launch(self._h, int(block_v), int(grid_v), int(grid_c)),
              "subfv_ns_batch_set_launch")

    def set_node_kernel(self, lanes: int):
        """0: one thread per vertex; 1: a group of lanes per vertex (8/16/32 as the mesh
        needs); 8, 16, 32: a group of at least that many lanes. Same results in all."""
        check(_lib.load().subfv_ns_batch_set_node_kernel(self._h, int(lanes)), "subfv_ns_batch_set_node_kernel")

    def close(self):
        if getattr(self, "_h", None):
            _lib.load().subfv_ns_batch_destroy(self._h)
            self._h = None
            self._meshes.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
