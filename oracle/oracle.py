"""Test infrastructure only: ctypes binding of the oracle (oracle/_build/liboracle.so).

The oracle is a serial CPU restatement of the reference Fortran (see oracle.h).
PARITY UNPINNED: no Fortran compiler exists here and the reference's tests hold no
golden vectors. Only tests/, the smoke check and bench.py's CPU-baseline leg use it.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "liboracle.so"

PD = C.POINTER(C.c_double)
PI = C.POINTER(C.c_int32)
_lib = None


def build() -> Path:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB_PATH


def load():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        lib = C.CDLL(str(LIB_PATH))
        lib.or_mesh_new.restype = C.c_void_p
        lib.or_mesh_new.argtypes = [C.c_int, PD, C.c_int, PI, PI, PI, C.c_int, PI, PI, PI, C.c_int, C.c_int]
        lib.or_mesh_new_ex.restype = C.c_void_p
        lib.or_mesh_new_ex.argtypes = [C.c_int, PD, C.c_int, PI, PI, PI, C.c_int, PI, PI, PI, C.c_int, C.c_int,
                                       C.c_int]
        lib.or_mesh_free.argtypes = [C.c_void_p]
        lib.or_topo_len.argtypes = [C.c_void_p, C.c_char_p]
        lib.or_topo_get.argtypes = [C.c_void_p, C.c_char_p, PI]
        lib.or_vert_is_bound.argtypes = [C.c_void_p, PI]
        lib.or_geometry.argtypes = [C.c_void_p, C.c_int]
        lib.or_geometry_ok.argtypes = [C.c_void_p]
        lib.or_set_coords.argtypes = [C.c_void_p, PD]
        lib.or_geom_get.argtypes = [C.c_void_p, C.c_char_p, PD]
        lib.or_lag_rhs.argtypes = [C.c_void_p, PD, PD, PD, C.c_int, PD]
        lib.or_lag_dt.restype = C.c_double
        lib.or_lag_dt.argtypes = [C.c_void_p, PD, C.c_double, PD]
        lib.or_lag_move.argtypes = [C.c_void_p, PD, C.c_double]
        lib.or_sedov_init.argtypes = [C.c_void_p, PD, C.c_double, C.c_double, PI]
        lib.or_lag_run.argtypes = [C.c_void_p, PD, PD, PD, PD, C.c_double, C.c_double, C.c_int, C.c_int, PD, PD]
        lib.or_lag_run_scheme.argtypes = [C.c_void_p, PD, PD, PD, PD, C.c_double, C.c_double, C.c_int, C.c_int, PD,
                                          PD, C.c_int, C.c_int]
        lib.or_lag_rhs_sidil.argtypes = [C.c_void_p, PD, PD, PD, C.c_int, PD, C.c_int]
        lib.or_inverse_3_by_3.argtypes = [PD, PD]
        lib.or_fnorm2.restype = C.c_double
        lib.or_fnorm2.argtypes = [PD, C.c_int]
        lib.or_ns_rhs.argtypes = [C.c_void_p, PI, PD, PI, PD, PD, PD, PD, PD, PD]
        lib.or_ns_rhs_diag.argtypes = [C.c_void_p, PI, PD, PI, PD, PD, PD, PD, PD]
        lib.or_ns_run.argtypes = [C.c_void_p, PI, PD, PI, PD, PD, C.c_int, C.c_double, PD, PI, PD, PD, PD]
        lib.or_ns_gresho.argtypes = [C.c_void_p, C.c_double, PD]
        lib.or_pinv3.argtypes = [PD]
        lib.or_euler_flux.argtypes = [C.c_void_p, PI, PD, PI, PD, PD, PD, C.c_int, PD, PD, PD]
        lib.or_cell_grads.argtypes = [C.c_void_p, PI, PD, PI, PD, PD, PD, PD]
        lib.or_flux_limiting.argtypes = [C.c_void_p, PD, PD, PD, PD, C.c_double]
        lib.or_add_timedisc.argtypes = [C.c_void_p, PI, PD, PI, PD, PD, PD, PD, PD, PD, PD, PD, C.c_double,
                                        C.c_double, C.c_double, PD]
        lib.or_set_lapack.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        lib.or_ns_flux.argtypes = [C.c_int, PD, PD, PD, PD, PD]
        lib.or_lu3.argtypes = [PD, PD, PD]
        lib.or_potential_flow.argtypes = [PD, C.c_int, PD]
        lib.or_lapack_inverse.argtypes = [C.c_int, PD]
        lib.or_lapack_solve.argtypes = [C.c_int, PD, PD]
        lib.or_ns_set_diffusion.argtypes = [C.c_int, C.c_int, PD, C.c_int, PI, PD, PI, PD]
        lib.or_bcsr_matmul.argtypes = [C.c_int, C.c_int, C.c_int, PI, PI, PD, PD, PD]
        lib.or_bcsr_diag.argtypes = [C.c_int, C.c_int, PI, PI, PD, PD, PD]
        lib.or_bcsr_pcgm.argtypes = [C.c_int, C.c_int, PI, PI, PD, PD, PD, C.c_double, PI, PD]
        lib.or_bcsr_parallel_lusgs.argtypes = [C.c_int, C.c_int, PI, PI, PD, C.c_int, PI, PD, PD]
        lib.or_bcsr_gmres_lusgs.argtypes = [C.c_int, C.c_int, PI, PI, PD, C.c_int, PI, PD, PD, C.c_double, C.c_int,
                                            PI, PD]
        lib.or_bcsr_gmres.argtypes = [C.c_int, C.c_int, PI, PI, PD, PD, PD, C.c_double, C.c_int, C.c_int, PI, PD, PD]
        lib.or_be_jacobian.restype = C.c_long
        lib.or_be_jacobian.argtypes = [C.c_void_p, PI, PD, PI, PD, PD, C.c_double, PI, PI, PD, C.c_long]
        _lib = lib
    return _lib


def _capsule_ptr(name):
    """The C function pointer behind scipy.linalg.cython_lapack's exported routine."""
    from scipy.linalg import cython_lapack
    cap = cython_lapack.__pyx_capi__[name]
    get_name = C.pythonapi.PyCapsule_GetName
    get_name.restype, get_name.argtypes = C.c_char_p, [C.py_object]
    get_ptr = C.pythonapi.PyCapsule_GetPointer
    get_ptr.restype, get_ptr.argtypes = C.c_void_p, [C.py_object, C.c_char_p]
    return get_ptr(cap, get_name(cap))


def use_lapack(on: bool):
    """Route the oracle's 3x3 pseudo-inverse and LU solve through scipy's bundled LAPACK
    (dgesvd, dgetrf, dgetrs), called as the reference calls system LAPACK
    (linear_solver_module.F90:643-715); off restores the restated algorithms that the
    GPU kernels follow."""
    if on:
        load().or_set_lapack(_capsule_ptr("dgesvd"), _capsule_ptr("dgetrf"), _capsule_ptr("dgetrs"))
    else:
        load().or_set_lapack(None, None, None)


def _pd(a):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(PD)


def _pi(a):
    assert a.dtype == np.int32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(PI)


class OracleMesh:
    """build_mesh + compute_geometry_mesh on the CPU, as the reference does them."""

    def __init__(self, raw, renumber="bfs"):
        lib = load()
        self._keep = [np.ascontiguousarray(raw.coords.reshape(-1), np.float64),
                      np.ascontiguousarray(raw.elem_kind, np.int32),
                      np.ascontiguousarray(raw.elem_vert_off, np.int32),
                      np.ascontiguousarray(raw.elem_vert, np.int32),
                      np.ascontiguousarray(raw.bface_off, np.int32),
                      np.ascontiguousarray(raw.bface_vert, np.int32),
                      np.ascontiguousarray(raw.bface_tag, np.int32)]
        c, k, o, v, bo, bv, bt = self._keep
        self.b2d = bool(raw.b2d)
        self._h = lib.or_mesh_new_ex(raw.n_vert, _pd(c), raw.n_elems, _pi(k), _pi(o), _pi(v), int(bo.size - 1),
                                     _pi(bo), _pi(bv), _pi(bt), int(raw.b2d), int(raw.periodic),
                                     {"bfs": 0, "hilbert": 1}[renumber])
        if not self._h:
            raise RuntimeError("oracle build_mesh failed")
        s = self.topo("sizes")
        self.n_vert, self.n_elems, self.n_faces, self.n_sub_faces, self.n_sub_elems = map(int, s[:5])

    def topo(self, name):
        lib = load()
        n = lib.or_topo_len(self._h, name.encode())
        if n < 0:
            raise KeyError(name)
        out = np.empty(n, np.int32)
        lib.or_topo_get(self._h, name.encode(), _pi(out))
        return out

    _N = {"vert_coord": ("n_vert", 3), "vert_volume": ("n_vert", 1), "face_coord": ("n_faces", 3),
          "face_norm": ("n_faces", 3), "face_area": ("n_faces", 1), "sub_face_norm": ("n_sub_faces", 3),
          "sub_face_area": ("n_sub_faces", 1), "elem_coord": ("n_elems", 3), "elem_volume": ("n_elems", 1),
          "sub_elem_volume": ("n_sub_elems", 1)}

    def geom(self, name):
        cnt, comp = self._N[name]
        n = getattr(self, cnt)
        out = np.empty(n * comp)
        if load().or_geom_get(self._h, name.encode(), _pd(out)) != 0:
            raise KeyError(name)
        return out.reshape(n, comp) if comp > 1 else out

    def vert_is_bound(self):
        out = np.empty(self.n_vert, np.int32)
        load().or_vert_is_bound(self._h, _pi(out))
        return out

    def geometry(self):
        return load().or_geometry(self._h, int(self.b2d))

    def geometry_ok(self):
        return bool(load().or_geometry_ok(self._h))

    def set_coords(self, c):
        c = np.ascontiguousarray(np.asarray(c).reshape(-1), np.float64)
        load().or_set_coords(self._h, _pd(c))

    # --- Lagrange
    def lag_rhs(self, sol, mass):
        sol = np.ascontiguousarray(sol, np.float64)
        mass = np.ascontiguousarray(mass, np.float64)
        vp = np.zeros((self.n_vert, 3))
        rhs = np.zeros((self.n_elems, 5))
        load().or_lag_rhs(self._h, _pd(sol), _pd(vp), _pd(rhs), int(self.b2d), _pd(mass))
        return vp, rhs

    def lag_rhs_sidil(self, sol, mass, method):
        """compute_rhs_lagrange_sidil: (status, vp, rhs)."""
        sol = np.ascontiguousarray(sol, np.float64)
        mass = np.ascontiguousarray(mass, np.float64)
        vp = np.zeros((self.n_vert, 3))
        rhs = np.zeros((self.n_elems, 5))
        st = load().or_lag_rhs_sidil(self._h, _pd(sol), _pd(vp), _pd(rhs), int(self.b2d), _pd(mass), int(method))
        return st, vp, rhs

    def lag_dt(self, sol, cfl, vp):
        sol = np.ascontiguousarray(sol, np.float64)
        vp = np.ascontiguousarray(vp, np.float64)
        return load().or_lag_dt(self._h, _pd(sol), float(cfl), _pd(vp))

    def lag_move(self, vp, dt):
        vp = np.ascontiguousarray(vp, np.float64)
        load().or_lag_move(self._h, _pd(vp), float(dt))

    def sedov_init(self, r_sedov=0.06, e_total=0.983909, mask=None):
        sol = np.zeros((self.n_elems, 5))
        m = None if mask is None else np.ascontiguousarray(mask, np.int32)
        rc = load().or_sedov_init(self._h, _pd(sol), float(r_sedov), float(e_total), None if m is None else _pi(m))
        if rc != 0:
            raise ValueError("r_sedov too small")
        return sol

    def lag_run(self, sol, mass, cfl, t_max, max_steps, t0=0.0, scheme=0, method=0):
        """Runs the reference time loop in place on sol (scheme 0 classic, 1 sidil with
        method_length `method`); returns (steps, t, last dt, vp)."""
        assert sol.dtype == np.float64 and sol.flags["C_CONTIGUOUS"]
        mass = np.ascontiguousarray(mass, np.float64)
        vp = np.zeros((self.n_vert, 3))
        rhs = np.zeros((self.n_elems, 5))
        t = C.c_double(t0)
        dt = C.c_double(0.0)
        n = load().or_lag_run_scheme(self._h, _pd(sol), _pd(vp), _pd(rhs), _pd(mass), float(cfl), float(t_max),
                                     int(max_steps), int(self.b2d), C.byref(t), C.byref(dt), int(scheme),
                                     int(method))
        return n, t.value, dt.value, vp

    # --- explicit Euler (subfvns)
    @staticmethod
    def _ns_args(cfg):
        nb = max(1, int(cfg.get("n_bc", 0)))
        dc = list(cfg.get("diff_dc", [1.329e-5, 1.716e-5, 273.15, 720.19471]))
        dc = dc + [0.71] * (5 - len(dc))
        dif = [np.ascontiguousarray(dc, np.float64),
               np.ascontiguousarray(cfg.get("bc_type_V", np.zeros(nb)), np.int32),
               np.ascontiguousarray(cfg.get("bc_val_V", np.zeros((nb, 3))), np.float64).reshape(-1),
               np.ascontiguousarray(cfg.get("bc_type_T", np.zeros(nb)), np.int32),
               np.ascontiguousarray(cfg.get("bc_val_T", np.zeros(nb)), np.float64)]
        load().or_ns_set_diffusion(int(cfg.get("activate_diffusion", 0)), int(cfg.get("use_sutherland", 0)),
                                   _pd(dif[0]), int(cfg.get("n_bc", 0)), _pi(dif[1]), _pd(dif[2]), _pi(dif[3]),
                                   _pd(dif[4]))
        ic = np.array([cfg["scheme"], cfg["second_order"], cfg["method"], cfg["bc_style"], cfg["b2d"],
                       cfg["exclude_bound_vert"], cfg["local_time_step"], cfg.get("n_bc", 0)], np.int32)
        dc = np.array([cfg["cfl"], cfg["tmax"]], np.float64)
        bt = np.ascontiguousarray(cfg.get("bc_type", np.zeros(1, np.int32)), np.int32)
        bv = np.ascontiguousarray(cfg.get("bc_val", np.zeros(5)), np.float64).reshape(-1)
        return ic, dc, bt, bv

    def be_jacobian(self, cfg, sol, dt):
        """Backward-Euler matrix V/dt I - d rhs/dU of the first-order two-wave residual
        (frozen wave speeds); returns (row, col, v (nnz, 5, 5) with v[j].T the block)."""
        ic, dc, bt, bv = self._ns_args(cfg)
        sol = np.ascontiguousarray(sol, np.float64)
        cap = 64 * self.n_elems
        row = np.zeros(self.n_elems + 1, np.int32)
        col = np.zeros(cap, np.int32)
        v = np.zeros(25 * cap)
        nnz = load().or_be_jacobian(self._h, _pi(ic), _pd(dc), _pi(bt), _pd(bv), _pd(sol), float(dt), _pi(row),
                                    _pi(col), _pd(v), cap)
        assert nnz > 0
        return row, col[:nnz].copy(), v[:25 * nnz].reshape(nnz, 5, 5).copy()

    def ns_gresho(self, mach):
        sol = np.zeros((self.n_elems, 5))
        load().or_ns_gresho(self._h, float(mach), _pd(sol))
        return sol

    def ns_rhs(self, cfg, sol):
        ic, dc, bt, bv = self._ns_args(cfg)
        sol = np.ascontiguousarray(sol, np.float64)
        rhs = np.zeros((self.n_elems, 5))
        sl = np.zeros(self.n_elems)
        vp = np.zeros((self.n_vert, 3))
        grad = np.zeros((self.n_elems, 15))
        st = load().or_ns_rhs(self._h, _pi(ic), _pd(dc), _pi(bt), _pd(bv), _pd(sol), _pd(rhs), _pd(sl), _pd(vp),
                              _pd(grad))
        return st, rhs, sl, vp, grad

    def ns_rhs_diag(self, cfg, sol):
        """compute_rhs_ns with the diffusion blocks: (status, rhs, sum_lambda, mat_diag (n, 5, 5))."""
        ic, dc, bt, bv = self._ns_args(cfg)
        sol = np.ascontiguousarray(sol, np.float64)
        rhs = np.zeros((self.n_elems, 5))
        sl = np.zeros(self.n_elems)
        diag = np.zeros((self.n_elems, 5, 5))
        st = load().or_ns_rhs_diag(self._h, _pi(ic), _pd(dc), _pi(bt), _pd(bv), _pd(sol), _pd(rhs), _pd(sl),
                                   _pd(diag))
        return st, rhs, sl, diag

    # --- the procedures one at a time (grad arrays (n, 5, 3) = the reference's (3, 5, n))
    @staticmethod
    def _g_to_oracle(g):
        return np.ascontiguousarray(np.asarray(g, np.float64).transpose(0, 2, 1).reshape(-1, 15))

    @staticmethod
    def _g_from_oracle(g):
        return np.ascontiguousarray(g.reshape(-1, 3, 5).transpose(0, 2, 1))

    def euler_flux(self, cfg, sol, grad, second_order):
        """compute_euler_flux: (status, rhs (n, 5), sum_lambda (n,), vp (nv, 3))."""
        ic, dc, bt, bv = self._ns_args(cfg)
        sol = np.ascontiguousarray(sol, np.float64)
        g = self._g_to_oracle(grad) if grad is not None else np.zeros((self.n_elems, 15))
        rhs, sl, vp = np.zeros((self.n_elems, 5)), np.zeros(self.n_elems), np.zeros((self.n_vert, 3))
        st = load().or_euler_flux(self._h, _pi(ic), _pd(dc), _pi(bt), _pd(bv), _pd(sol), _pd(g), int(second_order),
                                  _pd(rhs), _pd(sl), _pd(vp))
        return st, rhs, sl, vp

    def cell_grads(self, cfg, sol):
        """compute_cell_grad_from_nodal_grad: (grad (n, 5, 3), nodal_grad (nv, 5, 3))."""
        ic, dc, bt, bv = self._ns_args(cfg)
        sol = np.ascontiguousarray(sol, np.float64)
        g, ng = np.zeros((self.n_elems, 15)), np.zeros((self.n_vert, 15))
        load().or_cell_grads(self._h, _pi(ic), _pd(dc), _pi(bt), _pd(bv), _pd(sol), _pd(g), _pd(ng))
        return self._g_from_oracle(g), self._g_from_oracle(ng)

    def flux_limiting(self, sol, rhs, rhs_o2, sum_lambda, cfl):
        """flux_limiting on a copy of rhs; returns it."""
        r = np.array(rhs, np.float64)
        load().or_flux_limiting(self._h, _pd(np.ascontiguousarray(sol, np.float64)), _pd(r),
                                _pd(np.ascontiguousarray(rhs_o2, np.float64)),
                                _pd(np.ascontiguousarray(sum_lambda, np.float64)), float(cfl))
        return r

    def add_timedisc(self, cfg, sol, rhs, diag, sum_lambda, a1, a2, t):
        """add_timedisc_and_solve in place on sol, rhs, diag (n, 5, 5) or None, sum_lambda;
        returns (status, delta (n, 5), res, res_vect, dt)."""
        ic, dc, bt, bv = self._ns_args(cfg)
        delta, rv = np.zeros((self.n_elems, 5)), np.zeros(5)
        res, dt = C.c_double(), C.c_double()
        st = load().or_add_timedisc(self._h, _pi(ic), _pd(dc), _pi(bt), _pd(bv), _pd(sol), _pd(rhs),
                                    _pd(diag) if diag is not None else None, _pd(sum_lambda), _pd(delta),
                                    C.byref(res), _pd(rv), float(a1), float(a2), float(t), C.byref(dt))
        return st, delta, res.value, rv, dt.value

    def ns_run(self, cfg, sol, n_max_iter, final_res=-1.0, t0=0.0):
        """The ns_main time loop in place on sol (n_max_iter + 1 steps unless stopped)."""
        ic, dc, bt, bv = self._ns_args(cfg)
        assert sol.dtype == np.float64 and sol.flags["C_CONTIGUOUS"]
        t = C.c_double(t0)
        it = C.c_int32(0)
        res = C.c_double(0.0)
        rv = np.zeros(5)
        vp = np.zeros((self.n_vert, 3))
        st = load().or_ns_run(self._h, _pi(ic), _pd(dc), _pi(bt), _pd(bv), _pd(sol), int(n_max_iter),
                              float(final_res), C.byref(t), C.byref(it), C.byref(res), _pd(rv), _pd(vp))
        return st, it.value, t.value, res.value, rv, vp

    def close(self):
        if getattr(self, "_h", None):
            load().or_mesh_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class OracleBcsr:
    """bcsr_matmul / bcsr_diag / bcsr_gmres(_diag) on the CPU (restatement)."""

    def __init__(self, A):
        self.m, self.bs = A.m, A.blc_size
        self.row = np.ascontiguousarray(A.row, np.int32)
        self.col = np.ascontiguousarray(A.col, np.int32)
        self.v = np.ascontiguousarray(A.v.reshape(-1), np.float64)
        self.n = self.m * self.bs

    def matmul(self, x):
        x = np.ascontiguousarray(x, np.float64)
        y = np.empty(self.n)
        load().or_bcsr_matmul(self.m, self.m, self.bs, _pi(self.row), _pi(self.col), _pd(self.v), _pd(x), _pd(y))
        return y

    def diag(self, b):
        b = np.ascontiguousarray(b, np.float64)
        x = np.zeros(self.n)
        load().or_bcsr_diag(self.m, self.bs, _pi(self.row), _pi(self.col), _pd(self.v), _pd(x), _pd(b))
        return x

    def pcgm(self, b, tol, x0=None):
        """bcsr_pcgm from x0 (zeros if None): (x, iterations, status, res)."""
        b = np.ascontiguousarray(b, np.float64)
        x = np.zeros(self.n) if x0 is None else np.array(x0, np.float64)
        st = np.zeros(1, np.int32)
        res = np.zeros(1)
        it = load().or_bcsr_pcgm(self.m, self.bs, _pi(self.row), _pi(self.col), _pd(self.v), _pd(x), _pd(b),
                                 float(tol), _pi(st), _pd(res))
        return x, it, int(st[0]), float(res[0])

    def parallel_lusgs(self, b, ncs, color):
        b = np.ascontiguousarray(b, np.float64)
        c = np.ascontiguousarray(color, np.int32)
        x = np.zeros(self.n)
        load().or_bcsr_parallel_lusgs(self.m, self.bs, _pi(self.row), _pi(self.col), _pd(self.v), int(ncs), _pi(c),
                                      _pd(x), _pd(b))
        return x

    def gmres_lusgs(self, b, tol, m, ncs, color):
        b = np.ascontiguousarray(b, np.float64)
        c = np.ascontiguousarray(color, np.int32)
        x = np.empty(self.n)
        conv = np.zeros(1, np.int32)
        rho = np.zeros(1)
        it = load().or_bcsr_gmres_lusgs(self.m, self.bs, _pi(self.row), _pi(self.col), _pd(self.v), int(ncs),
                                        _pi(c), _pd(x), _pd(b), float(tol), int(m), _pi(conv), _pd(rho))
        return x, bool(conv[0]), it, float(rho[0])

    def gmres(self, b, tol, m=30, precond=True):
        b = np.ascontiguousarray(b, np.float64)
        x = np.empty(self.n)
        conv = np.zeros(1, np.int32)
        rho = np.zeros(1)
        H = np.zeros((m, m + 1))
        it = load().or_bcsr_gmres(self.m, self.bs, _pi(self.row), _pi(self.col), _pd(self.v), _pd(x), _pd(b),
                                  float(tol), int(m), int(precond), _pi(conv), _pd(rho), _pd(H))
        return x, bool(conv[0]), it, float(rho[0]), H
