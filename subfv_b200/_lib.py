"""ctypes binding of the native library (include/subfv.h).

The library is built in-tree (subfv_b200/_build/libsubfv_b200.so). There is no
fallback: if it is missing or was built without the entry points, loading fails with
an error naming the build command.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "_build" / "libsubfv_b200.so"

c_int = C.c_int
c_i64 = C.c_int64
c_dbl = C.c_double
c_char_p = C.c_char_p
P = C.c_void_p
PI32 = C.POINTER(C.c_int32)
PD = C.POINTER(C.c_double)

# name -> (restype, argtypes); every exported symbol of include/subfv.h
SIGNATURES = {
    "subfv_last_error": (c_char_p, []),
    "subfv_version": (c_int, []),
    "subfv_probe_fp64_fma": (c_int, [c_int, PD, PD]),
    "subfv_probe_div_const": (c_int, [PD, c_i64, C.POINTER(c_i64)]),
    "subfv_topology_build": (c_int, [c_int, PD, c_int, PI32, PI32, PI32, c_int, PI32, PI32, PI32, c_int, c_int,
                                     C.POINTER(P)]),
    "subfv_topology_build_ex": (c_int, [c_int, PD, c_int, PI32, PI32, PI32, c_int, PI32, PI32, PI32, c_int, c_int,
                                        c_int, C.POINTER(P)]),
    "subfv_topology_array_len": (c_i64, [P, c_char_p]),
    "subfv_topology_array_get": (c_int, [P, c_char_p, PI32]),
    "subfv_topology_coords": (c_int, [P, PD]),
    "subfv_topology_destroy": (None, [P]),
    "subfv_msh_read": (c_int, [c_char_p, c_int, C.POINTER(c_char_p), C.POINTER(P)]),
    "subfv_msh_sizes": (c_int, [P, C.POINTER(c_i64)]),
    "subfv_msh_get": (c_int, [P, PD, PI32, PI32, PI32, PI32, PI32, PI32]),
    "subfv_msh_destroy": (None, [P]),
    "subfv_lag_prepare": (c_int, [P]),
    "subfv_ns_prepare": (c_int, [P]),
    "subfv_write_sol_vtu": (c_int, [c_char_p, P, PD, PD, PD, PD, c_dbl, c_dbl]),
    "subfv_restart_from_vtu": (c_int, [c_char_p, c_i64, PD]),
    "subfv_write_sol_vtu_lag": (c_int, [c_char_p, P, PD, PD, PD, PD]),
    "subfv_mesh_create": (c_int, [P, C.POINTER(P)]),
    "subfv_mesh_create_from_topology": (c_int, [P, c_int, C.POINTER(P)]),
    "subfv_mesh_destroy": (c_int, [P]),
    "subfv_mesh_device_bytes": (c_i64, [P]),
    "subfv_mesh_set_coords": (c_int, [P, PD]),
    "subfv_mesh_get_coords": (c_int, [P, PD]),
    "subfv_mesh_get_geometry": (c_int, [P, c_char_p, PD]),
    "subfv_compute_geometry_mesh": (c_int, [P]),
    "subfv_compute_rhs_lagrange": (c_int, [P, PD, PD, PD, c_int, PD]),
    "subfv_compute_rhs_lagrange_sidil": (c_int, [P, PD, PD, PD, c_int, PD, c_int]),
    "subfv_lag_state_set_scheme": (c_int, [P, c_int, c_int]),
    "subfv_compute_dt": (c_int, [P, PD, c_dbl, PD, PD]),
    "subfv_compute_dt_noalloc": (c_int, [P, P, P, c_dbl, P]),
    "subfv_move_mesh": (c_int, [P, PD, c_dbl]),
    "subfv_lag_state_create": (c_int, [P, PD, PD, c_dbl, c_dbl, c_dbl, c_int, C.POINTER(P)]),
    "subfv_lag_state_destroy": (c_int, [P]),
    "subfv_lag_advance": (c_int, [P, c_int, C.POINTER(c_int), PD]),
    "subfv_lag_advance_async": (c_int, [P, c_int]),
    "subfv_lag_sync": (c_int, [P, C.POINTER(c_int), PD]),
    "subfv_lag_get_sol": (c_int, [P, PD]),
    "subfv_lag_set_sol": (c_int, [P, PD]),
    "subfv_lag_get_vp": (c_int, [P, PD]),
    "subfv_lag_last_dt": (c_int, [P, PD]),
    "subfv_lag_step_host": (c_int, [P, PD]),
    "subfv_lag_profile_steps": (c_int, [P, c_int, PD]),
    "subfv_compute_rhs_ns": (c_int, [P, P, PD, PD, PD, PD, PD]),
    "subfv_compute_rhs_ns_ex": (c_int, [P, P, PD, PD, PD, PD, PD, PD]),
    "subfv_compute_euler_flux": (c_int, [P, P, PD, PD, PD, PD, c_int, PD]),
    "subfv_compute_cell_grad_from_nodal_grad": (c_int, [P, P, PD, PD, PD]),
    "subfv_flux_limiting": (c_int, [P, PD, PD, PD, PD, c_dbl]),
    "subfv_add_timedisc_and_solve": (c_int, [P, PD, PD, PD, PD, PD, PD, PD, c_dbl, c_dbl, c_dbl, c_dbl, c_dbl,
                                             PD]),
    "subfv_ns_state_create": (c_int, [P, P, PD, c_dbl, C.POINTER(P)]),
    "subfv_ns_state_destroy": (c_int, [P]),
    "subfv_ns_state_set_node_kernel": (c_int, [P, c_int]),
    "subfv_ns_advance": (c_int, [P, c_int, C.POINTER(c_int), PD]),
    "subfv_ns_advance_async": (c_int, [P, c_int]),
    "subfv_ns_sync": (c_int, [P, C.POINTER(c_int), PD]),
    "subfv_ns_get_sol": (c_int, [P, PD]),
    "subfv_ns_residuals": (c_int, [P, PD, PD, PD]),
    "subfv_ns_init_gresho": (c_int, [P, c_dbl, PD]),
    "subfv_ns_implicit_step": (c_int, [P, c_dbl, c_int, c_dbl, c_int, P]),
    "subfv_ns_implicit_step_ex": (c_int, [P, c_dbl, c_int, c_dbl, c_int, c_int, P]),
    "subfv_ns_be_jacobian": (c_int, [P, c_dbl, PI32, PI32, PD, c_i64]),
    "subfv_ns_batch_create": (c_int, [P, c_int, c_i64, C.POINTER(P)]),
    "subfv_ns_batch_destroy": (c_int, [P]),
    "subfv_ns_batch_state_bytes": (c_i64, [P, P]),
    "subfv_ns_batch_time_steps": (c_int, [P, c_int, PD]),
    "subfv_ns_batch_free_bytes": (c_i64, [P]),
    "subfv_ns_batch_size": (c_int, [P, C.POINTER(c_int), C.POINTER(c_i64)]),
    "subfv_ns_batch_add": (c_int, [P, P, c_int, PD, c_dbl, c_dbl, C.POINTER(c_int)]),
    "subfv_ns_batch_remove": (c_int, [P, c_int]),
    "subfv_ns_batch_advance": (c_int, [P, c_int]),
    "subfv_ns_batch_poll": (c_int, [P, c_int]),
    "subfv_ns_batch_sync": (c_int, [P]),
    "subfv_ns_batch_slot_info": (c_int, [P, c_int, PD, C.POINTER(c_i64), C.POINTER(c_int), C.POINTER(C.c_uint)]),
    "subfv_ns_batch_get_sol": (c_int, [P, c_int, PD]),
    "subfv_ns_batch_set_launch": (c_int, [P, c_int, c_int, c_int]),
    "subfv_ns_batch_set_node_kernel": (c_int, [P, c_int]),
    "subfv_lag_batch_create": (c_int, [c_int, c_int, c_i64, C.POINTER(P)]),
    "subfv_lag_batch_destroy": (c_int, [P]),
    "subfv_lag_batch_state_bytes": (c_i64, [P, P]),
    "subfv_lag_batch_free_bytes": (c_i64, [P]),
    "subfv_lag_batch_size": (c_int, [P, C.POINTER(c_int), C.POINTER(c_i64)]),
    "subfv_lag_batch_add": (c_int, [P, P, c_int, PD, PD, c_dbl, c_dbl, c_dbl, C.POINTER(c_int)]),
    "subfv_lag_batch_remove": (c_int, [P, c_int]),
    "subfv_lag_batch_advance": (c_int, [P, c_int]),
    "subfv_lag_batch_time_steps": (c_int, [P, c_int, PD]),
    "subfv_lag_batch_poll": (c_int, [P, c_int]),
    "subfv_lag_batch_sync": (c_int, [P]),
    "subfv_lag_batch_slot_info": (c_int, [P, c_int, PD, C.POINTER(c_i64), C.POINTER(c_int), C.POINTER(C.c_uint)]),
    "subfv_lag_batch_get_sol": (c_int, [P, c_int, PD]),
    "subfv_lag_batch_set_grid": (c_int, [P, c_int]),
    "subfv_bcsr_create": (c_int, [c_int, c_int, PI32, PI32, PD, C.POINTER(P)]),
    "subfv_bcsr_destroy": (c_int, [P]),
    "subfv_bcsr_set_colors": (c_int, [P, c_int, PI32]),
    "subfv_bcsr_pcgm": (c_int, [P, PD, PD, c_dbl, C.POINTER(c_int), PD]),
    "subfv_bcsr_parallel_lusgs": (c_int, [P, PD, PD]),
    "subfv_bcsr_gmres_parallel_lusgs": (c_int, [P, PD, PD, c_dbl, c_int, C.POINTER(c_int), C.POINTER(c_int), PD]),
    "subfv_bcsr_set_values": (c_int, [P, PD]),
    "subfv_bcsr_matmul": (c_int, [P, PD, PD]),
    "subfv_bcsr_diag": (c_int, [P, PD, PD]),
    "subfv_bcsr_gmres_diag": (c_int, [P, PD, PD, c_dbl, c_int, C.POINTER(c_int), C.POINTER(c_int), PD]),
    "subfv_bcsr_gmres": (c_int, [P, PD, PD, c_dbl, c_int, C.POINTER(c_int), C.POINTER(c_int), PD]),
    "subfv_bcsr_gmres_ex": (c_int, [P, PD, PD, c_dbl, c_int, c_int, C.POINTER(c_int), C.POINTER(c_int), PD, PD]),
    "subfv_bcsr_gmres_refine": (c_int, [P, PD, PD, c_dbl, c_int, C.POINTER(c_int), C.POINTER(c_int), PD]),
    "subfv_bcsr_profile_spmv": (c_int, [P, c_int, c_int, PD]),
    "subfv_mesh_stream": (P, [P]),
}

_lib = None


class SubfvError(RuntimeError):
    pass


def load():
    """Load the native library once; raise if it is absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise SubfvError(f"native library missing: {LIB_PATH} (run `python -m subfv_b200.build`)")
    lib = C.CDLL(str(LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def last_error() -> str:
    e = load().subfv_last_error()
    return e.decode() if e else ""


def check(rc: int, what: str) -> int:
    """Raise on API/CUDA errors (rc < 0); return numerical status bits (rc >= 0)."""
    if rc < 0:
        raise SubfvError(f"{what} failed ({rc}): {last_error()}")
    return rc


def f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def i32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.int32)


def pd(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(PD)


def pi(a: np.ndarray):
    assert a.dtype == np.int32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(PI32)
