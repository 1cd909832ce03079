"""The C-ABI library loads without a GPU and exports every entry point include/subfv.h
declares (no compute calls here)."""
import re
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def declared_symbols():
    syms = set()
    for h in (ROOT / "include").glob("*.h"):
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(subfv_[a-z0-9_]+)\s*\(", text):
            syms.add(m.group(1))
    return syms


def test_all_declared_symbols_exported(native):
    syms = declared_symbols()
    assert len(syms) > 20
    missing = [s for s in sorted(syms) if not hasattr(native, s)]
    assert not missing, missing


def test_ctypes_signatures_cover_header(native):
    from subfv_b200 import _lib
    assert declared_symbols() <= set(_lib.SIGNATURES), declared_symbols() - set(_lib.SIGNATURES)


def test_version(native):
    assert native.subfv_version() >= 1


def test_host_entry_points_reject_bad_arguments(native, tmp_path):
    """Argument checks of entry points that need no GPU: API errors are negative codes
    with a message, never a crash."""
    import ctypes as C
    from subfv_b200 import _lib
    lib = _lib.load()
    h = C.c_void_p()
    assert lib.subfv_msh_read(None, 0, None, C.byref(h)) == -2
    assert lib.subfv_msh_read(str(tmp_path / "none.msh").encode(), 0, None, C.byref(h)) == -2
    assert b"cannot open" in lib.subfv_last_error()
    assert lib.subfv_msh_read(b"x.msh", -1, None, C.byref(h)) == -2
    assert lib.subfv_write_sol_vtu(None, None, None, None, None, None, 1.0, -1.0) == -2
    assert lib.subfv_write_sol_vtu_lag(None, None, None, None, None, None) == -2
    assert lib.subfv_restart_from_vtu(None, 1, None) == -2
    assert lib.subfv_restart_from_vtu(str(tmp_path / "none.vtu").encode(), 0, None) == -2
    assert lib.subfv_lag_prepare(None) == -2
    assert lib.subfv_ns_prepare(None) == -2
    assert lib.subfv_msh_sizes(None, None) == -2
