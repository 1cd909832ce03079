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
