"""The C-ABI library loads and exports every symbol the headers in include/ declare (no GPU calls)."""
import os
import re

import pytest

from xyce_b200 import _native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    syms = set()
    inc = os.path.join(ROOT, "include")
    for name in sorted(os.listdir(inc)):
        if name.endswith(".h"):
            text = re.sub(r"/\*.*?\*/", "", open(os.path.join(inc, name)).read(), flags=re.S)
            syms |= set(re.findall(r"\b(xd_[a-z0-9_]+)\s*\(", text))
    return sorted(syms)


def test_header_declares_the_entry_points():
    syms = header_symbols()
    for s in ("xd_create", "xd_destroy", "xd_update_state", "xd_load_vectors", "xd_load_matrices", "xd_load"):
        assert s in syms


def test_library_exports_every_declared_symbol():
    lib = _native.load()
    for s in header_symbols():
        assert hasattr(lib, s), s
        assert s in _native.SIGNATURES, f"{s} has no ctypes signature"


def test_last_error_is_empty_string_initially():
    lib = _native.load()
    assert isinstance(lib.xd_last_error(), bytes)


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    monkeypatch.setattr(_native, "_LIB", None)
    monkeypatch.setattr(_native, "LIB_PATH", str(tmp_path / "missing.so"))
    with pytest.raises(_native.NativeError):
        _native.load()
