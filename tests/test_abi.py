"""The C-ABI library loads and exports every entry point include/gvc.h declares
(no compute calls: runs without a GPU)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "gvc.h")


def declared():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(gvc_[a-z_0-9]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    import gvc_native
    lib = gvc_native.lib()
    names = declared()
    assert len(names) >= 14
    for n in names:
        assert hasattr(lib, n), n


def test_binding_table_matches_header():
    import gvc_native
    assert sorted(gvc_native.exported_symbols()) == declared()


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    import gvc_native
    monkeypatch.setattr(gvc_native, "LIB_PATH", str(tmp_path / "nope.so"))
    monkeypatch.setattr(gvc_native, "_lib", None)
    with pytest.raises(RuntimeError, match="libgvc.so not found"):
        gvc_native.lib()

