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


def _enum_values(pattern):
    src = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    return {m.group(1): int(m.group(2)) for m in re.finditer(r"\b(%s)\s*=\s*(\d+)" % pattern, src)}


def test_status_and_option_codes_match_header():
    """gvc_status and the option codes of include/gvc.h against the ctypes binding."""
    import gvc_native
    status = _enum_values(r"GVC_OK|GVC_ERR_[A-Z_]+")
    assert {v: k for k, v in status.items()} == gvc_native.STATUS_NAMES
    assert status["GVC_ERR_TRAVERSAL"] == gvc_native.GVC_ERR_TRAVERSAL
    assert status["GVC_ERR_TIMEOUT"] == gvc_native.GVC_ERR_TIMEOUT
    opts = _enum_values(r"GVC_OPT_[A-Z_]+")
    py = {"GVC_OPT_COV_GRAD": gvc_native.OPT_COV_GRAD, "GVC_OPT_BWD_MODE": gvc_native.OPT_BWD_MODE,
          "GVC_OPT_EVAL_PATH": gvc_native.OPT_EVAL_PATH, "GVC_OPT_COUNT_PAIRS": gvc_native.OPT_COUNT_PAIRS,
          "GVC_OPT_TIME_KERNELS": gvc_native.OPT_TIME_KERNELS, "GVC_OPT_TRAVERSAL": gvc_native.OPT_TRAVERSAL,
          "GVC_OPT_CAND_LOG": gvc_native.OPT_CAND_LOG}
    assert opts == py
