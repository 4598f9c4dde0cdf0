"""The C-ABI library loads and exports every entry point include/b200la.h
declares (no device work: these run without a GPU)."""
import ctypes as C
import os
import re

import pytest

from ba_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared(header):
    src = open(os.path.join(ROOT, "include", header)).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(b200la_\w+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    names = _declared("b200la.h")
    assert len(names) > 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert missing == []


def test_binding_covers_header():
    names = set(_declared("b200la.h"))
    assert names <= set(_lib.exported_symbols()) | {"b200la_version", "b200la_last_error"}


def test_version_and_errors_without_device():
    lib = _lib.load()
    assert lib.b200la_version().startswith(b"b200la")
    # null-argument checks happen before any device call
    assert lib.b200la_ctx_create(0, None) == -1
    assert b"null" in lib.b200la_last_error().lower()
    assert lib.b200la_vec_dot(None, None, None) == -1
    assert lib.b200la_spmv(None, None, None) == -1
    assert lib.b200la_cg_solve(None, None, None, None) == -1


def test_struct_layouts():
    assert C.sizeof(_lib.CgParams) == 40
    assert C.sizeof(_lib.CgResult) == 40


def test_load_fails_loudly_when_missing(monkeypatch):
    monkeypatch.setattr(_lib, "_lib", None)
    monkeypatch.setattr(_lib, "LIB_PATH", "/nonexistent/libb200la.so")
    with pytest.raises(RuntimeError, match="missing"):
        _lib.load()
