"""The C-ABI library loads and exports every entry point include/dgann.h declares
(no compute calls: this runs without a GPU)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for h in os.listdir(os.path.join(ROOT, "include")):
        if h.endswith(".h"):
            src = open(os.path.join(ROOT, "include", h)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names |= set(re.findall(r"\b(dg_[a-z0-9_]+)\s*\(", src))
    return names


def test_header_declares_entry_points():
    names = _declared()
    assert {"dg_index_create", "dg_search_batch", "dg_build_vamana", "dg_last_error"} <= names


def test_library_exports_every_declared_symbol():
    from pydiskann_b200 import _lib

    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in sorted(_declared()) if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_header():
    from pydiskann_b200 import _lib

    assert _declared() == set(_lib.EXPORTED)


def test_version_and_error_without_gpu():
    from pydiskann_b200 import _lib

    L = _lib.lib()
    assert L.dg_version() == 1
    assert isinstance(L.dg_last_error(), bytes)


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    from pydiskann_b200 import _lib

    monkeypatch.setattr(_lib, "LIB_PATH", str(tmp_path / "absent.so"))
    monkeypatch.setattr(_lib, "_lib", None)
    with pytest.raises(ImportError):
        _lib.lib()
