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


_C_TYPES = {"uint32_t": ctypes.c_uint32, "uint64_t": ctypes.c_uint64, "int32_t": ctypes.c_int32,
            "int64_t": ctypes.c_int64, "float": ctypes.c_float, "double": ctypes.c_double, "int": ctypes.c_int,
            "size_t": ctypes.c_size_t, "DgStatus": ctypes.c_int}


def _ctype(decl, is_return=False):
    """ctypes class of one C parameter or return declaration."""
    decl = " ".join(decl.split())
    if "*" in decl:
        return ctypes.c_char_p if is_return and decl.replace(" ", "") == "constchar*" else ctypes.c_void_p
    words = [w for w in decl.split() if w != "const"]
    base = words[0] if is_return else words[-2]
    return _C_TYPES[base]


def _prototypes():
    out = {}
    for h in os.listdir(os.path.join(ROOT, "include")):
        if h.endswith(".h"):
            src = open(os.path.join(ROOT, "include", h)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            for ret, name, params in re.findall(r"DG_API\s+([^;()]+?)\s*\b(dg_\w+)\s*\(([^)]*)\)\s*;", src):
                ps = [p for p in (x.strip() for x in params.split(",")) if p and p != "void"]
                out[name] = (_ctype(ret, True), [_ctype(p) for p in ps])
    return out


def test_ctypes_signatures_match_header():
    """Every prototype's return type and each parameter (pointers as void *)
    equal the ctypes signature the package binds, so no call passes an
    argument of the wrong width."""
    from pydiskann_b200 import _lib

    protos = _prototypes()
    assert set(protos) == _declared()
    sigs = _lib._signatures()
    for name, (ret, args) in protos.items():
        bret, bargs = sigs[name]
        assert bret is ret, f"{name}: return type"
        assert len(bargs) == len(args), f"{name}: {len(bargs)} arguments bound, {len(args)} declared"
        for i, (b, a) in enumerate(zip(bargs, args)):
            assert b is a, f"{name}: argument {i} bound as {b.__name__}, declared {a.__name__}"


# Methods and getters of each class of the reference binding
# (python/src/lib.rs:53-389).  SPFresh.snapshot / restore copy an index to and
# from an object store (remote storage, not the search path) and are not here.
BINDING = {
    "Filter": ["none", "eq", "in_", "lt", "gt", "range", "and_", "or_", "matches"],
    "DiskANN": ["build", "open", "from_bytes", "search", "search_with_dists", "search_batch", "get_vector",
                "num_vectors", "dim", "max_degree"],
    "IncrementalDiskANN": ["build", "open", "from_bytes", "add_vectors", "add_vectors_with_labels",
                           "delete_vectors", "is_deleted", "search", "search_with_dists", "search_filtered",
                           "search_batch", "get_vector", "should_compact", "compact", "stats"],
    "FilteredDiskANN": ["build", "open", "from_bytes", "search", "search_filtered", "search_filtered_with_dists",
                        "search_filtered_batch", "count_matching", "get_labels", "num_vectors", "num_fields"],
    "QuantizedDiskANN": ["build", "open", "save_quantized", "from_bytes", "search", "search_with_dists",
                         "search_batch", "num_vectors", "dim"],
    "SPFresh": ["build", "open", "save", "insert", "delete", "is_deleted", "search", "search_with_dists",
                "search_batch", "get_vector", "gc", "compact", "stats"],
}
MODULE_FUNCTIONS = ["read_fvecs", "read_ivecs", "read_bvecs_as_f32", "write_fvecs", "simd_info"]


def test_binding_surface():
    import pydiskann_b200 as dg
    from pydiskann_b200.spfresh import SPFresh

    for cls, names in BINDING.items():
        missing = [n for n in names if not hasattr(getattr(dg, cls), n)]
        assert not missing, f"{cls} lacks {missing}"
    assert not [f for f in MODULE_FUNCTIONS if not callable(getattr(dg, f, None))]
    # dim is an instance attribute of the updatable indexes
    assert SPFresh(4, device=None).dim == 4
    assert dg.simd_info().startswith("CUDA sm_100a")
