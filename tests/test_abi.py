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


def test_builder_library_exports_the_construction_subset():
    """libdgbuild.so (index construction only) exports the construction entry
    points and the error text, and none of the search or index calls."""
    from pydiskann_b200 import _lib

    lib = ctypes.CDLL(_lib.BUILD_LIB_PATH)
    assert all(hasattr(lib, n) for n in _lib.BUILDER)
    assert set(_lib.BUILDER) <= _declared()
    for n in ("dg_index_create", "dg_search_batch", "dg_server_create", "dg_spfresh_search_batch"):
        assert not hasattr(lib, n), n


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
    "DiskANN": ["build", "open", "from_bytes", "to_bytes", "search", "search_with_dists", "search_batch",
                "get_vector", "num_vectors", "dim", "max_degree"],
    "IncrementalDiskANN": ["build", "open", "from_bytes", "to_bytes", "add_vectors", "add_vectors_with_labels",
                           "delete_vectors", "is_deleted", "search", "search_with_dists", "search_filtered",
                           "search_batch", "get_vector", "should_compact", "compact", "stats"],
    "FilteredDiskANN": ["build", "open", "from_bytes", "to_bytes", "search", "search_filtered", "search_filtered_with_dists",
                        "search_filtered_batch", "count_matching", "get_labels", "num_vectors", "num_fields"],
    "QuantizedDiskANN": ["build", "open", "save_quantized", "from_bytes", "to_bytes", "search", "search_with_dists",
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


# Parameter names and defaults of the reference binding's methods, from their
# #[pyo3(signature = ...)] attributes (python/src/lib.rs:84-356); REQ marks a
# parameter without a default.
REQ = object()
_SEARCH = [("query", REQ), ("k", 10), ("beam_width", 128)]
_BATCH = [("queries", REQ), ("k", 10), ("beam_width", 128)]
_OPEN = [("path", REQ), ("metric", "l2")]
_BYTES = [("data", REQ), ("metric", "l2")]
SIGNATURES = {
    ("DiskANN", "build"): [("vectors", REQ), ("path", REQ), ("metric", "l2"), ("max_degree", 64),
                           ("build_beam_width", 128), ("alpha", 1.2)],
    ("DiskANN", "open"): _OPEN, ("DiskANN", "from_bytes"): _BYTES, ("DiskANN", "search"): _SEARCH,
    ("DiskANN", "search_with_dists"): _SEARCH, ("DiskANN", "search_batch"): _BATCH,
    ("IncrementalDiskANN", "build"): [("vectors", REQ), ("path", REQ), ("metric", "l2"), ("labels", None),
                                      ("quantizer", None), ("rerank_size", 0), ("pq_subspaces", 8),
                                      ("delta_threshold", 10_000), ("tombstone_ratio", 0.1)],
    ("IncrementalDiskANN", "open"): _OPEN, ("IncrementalDiskANN", "from_bytes"): _BYTES,
    ("IncrementalDiskANN", "search"): _SEARCH, ("IncrementalDiskANN", "search_with_dists"): _SEARCH,
    ("IncrementalDiskANN", "search_filtered"): [("query", REQ), ("filter", REQ), ("k", 10), ("beam_width", 128)],
    ("IncrementalDiskANN", "search_batch"): _BATCH,
    ("FilteredDiskANN", "build"): [("vectors", REQ), ("labels", REQ), ("path", REQ), ("metric", "l2"),
                                   ("max_degree", 64), ("build_beam_width", 128), ("alpha", 1.2)],
    ("FilteredDiskANN", "open"): _OPEN, ("FilteredDiskANN", "from_bytes"): _BYTES,
    ("FilteredDiskANN", "search"): _SEARCH,
    ("FilteredDiskANN", "search_filtered"): [("query", REQ), ("filter", REQ), ("k", 10), ("beam_width", 128)],
    ("FilteredDiskANN", "search_filtered_with_dists"): [("query", REQ), ("filter", REQ), ("k", 10),
                                                        ("beam_width", 128)],
    ("FilteredDiskANN", "search_filtered_batch"): [("queries", REQ), ("filter", REQ), ("k", 10),
                                                   ("beam_width", 128)],
    ("QuantizedDiskANN", "build"): [("vectors", REQ), ("path", REQ), ("quantizer", "f16"), ("metric", "l2"),
                                    ("rerank_size", 0), ("pq_subspaces", 8), ("max_degree", 64),
                                    ("build_beam_width", 128), ("alpha", 1.2)],
    ("QuantizedDiskANN", "open"): [("base_path", REQ), ("quantized_path", REQ), ("metric", "l2"),
                                   ("rerank_size", 0)],
    ("QuantizedDiskANN", "from_bytes"): [("data", REQ), ("metric", "l2"), ("rerank_size", 0)],
    ("QuantizedDiskANN", "search"): _SEARCH, ("QuantizedDiskANN", "search_with_dists"): _SEARCH,
    ("QuantizedDiskANN", "search_batch"): _BATCH,
    ("SPFresh", "build"): [("vectors", REQ), ("path", REQ), ("metric", "l2"), ("quantizer", None),
                           ("rerank_size", 0), ("pq_subspaces", 8), ("max_posting_size", 128),
                           ("min_posting_size", 16), ("reassign_neighbors", 16), ("probe_ratio", float("inf"))],
    ("SPFresh", "open"): _OPEN,
    ("SPFresh", "search"): [("query", REQ), ("k", 10), ("n_probe", 8)],
    ("SPFresh", "search_with_dists"): [("query", REQ), ("k", 10), ("n_probe", 8)],
    ("SPFresh", "search_batch"): [("queries", REQ), ("k", 10), ("n_probe", 8)],
}


@pytest.mark.parametrize("cls, method", list(SIGNATURES))
def test_binding_signatures(cls, method):
    """Each reference parameter sits at the same position under the same name
    with the same default, so positional and keyword calls written against the
    reference binding work unchanged.  (A parameter the reference requires may
    be optional here, e.g. `path`; parameters added after the reference's
    ones must have defaults.)"""
    import inspect

    import pydiskann_b200 as dg
    from pydiskann_b200.spfresh import SPFresh

    owner = SPFresh if cls == "SPFresh" else getattr(dg, cls)
    f = inspect.getattr_static(owner, method)
    f = f.__func__ if isinstance(f, (staticmethod, classmethod)) else f
    f = getattr(f, "__wrapped__", f)
    ps = [p for p in inspect.signature(f).parameters.values() if p.name != "self"]
    want = SIGNATURES[(cls, method)]
    assert len(ps) >= len(want), f"{cls}.{method} takes {len(ps)} parameters"
    for p, (name, default) in zip(ps, want):
        assert p.name == name, f"{cls}.{method}: {p.name} where the reference has {name}"
        if default is not REQ:
            assert p.default == default, f"{cls}.{method}({name}=) defaults to {p.default!r}, not {default!r}"
    assert all(p.default is not inspect.Parameter.empty for p in ps[len(want):])


def test_errors_raised_before_any_device_work(tmp_path):
    """The binding's error classes and messages (python/src/lib.rs:25-49): an
    unknown metric or quantizer is a ValueError, a missing file a RuntimeError
    carrying DiskAnnError::Io's text.  All of them are raised on the host,
    before any device work."""
    import numpy as np

    import pydiskann_b200 as dg
    from pydiskann_b200.spfresh import SPFresh

    X = np.zeros((4, 2), np.float32)
    bad_metric = [lambda: dg.DiskANN.build(X, None, metric="m"), lambda: dg.DiskANN.open("x", metric="m"),
                  lambda: dg.QuantizedDiskANN.build(X, None, metric="m"),
                  lambda: dg.FilteredDiskANN.build(X, np.zeros((4, 1), np.uint64), None, metric="m"),
                  lambda: dg.IncrementalDiskANN.build(X, None, metric="m"), lambda: SPFresh.build(X, None, metric="m"),
                  lambda: SPFresh.open("x", metric="m")]
    for f in bad_metric:
        with pytest.raises(ValueError, match="^unknown metric: m$"):
            f()
    for f in (lambda: dg.QuantizedDiskANN.build(X, None, quantizer="q"),
              lambda: dg.IncrementalDiskANN.build(X, None, quantizer="q"), lambda: SPFresh.build(X, None, quantizer="q")):
        with pytest.raises(ValueError, match="^unknown quantizer: q$"):
            f()
    gone = str(tmp_path / "absent")
    for f in (lambda: dg.DiskANN.open(gone), lambda: dg.FilteredDiskANN.open(gone),
              lambda: dg.QuantizedDiskANN.open(gone, gone + ".q"), lambda: dg.IncrementalDiskANN.open(gone),
              lambda: SPFresh.open(gone), lambda: dg.read_fvecs(gone)):
        with pytest.raises(RuntimeError, match=r"^I/O error: No such file or directory \(os error 2\)$"):
            f()


def test_build_validation_messages():
    """DiskAnnError::IndexError texts of the builders' input checks
    (src/lib.rs:412-424, src/filtered.rs:181-186), raised on the host."""
    import numpy as np

    import pydiskann_b200 as dg

    E, X = np.zeros((0, 3), np.float32), np.zeros((4, 3), np.float32)
    for f in (lambda: dg.DiskANN.build(E, None), lambda: dg.QuantizedDiskANN.build(E, None),
              lambda: dg.FilteredDiskANN.build(E, np.zeros((0, 1), np.uint64), None)):
        with pytest.raises(RuntimeError, match="^Index error: No vectors provided$"):
            f()
    with pytest.raises(RuntimeError, match="^Index error: Vector 2 has dimension 2 but expected 3$"):
        dg.DiskANN.build([[1, 2, 3], [4, 5, 6], [7, 8]], None)
    with pytest.raises(RuntimeError, match=r"^Index error: vectors.len\(\) \(4\) != labels.len\(\) \(3\)$"):
        dg.FilteredDiskANN.build(X, np.zeros((3, 1), np.uint64), None)


def test_insert_dimension_checks():
    """Inserts name the first vector of the wrong length, ragged lists
    included, with the reference's texts (SPFresh: src/spfresh.rs:417-421;
    IncrementalDiskANN: src/incremental.rs:834-843), and leave the index as it
    was (python/tests/test_spfresh.py:239-243)."""
    import numpy as np

    from pydiskann_b200 import _lib
    from pydiskann_b200.spfresh import SPFresh

    s = SPFresh.build(np.random.default_rng(0).standard_normal((300, 8)).astype(np.float32), None,
                      max_posting_size=24, device=None)
    st = s.stats()
    for bad, n in (([[0.0] * 9], 9), ([[0.0] * 8, [0.0] * 7], 7), (np.zeros((2, 9), np.float32), 9)):
        with pytest.raises(RuntimeError, match=f"^Index error: Vector dim {n} != index dim 8$"):
            s.insert(bad)
    assert s.stats() == st
    msg = lambda i, n: f"Index error: Vector {i} has dimension {n} but index expects 8"  # noqa: E731
    with pytest.raises(RuntimeError, match="^Index error: Vector 2 has dimension 3 but index expects 8$"):
        _lib.rows_f32([[0.0] * 8, [1.0] * 8, [2.0] * 3], 8, msg)
    assert _lib.rows_f32(np.zeros((0, 8)), 8, msg).shape == (0, 8)
    assert _lib.rows_f32([1.0] * 8, 8, msg).shape == (1, 8)


def test_query_shapes():
    """Host queries of the wrong length raise the reference's assertion text
    (src/lib.rs:684-690) as ValueError; a batch is never reshaped into other
    queries."""
    import numpy as np

    from pydiskann_b200 import _lib

    for bad, n in ((np.zeros((2, 3)), 3), ([[0.0] * 4, [0.0] * 3], 3), (np.zeros(8), 8)):
        with pytest.raises(ValueError, match=f"^Query dim {n} != index dim 4$"):
            _lib.query_rows(bad, 4)
    with pytest.raises(ValueError, match="2-D batch"):
        _lib.query_rows(np.zeros((2, 2, 4)), 4)
    assert _lib.query_rows(np.zeros(4), 4).shape == (1, 4)
    assert _lib.query_rows([], 4).shape == (0, 4) and _lib.query_rows(np.zeros((0, 4)), 4).shape == (0, 4)
    assert _lib.query_rows(np.ones((3, 4)), 4).shape == (3, 4)
