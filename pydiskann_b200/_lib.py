"""ctypes binding of libdgann.so (include/dgann.h).

The library is the only compute path: importing this module without a built
libdgann.so raises, and there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import functools
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# DGANN_LIBRARY points at a libdgann.so built elsewhere (e.g. another tuning)
LIB_PATH = os.environ.get("DGANN_LIBRARY", os.path.join(HERE, "libdgann.so"))

DG_OK, DG_EINVAL, DG_ENOMEM, DG_ETIMEOUT, DG_EDEVICE, DG_ENOTSUP = range(6)
L2SQ, L2, COSINE, DOT = 0, 1, 2, 3
TRAVERSE_F32, TRAVERSE_BF16, TRAVERSE_CODES, TRAVERSE_FP8 = 0, 1, 2, 3
Q_NONE, Q_PQ, Q_INT8, Q_RABITQ, Q_F16 = 0, 1, 2, 3, 4
F_TRUE, F_EQ, F_IN, F_LT, F_GT, F_RANGE, F_AND, F_OR = range(8)
FLAG_DEVICE_PTRS = 1
FLAG_STREAM = 2
PAD = 0xFFFFFFFF
PAD64 = 0xFFFFFFFFFFFFFFFF


class DgError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(msg)
        self.status = status


class FilterOp(C.Structure):
    _fields_ = [("op", C.c_uint32), ("field", C.c_uint32), ("a", C.c_uint64), ("b", C.c_uint64)]


class IndexDesc(C.Structure):
    _fields_ = [
        ("dim", C.c_uint32), ("max_degree", C.c_uint32), ("num_vectors", C.c_uint64),
        ("medoid", C.c_uint32), ("metric", C.c_int32), ("vectors", C.c_void_p),
        ("adjacency", C.c_void_p), ("device", C.c_int32), ("hbm_budget_bytes", C.c_uint64),
    ]


class SearchParams(C.Structure):
    _fields_ = [
        ("k", C.c_uint32), ("beam_width", C.c_uint32), ("rerank_size", C.c_uint32),
        ("traversal", C.c_int32), ("filter_ops", C.c_void_p), ("filter_nops", C.c_uint32),
        ("filter_offsets", C.c_void_p), ("filter_pool", C.c_void_p),
        ("filter_pool_len", C.c_uint32), ("per_query_beam", C.c_void_p), ("flags", C.c_uint32),
        ("stream", C.c_void_p), ("per_query_k", C.c_void_p),
    ]


class SpfreshDesc(C.Structure):
    _fields_ = [
        ("dim", C.c_uint32), ("metric", C.c_int32), ("device", C.c_int32), ("num_blocks", C.c_uint32),
        ("block_cap", C.c_uint32), ("centroids", C.c_void_p), ("block_live", C.c_void_p),
        ("block_len", C.c_void_p), ("entry_ids", C.c_void_p), ("entry_codes", C.c_void_p),
        ("code_size", C.c_uint32), ("quantizer", C.c_int32), ("pq_M", C.c_uint32), ("pq_K", C.c_uint32),
        ("pq_codebooks", C.c_void_p), ("int8_scale", C.c_float), ("int8_offset", C.c_float),
        ("rq_padded", C.c_uint32), ("rq_signs", C.c_void_p), ("id_capacity", C.c_uint64),
        ("num_raw", C.c_uint64), ("raw", C.c_void_p), ("deleted", C.c_void_p),
    ]


class SpfreshParams(C.Structure):
    _fields_ = [("k", C.c_uint32), ("nprobe", C.c_uint32), ("rerank_size", C.c_uint32),
                ("probe_ratio", C.c_float), ("flags", C.c_uint32), ("stream", C.c_void_p)]


class ServerConfig(C.Structure):
    _fields_ = [("max_batch", C.c_uint32), ("streams", C.c_uint32), ("max_k", C.c_uint32),
                ("max_filter_ops", C.c_uint32), ("max_wait_us", C.c_uint32), ("hbm_budget_bytes", C.c_uint64)]


class Request(C.Structure):
    _fields_ = [("k", C.c_uint32), ("beam_width", C.c_uint32), ("rerank_size", C.c_uint32),
                ("traversal", C.c_int32), ("filter_ops", C.c_void_p), ("filter_nops", C.c_uint32),
                ("filter_pool", C.c_void_p), ("filter_pool_len", C.c_uint32)]


# Every symbol include/dgann.h declares, with its ctypes signature.
def _signatures():
    vp, u32, u64, i32, f32 = C.c_void_p, C.c_uint32, C.c_uint64, C.c_int32, C.c_float
    st = C.c_int
    return {
        "dg_index_create": (st, [vp, vp]),
        "dg_index_destroy": (st, [vp]),
        "dg_index_enable_bf16": (st, [vp]),
        "dg_index_enable_fp8": (st, [vp]),
        "dg_index_attach_pq": (st, [vp, u32, u32, vp, vp]),
        "dg_index_attach_int8": (st, [vp, f32, f32, vp]),
        "dg_index_attach_f16": (st, [vp]),
        "dg_index_attach_f16_codes": (st, [vp, vp]),
        "dg_index_attach_rabitq": (st, [vp, u32, vp, vp, vp]),
        "dg_index_attach_labels": (st, [vp, u32, vp]),
        "dg_index_get_codes": (st, [vp, vp, u64, vp]),
        "dg_index_autotune": (st, [vp, vp, vp, u32, u32, vp, vp]),
        "dg_index_tuned_schedule": (st, [vp, vp, vp, vp, vp]),
        "dg_index_set_entry_points": (st, [vp, vp, u32]),
        "dg_index_set_code_limit": (st, [vp, u64]),
        "dg_index_set_tombstones": (st, [vp, vp, u64, i32, u64]),
        "dg_index_update_rows": (st, [vp, u64, u64, vp, vp, vp]),
        "dg_delta_insert": (st, [vp, u32, i32, u32, vp, u64, u64, vp]),
        "dg_search_batch": (st, [vp, vp, vp, u32, vp, vp, vp, vp]),
        "dg_search_batch_static": (st, [vp, vp, vp, u32, vp, vp, vp]),
        "dg_count_matching": (st, [vp, vp, u32, vp, u32, vp]),
        "dg_server_create": (st, [vp, vp, vp]),
        "dg_server_destroy": (st, [vp]),
        "dg_server_submit": (st, [vp, vp, vp, vp]),
        "dg_server_wait": (st, [vp, u64, C.c_int64, vp, vp, vp, vp]),
        "dg_server_stats": (st, [vp, vp, vp, vp]),
        "dg_server_run_trace": (st, [vp, vp, u32, vp, vp, C.c_int64, vp, vp, vp, vp, vp]),
        "dg_spfresh_create": (st, [vp, vp]),
        "dg_spfresh_destroy": (st, [vp]),
        "dg_spfresh_update_blocks": (st, [vp, vp, u32, vp, vp, vp, vp, vp]),
        "dg_spfresh_put_raw": (st, [vp, u64, vp, u64]),
        "dg_spfresh_set_deleted": (st, [vp, vp, u64, i32]),
        "dg_spfresh_set_centroids": (st, [vp, vp, u32, vp, vp]),
        "dg_spfresh_nearest": (st, [vp, vp, u32, u32, vp, vp]),
        "dg_spfresh_search_batch": (st, [vp, vp, vp, u32, vp, vp, vp]),
        "dg_medoid": (st, [vp, u64, u32, i32, i32, vp]),
        "dg_build_vamana": (st, [vp, u64, u32, i32, u32, u32, f32, u64, u32, i32, vp]),
        "dg_pq_train": (st, [vp, u64, u32, u32, u32, u32, u64, u64, i32, vp]),
        "dg_pq_encode": (st, [vp, u64, u32, u32, u32, vp, i32, vp]),
        "dg_fp8_encode": (st, [vp, u64, u32, i32, vp, vp]),
        "dg_rabitq_encode": (st, [vp, u64, u32, u32, vp, vp, i32, vp]),
        "dg_exact_knn": (st, [vp, u64, u32, vp, u32, u32, i32, i32, vp, vp]),
        "dg_last_error": (C.c_char_p, []),
        "dg_version": (i32, []),
    }


EXPORTED = tuple(_signatures().keys())

# The index-construction subset of the ABI, also linked on its own into
# libdgbuild.so (medoid, Vamana build, PQ training and encodes, exact kNN):
# a process that only prepares an index loads that library, not the search
# library.
BUILDER = ("dg_medoid", "dg_build_vamana", "dg_pq_train", "dg_pq_encode", "dg_fp8_encode", "dg_rabitq_encode",
           "dg_exact_knn", "dg_last_error", "dg_version")
BUILD_LIB_PATH = os.environ.get("DGANN_BUILD_LIBRARY", os.path.join(HERE, "libdgbuild.so"))

_lib = None
_builder = None


def lib():
    """Load libdgann.so; raises when it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"libdgann.so not found at {LIB_PATH}; build it with `python -m pydiskann_b200.build`"
            )
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _signatures().items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def builder():
    """Load libdgbuild.so (the index-construction library); raises when it has
    not been built."""
    global _builder
    if _builder is None:
        if not os.path.exists(BUILD_LIB_PATH):
            raise ImportError(
                f"libdgbuild.so not found at {BUILD_LIB_PATH}; build it with `python -m pydiskann_b200.build`"
            )
        L = C.CDLL(BUILD_LIB_PATH)
        sig = _signatures()
        for name in BUILDER:
            f = getattr(L, name)
            f.restype, f.argtypes = sig[name]
        _builder = L
    return _builder


def check(status, library=None):
    """Raise for a non-OK status with the error text of `library` (the
    library that returned it; default libdgann)."""
    if status != DG_OK:
        msg = (library or lib()).dg_last_error().decode(errors="replace")
        if status == DG_EINVAL:
            raise ValueError(msg)
        raise DgError(status, msg)


def ptr(a):
    """Address of a numpy array, torch tensor, or None."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data_as(C.c_void_p)
    if hasattr(a, "data_ptr"):
        return C.c_void_p(a.data_ptr())
    raise TypeError(type(a))


def locked(fn):
    """Run a method under its object's `_lock` (a threading.RLock).  Updates and
    searches of one index from several threads then see whole updates, as the
    reference's RwLock-guarded state gives (src/incremental.rs:521-534,
    src/spfresh.rs:778); a search never meets a device mirror that an insert
    is replacing."""

    @functools.wraps(fn)
    def run(self, *args, **kwargs):
        with self._lock:
            return fn(self, *args, **kwargs)

    return run


def rows_f32(vectors, dim, message):
    """Vectors for an insert into an index of dimension `dim`, as f32[n, dim].
    The first vector of another length (ragged lists included) raises
    RuntimeError(message(i, its_length)), the text of the reference's check."""
    try:
        X = np.ascontiguousarray(vectors, dtype=np.float32)
    except ValueError:
        for i, v in enumerate(vectors):
            if len(v) != dim:
                raise RuntimeError(message(i, len(v))) from None
        raise
    if X.size == 0:
        return X.reshape(0, dim)
    if X.ndim == 1:
        X = X.reshape(1, -1)
    if X.ndim != 2 or X.shape[1] != dim:
        raise RuntimeError(message(0, X.shape[-1]))
    return X


def query_rows(queries, dim):
    """Host queries as f32[nq, dim].  A query of another length (ragged lists
    included) raises ValueError with the text of the reference's assertion
    (src/lib.rs:684-690); a batch is never reinterpreted by reshaping it."""
    try:
        Q = np.ascontiguousarray(queries, dtype=np.float32)
    except ValueError:
        for q in queries:
            if len(q) != dim:
                raise ValueError(f"Query dim {len(q)} != index dim {dim}") from None
        raise
    if Q.size == 0 and Q.ndim <= 2 and (Q.ndim < 2 or Q.shape[1] in (0, dim)):
        return Q.reshape(0, dim)
    if Q.ndim == 1:
        Q = Q.reshape(1, -1)
    if Q.ndim != 2:
        raise ValueError(f"queries must be one query or a 2-D batch, not shape {Q.shape}")
    if Q.shape[1] != dim:
        raise ValueError(f"Query dim {Q.shape[1]} != index dim {dim}")
    return Q
