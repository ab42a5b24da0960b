"""Continuous-batching request loop over one index (dg_server_* in libdgann).

Requests are queued one at a time; a native dispatcher thread batches pending
requests of the same k / traversal / rerank size / filter presence and runs
each batch on the next free stream slot, so requests arriving while others
run are admitted as slots free up and their batches overlap on the device.
The reference has no serving loop: a query is a synchronous call
(DiskANN::search_with_dists, src/lib.rs:683-714) and its benches time
sequential request loops (benches/benchmark.rs:183-207).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check, lib, ptr

_TRAV = {"f32": _lib.TRAVERSE_F32, "bf16": _lib.TRAVERSE_BF16, "codes": _lib.TRAVERSE_CODES,
         "fp8": _lib.TRAVERSE_FP8}

# DgRequest as a numpy record (u32 k, beam, rerank; i32 traversal; ops pointer,
# u32 nops; pool pointer, u32 pool_len), so a trace of 10^5 requests is built
# without a Python loop over ctypes structures.
_REQ_DTYPE = np.dtype({
    "names": ["k", "beam", "rerank", "trav", "ops", "nops", "pool", "npool"],
    "formats": [np.uint32, np.uint32, np.uint32, np.int32, np.uint64, np.uint32, np.uint64, np.uint32],
    "offsets": [0, 4, 8, 12, 16, 24, 32, 40],
    "itemsize": C.sizeof(_lib.Request),
})


def _trav(index, traversal):
    if traversal is None:
        return _lib.TRAVERSE_CODES if getattr(index, "_quant", None) else _lib.TRAVERSE_F32
    return _TRAV[traversal] if isinstance(traversal, str) else int(traversal)


class Server:
    """Serving loop over `index` (a DiskANN / QuantizedDiskANN / FilteredDiskANN).

    max_batch requests per launch, `streams` batches in flight, requests up to
    max_k results and max_filter_ops filter ops; a partial batch waits at most
    max_wait_us for more requests.  Batches mix k, beams and filters; each
    batch is admitted by its own memory need into an arena of
    hbm_budget_bytes (0 = a full batch at max_k per stream).
    """

    def __init__(self, index, max_batch=1024, streams=4, max_k=100, max_filter_ops=64, max_wait_us=0,
                 hbm_budget_bytes=0):
        self.index = index
        cfg = _lib.ServerConfig(max_batch, streams, max_k, max_filter_ops, max_wait_us, hbm_budget_bytes)
        h = C.c_void_p()
        check(lib().dg_server_create(index._h, C.byref(cfg), C.byref(h)))
        self._h = h
        self.max_k = max_k
        self._pending = {}  # ticket -> k

    def close(self):
        if getattr(self, "_h", None):
            lib().dg_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def submit(self, query, k=10, beam_width=64, rerank_size=0, traversal=None, filter=None):  # noqa: A002
        q = np.ascontiguousarray(query, dtype=np.float32).reshape(-1)
        if q.shape[0] != self.index.dim:
            raise ValueError(f"Query dim {q.shape[0]} != index dim {self.index.dim}")
        r = _lib.Request(k, beam_width, rerank_size, _trav(self.index, traversal))
        keep = []
        if filter is not None and not filter.is_none():
            ops, pool = filter.program()
            arr = (_lib.FilterOp * len(ops))(*[_lib.FilterOp(*o) for o in ops])
            pl = np.asarray(pool if pool else [0], dtype=np.uint64)
            keep = [arr, pl]
            r.filter_ops, r.filter_nops = C.cast(arr, C.c_void_p), len(ops)
            r.filter_pool, r.filter_pool_len = pl.ctypes.data, len(pool)
        t = C.c_uint64()
        check(lib().dg_server_submit(self._h, ptr(q), C.byref(r), C.byref(t)))
        del keep  # the request's program was copied by submit
        self._pending[t.value] = k
        return t.value

    def wait(self, ticket, timeout=10.0):
        """(ids u32[count], dists f32[count], latency in µs) of a ticket."""
        k = self._pending[ticket]
        ids = np.empty(k, np.uint32)
        ds = np.empty(k, np.float32)
        cnt = C.c_uint32()
        lat = C.c_double()
        check(lib().dg_server_wait(self._h, ticket, int(timeout * 1e6), ptr(ids), ptr(ds), C.byref(cnt),
                                   C.byref(lat)))
        del self._pending[ticket]
        return ids[: cnt.value], ds[: cnt.value], lat.value

    def stats(self):
        b, s, m = C.c_uint64(), C.c_uint64(), C.c_uint32()
        check(lib().dg_server_stats(self._h, C.byref(b), C.byref(s), C.byref(m)))
        return {"batches": b.value, "served": s.value, "max_in_flight": m.value}

    def run_trace(self, queries, arrival_us, k=10, beam_width=64, rerank_size=0, traversal=None,
                  filters=None, timeout=120.0):
        """Replays requests at arrival_us (µs from the start) from a native thread.

        k, beam_width, rerank_size and traversal are scalars or per-request
        arrays; filters is None, one Filter or a list of one per request.
        Returns a dict with per-request `ids` / `dists` (trimmed to counts),
        `latency_us` (scheduled arrival to result) and `wall_us`.
        """
        Q = _lib.query_rows(queries, self.index.dim)
        n = Q.shape[0]
        arr = np.ascontiguousarray(arrival_us, dtype=np.float64)
        if arr.shape != (n,):
            raise ValueError("one arrival time per query")
        req = np.zeros(n, _REQ_DTYPE)
        req["k"] = np.broadcast_to(np.asarray(k, np.uint32), n)
        req["beam"] = np.broadcast_to(np.asarray(beam_width, np.uint32), n)
        req["rerank"] = np.broadcast_to(np.asarray(rerank_size, np.uint32), n)
        if traversal is None or isinstance(traversal, str):
            req["trav"] = _trav(self.index, traversal)
        else:
            req["trav"] = np.broadcast_to(np.asarray(traversal, np.int32), n)
        keep = []
        if filters is not None:
            fl = filters if isinstance(filters, (list, tuple)) else [filters] * n
            if len(fl) != n:
                raise ValueError("one filter per query")
            ops_all, pool_all, o_off, p_off, o_n, p_n = [], [], [], [], [], []
            for f in fl:
                ops, pool = ([], []) if f is None or f.is_none() else f.program()
                o_off.append(len(ops_all))
                p_off.append(len(pool_all))
                o_n.append(len(ops))
                p_n.append(len(pool))
                ops_all.extend(ops)
                pool_all.extend(pool)
            ops_arr = np.zeros(max(len(ops_all), 1), np.dtype(
                {"names": ["op", "field", "a", "b"], "formats": [np.uint32, np.uint32, np.uint64, np.uint64],
                 "offsets": [0, 4, 8, 16], "itemsize": C.sizeof(_lib.FilterOp)}))
            if ops_all:
                ops_arr[: len(ops_all)] = [tuple(o) for o in ops_all]
            pool_arr = np.asarray(pool_all if pool_all else [0], dtype=np.uint64)
            keep = [ops_arr, pool_arr]
            o_n, p_n = np.asarray(o_n, np.uint32), np.asarray(p_n, np.uint32)
            req["nops"], req["npool"] = o_n, p_n
            req["ops"] = np.where(o_n > 0, ops_arr.ctypes.data + np.asarray(o_off, np.uint64) * ops_arr.itemsize, 0)
            req["pool"] = np.where(p_n > 0, pool_arr.ctypes.data + np.asarray(p_off, np.uint64) * 8, 0)
        ks = req["k"].astype(np.int64)
        offs = np.concatenate([[0], np.cumsum(ks)])
        ids = np.empty(int(offs[-1]), np.uint32)
        ds = np.empty(int(offs[-1]), np.float32)
        cnt = np.empty(n, np.uint32)
        lat = np.empty(n, np.float64)
        wall = C.c_double()
        check(lib().dg_server_run_trace(self._h, ptr(Q), n, req.ctypes.data_as(C.c_void_p), ptr(arr),
                                        int(timeout * 1e6), ptr(ids), ptr(ds), ptr(cnt), ptr(lat), C.byref(wall)))
        del keep
        return {
            "ids": [ids[offs[i]: offs[i] + cnt[i]] for i in range(n)],
            "dists": [ds[offs[i]: offs[i] + cnt[i]] for i in range(n)],
            "counts": cnt,
            "latency_us": lat,
            "wall_us": wall.value,
        }


def poisson_arrivals(n, rate_per_s, seed=0):
    """Arrival times in µs of a Poisson stream of `rate_per_s` requests/s."""
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1e6 / rate_per_s, size=n))
