"""Host side of the base + delta (IncrementalDiskANN) index, on CPU.

dg_delta_insert (libdgann's host restatement of DeltaLayer::add_vectors,
src/incremental.rs:114-193) must write the same delta graph and entry point
as the oracle's pure-Python restatement (oracle/delta.py), batch after batch;
integer-valued vectors keep every distance exact.  The INCR v2 byte layout
(src/incremental.rs:1234-1327) is checked against a hand-assembled buffer.
"""
import ctypes as C
import struct

import numpy as np
import pytest

from oracle import delta as odelta
from pydiskann_b200 import _lib
from pydiskann_b200 import formats as F

PAD = 0xFFFFFFFF


def _insert(X, R, metric, batches):
    n = sum(batches)
    A = np.full((n, R), PAD, np.uint32)
    ep = C.c_int64(-1)
    done = 0
    for b in batches:
        rc = _lib.lib().dg_delta_insert(_lib.ptr(X), X.shape[1], metric, R, _lib.ptr(A), done, b, C.byref(ep))
        assert rc == 0, _lib.lib().dg_last_error()
        done += b
        yield A[:done].copy(), ep.value


@pytest.mark.parametrize("metric", [odelta.L2SQ, odelta.L2, odelta.DOT])
@pytest.mark.parametrize("R", [4, 8])
def test_delta_insert_matches_oracle(metric, R):
    rng = np.random.default_rng(5 + R)
    batches = [1, 40, 57, 3]
    X = rng.integers(-6, 7, size=(sum(batches), 8)).astype(np.float32)
    ref = odelta.DeltaLayer(8, R, metric)
    done = 0
    for (A, ep), b in zip(_insert(X, R, metric, batches), batches):
        ref.add_vectors(X[done:done + b])
        done += b
        assert ep == ref.entry
        assert np.array_equal(A, ref.adjacency()), np.nonzero((A != ref.adjacency()).any(1))[0][:5]
        deg = (A != PAD).sum(1)
        assert deg.max() <= R and all(i not in A[i] for i in range(done))


def test_delta_insert_rejects_bad_input():
    X = np.zeros((4, 3), np.float32)
    A = np.full((4, 2), PAD, np.uint32)
    ep = C.c_int64(5)
    assert _lib.lib().dg_delta_insert(_lib.ptr(X), 3, 0, 2, _lib.ptr(A), 2, 2, C.byref(ep)) == _lib.DG_EINVAL
    ep = C.c_int64(-1)
    A[0, 0] = 3  # an id past the inserted rows
    assert _lib.lib().dg_delta_insert(_lib.ptr(X), 3, 0, 2, _lib.ptr(A), 2, 2, C.byref(ep)) == _lib.DG_EINVAL
    assert _lib.lib().dg_delta_insert(_lib.ptr(X), 3, 9, 2, _lib.ptr(A), 0, 2, C.byref(ep)) == _lib.DG_EINVAL


def test_incremental_bytes_with_base_labels_tombstones():
    core = F.core_bytes(np.ones((2, 2), np.float32), np.full((2, 3), PAD, np.uint32), 0)
    V = np.array([[1, 2], [3, 4]], np.float32)
    BL = np.array([[7], [8]], np.uint64)
    DL = np.array([[9], [10]], np.uint64)
    raw = F.incremental_bytes(V, [[1], [0]], 0, 32, [5, (1 << 48) + 1], base=core, labels=(1, BL, DL))
    want = (struct.pack("<II", 0x494E4352, 2) + b"\x01" + struct.pack("<Q", len(core)) + core
            + struct.pack("<QQ", 2, 2) + V.tobytes() + struct.pack("<Q", 2) + struct.pack("<II", 1, 1)
            + struct.pack("<II", 1, 0) + struct.pack("<qQQ", 0, 32, 2) + struct.pack("<QQ", 5, (1 << 48) + 1)
            + b"\x01" + struct.pack("<QQ", 1, 2) + BL.tobytes() + struct.pack("<Q", 2) + DL.tobytes() + b"\x00")
    assert raw == want
    p = F.parse_incremental(raw)
    assert bytes(p["base"]) == core and p["graph"] == [[1], [0]] and p["entry_point"] == 0
    assert p["tombstones"] == [5, (1 << 48) + 1] and p["max_degree"] == 32 and p["dim"] == 2
    assert np.array_equal(p["vectors"], V) and p["labels"][0] == 1
    assert np.array_equal(p["labels"][1], BL) and np.array_equal(p["labels"][2], DL)
    with pytest.raises(RuntimeError, match="truncated"):
        F.parse_incremental(raw[:-20])
    with pytest.raises(RuntimeError, match="truncated"):
        F.parse_incremental(raw[:-1] + b"\x01")  # a quantizer flag with no section
    # quantizer section (src/incremental.rs:1308-1324): code size, rerank size,
    # bincode QuantizerState, base codes
    st = F.QuantizerState("int8", 2, scale=0.5, offset=-1.0)
    codes = np.array([[1, 2], [3, 4]], np.uint8)
    rq = F.incremental_bytes(V, [[1], [0]], 0, 32, [], base=core, quantizer=(2, 7, st, codes))
    qbody = struct.pack("<IQff", 2, 2, 0.5, -1.0)
    assert rq.endswith(b"\x00" + b"\x01" + struct.pack("<QQQ", 2, 7, len(qbody)) + qbody + struct.pack("<Q", 4)
                       + codes.tobytes())
    pq = F.parse_incremental(rq)
    cs, rr, st2, c2 = pq["quantizer"]
    assert (cs, rr, st2.kind, st2.scale, st2.offset) == (2, 7, "int8", 0.5, -1.0) and np.array_equal(c2, codes.ravel())
    with pytest.raises(RuntimeError, match="Unsupported incremental format version: 1"):
        F.parse_incremental(struct.pack("<II", 0x494E4352, 1) + raw[8:])


def test_should_compact_rule():
    """IncrementalDiskANN::should_compact (src/incremental.rs:1100-1122): the
    delta threshold, or tombstones / (base + delta) >= the ratio in f32.  The
    object is made without its device mirror; the rule reads only sizes."""
    import threading

    from pydiskann_b200.incremental import IncrementalDiskANN

    class Sized:
        def __init__(self, n):
            self.n = n

        def __len__(self):
            return self.n

    def ix(base, delta, tomb, threshold=10_000, ratio=0.1):
        o = object.__new__(IncrementalDiskANN)
        o._lock = threading.RLock()
        o._bX, o._dn, o.tombstones = Sized(base), delta, Sized(tomb)
        o.delta_threshold, o.tombstone_ratio = threshold, ratio
        return o

    assert ix(100, 10_000, 0).should_compact()
    assert not ix(100, 9_999, 0).should_compact()
    assert ix(90, 10, 10).should_compact() and not ix(90, 10, 9).should_compact()
    assert not ix(0, 0, 0).should_compact()
    # 99 999 999 / 10^9 is below 0.1 in f64 but rounds to 0.1f in f32, so it compacts
    assert ix(10**9, 0, 99_999_999).should_compact()
    assert 99_999_999 / 10**9 < 0.1
