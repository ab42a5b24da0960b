"""The reference's on-disk formats (pydiskann_b200/formats.py), on CPU.

Each fixture is assembled here byte by byte with `struct`, from the layouts in
the reference's source (DANN core file, src/lib.rs:355-680; QANN sidecar v2,
src/quantized.rs:420-575; labels, src/filtered.rs:322-425; bincode 1.3
default encoding), not with the writer under test.  The readers must recover
every field and array, the writers must reproduce the bytes exactly, and each
malformed input must raise the reference's error message.
"""
import struct

import numpy as np
import pytest

from pydiskann_b200 import formats as F

MiB = 1024 * 1024


def _bc_str(s):
    b = s.encode()
    return struct.pack("<Q", len(b)) + b


def _bc_vec_f32(a):
    a = np.asarray(a, dtype="<f4")
    return struct.pack("<Q", a.size) + a.tobytes()


def _core_fixture(n=5, d=3, R=4, med=2, name="diskann_rs::metric::DistL2Sq", legacy=False, version=1):
    X = (np.arange(n * d, dtype=np.float32) * 0.5 - 3).reshape(n, d)
    A = np.full((n, R), 0xFFFFFFFF, np.uint32)
    for i in range(n):
        nb = [(i + 1) % n, (i + 2) % n][: 1 + i % 2]
        A[i, : len(nb)] = nb
    md = struct.pack("<QQQIQQ", d, n, R, med, MiB, MiB + n * d * 4) + _bc_str(name)
    head = b"" if legacy else struct.pack("<II", 0x44414E4E, version)
    head += struct.pack("<Q", len(md)) + md
    raw = head + bytes(MiB - len(head)) + X.astype("<f4").tobytes() + A.astype("<u4").tobytes()
    return raw, X, A, med


def test_core_reads_hand_built_file():
    raw, X, A, med = _core_fixture()
    m, Xr, Ar = F.parse_core(raw)
    assert (m.dim, m.num_vectors, m.max_degree, m.medoid_id) == (3, 5, 4, med)
    assert (m.vectors_offset, m.adjacency_offset) == (MiB, MiB + 5 * 3 * 4)
    assert m.distance_name == "diskann_rs::metric::DistL2Sq" and m.metric == "l2" and not m.legacy
    assert np.array_equal(Xr, X) and np.array_equal(Ar, A)


def test_core_writer_reproduces_bytes():
    raw, X, A, med = _core_fixture()
    assert F.core_bytes(X, A, med, "l2") == raw
    raw_c, *_ = _core_fixture(name="diskann_rs::metric::DistCosine")
    assert F.core_bytes(X, A, med, "cosine") == raw_c


def test_core_legacy_layout():
    """The older layout has no magic / version words (src/lib.rs:528-532)."""
    raw, X, A, med = _core_fixture(legacy=True)
    m, Xr, Ar = F.parse_core(raw)
    assert m.legacy and np.array_equal(Xr, X) and np.array_equal(Ar, A) and m.medoid_id == med
    assert F.core_bytes(X, A, med, "l2", legacy=True) == raw


def test_core_file_roundtrip(tmp_path):
    raw, X, A, med = _core_fixture(n=40, d=8, R=6)
    p = tmp_path / "idx.bin"
    F.write_core(str(p), X, A, med, "dot")
    m, Xr, Ar = F.read_core(str(p))
    assert m.metric == "dot" and np.array_equal(Xr, X) and np.array_equal(Ar, A)
    assert p.read_bytes() == F.core_bytes(X, A, med, "dot")


@pytest.mark.parametrize("name,metric", [
    ("diskann_rs::metric::DistL2Sq", "l2"), ("diskann_rs::metric::DistL2", "euclidean"),
    ("diskann_rs::metric::DistCosine", "cosine"), ("diskann_rs::metric::DistDot", "dot"),
    ("other_crate::DistDot", "dot"), ("diskann_rs::metric::Hamming", None)])
def test_distance_names(name, metric):
    assert F.metric_of_distance_name(name) == metric


def test_core_errors(tmp_path):
    raw, X, A, med = _core_fixture()
    with pytest.raises(RuntimeError, match="Unsupported core format version: 2"):
        F.parse_core(_core_fixture(version=2)[0])
    with pytest.raises(RuntimeError, match="Buffer too small for metadata length"):
        F.parse_core(raw[:7])
    bad = bytearray(raw)
    struct.pack_into("<Q", bad, 8, MiB + 1)
    with pytest.raises(RuntimeError, match="Invalid metadata length"):
        F.parse_core(bytes(bad))
    with pytest.raises(RuntimeError, match="past the end"):
        F.parse_core(raw[:-4])  # last adjacency word missing
    bad = bytearray(raw)
    struct.pack_into("<Q", bad, 8, 40)  # metadata cut inside distance_name
    with pytest.raises(RuntimeError, match="Serialization error"):
        F.parse_core(bytes(bad))
    bad = bytearray(raw)
    struct.pack_into("<I", bad, 16 + 24, 5)  # medoid = n
    with pytest.raises(RuntimeError, match="medoid 5 out of range"):
        F.parse_core(bytes(bad))
    with pytest.raises(RuntimeError, match="I/O error"):
        F.read_core(str(tmp_path / "missing.idx"))


# ------------------------------------------------------------------ sidecar
def _state_fixture(kind, d=8):
    rng = np.random.default_rng(3)
    if kind == "pq":
        M, K, ds = 4, 16, 2
        cb = rng.standard_normal(M * K * ds).astype(np.float32)
        body = struct.pack("<IQQQQ", 0, d, M, K, ds) + _bc_vec_f32(cb)
        st = F.QuantizerState("pq", d, M, K, ds, codebooks=cb)
        cs = M
    elif kind == "f16":
        body = struct.pack("<IQ", 1, d)
        st = F.QuantizerState("f16", d)
        cs = 2 * d
    elif kind == "int8":
        body = struct.pack("<IQff", 2, d, 0.25, -1.5)
        st = F.QuantizerState("int8", d, scale=0.25, offset=-1.5)
        cs = d
    else:
        P = 64
        cen = rng.standard_normal(d).astype(np.float32)
        sg = np.where(rng.random(3 * P) < 0.5, -0.125, 0.125).astype(np.float32)
        body = struct.pack("<IQQ", 3, d, P) + _bc_vec_f32(cen) + _bc_vec_f32(sg)
        st = F.QuantizerState("rabitq", d, padded=P, centroid=cen, signs=sg)
        cs = P // 8 + 8
    return body, st, cs


def _sidecar_fixture(kind, n=6, version=2, type_byte=None):
    body, st, cs = _state_fixture(kind)
    codes = (np.arange(n * cs) % 13).astype(np.uint8).reshape(n, cs)
    tb = F.QUANTIZER_TYPES.index(kind) if type_byte is None else type_byte
    raw = struct.pack("<IIBQQQ", 0x51414E4E, version, tb, n, cs, len(body)) + body + codes.tobytes()
    return raw, st, codes


@pytest.mark.parametrize("kind", ["pq", "f16", "int8", "rabitq"])
def test_sidecar_reads_and_writes(kind, tmp_path):
    raw, st, codes = _sidecar_fixture(kind)
    s, c = F.parse_sidecar(raw, 6)
    assert s.kind == kind and s.dim == st.dim and s.code_size == codes.shape[1]
    assert np.array_equal(c, codes)
    for f in ("num_subspaces", "num_centroids", "subspace_dim", "scale", "offset", "padded"):
        assert getattr(s, f) == getattr(st, f), f
    for f in ("codebooks", "centroid", "signs"):
        a, b = getattr(s, f), getattr(st, f)
        assert (a is None and b is None) or np.array_equal(a, b), f
    assert F.sidecar_bytes(s, c) == raw
    p = tmp_path / "q.qann"
    F.write_sidecar(str(p), s, c)
    assert p.read_bytes() == raw
    s2, c2 = F.read_sidecar(str(p), 6)
    assert s2.kind == kind and np.array_equal(c2, codes)


def test_sidecar_errors():
    raw, _, _ = _sidecar_fixture("int8")
    with pytest.raises(RuntimeError, match="Quantized data too small"):
        F.parse_sidecar(raw[:32])
    bad = bytearray(raw)
    struct.pack_into("<I", bad, 0, 0x12345678)
    with pytest.raises(RuntimeError, match="Invalid magic: expected 0x51414E4E, got 0x12345678"):
        F.parse_sidecar(bytes(bad))
    with pytest.raises(RuntimeError, match="Unsupported version: 1"):
        F.parse_sidecar(_sidecar_fixture("int8", version=1)[0])
    with pytest.raises(RuntimeError, match="Sidecar has 6 vectors, base index has 7"):
        F.parse_sidecar(raw, 7)
    with pytest.raises(RuntimeError, match="Quantizer type mismatch"):
        F.parse_sidecar(_sidecar_fixture("int8", type_byte=0)[0])
    with pytest.raises(RuntimeError, match="Truncated codes data"):
        F.parse_sidecar(raw[:-1])
    with pytest.raises(RuntimeError, match="Truncated quantizer data"):
        F.parse_sidecar(raw[:40])
    bad = bytearray(raw)
    struct.pack_into("<I", bad, 33, 7)  # variant index 7
    with pytest.raises(RuntimeError, match="Serialization error"):
        F.parse_sidecar(bytes(bad))
    bad = bytearray(_sidecar_fixture("pq")[0])
    struct.pack_into("<Q", bad, 17, 3)  # code_size disagrees with num_subspaces
    with pytest.raises(RuntimeError, match="code_size 3 != pq code size 4"):
        F.parse_sidecar(bytes(bad))


# ------------------------------------------------------------------- labels
def _labels_fixture(n=4, nf=3):
    L = (np.arange(n * nf, dtype=np.uint64) * 7 + (1 << 40)).reshape(n, nf)
    md = struct.pack("<QQ", n, nf)
    return struct.pack("<Q", len(md)) + md + L.astype("<u8").tobytes(), L


def test_labels_read_write(tmp_path):
    raw, L = _labels_fixture()
    assert np.array_equal(F.parse_labels(raw), L)
    assert F.labels_bytes(L) == raw
    p = tmp_path / "x.labels"
    F.write_labels(str(p), L)
    assert np.array_equal(F.read_labels(str(p)), L)
    raw0, L0 = _labels_fixture(n=3, nf=0)
    assert F.parse_labels(raw0).shape == (3, 0)


def test_labels_errors():
    raw, _ = _labels_fixture()
    with pytest.raises(RuntimeError, match="Labels buffer too small"):
        F.parse_labels(raw[:4])
    with pytest.raises(RuntimeError, match="Labels buffer too small for metadata"):
        F.parse_labels(raw[:12])
    with pytest.raises(RuntimeError, match="Labels data truncated"):
        F.parse_labels(raw[:-8])


def test_prefixed_forms():
    """[len u64][first][rest]: QuantizedDiskANN / FilteredDiskANN to_bytes."""
    core, X, A, med = _core_fixture()
    lab, L = _labels_fixture(n=5)
    blob = F.join_prefixed(core, lab)
    assert blob[:8] == struct.pack("<Q", len(core))
    a, b = F.split_prefixed(blob)
    assert bytes(a) == core and bytes(b) == lab
    m, Xr, _ = F.parse_core(a)
    assert np.array_equal(Xr, X) and F.parse_labels(b).shape == (5, 3)
    with pytest.raises(RuntimeError, match="Buffer too small"):
        F.split_prefixed(b"\x01")
    with pytest.raises(RuntimeError, match="Buffer too small for base index"):
        F.split_prefixed(blob[:100])


# ------------------------------------------------------------------ SPFresh
def _spf_fixture():
    """A 2-block int8 SPFresh Meta, bincode by hand (src/spfresh.rs:25-72)."""
    d = 4
    cfg = struct.pack("<QQfQQQ", 8, 2, float("inf"), 5, 16, 64)
    q = b"\x01" + struct.pack("<IQff", 2, d, 0.5, -2.0)  # Some(Int8)
    cid = struct.pack("<QQQ", 2, (1 << 48) + 0, 0xFFFFFFFFFFFFFFFF)
    cents = struct.pack("<Q", 2) + _bc_vec_f32([1, 2, 3, 4]) + _bc_vec_f32([])
    tail = struct.pack("<Q", 9) + struct.pack("<QQ", 1, 3) + struct.pack("<Q", 8)
    return struct.pack("<Q", d) + cfg + q + cid + cents + tail


def test_spf_meta_reads_and_writes():
    raw = _spf_fixture()
    m = F.parse_spf(raw)
    assert m.dim == 4 and m.cfg == F.SPFreshConfig(8, 2, float("inf"), 5, 16, 64)
    assert m.quantizer.kind == "int8" and (m.quantizer.scale, m.quantizer.offset) == (0.5, -2.0)
    assert m.block_cid.tolist() == [1 << 48, F.SPF_FREE]
    assert m.block_centroid[0].tolist() == [1, 2, 3, 4] and m.block_centroid[1].size == 0
    assert (m.next_id, m.deleted.tolist(), m.live) == (9, [3], 8)
    assert F.spf_bytes(m) == raw
    assert F.spf_block_bytes(m.cfg, m.quantizer, 4) == 4 + 2 * 8 * (8 + 4)
    assert F.spf_block_bytes(F.SPFreshConfig(1), None, 4) == 4 + 2 * 2 * (8 + 16)  # max(2) clamp
    bad = bytearray(raw)
    bad[8 + 44] = 7  # Option tag
    with pytest.raises(RuntimeError, match="Serialization error"):
        F.parse_spf(bytes(bad))


def test_postings_blocks():
    cs, block = 3, 4 + 4 * (8 + 3)
    blocks = [(np.array([5, 1 << 40], np.uint64), np.arange(6, dtype=np.uint8).reshape(2, 3)),
              (np.zeros(0, np.uint64), np.zeros((0, 3), np.uint8))]
    raw = F.postings_bytes(blocks, block, cs)
    want = (struct.pack("<I", 2) + struct.pack("<Q", 5) + bytes([0, 1, 2]) + struct.pack("<Q", 1 << 40)
            + bytes([3, 4, 5]))
    assert raw[:block] == want + bytes(block - len(want)) and raw[block:] == bytes(block)
    got = F.parse_postings(raw, 2, block, cs)
    assert got[0][0].tolist() == [5, 1 << 40] and np.array_equal(got[0][1], blocks[0][1]) and len(got[1][0]) == 0
    bad = bytearray(raw)
    struct.pack_into("<I", bad, 0, 5)
    with pytest.raises(RuntimeError, match="capacity 4"):
        F.parse_postings(bytes(bad), 2, block, cs)
    with pytest.raises(RuntimeError, match="postings file holds 1 blocks"):
        F.parse_postings(raw[:block], 2, block, cs)


def test_incremental_bytes_layout():
    V = np.arange(6, dtype=np.float32).reshape(3, 2)
    raw = F.incremental_bytes(V, [[1, 2], [0], []], 1, 32)
    want = (struct.pack("<IIBQQ", 0x494E4352, 2, 0, 2, 3) + V.tobytes() + struct.pack("<Q", 3)
            + struct.pack("<III", 2, 1, 2) + struct.pack("<II", 1, 0) + struct.pack("<I", 0)
            + struct.pack("<qQQ", 1, 32, 0) + b"\x00\x00")
    assert raw == want
    F.check_incremental_header(raw)
    with pytest.raises(RuntimeError):
        F.check_incremental_header(struct.pack("<II", 0x494E4352, 1))


@pytest.mark.parametrize("quantizer", [None, "int8", "f16", "rabitq"])
def test_spfresh_save_open_host(tmp_path, quantizer):
    """A host-side SPFresh (no device mirror) saved and reopened keeps its state."""
    from pydiskann_b200.spfresh import SPFresh

    rng = np.random.default_rng(1)
    X = rng.integers(-8, 8, size=(600, 16)).astype(np.float32)
    s = SPFresh.build(X, metric="l2", quantizer=quantizer, max_posting_size=24, device=None)
    s.delete([3, 50, 51])
    s.gc()
    p = str(tmp_path / "sp")
    s.save(p)
    for suffix in ("spf", "postings", "vectors", "centroids"):
        assert (tmp_path / f"sp.{suffix}").exists()
    t = SPFresh.open(p, device=None)
    assert (t.dim, t.next_id, t.live, t.deleted) == (s.dim, s.next_id, s.live, s.deleted)
    assert (t.max_posting, t.min_posting, t.rerank_size, t.codec.kind) == (24, 16, 0, quantizer)
    assert np.array_equal(t.live_b, s.live_b)
    for b in np.nonzero(s.live_b)[0]:
        assert np.array_equal(t.cent[b], s.cent[b])
        assert np.array_equal(t.ids[b], s.ids[b]) and np.array_equal(t.codes[b], s.codes[b])
    assert np.array_equal(t.raw, s.raw[: s.next_id])
    assert t.stats() == s.stats()
    t.save(str(tmp_path / "again"))
    for suffix in ("spf", "postings", "vectors"):
        assert (tmp_path / f"again.{suffix}").read_bytes() == (tmp_path / f"sp.{suffix}").read_bytes()


def _vecs_bytes(rows, fmt):
    out = b""
    for r in rows:
        out += struct.pack("<I", len(r)) + b"".join(struct.pack(fmt, x) for x in r)
    return out


def test_vecs_readers(tmp_path):
    """read_fvecs / read_ivecs / read_bvecs_as_f32 (src/formats.rs:7-122):
    records of a u32 count and that many elements, lengths may differ; a 1-3
    byte tail ends the file; a record cut short is an I/O error."""
    import pydiskann_b200 as dg

    rows = [[1.5, -2.0, 3.25], [], [7.0], [0.5, 0.25, 0.125, 2.0 ** 100]]
    p = tmp_path / "ragged.fvecs"
    p.write_bytes(_vecs_bytes(rows, "<f"))
    assert dg.read_fvecs(str(p)) == rows
    X = np.arange(20, dtype=np.float32).reshape(5, 4) - 7.5
    dg.write_fvecs(str(tmp_path / "u.fvecs"), X)
    assert dg.read_fvecs(str(tmp_path / "u.fvecs")) == X.tolist()
    (tmp_path / "tail.fvecs").write_bytes(_vecs_bytes(rows, "<f") + b"\x03\x00")
    assert dg.read_fvecs(str(tmp_path / "tail.fvecs")) == rows
    (tmp_path / "cut.fvecs").write_bytes(_vecs_bytes(rows, "<f")[:-2])
    with pytest.raises(RuntimeError, match="I/O error: failed to fill whole buffer"):
        dg.read_fvecs(str(tmp_path / "cut.fvecs"))
    with pytest.raises(RuntimeError, match="I/O error"):
        dg.read_fvecs(str(tmp_path / "absent.fvecs"))
    (tmp_path / "empty.ivecs").write_bytes(b"")
    assert dg.read_ivecs(str(tmp_path / "empty.ivecs")) == []
    irows = [[1, -2, 2147483647], [-2147483648], []]
    (tmp_path / "g.ivecs").write_bytes(_vecs_bytes(irows, "<i"))
    assert dg.read_ivecs(str(tmp_path / "g.ivecs")) == irows
    brows = [[0, 1, 128, 255], [17]]
    (tmp_path / "b.bvecs").write_bytes(_vecs_bytes(brows, "<B"))
    got = dg.read_bvecs_as_f32(str(tmp_path / "b.bvecs"))
    want = [[float(np.float32(b) / np.float32(255.0)) for b in r] for r in brows]
    assert got == want and got[0][3] == 1.0 and got[0][0] == 0.0


def test_spfresh_compact_host():
    """compact keeps the index's state and answers: routing here is exact over
    the live centroids, so there is no centroid graph to go stale."""
    from pydiskann_b200.spfresh import SPFresh

    rng = np.random.default_rng(5)
    X = rng.integers(-8, 8, size=(500, 8)).astype(np.float32)
    s = SPFresh.build(X, metric="l2", max_posting_size=24, device=None)
    s.delete(range(0, 500, 9))
    s.gc()
    before = (s.stats(), [ids.copy() for ids in s.ids])
    s.compact()
    assert s.stats() == before[0]
    assert set(before[0]) == {"live", "deleted", "postings", "max_posting"}  # python/src/lib.rs:341-344
    assert all(np.array_equal(a, b) for a, b in zip(s.ids, before[1]))
