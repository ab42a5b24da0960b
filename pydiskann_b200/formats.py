"""Readers and writers for the reference's on-disk index formats.

Files written by the reference (diskann-rs 0.5.x) open here unchanged, and
files written here open in the reference:

* DANN core file -- DiskANN::build_index_with_params / open_index_with /
  from_bytes / to_bytes (src/lib.rs:355-680): ``[magic u32 = 0x44414E4E]
  [version u32 = 1][md_len u64][bincode Metadata]`` at offset 0 (or, in the
  older layout, ``[md_len u64][Metadata]``), the f32 rows at
  ``vectors_offset`` (1 MiB) and the adjacency rows, ``max_degree`` u32 each
  padded with 0xFFFFFFFF, at ``adjacency_offset``.
* QANN sidecar, version 2 -- QuantizedDiskANN::save_quantized /
  from_quantized_bytes (src/quantized.rs:420-575): a 33-byte header
  ``[magic u32 = 0x51414E4E][version u32 = 2][quantizer_type u8][num_vectors
  u64][code_size u64][quantizer_data_len u64]``, the bincode QuantizerState
  and then ``num_vectors * code_size`` code bytes.
* Labels -- FilteredDiskANN::save_labels / load_labels (src/filtered.rs:
  322-425): ``[meta_len u64][bincode {num_vectors, num_fields}]`` and then the
  u64 labels row by row.
* The combined byte forms QuantizedDiskANN::to_bytes and
  FilteredDiskANN::to_bytes: ``[base_len u64][core bytes][sidecar or labels]``.

bincode 1.x with its default options (the reference calls
``bincode::serialize``): little-endian fixed-width integers, usize as u64,
f32 as its IEEE bits, String and Vec as a u64 length and the items, an enum
as its u32 variant index and the variant's fields, Option as a u8 tag.

Errors carry the reference's messages and are RuntimeError, like the
reference binding's (python/src/lib.rs:36-38).
"""
from __future__ import annotations

import os
import struct
from dataclasses import dataclass

import numpy as np

CORE_MAGIC = 0x44414E4E
CORE_FORMAT_VERSION = 1
CORE_VECTORS_OFFSET = 1024 * 1024
QANN_MAGIC = 0x51414E4E
QANN_VERSION = 2
QANN_HEADER = 33
PAD_U32 = 0xFFFFFFFF

# std::any::type_name of the reference's distance types (src/metric.rs:8-14)
# against this package's metric names; "l2" is squared L2 as in the binding.
DISTANCE_NAMES = {
    "l2": "diskann_rs::metric::DistL2Sq",
    "euclidean": "diskann_rs::metric::DistL2",
    "cosine": "diskann_rs::metric::DistCosine",
    "dot": "diskann_rs::metric::DistDot",
}
_SUFFIX_METRIC = {"DistL2Sq": "l2", "DistL2": "euclidean", "DistCosine": "cosine", "DistDot": "dot"}

# QuantizerState variant index = quantizer_type byte (src/quantized.rs:150-165)
QUANTIZER_TYPES = ("pq", "f16", "int8", "rabitq")


def _index_error(msg):
    return RuntimeError(f"Index error: {msg}")


def io_error(e: OSError) -> RuntimeError:
    """DiskAnnError::Io as the binding raises it: `I/O error: ` and Rust's
    io::Error text, e.g. `No such file or directory (os error 2)`."""
    if e.strerror and e.errno is not None:
        return RuntimeError(f"I/O error: {e.strerror} (os error {e.errno})")
    return RuntimeError(f"I/O error: {e}")


def _ser_error(msg):
    return RuntimeError(f"Serialization error: {msg}")


def metric_of_distance_name(name: str) -> str | None:
    """The package metric a recorded distance_name denotes (None if unknown)."""
    return _SUFFIX_METRIC.get(name.rsplit("::", 1)[-1])


# ------------------------------------------------------------------ bincode
class _Reader:
    def __init__(self, buf, pos=0, end=None):
        self.b = memoryview(buf).cast("B")
        self.p = pos
        self.end = len(self.b) if end is None else end

    def _take(self, n):
        if n < 0 or self.p + n > self.end:
            raise _ser_error("io error: unexpected end of file")
        s = self.p
        self.p += n
        return s

    def u8(self):
        return self.b[self._take(1)]

    def u32(self):
        return struct.unpack_from("<I", self.b, self._take(4))[0]

    def u64(self):
        return struct.unpack_from("<Q", self.b, self._take(8))[0]

    usize = u64

    def f32(self):
        return struct.unpack_from("<f", self.b, self._take(4))[0]

    def string(self):
        n = self.u64()
        s = self._take(n)
        try:
            return bytes(self.b[s:s + n]).decode("utf-8")
        except UnicodeDecodeError as e:
            raise _ser_error(f"invalid utf-8: {e}") from None

    def vec(self, dtype):
        n = self.u64()
        dt = np.dtype(dtype).newbyteorder("<")
        if n > (self.end - self.p) // dt.itemsize:
            raise _ser_error("io error: unexpected end of file")
        s = self._take(n * dt.itemsize)
        return np.frombuffer(self.b, dtype=dt, count=n, offset=s).astype(dt.newbyteorder("="))

    def option(self, read):
        tag = self.u8()
        if tag == 0:
            return None
        if tag == 1:
            return read()
        raise _ser_error(f"invalid value: integer `{tag}`, expected option tag")


class _Writer:
    def __init__(self):
        self.parts = []

    def u8(self, v):
        self.parts.append(struct.pack("<B", v))

    def u32(self, v):
        self.parts.append(struct.pack("<I", v))

    def u64(self, v):
        self.parts.append(struct.pack("<Q", v))

    usize = u64

    def f32(self, v):
        self.parts.append(struct.pack("<f", v))

    def string(self, s):
        b = s.encode("utf-8")
        self.u64(len(b))
        self.parts.append(b)

    def vec(self, a, dtype):
        a = np.ascontiguousarray(a, dtype=np.dtype(dtype).newbyteorder("<")).reshape(-1)
        self.u64(a.size)
        self.parts.append(a.tobytes())

    def option(self, v, write):
        if v is None:
            self.u8(0)
        else:
            self.u8(1)
            write(v)

    def bytes(self):
        return b"".join(self.parts)


# ---------------------------------------------------------------- core file
@dataclass
class CoreMetadata:
    """Metadata (src/lib.rs:88-98)."""
    dim: int
    num_vectors: int
    max_degree: int
    medoid_id: int
    vectors_offset: int
    adjacency_offset: int
    distance_name: str
    legacy: bool = False  # written without the magic / version words

    @property
    def metric(self):
        return metric_of_distance_name(self.distance_name)


def _metadata_bytes(m: CoreMetadata) -> bytes:
    w = _Writer()
    w.usize(m.dim)
    w.usize(m.num_vectors)
    w.usize(m.max_degree)
    w.u32(m.medoid_id)
    w.u64(m.vectors_offset)
    w.u64(m.adjacency_offset)
    w.string(m.distance_name)
    return w.bytes()


def parse_core_metadata(buf) -> tuple[CoreMetadata, int]:
    """DiskANN::parse_metadata (src/lib.rs:636-680): (metadata, its end offset)."""
    b = memoryview(buf).cast("B")
    if len(b) < 8:
        raise _index_error("Buffer too small for metadata length")
    legacy = struct.unpack_from("<I", b, 0)[0] != CORE_MAGIC
    if legacy:
        off = 0
    else:
        if len(b) < 16:
            raise _index_error("Buffer too small for header")
        ver = struct.unpack_from("<I", b, 4)[0]
        if ver != CORE_FORMAT_VERSION:
            raise _index_error(f"Unsupported core format version: {ver}")
        off = 8
    md_len = struct.unpack_from("<Q", b, off)[0]
    # open_index_with's bound (src/lib.rs:540-547): under 1 MiB and in the file
    if md_len > CORE_VECTORS_OFFSET or off + 8 + md_len > len(b):
        raise _index_error(f"Invalid metadata length {md_len} (file size {len(b)})")
    r = _Reader(b, off + 8, off + 8 + md_len)
    m = CoreMetadata(r.usize(), r.usize(), r.usize(), r.u32(), r.u64(), r.u64(), r.string(), legacy)
    return m, off + 8 + md_len


def parse_core(buf):
    """(metadata, vectors f32[n, dim], adjacency u32[n, max_degree]) of a core
    file's bytes; the arrays are views of `buf` (a memmap stays a memmap)."""
    m, _ = parse_core_metadata(buf)
    n, d, R = m.num_vectors, m.dim, m.max_degree
    size = len(memoryview(buf).cast("B"))
    if n == 0 or d == 0 or R == 0:
        raise _index_error(f"empty index (num_vectors {n}, dim {d}, max_degree {R})")
    if m.vectors_offset + n * d * 4 > size:
        raise _index_error(f"vectors [{m.vectors_offset}, +{n * d * 4}) past the end ({size} bytes)")
    if m.adjacency_offset + n * R * 4 > size:
        raise _index_error(f"adjacency [{m.adjacency_offset}, +{n * R * 4}) past the end ({size} bytes)")
    if m.vectors_offset % 4 or m.adjacency_offset % 4:
        raise _index_error("vectors / adjacency offsets are not 4-byte aligned")
    if m.medoid_id >= n:
        raise _index_error(f"medoid {m.medoid_id} out of range (num_vectors {n})")
    X = np.frombuffer(buf, dtype="<f4", count=n * d, offset=m.vectors_offset).reshape(n, d)
    A = np.frombuffer(buf, dtype="<u4", count=n * R, offset=m.adjacency_offset).reshape(n, R)
    return m, X, A


def read_core(path):
    """parse_core over a read-only memory map of `path` (open_index_with)."""
    try:
        buf = np.memmap(path, dtype=np.uint8, mode="r")
    except OSError as e:
        raise io_error(e) from None
    except ValueError as e:  # empty file
        raise _index_error(f"Invalid metadata length (file size 0): {e}") from None
    return parse_core(buf)


def core_bytes(vectors, adjacency, medoid_id, metric="l2", legacy=False) -> bytes:
    """The core file build_index_with_params writes (src/lib.rs:425-498):
    metadata at 0, zeros up to 1 MiB, the rows, the padded adjacency."""
    X = np.ascontiguousarray(vectors, dtype="<f4")
    A = np.ascontiguousarray(adjacency, dtype="<u4")
    n, d = X.shape
    if A.shape[0] != n:
        raise ValueError(f"adjacency has {A.shape[0]} rows, vectors {n}")
    name = DISTANCE_NAMES[metric] if metric in DISTANCE_NAMES else metric
    m = CoreMetadata(d, n, A.shape[1], int(medoid_id), CORE_VECTORS_OFFSET,
                     CORE_VECTORS_OFFSET + n * d * 4, name, legacy)
    md = _metadata_bytes(m)
    head = (b"" if legacy else struct.pack("<II", CORE_MAGIC, CORE_FORMAT_VERSION)) + struct.pack("<Q", len(md)) + md
    if len(head) > CORE_VECTORS_OFFSET:
        raise ValueError("metadata does not fit below the vectors offset")
    return b"".join([head, bytes(CORE_VECTORS_OFFSET - len(head)), X.tobytes(), A.tobytes()])


def write_core(path, vectors, adjacency, medoid_id, metric="l2"):
    _write(path, core_bytes(vectors, adjacency, medoid_id, metric))


def _write(path, data: bytes):
    with open(path, "wb") as f:
        f.write(data)
        f.flush()
        os.fsync(f.fileno())


# ------------------------------------------------------------- QANN sidecar
@dataclass
class QuantizerState:
    """QuantizerState (src/quantized.rs:150-155) with its variant's fields:
    pq: dim, num_subspaces, num_centroids, subspace_dim, codebooks f32[M*K*ds]
    (src/pq.rs:35-47); f16: dim (src/sq.rs:36-38); int8: dim, scale, offset
    (src/sq.rs:121-125); rabitq: dim, padded, centroid f32[dim], signs
    f32[3*padded] (src/rabitq.rs:12-18)."""
    kind: str
    dim: int
    num_subspaces: int = 0
    num_centroids: int = 0
    subspace_dim: int = 0
    codebooks: np.ndarray | None = None
    scale: float = 0.0
    offset: float = 0.0
    padded: int = 0
    centroid: np.ndarray | None = None
    signs: np.ndarray | None = None

    @property
    def type_id(self) -> int:
        return QUANTIZER_TYPES.index(self.kind)

    @property
    def code_size(self) -> int:
        """Bytes per code: PQ one per subspace, F16 2*dim, Int8 dim, RaBitQ
        padded/8 + 8 (src/rabitq.rs:117-119)."""
        return {"pq": self.num_subspaces, "f16": 2 * self.dim, "int8": self.dim,
                "rabitq": self.padded // 8 + 8}[self.kind]


def _read_state(r: _Reader) -> QuantizerState:
    tag = r.u32()
    if tag == 0:
        d, M, K, ds = r.usize(), r.usize(), r.usize(), r.usize()
        return QuantizerState("pq", d, M, K, ds, codebooks=r.vec("f4"))
    if tag == 1:
        return QuantizerState("f16", r.usize())
    if tag == 2:
        d = r.usize()
        return QuantizerState("int8", d, scale=r.f32(), offset=r.f32())
    if tag == 3:
        d, P = r.usize(), r.usize()
        return QuantizerState("rabitq", d, padded=P, centroid=r.vec("f4"), signs=r.vec("f4"))
    raise _ser_error(f"invalid value: integer `{tag}`, expected variant index 0 <= i < 4")


def _write_state(w: _Writer, s: QuantizerState):
    w.u32(s.type_id)
    w.usize(s.dim)
    if s.kind == "pq":
        w.usize(s.num_subspaces)
        w.usize(s.num_centroids)
        w.usize(s.subspace_dim)
        w.vec(s.codebooks, "f4")
    elif s.kind == "int8":
        w.f32(s.scale)
        w.f32(s.offset)
    elif s.kind == "rabitq":
        w.usize(s.padded)
        w.vec(s.centroid, "f4")
        w.vec(s.signs, "f4")


def quantizer_state_bytes(s: QuantizerState) -> bytes:
    w = _Writer()
    _write_state(w, s)
    return w.bytes()


def parse_quantizer_state(buf) -> QuantizerState:
    return _read_state(_Reader(buf))


def _check_state(s: QuantizerState):
    """The invariants the reference's quantizers hold after train()."""
    if s.kind == "pq":
        if s.num_subspaces == 0 or s.num_subspaces * s.subspace_dim != s.dim:
            raise _index_error(f"PQ: num_subspaces {s.num_subspaces} * subspace_dim {s.subspace_dim} != dim {s.dim}")
        if s.codebooks.size != s.num_subspaces * s.num_centroids * s.subspace_dim:
            raise _index_error("PQ: codebooks size != num_subspaces * num_centroids * subspace_dim")
    elif s.kind == "rabitq":
        if s.centroid.size != s.dim or s.signs.size != 3 * s.padded:
            raise _index_error("RaBitQ: centroid / signs sizes do not match dim / padded")


def parse_sidecar(buf, num_vectors=None):
    """QuantizedDiskANN::from_quantized_bytes (src/quantized.rs:511-574):
    (QuantizerState, codes u8[num_vectors, code_size])."""
    b = memoryview(buf).cast("B")
    if len(b) < QANN_HEADER:
        raise _index_error("Quantized data too small")
    magic, ver, qtype, n, code_size, qlen = struct.unpack_from("<IIBQQQ", b, 0)
    if magic != QANN_MAGIC:
        raise _index_error(f"Invalid magic: expected 0x{QANN_MAGIC:08X}, got 0x{magic:08X}")
    if ver != QANN_VERSION:
        raise _index_error(f"Unsupported version: {ver}")
    if num_vectors is not None and n != num_vectors:
        raise _index_error(f"Sidecar has {n} vectors, base index has {num_vectors}")
    pos = QANN_HEADER
    if len(b) < pos + qlen:
        raise _index_error("Truncated quantizer data")
    s = _read_state(_Reader(b, pos, pos + qlen))
    if s.type_id != qtype:
        raise _index_error("Quantizer type mismatch")
    pos += qlen
    if len(b) < pos + n * code_size:
        raise _index_error("Truncated codes data")
    _check_state(s)
    if code_size != s.code_size:
        raise _index_error(f"code_size {code_size} != {s.kind} code size {s.code_size}")
    codes = np.frombuffer(b, dtype=np.uint8, count=n * code_size, offset=pos).reshape(n, code_size)
    return s, codes


def sidecar_bytes(state: QuantizerState, codes) -> bytes:
    """QuantizedDiskANN::quantized_to_bytes (src/quantized.rs:490-509)."""
    c = np.ascontiguousarray(codes, dtype=np.uint8)
    if c.ndim != 2 or c.shape[1] != state.code_size:
        raise ValueError(f"codes must be u8[n, {state.code_size}]")
    q = quantizer_state_bytes(state)
    return struct.pack("<IIBQQQ", QANN_MAGIC, QANN_VERSION, state.type_id, c.shape[0], c.shape[1], len(q)) + q + c.tobytes()


def read_sidecar(path, num_vectors=None):
    try:
        with open(path, "rb") as f:
            data = f.read()
    except OSError as e:
        raise io_error(e) from None
    return parse_sidecar(data, num_vectors)


def write_sidecar(path, state: QuantizerState, codes):
    _write(path, sidecar_bytes(state, codes))


# ------------------------------------------------------------------- labels
def parse_labels(buf) -> np.ndarray:
    """FilteredDiskANN::deserialize_labels (src/filtered.rs:339-370): u64[n, num_fields]."""
    b = memoryview(buf).cast("B")
    if len(b) < 8:
        raise _index_error("Labels buffer too small")
    meta_len = struct.unpack_from("<Q", b, 0)[0]
    if len(b) < 8 + meta_len:
        raise _index_error("Labels buffer too small for metadata")
    r = _Reader(b, 8, 8 + meta_len)
    n, nf = r.usize(), r.usize()
    data = len(b) - 8 - meta_len
    if n * nf * 8 > data:
        raise _index_error("Labels data truncated")
    return np.frombuffer(b, dtype="<u8", count=n * nf, offset=8 + meta_len).reshape(n, nf).astype(np.uint64)


def labels_bytes(labels) -> bytes:
    """FilteredDiskANN::serialize_labels (src/filtered.rs:322-337)."""
    L = np.ascontiguousarray(labels, dtype="<u8")
    if L.ndim != 2:
        raise ValueError("labels must be u64[n, num_fields]")
    w = _Writer()
    w.usize(L.shape[0])
    w.usize(L.shape[1])
    md = w.bytes()
    return struct.pack("<Q", len(md)) + md + L.tobytes()


def read_labels(path) -> np.ndarray:
    try:
        with open(path, "rb") as f:
            data = f.read()
    except OSError as e:
        raise io_error(e) from None
    return parse_labels(data)


def write_labels(path, labels):
    _write(path, labels_bytes(labels))


# ------------------------------------------------------------ combined forms
def split_prefixed(buf, what="base index"):
    """``[len u64][first][rest]`` (QuantizedDiskANN::from_bytes,
    src/quantized.rs:468-488; FilteredDiskANN::from_bytes, src/filtered.rs:257-270)."""
    b = memoryview(buf).cast("B")
    if len(b) < 8:
        raise _index_error("Buffer too small")
    n = struct.unpack_from("<Q", b, 0)[0]
    if len(b) < 8 + n:
        raise _index_error(f"Buffer too small for {what}")
    return b[8:8 + n], b[8 + n:]


def join_prefixed(first: bytes, rest: bytes) -> bytes:
    return struct.pack("<Q", len(first)) + first + rest



# ------------------------------------------------------------------ SPFresh
# SPFresh::save / open (src/spfresh.rs:819-859) keep an index in four files:
#   {path}.spf        bincode Meta {dim, cfg, quantizer, block_cid, block_centroid,
#                     next_id, deleted, live} (src/spfresh.rs:62-72)
#   {path}.postings   fixed-size blocks [len u32][len x (id u64, code)] zero-padded
#                     to 4 + 2 * max_posting_size * (8 + code_size) bytes
#                     (src/spfresh.rs:109-111, 258-270)
#   {path}.vectors    the raw f32 rows by id (src/spfresh.rs:271-273)
#   {path}.centroids  IncrementalDiskANN bytes over the posting centroids; a
#                     block's entry in block_cid is its centroid's id there,
#                     u64::MAX for a free block (src/spfresh.rs:18, 395-415)
SPF_FREE = 0xFFFFFFFFFFFFFFFF
INCR_MAGIC = 0x494E4352
INCR_FORMAT_VERSION = 2
DELTA_ID_OFFSET = 1 << 48  # delta-layer ids of IncrementalDiskANN (src/incremental.rs:334)


@dataclass
class SPFreshConfig:
    """SPFreshConfig (src/spfresh.rs:25-52), field order as serialized."""
    max_posting_size: int = 128
    min_posting_size: int = 16
    probe_ratio: float = float("inf")
    rerank_size: int = 0
    reassign_neighbors: int = 16
    centroid_beam: int = 64


@dataclass
class SPFreshMeta:
    dim: int
    cfg: SPFreshConfig
    quantizer: QuantizerState | None
    block_cid: np.ndarray        # u64[nblocks]
    block_centroid: list         # f32[dim] per live block, empty for a free one
    next_id: int
    deleted: np.ndarray          # u64[]
    live: int


def spf_code_size(quantizer: QuantizerState | None, dim: int) -> int:
    """code_size (src/spfresh.rs:99-107): raw f32 rows without a quantizer."""
    return 4 * dim if quantizer is None else quantizer.code_size


def spf_block_bytes(cfg: SPFreshConfig, quantizer, dim: int) -> int:
    """block_bytes (src/spfresh.rs:109-111) after Inner::new's max(2) clamp."""
    return 4 + 2 * max(cfg.max_posting_size, 2) * (8 + spf_code_size(quantizer, dim))


def parse_spf(buf) -> SPFreshMeta:
    r = _Reader(buf)
    dim = r.usize()
    cfg = SPFreshConfig(r.usize(), r.usize(), r.f32(), r.usize(), r.usize(), r.usize())
    q = r.option(lambda: _read_state(r))
    if q is not None:
        _check_state(q)
        if q.dim != dim:
            raise _index_error(f"quantizer dim {q.dim} != index dim {dim}")
    cid = r.vec("u8")
    ncent = r.u64()
    if ncent != len(cid):
        raise _index_error(f"{ncent} block centroids for {len(cid)} blocks")
    cents = [r.vec("f4") for _ in range(ncent)]
    for b, c in enumerate(cents):
        if cid[b] != SPF_FREE and c.size != dim:
            raise _index_error(f"block {b}: centroid of {c.size} values, dim {dim}")
    return SPFreshMeta(dim, cfg, q, cid, cents, r.u64(), r.vec("u8"), r.usize())


def spf_bytes(m: SPFreshMeta) -> bytes:
    w = _Writer()
    w.usize(m.dim)
    c = m.cfg
    w.usize(c.max_posting_size)
    w.usize(c.min_posting_size)
    w.f32(c.probe_ratio)
    w.usize(c.rerank_size)
    w.usize(c.reassign_neighbors)
    w.usize(c.centroid_beam)
    w.option(m.quantizer, lambda q: _write_state(w, q))
    w.vec(m.block_cid, "u8")
    w.u64(len(m.block_centroid))
    for v in m.block_centroid:
        w.vec(v, "f4")
    w.u64(m.next_id)
    w.vec(m.deleted, "u8")
    w.usize(m.live)
    return w.bytes()


def parse_postings(buf, nblocks: int, block: int, code_size: int):
    """(ids u64[len], codes u8[len, code_size]) per block (Inner::len / entry,
    src/spfresh.rs:258-270)."""
    b = np.frombuffer(buf, dtype=np.uint8)
    if b.size < nblocks * block:
        raise _index_error(f"postings file holds {b.size // block} blocks, metadata {nblocks}")
    entry = 8 + code_size
    cap = (block - 4) // entry
    out = []
    for k in range(nblocks):
        blk = b[k * block:(k + 1) * block]
        n = int(blk[:4].view("<u4")[0])
        if n > cap:
            raise _index_error(f"block {k}: {n} entries, capacity {cap}")
        e = blk[4:4 + n * entry].reshape(n, entry)
        out.append((np.ascontiguousarray(e[:, :8]).view("<u8").reshape(n).astype(np.uint64),
                    np.ascontiguousarray(e[:, 8:])))
    return out


def postings_bytes(blocks, block: int, code_size: int) -> bytes:
    """The postings file for [(ids, codes)] per block (Inner::rewrite, src/spfresh.rs:304-314)."""
    entry = 8 + code_size
    out = np.zeros((len(blocks), block), np.uint8)
    for k, (ids, codes) in enumerate(blocks):
        n = len(ids)
        if 4 + n * entry > block:
            raise ValueError(f"block {k}: {n} entries do not fit in {block} bytes")
        out[k, :4] = np.frombuffer(struct.pack("<I", n), np.uint8)
        e = out[k, 4:4 + n * entry].reshape(n, entry)
        e[:, :8] = np.asarray(ids, dtype="<u8").view(np.uint8).reshape(n, 8)
        e[:, 8:] = np.asarray(codes, dtype=np.uint8).reshape(n, code_size)
    return out.tobytes()


def incremental_bytes(vectors, graph, entry_point, max_degree, tombstones=(), base=None, labels=None,
                      dim=None, quantizer=None) -> bytes:
    """IncrementalDiskANN::to_bytes (src/incremental.rs:1234-1327): the base core
    bytes (or none), the delta rows, their adjacency lists (local indexes),
    entry point (-1 = none), max degree, tombstones, labels as (num_fields,
    base_labels, delta_labels) or None, and the quantizer as (code_size,
    rerank_size, QuantizerState, base codes) or None."""
    V = np.ascontiguousarray(vectors, dtype="<f4")
    d = V.shape[1] if V.ndim == 2 and V.shape[1] else int(dim or 0)
    V = V.reshape(-1, d) if d else V.reshape(0, 0)
    parts = [struct.pack("<II", INCR_MAGIC, INCR_FORMAT_VERSION)]
    parts += [b"\x00"] if base is None else [b"\x01", struct.pack("<Q", len(base)), bytes(base)]
    parts += [struct.pack("<QQ", d, V.shape[0]), V.tobytes(), struct.pack("<Q", len(graph))]
    for nb in graph:
        a = np.asarray(nb, dtype="<u4")
        parts += [struct.pack("<I", a.size), a.tobytes()]
    ts = np.asarray(list(tombstones), dtype="<u8")
    parts += [struct.pack("<qQQ", -1 if entry_point is None else int(entry_point), max_degree, ts.size), ts.tobytes()]
    if labels is None:
        parts.append(b"\x00")
    else:
        nf, bl, dl = labels
        bl = np.ascontiguousarray(bl, dtype="<u8").reshape(-1, nf) if nf else np.zeros((len(bl), 0), "<u8")
        dl = np.ascontiguousarray(dl, dtype="<u8").reshape(-1, nf) if nf else np.zeros((len(dl), 0), "<u8")
        parts += [b"\x01", struct.pack("<QQ", nf, len(bl)), bl.tobytes(), struct.pack("<Q", len(dl)), dl.tobytes()]
    if quantizer is None:
        parts.append(b"\x00")
    else:
        cs, rr, st, codes = quantizer
        q = quantizer_state_bytes(st)
        c = np.ascontiguousarray(codes, dtype=np.uint8).reshape(-1)
        parts += [b"\x01", struct.pack("<QQQ", cs, rr, len(q)), q, struct.pack("<Q", c.size), c.tobytes()]
    return b"".join(parts)


def parse_incremental(buf) -> dict:
    """IncrementalDiskANN::from_bytes_v1 (src/incremental.rs:1451-1611): base
    bytes (or None), dim, delta vectors f32[n, dim], adjacency lists, entry
    point, max degree, tombstones, labels as (num_fields, base, delta) or None,
    quantizer as (code_size, rerank_size, QuantizerState, codes u8[]) or None.
    The older layout without the magic is refused."""
    b = memoryview(buf).cast("B")
    r = _Reader(b)

    def trunc(fn):
        try:
            return fn()
        except RuntimeError:
            raise _index_error("Incremental buffer truncated") from None

    if len(b) < 4:
        raise _index_error("Incremental buffer too small")
    if struct.unpack_from("<I", b, 0)[0] != INCR_MAGIC:
        raise _index_error("incremental buffers without the INCR magic (the older layout) are not supported")
    r.u32()
    ver = trunc(r.u32)
    if ver != INCR_FORMAT_VERSION:
        raise _index_error(f"Unsupported incremental format version: {ver}")
    base = None
    if trunc(r.u8) == 1:
        n = trunc(r.u64)
        s = trunc(lambda: r._take(n))
        base = b[s:s + n]
    dim = trunc(r.u64)
    nd = trunc(r.u64)
    s = trunc(lambda: r._take(nd * dim * 4))
    V = np.frombuffer(b, dtype="<f4", count=nd * dim, offset=s).reshape(nd, dim).astype(np.float32)
    ng = trunc(r.u64)
    graph = []
    for _ in range(ng):
        deg = trunc(r.u32)
        s = trunc(lambda: r._take(deg * 4))
        graph.append(np.frombuffer(b, dtype="<u4", count=deg, offset=s).astype(np.uint32).tolist())
    ep = struct.unpack("<q", bytes(b[trunc(lambda: r._take(8)):][:8]))[0]
    max_degree = trunc(r.u64)
    nt = trunc(r.u64)
    s = trunc(lambda: r._take(nt * 8))
    tomb = np.frombuffer(b, dtype="<u8", count=nt, offset=s).astype(np.uint64).tolist()
    labels = None
    if trunc(r.u8) == 1:
        nf = trunc(r.u64)
        nbl = trunc(r.u64)
        s = trunc(lambda: r._take(nbl * nf * 8))
        bl = np.frombuffer(b, dtype="<u8", count=nbl * nf, offset=s).reshape(nbl, nf).astype(np.uint64)
        ndl = trunc(r.u64)
        s = trunc(lambda: r._take(ndl * nf * 8))
        dl = np.frombuffer(b, dtype="<u8", count=ndl * nf, offset=s).reshape(ndl, nf).astype(np.uint64)
        labels = (nf, bl, dl)
    quant = None
    if trunc(r.u8) == 1:
        cs, rr, ql = trunc(r.u64), trunc(r.u64), trunc(r.u64)
        s = trunc(lambda: r._take(ql))
        st = _read_state(_Reader(b, s, s + ql))
        _check_state(st)
        if st.code_size != cs:
            raise _index_error(f"code_size {cs} != {st.kind} code size {st.code_size}")
        nc = trunc(r.u64)
        s = trunc(lambda: r._take(nc))
        quant = (cs, rr, st, np.frombuffer(b, dtype=np.uint8, count=nc, offset=s).copy())
    if len(graph) != nd:
        raise _index_error(f"{len(graph)} adjacency lists for {nd} delta vectors")
    return {"base": base, "dim": dim, "vectors": V, "graph": graph, "entry_point": None if ep < 0 else ep,
            "max_degree": max_degree, "tombstones": tomb, "labels": labels, "quantizer": quant}


def check_incremental_header(buf):
    """IncrementalDiskANN::from_bytes's format probe (src/incremental.rs:1332-1351):
    the INCR magic and version 2, or the older layout's has_base byte."""
    b = memoryview(buf).cast("B")
    if len(b) < 4:
        raise _index_error("Incremental buffer too small")
    if struct.unpack_from("<I", b, 0)[0] == INCR_MAGIC:
        if len(b) < 8 or struct.unpack_from("<I", b, 4)[0] != INCR_FORMAT_VERSION:
            raise _index_error("Unsupported incremental format version")
    elif b[0] not in (0, 1):
        raise _index_error("Incremental buffer: unknown format")
