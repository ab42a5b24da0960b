"""Malformed files fail the way the reference fails (CPU).

The reference reads its formats with bincode and explicit bounds checks, so a
truncated or corrupted file returns DiskAnnError (`Index error: ...`,
`Serialization error: ...`, surfaced by the binding as RuntimeError), never a
crash.  Here every proper prefix of a valid blob, and blobs with bytes
overwritten at random, must parse or raise RuntimeError -- not IndexError,
struct.error, a numpy error or MemoryError from a corrupted length prefix.
"""
import numpy as np
import pytest

from pydiskann_b200 import formats as F
from test_formats import _spf_fixture

PAD = 0xFFFFFFFF


def _blobs():
    rng = np.random.default_rng(0)
    X = rng.standard_normal((6, 4)).astype(np.float32)
    A = np.full((6, 3), PAD, np.uint32)
    A[:, 0] = (np.arange(6) + 1) % 6
    core = F.core_bytes(X, A, 2, "l2")
    pq = F.QuantizerState("pq", 4, 2, 4, 2, codebooks=rng.standard_normal(16).astype(np.float32))
    i8 = F.QuantizerState("int8", 4, scale=0.5, offset=-1.0)
    lab = rng.integers(0, 9, (9, 2)).astype(np.uint64)
    incr = F.incremental_bytes(X[:3], [[1, 2], [0], []], 1, 32, tombstones=[4, (1 << 48) + 1], base=core,
                               labels=(2, lab[:6], lab[6:]),
                               quantizer=(4, 8, i8, rng.integers(0, 255, (6, 4)).astype(np.uint8)))
    cs, block = 3, 4 + 4 * (8 + 3)
    posts = F.postings_bytes([(np.array([5, 7], np.uint64), np.arange(6, dtype=np.uint8).reshape(2, 3)),
                              (np.zeros(0, np.uint64), np.zeros((0, 3), np.uint8))], block, cs)
    return {
        "core": (F.parse_core, core),
        "sidecar": (F.parse_sidecar, F.sidecar_bytes(pq, rng.integers(0, 4, (6, 2)).astype(np.uint8))),
        "labels": (F.parse_labels, F.labels_bytes(lab[:6])),
        "quantizer_state": (F.parse_quantizer_state, F.quantizer_state_bytes(pq)),
        "spf": (F.parse_spf, _spf_fixture()),
        "postings": (lambda b: F.parse_postings(b, 2, block, cs), posts),
        "incremental": (F.parse_incremental, incr),
    }


BLOBS = _blobs()


def _lengths(n):
    """Every prefix length for small blobs; for the 1 MiB-padded core files the
    header region, a stride through the padding and the tail."""
    if n <= 4096:
        return range(n)
    return sorted(set(range(0, 2048)) | set(range(2048, n, 4093)) | set(range(n - 512, n)))


@pytest.mark.parametrize("name", list(BLOBS))
def test_valid_blob_parses(name):
    parse, raw = BLOBS[name]
    parse(raw)


@pytest.mark.parametrize("name", list(BLOBS))
def test_every_truncation_is_an_error(name):
    parse, raw = BLOBS[name]
    for n in _lengths(len(raw)):
        try:
            parse(raw[:n])
        except RuntimeError:
            continue
        pytest.fail(f"{name}: a {n}-byte prefix of {len(raw)} bytes parsed without error")


@pytest.mark.parametrize("name", list(BLOBS))
def test_corrupted_bytes_parse_or_raise(name):
    parse, raw = BLOBS[name]
    rng = np.random.default_rng(len(raw))
    # where headers, length prefixes and tags sit: the first 256 bytes and the
    # last KiB (the delta, label and quantizer sections after a padded core file)
    n = len(raw)
    where = np.unique(np.concatenate([np.arange(min(n, 256)), np.arange(max(0, n - 1024), n)]))
    for _ in range(300):
        bad = bytearray(raw)
        for pos in rng.choice(where, size=rng.integers(1, 4)):
            bad[pos] = int(rng.integers(0, 256))
        try:
            parse(bytes(bad))
        except RuntimeError:
            pass
