"""The SPFresh posting lists kept on the host follow the reference's update
path exactly: after every batch of a stream of inserts and deletes (and a gc
every few batches), each live posting slot holds the same entries in the same
order with the same codes, under the same centroid, as the oracle's
restatement of src/spfresh.rs:380-643 (oracle/spfresh_updates.py), and the
free slot lists agree.  Host-only instances (no GPU): searches over these
postings are compared with the oracle in tests/test_gpu_spfresh.py."""
import numpy as np
import pytest

import oracle
from oracle.spfresh_updates import RefSpfresh
from pydiskann_b200 import synth
from pydiskann_b200.spfresh import SPFresh


def _same_state(s, ref, tag):
    live = [b for b in range(len(s.live_b)) if s.live_b[b]]
    assert live == ref.live_slots(), tag
    post = ref.postings()
    for b in live:
        ids, codes = post[b]
        assert np.array_equal(s.ids[b], ids), f"{tag}: slot {b} entries differ"
        if len(ids):
            assert np.array_equal(s.codes[b], codes), f"{tag}: slot {b} codes"
        assert np.array_equal(s.cent[b], ref.centroid[b]), f"{tag}: slot {b} centroid"
    assert sorted(s.free) == sorted(ref.free), tag
    assert s.next_id == ref.next_id and s.live == ref.live and s.deleted == ref.deleted, tag


def _build_both(X, max_posting, min_posting, quantizer=None, seed=0):
    s = SPFresh.build(X, None, quantizer=quantizer, max_posting_size=max_posting, min_posting_size=min_posting,
                      seed=seed, device=None)
    enc = None
    if quantizer == "int8":
        sc, off = s.codec.p["scale"], s.codec.p["offset"]
        enc = lambda V: oracle.int8_encode(V, sc, off)  # noqa: E731
    ref = RefSpfresh(X.shape[1], max_posting, min_posting, encode=enc)
    k = max(1, len(X) // max(max_posting // 2, 1))
    rng = np.random.default_rng([seed, 0x5EED])
    for i in rng.choice(len(X), size=min(k, len(X)), replace=False):
        ref.new_posting(X[i])
    ref.insert(X)
    return s, ref


@pytest.mark.parametrize("quantizer", [None, "int8"])
def test_update_stream_matches_restatement(quantizer):
    # integer-valued Zipf(1.1)-weighted mixture, the SPFresh workload's recipe at a small size
    X = synth.mixture(6000, 32, 64, seed=3, clip=False, zipf=1.1)
    s, ref = _build_both(X, 48, 8, quantizer)
    _same_state(s, ref, "build")
    rng = np.random.default_rng(17)
    for batch in range(8):
        new = synth.mixture(600, 32, 64, seed=3, stream=synth.STREAM_MISC + 10 + batch, clip=False, zipf=1.1)
        a = s.insert(new)
        b = ref.insert(new)
        assert a == b
        live_ids = np.array(sorted(set(range(s.next_id)) - s.deleted))
        gone = rng.choice(live_ids, size=300, replace=False)
        s.delete(gone)
        ref.delete(gone)
        if batch % 3 == 2:
            s.gc()
            ref.gc()
        _same_state(s, ref, f"batch {batch}")
