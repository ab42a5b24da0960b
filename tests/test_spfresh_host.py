"""SPFresh host-side update path (insert / split / relocate / delete / gc) on
CPU: structural invariants of src/spfresh.rs's posting lists."""
import numpy as np
import pytest

from pydiskann_b200 import SPFresh, synth
from pydiskann_b200.spfresh import kmeans2


def _check(s, all_ids):
    seen = {}
    for b in range(len(s.live_b)):
        if not s._is_live(b):
            assert len(s.ids[b]) == 0
            continue
        assert len(s.ids[b]) == len(s.codes[b])
        assert len(s.ids[b]) < 2 * s.max_posting
        for i in s.ids[b]:
            assert int(i) not in seen, "an id lives in two postings"
            seen[int(i)] = b
    live = {i for i in all_ids if i not in s.deleted}
    assert live <= set(seen), "a live id is in no posting"
    return seen


@pytest.mark.parametrize("quant", [None, "int8", "f16", "rabitq"])
def test_build_insert_delete_gc_invariants(quant):
    X = synth.mixture(3000, 32, 24, seed=5, clip=False)
    s = SPFresh.build(X, metric="l2", quantizer=quant, max_posting_size=40, min_posting_size=8, device=None)
    _check(s, range(3000))
    assert s.stats()["live"] == 3000
    Y = synth.mixture(600, 32, 24, seed=6, clip=False)
    new = s.insert(Y)
    assert new == list(range(3000, 3600))
    _check(s, range(3600))
    s.delete(list(range(0, 3600, 7)))
    assert s.is_deleted(0) and not s.is_deleted(1)
    assert s.get_vector(0) is None and s.get_vector(1) is not None
    s.gc()
    seen = _check(s, range(3600))
    assert all(i not in s.deleted for i in seen), "gc purges tombstones"
    st = s.stats()
    assert st["live"] == 3600 - len(range(0, 3600, 7))
    assert st["max_posting"] < 2 * s.max_posting


def test_codes_follow_their_posting():
    """RaBitQ codes are residuals against their posting's centroid (src/spfresh.rs:324-339)."""
    X = synth.mixture(1500, 32, 12, seed=8, clip=False)
    s = SPFresh.build(X, quantizer="rabitq", max_posting_size=30, device=None)
    for b in range(len(s.live_b)):
        if s._is_live(b) and len(s.ids[b]):
            want = s.codec.encode(s.raw[s.ids[b].astype(np.int64)], s.cent[b])
            assert np.array_equal(want, s.codes[b])


def test_kmeans2_degenerate_split():
    vs = np.ones((10, 4), dtype=np.float32)
    c1, c2, side = kmeans2(vs, 0)
    assert side.sum() == 5  # index split when every point is identical


def test_non_converging_updates_raise():
    """1 - dot on unnormalised data sends every vector to the largest centroid;
    the update path stops with an error instead of splitting forever."""
    X = synth.mixture(2000, 32, 20, seed=12, clip=False)
    with pytest.raises(RuntimeError):
        SPFresh.build(X, metric="dot", max_posting_size=40, min_posting_size=8, device=None)
