"""The SPFresh update stream of the 2M x 96 workload, at a small size: a
Zipf(1.1)-weighted, integer-valued 96-d mixture bulk-loaded into more than
512 postings, then batches of 1 % inserts and 0.5 % deletes, each followed by
a batch of searches at n_probe 64.  After every batch the posting lists equal
those of the oracle's restatement of the update path (src/spfresh.rs:380-643)
slot by slot, and the GPU search -- routed over more than 512 live postings,
so the batched posting-major scan with its tensor-core tiles runs -- returns
the oracle's ids, distances and counts bit for bit."""
import numpy as np
import pytest

import pydiskann_b200 as dg
from oracle.spfresh_updates import RefSpfresh
from pydiskann_b200 import synth

pytestmark = pytest.mark.gpu


def _ref_from(s):
    """A restatement instance holding the product's current slots."""
    ref = RefSpfresh(s.dim, s.max_posting, s.min_posting, s.reassign_neighbors)
    ref.live_slot = [bool(x) for x in s.live_b]
    ref.centroid = [s.cent[b].copy() if s.live_b[b] else None for b in range(len(s.live_b))]
    ref.entries = [[(int(i), bytes(c)) for i, c in zip(s.ids[b], s.codes[b])] for b in range(len(s.live_b))]
    ref.free = list(s.free)
    ref.epoch = s.epoch
    ref.raw = [r.copy() for r in s.raw[: s.next_id]]
    ref.next_id, ref.deleted, ref.live = s.next_id, set(s.deleted), s.live
    return ref


def test_update_stream_membership_and_search(oracle):
    from test_gpu_spfresh import oracle_view

    X = synth.mixture(24_000, 96, 256, seed=5, clip=False, zipf=1.1)
    s = dg.SPFresh.bulk_load(X, max_posting_size=32, min_posting_size=4, seed=1)
    assert int(s.live_b.sum()) > 512
    ref = _ref_from(s)
    Q = synth.mixture(768, 96, 256, seed=5, stream=synth.STREAM_QUERY, clip=False, zipf=1.1)
    rng = np.random.default_rng(9)
    for batch in range(4):
        new = synth.mixture(240, 96, 256, seed=5, stream=synth.STREAM_MISC + 20 + batch, clip=False, zipf=1.1)
        assert s.insert(new) == ref.insert(new)
        live_ids = np.array(sorted(set(range(s.next_id)) - s.deleted))
        gone = rng.choice(live_ids, size=120, replace=False)
        s.delete(gone)
        ref.delete(gone)
        post = ref.postings()
        assert [b for b in range(len(s.live_b)) if s.live_b[b]] == sorted(post)
        for b, (ids, codes) in post.items():
            assert np.array_equal(s.ids[b], ids), (batch, b)
            assert np.array_equal(s.cent[b], ref.centroid[b]), (batch, b)
        view, keep = oracle_view(oracle, s)
        gi, gd, gc = s.search_arrays(Q, 10, 64)
        oi, od, oc = oracle.spfresh_search(view, Q, 10, 64)
        assert np.array_equal(gc, oc), batch
        assert np.array_equal(gi, oi), (batch, np.nonzero((gi != oi).any(1))[0][:5])
        assert np.array_equal(gd, od), batch
    s.close()
