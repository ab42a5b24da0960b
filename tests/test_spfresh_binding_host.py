"""SPFresh update semantics of the reference's binding tests, on a host-only
instance (no GPU; searches are covered by tests/test_gpu_spfresh.py).

The assertions follow python/tests/test_spfresh.py:72-160 -- build stats and
posting bounds, contiguous insert ids, delete / re-delete / unknown ids, gc,
repeated inserts -- on seeded data of the same shape: 32 dimensions, postings
of at most 64 entries (min 8), 2000 points around 25 centres.
"""
import numpy as np
import pytest

from pydiskann_b200.spfresh import SPFresh

DIM, MAX_POSTING = 32, 64


def _clustered(n, seed, spread=0.12):
    centres = np.random.default_rng(1234).uniform(-1.0, 1.0, (25, DIM))
    rng = np.random.default_rng(seed)
    return (centres[np.arange(n) % 25] + rng.normal(0.0, spread, (n, DIM))).astype(np.float32)


def _uniform(n, seed):
    return np.random.default_rng(seed).uniform(-1.0, 1.0, (n, DIM)).astype(np.float32)


def _bounded(s):
    st = s.stats()
    assert st["max_posting"] < MAX_POSTING, st
    assert st["postings"] >= 1


@pytest.fixture()
def built():
    X = _clustered(2000, 1)
    return SPFresh.build(X, None, max_posting_size=MAX_POSTING, min_posting_size=8, device=None), X


def test_build_stats_and_bounds(built):
    s, X = built
    st = s.stats()
    assert (st["live"], st["deleted"]) == (len(X), 0)
    assert st["postings"] >= len(X) // MAX_POSTING and s.dim == DIM
    _bounded(s)
    for i in (0, 7, 1999):
        assert s.get_vector(i) == X[i].tolist()


def test_insert_ids_contiguous(built):
    s, X = built
    new = _clustered(300, 4)
    ids = s.insert(new)
    assert ids == list(range(len(X), len(X) + 300))
    assert s.stats()["live"] == len(X) + 300
    _bounded(s)
    for i in ids[::30]:
        assert s.get_vector(i) == new[i - len(X)].tolist()


def test_delete_then_gc(built):
    s, X = built
    dead = list(range(0, 500, 10))
    s.delete(dead)
    st = s.stats()
    assert (st["deleted"], st["live"]) == (len(dead), len(X) - len(dead))
    assert all(s.is_deleted(i) and s.get_vector(i) is None for i in dead)
    s.delete(dead)
    s.delete([10**9])  # past next_id: ignored
    assert s.stats()["live"] == len(X) - len(dead)
    assert not s.is_deleted(10**9)
    s.gc()
    assert s.stats()["live"] == len(X) - len(dead)
    _bounded(s)
    live_entries = {int(i) for b in range(len(s.ids)) if s.live_b[b] for i in s.ids[b]}
    assert not live_entries & set(dead)  # gc purged the tombstoned entries
    assert live_entries == set(range(len(X))) - set(dead)


def test_many_inserts_keep_bounds():
    X = _uniform(1000, 6)
    s = SPFresh.build(X, None, max_posting_size=MAX_POSTING, min_posting_size=8, device=None)
    n = len(X)
    for b in range(5):
        ids = s.insert(_uniform(600, 10 + b))
        assert ids[0] == n
        n += 600
        _bounded(s)
    assert s.stats()["live"] == n
    held = sorted(int(i) for b in range(len(s.ids)) if s.live_b[b] for i in s.ids[b])
    assert held == list(range(n))  # every id in exactly one posting
