"""Concurrent inserts and searches of one IncrementalDiskANN on the GPU.

The reference guards the delta layer and tombstones with RwLocks
(src/incremental.rs:521-534) and its binding releases the GIL around inserts
and searches (python/src/lib.rs:161-189), so one thread may insert while
others search.  Tolerance: none (the final state's ids, counts and FP32
distances bit-identical to the oracle; integer-valued data).
"""
import threading
import time

import pytest

import pydiskann_b200 as dg
from pydiskann_b200.incremental import DELTA_ID_OFFSET
from test_gpu_incremental import _check

pytestmark = pytest.mark.gpu


@pytest.fixture()
def inc(small_data):
    import oracle as o

    X, _ = small_data
    base = X[:3000]
    badj, bmed = o.build_vamana(base, R=32, L_build=64, alpha=1.2, seed=3)
    ix = dg.IncrementalDiskANN(base, badj, bmed)
    yield ix, X
    ix.close()


def test_inserts_while_searching(inc, small_data, oracle):
    """One thread inserts (growing the device mirror past its spare rows) and
    deletes while three threads search, as the reference's RwLocks and the
    binding's released GIL allow (python/src/lib.rs:161-189).  No search fails
    or returns an id the index does not hold, and the final state searches as
    the oracle does."""
    ix, X = inc
    _, Q = small_data
    errors, stop = [], threading.Event()

    def searcher():
        try:
            while not stop.is_set():
                ids, _, cnt = ix.search_arrays(Q[:32], 10, 64)
                time.sleep(0.002)  # the lock is not fair: leave the inserter room
                for q in range(len(cnt)):
                    for g in ids[q, : cnt[q]]:
                        g = int(g)
                        if not (g < ix.base_count or DELTA_ID_OFFSET <= g < DELTA_ID_OFFSET + 1200):
                            errors.append(g)
        except Exception as e:  # noqa: BLE001
            errors.append(e)

    threads = [threading.Thread(target=searcher) for _ in range(3)]
    for t in threads:
        t.start()
    batches = [X[c:c + 200] for c in range(3000, 4000, 200)] + [X[:200] + 1.0]  # 1200 rows > 1024 spare
    try:
        for j, B in enumerate(batches):
            ix.add_vectors(B)
            ix.delete_vectors([200 * j + 1, DELTA_ID_OFFSET + 200 * j])
    finally:
        stop.set()
        for t in threads:
            t.join()
    assert not errors, errors[:3]
    assert ix.stats()["delta_vectors"] == 1200
    _check(ix, oracle, Q, 10, 64)
