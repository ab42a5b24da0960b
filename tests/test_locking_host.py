"""Thread safety of the updatable indexes (host logic, no GPU).

The reference guards IncrementalDiskANN's delta layer, tombstones and labels
(src/incremental.rs:521-534) and SPFresh's state (src/spfresh.rs:778) with
RwLocks, and its binding releases the GIL around inserts and searches
(python/src/lib.rs:161-189), so one thread may insert while another searches.
The mirrors serialise every public update and search of one object on a
per-object lock; these tests check the lock's semantics on a stand-in object
and that every such method is wrapped.
"""
import threading
import time

import pytest

from pydiskann_b200._lib import locked
from pydiskann_b200.incremental import IncrementalDiskANN
from pydiskann_b200.spfresh import SPFresh


class _Counter:
    def __init__(self):
        self._lock = threading.RLock()
        self.inside = 0
        self.most = 0
        self.calls = 0

    @locked
    def work(self):
        self.inside += 1
        self.most = max(self.most, self.inside)
        time.sleep(0.001)
        self.calls += 1
        self.inside -= 1

    @locked
    def nested(self):  # a locked method calling another one (compact -> _mirror paths)
        self.work()
        return self.calls


def test_locked_excludes_and_reenters():
    c = _Counter()
    threads = [threading.Thread(target=lambda: [c.work() for _ in range(20)]) for _ in range(6)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert c.calls == 120 and c.most == 1
    assert c.nested() == 121
    assert c.work.__name__ == "work" and c.work.__wrapped__ is _Counter.work.__wrapped__


@pytest.mark.parametrize("cls, names", [
    (IncrementalDiskANN, ["_add", "delete_vectors", "is_deleted", "search_arrays", "enable_bf16", "get_vector",
                          "should_compact", "compact", "stats", "to_bytes", "close"]),
    (SPFresh, ["insert", "delete", "is_deleted", "get_vector", "gc", "compact", "stats", "save", "close",
               "search_arrays"]),
])
def test_public_methods_are_locked(cls, names):
    for n in names:
        assert hasattr(getattr(cls, n), "__wrapped__"), f"{cls.__name__}.{n} runs without the object's lock"
