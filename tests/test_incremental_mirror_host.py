"""IncrementalDiskANN's device mirror, simulated on the host (no GPU).

The device index is replaced by host arrays, and the entry points that
publish rows, adjacency, labels, seeds and tombstones write into them.
dg_delta_insert runs for real (it is host code).  After inserts that grow
past the spare rows, labelled inserts and deletes, the simulated device
holds exactly the reference's unified view (UnifiedView,
src/incremental.rs:349-471): base rows, then delta rows with their
adjacency shifted by base_count, the two seeds, and the tombstoned rows.
"""
import ctypes as C

import numpy as np
import pytest

import pydiskann_b200 as dg
import pydiskann_b200.incremental as inc_mod
from pydiskann_b200 import _lib
from pydiskann_b200.incremental import DELTA_ID_OFFSET, IncrementalDiskANN

PAD = 0xFFFFFFFF


class FakeIndex:
    def __init__(self, X, A, medoid, metric, device):
        self.X, self.A = X.copy(), A.copy()
        self._h = self
        self.seeds, self.dead, self.labels = None, set(), None
        self.n, self.dim, self.R = X.shape[0], X.shape[1], A.shape[1]

    def close(self):
        pass


def _arr(p, ctype, shape):
    return np.ctypeslib.as_array(C.cast(p, C.POINTER(ctype)), shape).copy()


class FakeLib:
    """The index entry points the mirror calls, applied to a FakeIndex."""

    def __init__(self):
        self.real = _lib.lib()

    def dg_delta_insert(self, *args):
        return self.real.dg_delta_insert(*args)

    def dg_index_update_rows(self, h, first, count, vec, adj, lab):
        assert 0 <= first and first + count <= h.n
        if vec is not None:
            h.X[first:first + count] = _arr(vec, C.c_float, (count, h.dim))
        if adj is not None:
            h.A[first:first + count] = _arr(adj, C.c_uint32, (count, h.R))
        if lab is not None:
            h.labels[first:first + count] = _arr(lab, C.c_uint64, (count, h.labels.shape[1]))
        return 0

    def dg_index_set_entry_points(self, h, ids, n):
        h.seeds = _arr(ids, C.c_uint32, (n,)).tolist()
        return 0

    def dg_index_set_tombstones(self, h, ids, n, deleted, count):
        rows = _arr(ids, C.c_uint32, (max(n, 1),))[:n].tolist()
        (h.dead.update if deleted else h.dead.difference_update)(rows)
        return 0

    def dg_index_attach_labels(self, h, nf, labels):
        h.labels = _arr(labels, C.c_uint64, (h.n, nf))
        return 0


@pytest.fixture()
def sim(monkeypatch):
    monkeypatch.setattr(dg, "_Index", FakeIndex)
    fake = FakeLib()
    monkeypatch.setattr(inc_mod, "lib", lambda: fake)


def _expect(ix):
    """The unified view from the object's own state."""
    nb, dn = ix.base_count, ix._dn
    X = np.concatenate([ix._bX, ix._dX[:dn]])
    A = np.full((nb + dn, ix._Ru), PAD, np.uint32)
    A[:nb, : ix._bA.shape[1]] = ix._bA
    dA = ix._dA[:dn]
    A[nb:, : dA.shape[1]] = np.where(dA != PAD, dA + nb, PAD)
    seeds = [ix._bmed] + ([nb + ix._ep] if ix._ep >= 0 else [])
    dead = {r for r in (ix._row_of(g) for g in ix.tombstones) if r is not None}
    return X, A, seeds, dead


def _check(ix):
    h = ix._h
    X, A, seeds, dead = _expect(ix)
    n = len(X)
    assert np.array_equal(h.X[:n], X) and np.array_equal(h.A[:n], A)
    assert np.all(h.A[n:] == PAD)  # spare rows link nowhere
    assert h.seeds == seeds and h.dead == dead


def test_mirror_tracks_inserts_growth_and_deletes(sim):
    rng = np.random.default_rng(3)
    base = rng.integers(0, 50, (300, 8)).astype(np.float32)
    badj = np.where(rng.random((300, 12)) < 0.8, rng.integers(0, 300, (300, 12)), PAD).astype(np.uint32)
    ix = IncrementalDiskANN(base, badj, 7)
    _check(ix)
    first_h = ix._h
    ids = ix.add_vectors(rng.integers(0, 50, (600, 8)).astype(np.float32))
    assert ids == [DELTA_ID_OFFSET + j for j in range(600)]
    _check(ix)
    ix.delete_vectors([3, 5, DELTA_ID_OFFSET + 10, DELTA_ID_OFFSET + 700])  # 700 not inserted yet
    _check(ix)
    ix.add_vectors(rng.integers(0, 50, (500, 8)).astype(np.float32))  # 1100 > 1024 spare rows: a new mirror
    assert ix._h is not first_h and ix._cap >= 1100
    _check(ix)  # delta id 700 now exists and is dead
    assert ix._row_of(DELTA_ID_OFFSET + 700) in ix._h.dead
    ix.add_vectors([[1.0] * 8])
    _check(ix)


def test_mirror_labels(sim):
    rng = np.random.default_rng(4)
    base = rng.integers(0, 50, (200, 6)).astype(np.float32)
    badj = rng.integers(0, 200, (200, 8)).astype(np.uint32)
    lab = rng.integers(0, 9, (200, 2)).astype(np.uint64)
    ix = IncrementalDiskANN(base, badj, 0, labels=lab)
    new_lab = rng.integers(0, 9, (50, 2)).astype(np.uint64)
    ix.add_vectors_with_labels(rng.integers(0, 50, (50, 6)).astype(np.float32), new_lab)
    ix.add_vectors(rng.integers(0, 50, (10, 6)).astype(np.float32))  # labels default to zeros
    _check(ix)
    h = ix._h
    assert np.array_equal(h.labels[:200], lab)
    assert np.array_equal(h.labels[200:250], new_lab)
    assert np.all(h.labels[250:260] == 0)
    with pytest.raises(RuntimeError, match="vectors.len\\(\\) \\(2\\) != labels.len\\(\\) \\(1\\)"):
        ix.add_vectors_with_labels(np.zeros((2, 6), np.float32), [[1, 2]])
    with pytest.raises(RuntimeError, match="Vector 1 has dimension 5 but index expects 6"):
        ix.add_vectors([[0.0] * 6, [0.0] * 5])
    assert ix.stats()["delta_vectors"] == 60
