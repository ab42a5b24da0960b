"""SPFresh's device mirror, simulated on the host (no GPU).

The dg_spfresh_* entry points are replaced by host arrays that they write, so
the host-to-device publishing of an SPFresh -- whole-mirror creation, dirty
posting slots, new raw rows, new tombstones, and re-creation when postings or
ids outgrow the mirror -- can be followed through inserts, deletes and gc.
After each step the simulated device must hold the host's posting slots
(host_arrays), raw rows and tombstone set.
"""
import ctypes as C

import numpy as np
import pytest

import pydiskann_b200.spfresh as spf_mod
from pydiskann_b200.spfresh import SPFresh


def _arr(p, ctype, shape):
    return _view(p, ctype, shape).copy()


def _view(p, ctype, shape):
    return np.ctypeslib.as_array(C.cast(C.c_void_p(p), C.POINTER(ctype)), shape)


class FakeSpfLib:
    def __init__(self):
        self.dev, self.next, self.created = {}, 1, 0

    def dg_spfresh_create(self, desc, out):
        d = desc._obj
        nb, cap, cs, dim = d.num_blocks, d.block_cap, d.code_size, d.dim
        st = {
            "cent": _arr(d.centroids, C.c_float, (nb, dim)), "live": _arr(d.block_live, C.c_uint8, (nb,)),
            "lens": _arr(d.block_len, C.c_uint32, (nb,)), "ids": _arr(d.entry_ids, C.c_uint64, (nb, cap)),
            "codes": _arr(d.entry_codes, C.c_uint8, (nb, cap, cs)), "raw": np.zeros((d.id_capacity, dim), np.float32),
            "deleted": _arr(d.deleted, C.c_uint8, (d.id_capacity,)).astype(bool), "cap": cap, "dim": dim, "cs": cs,
            "metric": d.metric,
        }
        if d.num_raw:
            st["raw"][: d.num_raw] = _arr(d.raw, C.c_float, (d.num_raw, dim))
        self.dev[self.next] = st
        out._obj.value = self.next
        self.next += 1
        self.created += 1
        return 0

    def _st(self, h):
        return self.dev[h.value]

    def dg_spfresh_destroy(self, h):
        del self.dev[h.value]
        return 0

    def dg_spfresh_update_blocks(self, h, blocks, n, cent, live, lens, ids, codes):
        st = self._st(h)
        b = _arr(blocks.value, C.c_uint32, (n,))
        st["cent"][b] = _arr(cent.value, C.c_float, (n, st["dim"]))
        st["live"][b] = _arr(live.value, C.c_uint8, (n,))
        st["lens"][b] = _arr(lens.value, C.c_uint32, (n,))
        st["ids"][b] = _arr(ids.value, C.c_uint64, (n, st["cap"]))
        st["codes"][b] = _arr(codes.value, C.c_uint8, (n, st["cap"], st["cs"]))
        return 0

    def dg_spfresh_put_raw(self, h, first, rows, n):
        st = self._st(h)
        st["raw"][first:first + n] = _arr(rows.value, C.c_float, (n, st["dim"]))
        return 0

    def dg_spfresh_set_centroids(self, h, blocks, n, cent, live):
        st = self._st(h)
        b = _arr(blocks.value, C.c_uint32, (n,))
        st["cent"][b] = _arr(cent.value, C.c_float, (n, st["dim"]))
        st["live"][b] = _arr(live.value, C.c_uint8, (n,))
        return 0

    def dg_spfresh_nearest(self, h, V, nv, n, slots, dists):
        """Routes against this stand-in's own copy of the centroids, so a
        centroid the host did not publish routes differently."""
        st = self._st(h)
        live = np.nonzero(st["live"])[0]
        D = spf_mod._seq_matrix(st["metric"], _arr(V.value, C.c_float, (nv, st["dim"])), st["cent"][live])
        order = np.lexsort((np.broadcast_to(live, D.shape), D), axis=1)[:, :n]
        _view(slots.value, C.c_uint32, (nv, n))[:] = live[order]
        _view(dists.value, C.c_float, (nv, n))[:] = np.take_along_axis(D, order, axis=1)
        return 0

    def dg_spfresh_set_deleted(self, h, ids, n, deleted):
        self._st(h)["deleted"][_arr(ids.value, C.c_uint64, (n,))] = bool(deleted)
        return 0


@pytest.fixture()
def fake(monkeypatch):
    f = FakeSpfLib()
    monkeypatch.setattr(spf_mod, "lib", lambda: f)
    return f


def _check(s, fake):
    st = fake.dev[s._h.value]
    cent, live, lens, ids, codes = s.host_arrays(s._dev_blocks)
    assert np.array_equal(st["live"], live) and np.array_equal(st["lens"], lens)
    for b in np.nonzero(live)[0]:  # free slots' contents are never read
        n = lens[b]
        assert np.array_equal(st["cent"][b], cent[b])
        assert np.array_equal(st["ids"][b, :n], ids[b, :n]) and np.array_equal(st["codes"][b, :n], codes[b, :n])
    assert np.array_equal(st["raw"][: s.next_id], s.raw[: s.next_id])
    assert set(np.nonzero(st["deleted"])[0].tolist()) == s.deleted


@pytest.mark.parametrize("quantizer", [None, "int8"])
def test_mirror_follows_updates(fake, quantizer):
    rng = np.random.default_rng(8)
    X = rng.standard_normal((1500, 16)).astype(np.float32)
    s = SPFresh.build(X, None, quantizer=quantizer, max_posting_size=32, min_posting_size=6, device=0)
    try:
        _check(s, fake)
        created = fake.created
        s.insert(rng.standard_normal((200, 16)).astype(np.float32))  # fits: dirty slots and raw rows only
        _check(s, fake)
        s.delete(list(range(0, 1700, 7)) + [10**9])
        _check(s, fake)
        s.gc()
        _check(s, fake)
        s.insert(rng.standard_normal((3000, 16)).astype(np.float32) * 3.0)  # outgrows the mirror
        assert fake.created > created
        _check(s, fake)
        s.compact()
        _check(s, fake)
        s.close()
        assert not fake.dev
    finally:
        s._h = None  # the handle is the stand-in's: the real library must never see it
