"""Known-answer checks of the reference test-suite (tests/golden/reference_kats.json),
written once and run against two backends: the CPU oracle and the GPU library."""
import json
import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def load_kats():
    with open(os.path.join(HERE, "golden", "reference_kats.json")) as f:
        return json.load(f)


def euclid(a, b):
    return math.sqrt(sum((x - y) ** 2 for x, y in zip(a, b)))


def build_filter(spec, Filter):
    kind = spec[0]
    if kind == "none":
        return Filter.none()
    if kind in ("and", "or"):
        subs = [build_filter(s, Filter) for s in spec[1]]
        return Filter.and_(subs) if kind == "and" else Filter.or_(subs)
    if kind == "in":
        return Filter.in_(spec[1], spec[2])
    if kind == "range":
        return Filter.range(spec[1], spec[2], spec[3])
    return getattr(Filter, kind)(spec[1], spec[2])


def grid_vectors(g):
    return [[float(i), float(j)] for i in range(g) for j in range(g)]


def check_index_kats(kats, build_and_search):
    """build_and_search(vectors, metric, R, Lb, alpha, queries, k, L) -> list of [(id, dist)]."""
    c = kats["square_best"]
    r = build_and_search(c["vectors"], c["metric"], 64, 128, 1.2, [c["query"]], c["k"], c["beam_width"])[0]
    assert r[0][0] == c["expect_first"], r

    c = kats["small_index_l2"]
    r = build_and_search(c["vectors"], c["metric"], 64, 128, 1.2, [c["query"]], c["k"], c["beam_width"])[0]
    assert len(r) == c["expect_len"]
    assert euclid(c["query"], c["vectors"][r[0][0]]) < c["first_within"]

    c = kats["cosine_direction"]
    r = build_and_search(c["vectors"], c["metric"], 64, 128, 1.2, [c["query"]], c["k"], c["beam_width"])[0]
    assert len(r) == c["k"]
    v, q = np.asarray(c["vectors"][r[0][0]]), np.asarray(c["query"])
    assert float(v @ q / (np.linalg.norm(v) * np.linalg.norm(q))) > c["min_cos_first"]

    c = kats["grid_connectivity"]
    vecs = grid_vectors(c["grid"])
    res = build_and_search(vecs, c["metric"], c["max_degree"], c["build_beam_width"], c["alpha"], vecs, c["k"],
                           c["beam_width"])
    for t, r in enumerate(res):
        ids = [i for i, _ in r]
        if t not in ids:
            assert euclid(vecs[t], vecs[ids[0]]) < c["miss_first_within"]
        for i in ids[:5]:
            assert euclid(vecs[t], vecs[i]) < c["top5_within"]

    c = kats["single_vector"]
    for q, k, exp in zip(c["queries"], c["ks"], c["expect"]):
        r = build_and_search(c["vectors"], c["metric"], 64, 128, 1.2, [q], k, c["beam_width"])[0]
        assert [i for i, _ in r] == exp

    c = kats["two_vectors"]
    res = build_and_search(c["vectors"], c["metric"], 64, 128, 1.2, c["queries"], c["k"], c["beam_width"])
    assert [[i for i, _ in r] for r in res] == c["expect"]

    c = kats["identical_vectors"]
    r = build_and_search(c["vectors"], c["metric"], 64, 128, 1.2, [c["query"]], c["k"], c["beam_width"])[0]
    assert len(r) == c["expect_len"]
    assert all(d < c["max_dist"] for _, d in r)


def check_result_invariants(rows, k, n):
    """tests/correctness.rs:58-99: count min(k, n), no duplicates, finite, non-negative, sorted."""
    for r in rows:
        assert len(r) == min(k, n)
        ids = [i for i, _ in r]
        assert len(set(ids)) == len(ids)
        ds = [d for _, d in r]
        assert all(math.isfinite(d) and d >= 0 for d in ds)
        assert ds == sorted(ds)
