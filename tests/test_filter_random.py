"""Random label filters (CPU): the Python restatement of Filter::matches
(src/filtered.rs:112-128) and the oracle's evaluator of the compiled postfix
program -- the program the kernels run -- agree on every label vector.

Edge cases the reference defines: a field past the vector's labels is false
(`labels.get(field).map_or(false, ..)`), And([]) is true and Or([]) false,
In with no values is false, Range with min > max is false, Filter::None
nested inside And / Or is true, and values at 0 and 2^64 - 1.  Per-query
programs packed into one array (pack_filters) keep each query's meaning.
"""
import numpy as np
import pytest

from pydiskann_b200 import Filter

U64_MAX = (1 << 64) - 1
VALUES = [0, 1, 2, 3, 5, 8, U64_MAX - 1, U64_MAX]


def _leaf(rng, nf):
    field = int(rng.integers(0, nf + 2))  # sometimes past the vector's labels
    v = lambda: VALUES[int(rng.integers(0, len(VALUES)))]  # noqa: E731
    kind = int(rng.integers(0, 6))
    if kind == 0:
        return Filter.eq(field, v())
    if kind == 1:
        return Filter.in_(field, [v() for _ in range(int(rng.integers(0, 4)))])
    if kind == 2:
        return Filter.lt(field, v())
    if kind == 3:
        return Filter.gt(field, v())
    if kind == 4:
        return Filter.range(field, v(), v())  # min > max half the time
    return Filter.none()


def _tree(rng, nf, depth):
    if depth == 0 or rng.random() < 0.3:
        return _leaf(rng, nf)
    kids = [_tree(rng, nf, depth - 1) for _ in range(int(rng.integers(0, 5)))]
    return Filter.and_(kids) if rng.random() < 0.5 else Filter.or_(kids)


@pytest.mark.parametrize("seed", range(4))
def test_compiled_program_matches_tree(oracle, seed):
    rng = np.random.default_rng(seed)
    checked = 0
    for _ in range(400):
        nf = int(rng.integers(1, 4))
        f = _tree(rng, nf, 3)
        ops, pool = f.program()
        for _ in range(8):
            lab = [VALUES[int(rng.integers(0, len(VALUES)))] for _ in range(nf)]
            assert f.matches(lab) == oracle.filter_matches(ops, pool, lab), (f, lab)
            checked += 1
    assert checked == 3200


def test_reference_edge_cases(oracle):
    lab = [3, U64_MAX]
    cases = [
        (Filter.and_([]), True), (Filter.or_([]), False), (Filter.in_(0, []), False),
        (Filter.range(0, 5, 1), False), (Filter.eq(2, 3), False), (Filter.lt(7, U64_MAX), False),
        (Filter.and_([Filter.none(), Filter.eq(0, 3)]), True), (Filter.or_([Filter.none()]), True),
        (Filter.gt(1, U64_MAX - 1), True), (Filter.range(1, U64_MAX, U64_MAX), True),
    ]
    for f, want in cases:
        ops, pool = f.program()
        assert f.matches(lab) is want, f
        assert oracle.filter_matches(ops, pool, lab) is want, f


def test_packed_per_query_programs(oracle):
    """pack_filters: query q's slice ops[offs[q]:offs[q+1]] of the packed
    program, with IN offsets rebased into the shared value pool, evaluates as
    that query's own filter (the layout dg_search_batch reads through
    filter_offsets)."""
    from pydiskann_b200 import pack_filters

    rng = np.random.default_rng(11)
    nf = 3
    filters = [_tree(rng, nf, 3) for _ in range(300)]
    pk = pack_filters(filters)
    assert pk.n == 300 and len(pk.offs) == 301 and pk.offs[0] == 0
    assert np.all(np.diff(pk.offs.astype(np.int64)) >= 0)
    ops = [(o.op, o.field, o.a, o.b) for o in pk.arr]
    pool = [int(v) for v in pk.pool[: pk.plen]]
    for q, f in enumerate(filters):
        mine = ops[pk.offs[q]: pk.offs[q + 1]]
        assert len(mine) == len(f.program()[0])
        for _ in range(6):
            lab = [VALUES[int(rng.integers(0, len(VALUES)))] for _ in range(nf)]
            assert oracle.filter_matches(mine, pool, lab) == f.matches(lab), (q, f, lab)
