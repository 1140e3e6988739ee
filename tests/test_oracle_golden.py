"""Pins the CPU oracle to libcudf's own known answers (CPU only)."""
import numpy as np
import pytest

import golden_harness as GH
from oracle import oracle as O

CASES = list(GH.expand())


@pytest.mark.parametrize("cid,case,keys,vals,kinds", CASES, ids=[c[0] for c in CASES])
def test_oracle_matches_reference_golden_vectors(cid, case, keys, vals, kinds):
    if case["error"]:
        with pytest.raises(ValueError):
            O.groupby([keys], [(vals, kinds)], include_null_keys=case["include_null_keys"])
        return
    r = O.groupby([keys], [(vals, kinds)], include_null_keys=case["include_null_keys"])
    out = [(v, valid) for (v, valid, _tol) in r.results[0]]
    GH.check(case, keys, vals, kinds, r.keys[0], out)


def _by_key(r):
    order = O.sort_order(r.keys)
    return order, [(np.asarray(d)[order], None if v is None else np.asarray(v)[order]) for d, v in r.keys]


@pytest.mark.parametrize("case", ["one_key", "two_keys_include", "two_keys_exclude"])
def test_oracle_partitioned_path_equals_single_threaded(case):
    """The multi-threaded oracle hash-partitions rows by key and aggregates each
    partition in row order, so every group sees its rows in the same order as
    the single-threaded path: results are identical bit for bit (floats too),
    only the order of the groups differs."""
    rng = np.random.default_rng(7)
    n = 300_000
    if case == "one_key":
        keys = [O.HostColumn(O.INT64, rng.integers(0, 5000, n))]
        inc = False
    else:
        keys = [O.HostColumn(O.INT32, rng.integers(0, 300, n), rng.random(n) > 0.05),
                O.HostColumn(O.FLOAT64, rng.integers(0, 40, n) * 0.5, rng.random(n) > 0.05)]
        inc = case == "two_keys_include"
    f2 = rng.normal(size=n)
    f2[rng.random(n) < 0.01] = np.nan
    v1 = O.HostColumn(O.INT64, rng.integers(-10**9, 10**9, n), rng.random(n) > 0.1)
    v2 = O.HostColumn(O.FLOAT64, f2, rng.random(n) > 0.1)
    v3 = O.HostColumn(O.FLOAT32, rng.lognormal(size=n).astype(np.float32))
    kinds = [O.SUM, O.MIN, O.MAX, O.COUNT_VALID, O.COUNT_ALL, O.MEAN, O.VARIANCE, O.STD,
             O.ARGMIN, O.ARGMAX, O.SUM_OF_SQUARES]
    reqs = [(v1, kinds), (v2, kinds), (v3, kinds)]
    a = O.groupby(keys, reqs, include_null_keys=inc, nthreads=1)
    b = O.groupby(keys, reqs, include_null_keys=inc, nthreads=8)
    assert a.num_groups == b.num_groups
    oa, ka = _by_key(a)
    ob, kb = _by_key(b)
    for (da, va), (db, vb) in zip(ka, kb):
        assert (va is None) == (vb is None)
        if va is not None:
            assert np.array_equal(va, vb)
            da, db = da[va], db[vb]
        assert np.array_equal(da, db)
    assert np.array_equal(a.group_rows[oa], b.group_rows[ob])
    for ra, rb in zip(a.results, b.results):
        for (xa, va, ta), (xb, vb, tb) in zip(ra, rb):
            assert np.array_equal(va[oa], vb[ob])
            assert np.array_equal(xa[oa], xb[ob], equal_nan=xa.dtype.kind == "f")
            assert np.array_equal(ta[oa], tb[ob], equal_nan=True)
