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


def test_oracle_multithreaded_equals_single_threaded():
    rng = np.random.default_rng(7)
    n = 300_000
    k = O.HostColumn(O.INT64, rng.integers(0, 5000, n))
    v1 = O.HostColumn(O.INT64, rng.integers(-10**9, 10**9, n), rng.random(n) > 0.1)
    v2 = O.HostColumn(O.FLOAT64, rng.normal(size=n), rng.random(n) > 0.1)
    kinds = [O.SUM, O.MIN, O.MAX, O.COUNT_VALID, O.MEAN]
    a = O.groupby([k], [(v1, kinds), (v2, kinds)], nthreads=1)
    b = O.groupby([k], [(v1, kinds), (v2, kinds)], nthreads=8)
    assert np.array_equal(a.group_rows, b.group_rows)
    for ra, rb in zip(a.results, b.results):
        for (xa, va, ta), (xb, vb, tb) in zip(ra, rb):
            assert np.array_equal(va, vb)
            if xa.dtype.kind == "f":
                assert np.all(np.abs(xa - xb) <= ta + tb + 1e-300)
            else:
                assert np.array_equal(xa, xb)
