"""Cross-checks the CPU oracle against pandas' groupby on seeded random data
(the pattern of python/cudf/cudf/tests/test_groupby.py:48-69 and :1438-1480).

pandas gives 0 for the SUM of an all-null group and NaN for its MIN/MAX/MEAN;
libcudf gives null for all of them, so those groups are compared on validity.
"""
import numpy as np
import pandas as pd
import pytest

from oracle import oracle as O


def _frame(n, seed, card, null_frac):
    rng = np.random.default_rng(seed)
    key = rng.integers(0, card, n).astype(np.int32)
    v1 = rng.integers(0, 1_000_000, n, endpoint=True).astype(np.int64)
    v2 = rng.random(n)
    m1 = rng.random(n) >= null_frac
    m2 = rng.random(n) >= null_frac
    return key, v1, v2, m1, m2


@pytest.mark.parametrize("n,card,null_frac,seed", [(20_000, 1000, 0.0, 0), (50_000, 37, 0.1, 1),
                                                   (5_000, 4000, 0.3, 2)])
def test_oracle_vs_pandas(n, card, null_frac, seed):
    key, v1, v2, m1, m2 = _frame(n, seed, card, null_frac)
    kinds1 = [O.SUM, O.COUNT_VALID, O.MIN, O.MAX, O.MEAN]
    kinds2 = [O.MEAN, O.SUM]
    r = O.groupby([O.HostColumn(O.INT32, key)],
                  [(O.HostColumn(O.INT64, v1, m1 if null_frac else None), kinds1),
                   (O.HostColumn(O.FLOAT64, v2, m2 if null_frac else None), kinds2)])
    df = pd.DataFrame({"key": key,
                       "v1": pd.Series(pd.array(v1, dtype="Int64")).where(m1 if null_frac else np.ones(n, bool)),
                       "v2": pd.Series(np.where(m2, v2, np.nan) if null_frac else v2)})
    g = df.groupby("key", sort=True)
    exp = pd.DataFrame({"sum": g["v1"].sum(min_count=1), "count": g["v1"].count(),
                        "min": g["v1"].min(), "max": g["v1"].max(), "mean": g["v1"].mean(),
                        "mean2": g["v2"].mean(), "sum2": g["v2"].sum(min_count=1)})
    order = np.argsort(r.keys[0][0], kind="stable")
    assert np.array_equal(r.keys[0][0][order], exp.index.to_numpy())
    (s, sv, _), (c, _, _), (mn, mnv, _), (mx, _, _), (me, mev, _) = r.results[0]
    (me2, me2v, tol2), (s2, s2v, tol3) = r.results[1]
    sv, s = sv[order], s[order]
    assert np.array_equal(sv, exp["sum"].notna().to_numpy())
    assert np.array_equal(s[sv], exp["sum"].to_numpy()[sv].astype(np.int64))
    assert np.array_equal(c[order], exp["count"].to_numpy())
    assert np.array_equal(mn[order][sv], exp["min"].to_numpy()[sv].astype(np.int64))
    assert np.array_equal(mx[order][sv], exp["max"].to_numpy()[sv].astype(np.int64))
    assert np.allclose(me[order][sv], exp["mean"].to_numpy()[sv].astype(float), rtol=1e-12)
    v = me2v[order]
    assert np.array_equal(v, exp["mean2"].notna().to_numpy())
    assert np.all(np.abs(me2[order][v] - exp["mean2"].to_numpy()[v]) <= tol2[order][v] + 1e-15)
    assert np.all(np.abs(s2[order][v] - exp["sum2"].to_numpy()[v]) <= tol3[order][v] + 1e-12)


def test_oracle_include_null_keys_vs_pandas_dropna_false():
    rng = np.random.default_rng(5)
    n = 10_000
    k1 = rng.integers(0, 50, n).astype(np.int32)
    k2 = rng.integers(0, 7, n).astype(np.int64)
    kv1 = rng.random(n) >= 0.05
    kv2 = rng.random(n) >= 0.05
    v = rng.integers(0, 10**6, n).astype(np.int64)
    r = O.groupby([O.HostColumn(O.INT32, k1, kv1), O.HostColumn(O.INT64, k2, kv2)],
                  [(O.HostColumn(O.INT64, v), [O.SUM, O.COUNT_VALID, O.MAX])],
                  include_null_keys=True)
    df = pd.DataFrame({"k1": pd.Series(pd.array(k1, dtype="Int32")).where(kv1),
                       "k2": pd.Series(pd.array(k2, dtype="Int64")).where(kv2), "v": v})
    g = df.groupby(["k1", "k2"], dropna=False, sort=True)["v"]
    assert r.num_groups == g.ngroups
    exp = g.agg(["sum", "count", "max"]).reset_index()
    got = {}
    (s, _, _), (c, _, _), (mx, _, _) = r.results[0]
    for i in range(r.num_groups):
        a = int(r.keys[0][0][i]) if r.keys[0][1][i] else None
        b = int(r.keys[1][0][i]) if r.keys[1][1][i] else None
        got[(a, b)] = (int(s[i]), int(c[i]), int(mx[i]))
    for row in exp.itertuples(index=False):
        a = None if pd.isna(row.k1) else int(row.k1)
        b = None if pd.isna(row.k2) else int(row.k2)
        assert got[(a, b)] == (int(row.sum), int(row.count), int(row.max))
