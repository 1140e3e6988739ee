"""DataFrame.groupby(...).agg on the engine against pandas on the same data
(the pattern of python/cudf/cudf/tests/test_groupby.py:48-69, which compares
cudf's groupby with pandas' on random frames).  Groups hold enough rows that
no group's values are all null (where cudf's null SUM and pandas' 0 differ)."""
import numpy as np
import pandas as pd
import pytest

pytestmark = pytest.mark.gpu


def _frames(n=200_000, card=2000, seed=0):
    rng = np.random.default_rng(seed)
    k1 = rng.integers(0, card, n).astype(np.int32)
    k2 = rng.integers(0, 4, n).astype(np.int64)
    df = pd.DataFrame({
        "k1": pd.array(k1, dtype="Int32"),
        "k2": k2,
        "v1": pd.array(rng.integers(-10**6, 10**6, n), dtype="Int64"),
        "v2": rng.normal(size=n),
        "v3": rng.random(n).astype(np.float32),
    })
    df.loc[rng.random(n) < 0.02, "k1"] = pd.NA
    df.loc[rng.random(n) < 0.1, "v1"] = pd.NA
    df.loc[rng.random(n) < 0.1, "v2"] = np.nan
    return df


def _as_float(s):
    return pd.to_numeric(pd.Series(s), errors="coerce").astype("float64").to_numpy()


def _compare(got, exp, rtol=1e-9):
    got = got.sort_index()
    exp = exp.sort_index()
    assert list(got.columns) == list(exp.columns), (list(got.columns), list(exp.columns))
    assert len(got) == len(exp)
    gi, ei = got.index.to_frame(index=False), exp.index.to_frame(index=False)
    for c in gi.columns:
        a, b = gi[c], ei[c]
        assert np.array_equal(a.isna().to_numpy(), b.isna().to_numpy())
        assert np.array_equal(_as_float(a[~a.isna()]), _as_float(b[~b.isna()]))
    for c in got.columns:
        a, b = _as_float(got[c]), _as_float(exp[c])
        assert np.array_equal(np.isnan(a), np.isnan(b)), c
        m = ~np.isnan(a)
        assert np.allclose(a[m], b[m], rtol=rtol, atol=1e-9), c


@pytest.mark.parametrize("dropna", [True, False])
@pytest.mark.parametrize("spec", ["sum", ["sum", "min", "max", "mean", "count"],
                                  {"v1": "sum", "v2": ["min", "mean"], "v3": "max"}])
def test_agg_matches_pandas(spec, dropna):
    import cudf_b200 as cb
    pdf = _frames()
    gdf = cb.DataFrame.from_pandas(pdf)
    got = gdf.groupby(["k1", "k2"], sort=True, dropna=dropna).agg(spec).to_pandas()
    exp = pdf.groupby(["k1", "k2"], sort=True, dropna=dropna).agg(spec)
    _compare(got, exp, rtol=1e-5)
    # sort=True: groups come out in key order, nulls last
    idx = got.index.to_frame(index=False)
    k1 = idx["k1"].astype("float64").to_numpy()
    k1 = np.where(np.isnan(k1), 1e18, k1)
    assert np.all(np.diff(k1) >= 0)


def test_count_and_size_are_int64():
    import cudf_b200 as cb
    pdf = _frames(50_000, 100, 1)
    gdf = cb.DataFrame.from_pandas(pdf)
    got = gdf.groupby("k2", sort=True).agg({"v1": ["count", "size"]}).to_pandas()
    assert str(got[("v1", "count")].dtype) == "int64" and str(got[("v1", "size")].dtype) == "int64"
    exp = pdf.groupby("k2", sort=True).agg({"v1": ["count", "size"]})
    _compare(got, exp)
    s = gdf.groupby("k2", sort=True).size().to_pandas()
    assert np.array_equal(s.iloc[:, 0].to_numpy(), pdf.groupby("k2").size().to_numpy())


def test_series_selection_and_as_index_false():
    import cudf_b200 as cb
    pdf = _frames(80_000, 300, 2)
    gdf = cb.DataFrame.from_pandas(pdf)
    got = gdf.groupby("k2", sort=True)["v2"].mean().to_pandas()
    exp = pdf.groupby("k2", sort=True)[["v2"]].mean()
    _compare(got, exp)
    flat = gdf.groupby("k2", sort=True, as_index=False).agg({"v1": "max"}).to_pandas()
    assert list(flat.columns) == ["k2", "v1"]
    e = pdf.groupby("k2", sort=True, as_index=False).agg({"v1": "max"})
    assert np.array_equal(flat["k2"].to_numpy(), e["k2"].to_numpy())
    assert np.array_equal(_as_float(flat["v1"]), _as_float(e["v1"]))


def test_var_std_prod_and_unsorted_order():
    import cudf_b200 as cb
    rng = np.random.default_rng(5)
    pdf = pd.DataFrame({"k": rng.integers(0, 50, 20_000), "x": rng.normal(size=20_000),
                        "p": rng.choice([1.0, 1.0001, 0.9999], 20_000)})
    gdf = cb.DataFrame.from_pandas(pdf)
    got = gdf.groupby("k").agg({"x": ["var", "std"], "p": "prod"}).to_pandas()  # sort=False default
    exp = pdf.groupby("k").agg({"x": ["var", "std"], "p": "prod"})
    _compare(got, exp, rtol=1e-8)


def test_arrow_table_groupby():
    import pyarrow as pa
    import cudf_b200 as cb
    t = pa.table({"k": pa.array([1, 2, 1, None, 2, 1], pa.int64()),
                  "v": pa.array([1.0, 2.0, None, 4.0, 5.0, 6.0])})
    out = cb.DataFrame.from_arrow(t).groupby("k", sort=True, dropna=False).agg(["sum", "count"]).to_arrow()
    assert out.column("k").to_pylist() == [1, 2, None]
    assert out.column(1).to_pylist() == [7.0, 7.0, 4.0]
    assert out.column(2).to_pylist() == [2, 2, 1]


def test_host_staging_round_trips_and_reuses_buffers():
    """HostStaging copies device results into reused pinned buffers; each call's
    arrays hold that call's data."""
    import torch
    import cudf_b200 as cb
    st = cb.HostStaging()
    for seed in (1, 2):
        g = torch.Generator(device="cuda")
        g.manual_seed(seed)
        ts = [torch.randint(-2**40, 2**40, (1000,), device="cuda", generator=g, dtype=torch.int64),
              torch.rand(777, device="cuda", generator=g, dtype=torch.float32),
              torch.rand(33, device="cuda", generator=g) > 0.5,
              torch.empty(0, device="cuda", dtype=torch.float64)]
        out = st.to_host(ts)
        for t, h in zip(ts, out):
            assert h.dtype == t.cpu().numpy().dtype and np.array_equal(h, t.cpu().numpy())
