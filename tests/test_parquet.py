"""Parquet input: a file written by Arrow, read back in batches and grouped in
a streaming fashion (partials per batch, merged when they grow, finalised at
the end).  On CPU the local aggregation is the oracle; on the GPU it is the
engine.  Either way the result must equal the groupby of the whole table."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from parity import compare

KINDS = [O.SUM, O.MIN, O.MAX, O.MEAN, O.COUNT_VALID, O.COUNT_ALL]
NAMES = ["sum", "min", "max", "mean", "count", "size"]


def _write(path, n, seed, row_group):
    import pyarrow as pa
    import pyarrow.parquet as pq
    rng = np.random.default_rng(seed)
    k1 = rng.integers(0, 700, n).astype(np.int64)
    k2 = rng.integers(0, 4, n).astype(np.int32)
    k2v = rng.random(n) > 0.05
    v1 = rng.integers(-10**9, 10**9, n).astype(np.int64)
    v1v = rng.random(n) > 0.1
    v2 = rng.normal(size=n)
    v2v = rng.random(n) > 0.2
    t = pa.table({"k1": pa.array(k1), "k2": pa.array(k2, mask=~k2v), "v1": pa.array(v1, mask=~v1v),
                  "v2": pa.array(v2, mask=~v2v), "junk": pa.array(rng.random(n))})
    pq.write_table(t, path, row_group_size=row_group)
    return k1, k2, k2v, v1, v1v, v2, v2v


def _check(df, cols, dropna):
    k1, k2, k2v, v1, v1v, v2, v2v = cols
    o = O.groupby([O.HostColumn(O.INT64, k1), O.HostColumn(O.INT32, k2, k2v)],
                  [(O.HostColumn(O.INT64, v1, v1v), KINDS), (O.HostColumn(O.FLOAT64, v2, v2v), KINDS)],
                  include_null_keys=not dropna)
    keys = [c.to_numpy() for _, c in df.index]
    res = [[df[(c, nm)].to_numpy() for nm in NAMES] for c in ("v1", "v2")]
    compare(o, keys, res, [KINDS, KINDS], None)


@pytest.mark.parametrize("dropna", [True, False])
def test_streaming_groupby_matches_whole_table_cpu(tmp_path, dropna):
    from cudf_b200.io import groupby_parquet
    from test_distributed_gloo import oracle_local_aggregate
    path = str(tmp_path / "t.parquet")
    cols = _write(path, 60_000, 3, 7_000)
    df = groupby_parquet(path, ["k1", "k2"], {"v1": NAMES, "v2": NAMES}, dropna=dropna,
                         batch_rows=9_000, merge_rows=5_000, device="cpu", local=oracle_local_aggregate)
    _check(df, cols, dropna)


def test_unsupported_column_is_rejected(tmp_path):
    import pyarrow as pa
    import pyarrow.parquet as pq
    from cudf_b200.io import parquet_schema
    path = str(tmp_path / "s.parquet")
    pq.write_table(pa.table({"s": pa.array(["a", "b"]), "x": pa.array([1, 2])}), path)
    assert int(parquet_schema(path, ["x"])["x"]) == O.INT64
    with pytest.raises(NotImplementedError):
        parquet_schema(path)


@pytest.mark.gpu
@pytest.mark.parametrize("dropna", [True, False])
def test_streaming_groupby_on_the_engine(tmp_path, dropna):
    from cudf_b200.io import groupby_parquet, read_parquet
    path = str(tmp_path / "g.parquet")
    cols = _write(path, 1_500_000, 4, 200_000)
    df = groupby_parquet(path, ["k1", "k2"], {"v1": NAMES, "v2": NAMES}, dropna=dropna,
                         batch_rows=250_000, merge_rows=4_000)
    _check(df, cols, dropna)
    whole = read_parquet(path, columns=["k1", "v2"])
    d, v = whole["v2"].to_numpy()
    assert np.array_equal(v, cols[6]) and np.array_equal(d[v], cols[5][cols[6]])
