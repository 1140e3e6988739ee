"""Host-side logic of the DataFrame binding and Arrow interop (no GPU):
aggregation-spec normalisation and labels as cudf's groupby.agg produces
them (python/cudf/cudf/core/groupby/groupby.py:518-702), key ordering for
sort=True, and pandas/Arrow round trips of device-layout columns."""
import numpy as np
import pandas as pd
import pyarrow as pa
import pytest
import torch

from cudf_b200 import frame as F
from cudf_b200 import interop as I
from cudf_b200.column import Column
from cudf_b200.types import TypeId


def test_is_multi_agg_matches_cudf_rules():
    assert not F.is_multi_agg("sum")
    assert F.is_multi_agg(["sum"])
    assert not F.is_multi_agg({"a": "sum", "b": "min"})
    assert F.is_multi_agg({"a": "sum", "b": ["min"]})


def test_normalize_aggs_orders_like_cudf():
    assert F.normalize_aggs("sum", ["b", "c"]) == [("b", ["sum"]), ("c", ["sum"])]
    assert F.normalize_aggs(["sum", "min"], ["b"]) == [("b", ["sum", "min"])]
    assert F.normalize_aggs({"c": "max", "b": ["min", "mean"]}, ["b", "c"]) == [("c", ["max"]), ("b", ["min", "mean"])]
    with pytest.raises(NotImplementedError):
        F.normalize_aggs("median", ["b"])


def test_key_order_sorts_lexicographically_with_nulls_last():
    k1 = Column.from_numpy(np.array([2, 1, 2, 1, 3], np.int32), np.array([1, 1, 1, 1, 0], bool), device="cpu")
    k2 = Column.from_numpy(np.array([5, 9, 4, 9, 0], np.int64), np.array([1, 0, 1, 1, 1], bool), device="cpu")
    order = F.key_order([k1, k2]).tolist()
    # (1, 9), (1, null), (2, 4), (2, 5), (null, 0)
    assert order == [3, 1, 2, 0, 4]


def test_key_order_unsigned_and_float():
    u = Column.from_numpy(np.array([2**63 + 5, 1, 2**64 - 1, 0], np.uint64), device="cpu")
    assert F.key_order([u]).tolist() == [3, 1, 0, 2]
    f = Column.from_numpy(np.array([0.5, -1.0, 3.0], np.float64), device="cpu")
    assert F.key_order([f]).tolist() == [1, 0, 2]


def test_from_pandas_to_pandas_round_trip_cpu():
    df = pd.DataFrame({
        "i": pd.array([1, None, 3], dtype="Int64"),
        "f": [1.5, np.nan, -2.0],
        "u": np.array([1, 2, 3], np.uint16),
        "t": pd.to_datetime(["2020-01-01", None, "2021-06-01"]).as_unit("ms"),
        "d": pd.to_timedelta([1, 2, None], unit="s").as_unit("s"),
        "b": pd.array([True, None, False], dtype="boolean"),
    })
    g = F.DataFrame.from_pandas(df, device="cpu")
    assert g["f"].type_id == TypeId.FLOAT64 and g["f"].null_count == 1  # NaN -> null
    assert g["t"].type_id == TypeId.TIMESTAMP_MILLISECONDS and g["t"].null_count == 1
    assert g["d"].type_id == TypeId.DURATION_SECONDS
    out = g.to_pandas()
    assert out["i"].isna().tolist() == [False, True, False] and out["i"].iloc[2] == 3
    assert out["f"].isna().tolist() == [False, True, False]
    assert (out["u"].to_numpy() == np.array([1, 2, 3])).all()
    assert out["t"].isna().tolist() == [False, True, False]
    assert out["t"].iloc[2] == pd.Timestamp("2021-06-01")
    assert out["d"].iloc[1] == pd.Timedelta(seconds=2)
    assert out["b"].isna().tolist() == [False, True, False] and bool(out["b"].iloc[0])


def test_arrow_validity_words_with_offset():
    arr = pa.array([1, None, 3, None, 5, 6, None] * 7, type=pa.int32()).slice(3, 40)
    vals, valid, tid = I.host_arrays(arr)
    assert tid == TypeId.INT32
    exp_valid = np.array([x is not None for x in arr.to_pylist()])
    assert np.array_equal(valid, exp_valid)
    assert np.array_equal(vals[valid], np.array([x for x in arr.to_pylist() if x is not None]))
    words = I.validity_words(arr.buffers()[0], arr.offset, len(arr))
    bits = np.unpackbits(words.view(np.uint8), bitorder="little")[:len(arr)].astype(bool)
    assert np.array_equal(bits, exp_valid)


@pytest.mark.parametrize("typ", [pa.int8(), pa.uint64(), pa.float32(), pa.bool_(), pa.date32(),
                                 pa.timestamp("us"), pa.duration("ns")])
def test_arrow_column_round_trip_cpu(typ):
    rng = np.random.default_rng(3)
    n = 100
    if typ == pa.bool_():
        py = [bool(x) if rng.random() > 0.2 else None for x in rng.integers(0, 2, n)]
    elif typ == pa.float32():
        py = [float(x) if rng.random() > 0.2 else None for x in rng.normal(size=n)]
    else:
        py = [int(x) if rng.random() > 0.2 else None for x in rng.integers(0, 100, n)]
    arr = pa.array(py, type=pa.int32() if typ == pa.date32() else None)
    arr = arr.cast(typ) if arr.type != typ else arr
    col = I.column_from_arrow(pa.chunked_array([arr.slice(0, 37), arr.slice(37)]), device="cpu")
    back = I.column_to_arrow(col)
    assert back.type == typ
    assert back.to_pylist() == arr.to_pylist()


def test_dataframe_from_arrow_cpu():
    t = pa.table({"k": pa.array([1, 2, None], pa.int64()), "v": pa.array([0.5, None, 2.0])})
    df = F.DataFrame.from_arrow(t, device="cpu")
    assert df.columns == ["k", "v"]
    assert df["k"].null_count == 1 and df["v"].null_count == 1
    assert df.to_arrow().to_pylist() == t.to_pylist()
