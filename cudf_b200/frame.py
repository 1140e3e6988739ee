"""DataFrame-level groupby on the engine: the role of cudf's
``DataFrame.groupby(by, sort=, dropna=, as_index=).agg(func)``
(python/cudf/cudf/core/groupby/groupby.py:518-702) for the hash-groupby
aggregations.

A ``DataFrame`` is an ordered mapping of names to device ``Column``s (plus an
optional index of key columns, which is what a groupby result carries).
``agg`` accepts what cudf accepts for these aggregations -- a name, a list of
names, or a dict of column -> name(s) -- runs one engine call with one request
per value column, and assembles the result the way cudf does:

* COUNT, SIZE, IDXMIN and IDXMAX results are int64 (groupby.py:651-652);
* a list, or a dict with any list value, gives (column, aggregation) labels,
  otherwise plain column labels (``_is_multi_agg``);
* ``sort=True`` orders the groups by key, nulls last (``result.sort_index()``,
  groupby.py:671-672); ``sort=False`` leaves the engine's order;
* ``dropna`` maps to the key null policy (True: EXCLUDE, False: INCLUDE);
* ``as_index=False`` turns the key index into leading columns.

``from_pandas`` turns NaN in float columns into nulls, as cudf's
``nan_as_null`` default does, so pandas' NaN-as-missing semantics carry over.
"""
from __future__ import annotations

from collections.abc import Mapping
from typing import Dict, List, Optional, Sequence, Tuple, Union

import numpy as np
import torch

from . import aggregation as _agg
from .column import Column, Table, pack_mask, unpack_mask
from .groupby import GroupBy, GroupByRequest
from .types import Kind, NullPolicy, TypeId

# pandas/cudf aggregation names -> engine aggregation factory
_AGG_NAMES = {
    "sum": _agg.sum,
    "min": _agg.min,
    "max": _agg.max,
    "mean": _agg.mean,
    "count": lambda: _agg.count(NullPolicy.EXCLUDE),
    "size": lambda: _agg.count(NullPolicy.INCLUDE),
    "prod": _agg.product,
    "product": _agg.product,
    "var": lambda: _agg.variance(1),
    "std": lambda: _agg.std(1),
    "idxmin": _agg.argmin,
    "idxmax": _agg.argmax,
}
_INT64_RESULTS = {Kind.COUNT_VALID, Kind.COUNT_ALL, Kind.ARGMIN, Kind.ARGMAX}

_NUMPY_TO_TYPE = {
    np.dtype(np.int8): TypeId.INT8, np.dtype(np.int16): TypeId.INT16, np.dtype(np.int32): TypeId.INT32,
    np.dtype(np.int64): TypeId.INT64, np.dtype(np.uint8): TypeId.UINT8, np.dtype(np.uint16): TypeId.UINT16,
    np.dtype(np.uint32): TypeId.UINT32, np.dtype(np.uint64): TypeId.UINT64,
    np.dtype(np.float32): TypeId.FLOAT32, np.dtype(np.float64): TypeId.FLOAT64, np.dtype(np.bool_): TypeId.BOOL8,
}
_TIME_UNITS = {"s": 0, "ms": 1, "us": 2, "ns": 3}
_TS_TYPES = [TypeId.TIMESTAMP_SECONDS, TypeId.TIMESTAMP_MILLISECONDS, TypeId.TIMESTAMP_MICROSECONDS,
             TypeId.TIMESTAMP_NANOSECONDS]
_DUR_TYPES = [TypeId.DURATION_SECONDS, TypeId.DURATION_MILLISECONDS, TypeId.DURATION_MICROSECONDS,
              TypeId.DURATION_NANOSECONDS]
_UNIT_OF = {t: u for u, i in _TIME_UNITS.items() for t in (_TS_TYPES[i], _DUR_TYPES[i])}


def _is_list_like(x) -> bool:
    return isinstance(x, (list, tuple))


def is_multi_agg(func) -> bool:
    """cudf's ``_is_multi_agg``: does ``func`` produce (column, agg) labels?"""
    if isinstance(func, Mapping):
        return any(_is_list_like(v) for v in func.values())
    return _is_list_like(func)


def normalize_aggs(func, value_names: Sequence[str]) -> List[Tuple[str, List[str]]]:
    """(column, [aggregation names]) in output order, as cudf's
    ``_normalize_aggs`` orders them: dict order for a dict, else every value
    column with the same list."""
    if isinstance(func, Mapping):
        out = []
        for col, f in func.items():
            names = list(f) if _is_list_like(f) else [f]
            out.append((col, [_agg_name(n) for n in names]))
        return out
    names = list(func) if _is_list_like(func) else [func]
    names = [_agg_name(n) for n in names]
    return [(c, list(names)) for c in value_names]


def _agg_name(n) -> str:
    if callable(n) and not isinstance(n, str):
        n = getattr(n, "__name__", repr(n))
    if n not in _AGG_NAMES:
        raise NotImplementedError(f"aggregation {n!r} is not on the hash groupby path")
    return n


def _gather_column(col: Column, order: torch.Tensor) -> Column:
    data = col.values().index_select(0, order)
    valid = col.valid()
    mask = None if valid is None else pack_mask(valid.index_select(0, order))
    return Column(col.type_id, data, mask)


def _sort_key(col: Column) -> torch.Tensor:
    """Values of a key column in an order-preserving signed/float torch dtype."""
    v = col.values()
    if v.dtype == torch.bool:
        return v.to(torch.int8)
    if v.dtype in (torch.uint16, torch.uint32):
        return v.to(torch.int64)
    if v.dtype == torch.uint64:
        return v.view(torch.int64) ^ torch.iinfo(torch.int64).min
    return v


def key_order(keys: Sequence[Column]) -> torch.Tensor:
    """Permutation sorting rows by the key columns (first column major),
    ascending, nulls after all values: a stable sort per column from the last
    to the first."""
    n = keys[0].size if keys else 0
    dev = keys[0].data.device if keys else torch.device("cpu")
    order = torch.arange(n, device=dev)
    for col in reversed(list(keys)):
        k = _sort_key(col).index_select(0, order)
        o = torch.argsort(k, stable=True)
        order = order.index_select(0, o)
        valid = col.valid()
        if valid is not None:
            nulls = (~valid.index_select(0, order)).to(torch.int8)
            order = order.index_select(0, torch.argsort(nulls, stable=True))
    return order


class DataFrame:
    """An ordered set of named device columns, with an optional index of
    named key columns."""

    def __init__(self, data: Optional[Mapping[str, Column]] = None,
                 index: Optional[Sequence[Tuple[str, Column]]] = None, multilevel: bool = False):
        self._data: Dict[object, Column] = dict(data or {})
        self.index: List[Tuple[str, Column]] = list(index or [])
        self.multilevel = multilevel
        sizes = {c.size for c in self._data.values()} | {c.size for _, c in self.index}
        if len(sizes) > 1:
            raise ValueError("columns have different lengths")

    # -- construction ---------------------------------------------------
    @staticmethod
    def from_pandas(df, device="cuda", nan_as_null: bool = True) -> "DataFrame":
        import pandas as pd
        cols = {}
        for name in df.columns:
            cols[name] = _column_from_pandas(df[name], device, nan_as_null)
        out = DataFrame(cols)
        if not isinstance(df.index, pd.RangeIndex) or df.index.start != 0 or df.index.step != 1:
            names = list(df.index.names)
            out.index = [(nm, _column_from_pandas(pd.Series(df.index.get_level_values(i)), device, nan_as_null))
                         for i, nm in enumerate(names)]
        return out

    @staticmethod
    def from_arrow(table, device="cuda") -> "DataFrame":
        from .interop import column_from_arrow
        return DataFrame({name: column_from_arrow(table.column(name), device) for name in table.column_names})

    # -- access ---------------------------------------------------------
    @property
    def columns(self) -> list:
        return list(self._data.keys())

    def __getitem__(self, name) -> Column:
        return self._data[name]

    def __len__(self) -> int:
        for c in self._data.values():
            return c.size
        for _, c in self.index:
            return c.size
        return 0

    def groupby(self, by, sort: bool = False, dropna: bool = True, as_index: bool = True) -> "DataFrameGroupBy":
        by = [by] if not _is_list_like(by) else list(by)
        return DataFrameGroupBy(self, by, sort=sort, dropna=dropna, as_index=as_index)

    # -- export ---------------------------------------------------------
    def to_pandas(self, nullable: bool = True):
        import pandas as pd
        data = {name: _column_to_pandas(c, nullable) for name, c in self._data.items()}
        index = None
        if self.index:
            if len(self.index) == 1:
                nm, c = self.index[0]
                index = pd.Index(_column_to_pandas(c, nullable), name=nm)
            else:
                arrays = [pd.Index(_column_to_pandas(c, nullable)) for _, c in self.index]
                index = pd.MultiIndex.from_arrays(arrays, names=[nm for nm, _ in self.index])
        cols = list(data.keys())
        if self.multilevel:
            cols = pd.MultiIndex.from_tuples(cols)
        df = pd.DataFrame({i: v for i, v in enumerate(data.values())}, index=index)
        df.columns = cols
        return df

    def to_arrow(self):
        import pyarrow as pa
        from .interop import column_to_arrow
        names = [str(nm) for nm, _ in self.index] + ["_".join(map(str, n)) if isinstance(n, tuple) else str(n)
                                                      for n in self._data.keys()]
        arrays = [column_to_arrow(c) for _, c in self.index] + [column_to_arrow(c) for c in self._data.values()]
        return pa.table(arrays, names=names)

    def __repr__(self):
        return f"DataFrame({len(self)} rows, columns={self.columns}, index={[n for n, _ in self.index]})"


class DataFrameGroupBy:
    """``df.groupby(by, ...)``: aggregations over the groups of the key columns."""

    def __init__(self, frame: DataFrame, by: List[str], sort: bool, dropna: bool, as_index: bool,
                 selection: Optional[List[str]] = None, series: bool = False):
        for b in by:
            if b not in frame._data:
                raise KeyError(b)
        self.frame = frame
        self.by = by
        self.sort = sort
        self.dropna = dropna
        self.as_index = as_index
        self.selection = selection
        self.series = series

    def __getitem__(self, key) -> "DataFrameGroupBy":
        sel = list(key) if _is_list_like(key) else [key]
        return DataFrameGroupBy(self.frame, self.by, self.sort, self.dropna, self.as_index, sel,
                                series=not _is_list_like(key))

    def _value_names(self) -> List[str]:
        if self.selection is not None:
            return list(self.selection)
        return [c for c in self.frame.columns if c not in self.by]

    def agg(self, func) -> DataFrame:
        spec = normalize_aggs(func, self._value_names())
        multilevel = is_multi_agg(func)
        keys = [self.frame[b] for b in self.by]
        gb = GroupBy(Table(keys), NullPolicy.EXCLUDE if self.dropna else NullPolicy.INCLUDE)
        reqs = [GroupByRequest(self.frame[col], [_AGG_NAMES[n]() for n in names]) for col, names in spec]
        uniq, results = gb.aggregate(reqs)
        key_cols = list(uniq.columns)
        out: Dict[object, Column] = {}
        for (col, names), res in zip(spec, results):
            for name, c, req in zip(names, res.columns, _AGG_NAMES_kinds(names)):
                if req in _INT64_RESULTS and c.type_id != TypeId.INT64:
                    v = c.values().to(torch.int64)
                    c = Column(TypeId.INT64, v, None if c.mask is None else pack_mask(c.valid()))
                out[(col, name) if multilevel else col] = c
        if self.sort and key_cols and key_cols[0].size > 1:
            order = key_order(key_cols)
            key_cols = [_gather_column(c, order) for c in key_cols]
            out = {k: _gather_column(c, order) for k, c in out.items()}
        index = list(zip(self.by, key_cols))
        if not self.as_index:
            lead = {(b, "") if multilevel else b: c for b, c in index}
            lead.update(out)
            return DataFrame(lead, multilevel=multilevel)
        res = DataFrame(out, index=index, multilevel=multilevel)
        res.series = self.series
        return res

    aggregate = agg

    def sum(self):
        return self.agg("sum")

    def min(self):
        return self.agg("min")

    def max(self):
        return self.agg("max")

    def mean(self):
        return self.agg("mean")

    def count(self):
        return self.agg("count")

    def size(self):
        """Rows per group (nulls included), as int64."""
        name = self.by[0]
        g = DataFrameGroupBy(self.frame, self.by, self.sort, self.dropna, self.as_index, [name], series=True)
        return g.agg({name: "size"})

    def prod(self):
        return self.agg("prod")

    def var(self):
        return self.agg("var")

    def std(self):
        return self.agg("std")


def _AGG_NAMES_kinds(names: Sequence[str]) -> List[Kind]:
    return [_AGG_NAMES[n]().kind for n in names]


# -- pandas conversion ------------------------------------------------------
def _column_from_pandas(s, device, nan_as_null: bool) -> Column:
    import pandas as pd
    dt = s.dtype
    valid = None
    if isinstance(dt, pd.api.extensions.ExtensionDtype) and not isinstance(dt, pd.DatetimeTZDtype):
        na = s.isna().to_numpy()
        if dt == "boolean":
            arr = s.fillna(False).to_numpy(dtype=np.bool_)
        else:
            arr = s.to_numpy(dtype=dt.numpy_dtype, na_value=0)
        valid = ~na if na.any() else None
    else:
        arr = s.to_numpy()
    if arr.dtype.kind == "M" or arr.dtype.kind == "m":
        unit = np.datetime_data(arr.dtype)[0]
        if unit not in _TIME_UNITS:
            raise NotImplementedError(f"time unit {unit!r}")
        tid = (_TS_TYPES if arr.dtype.kind == "M" else _DUR_TYPES)[_TIME_UNITS[unit]]
        nat = np.isnat(arr)
        if nat.any():
            valid = ~nat if valid is None else valid & ~nat
        return Column.from_numpy(arr.view(np.int64), valid, tid, device)
    if arr.dtype.kind == "f" and nan_as_null:
        nan = np.isnan(arr)
        if nan.any():
            valid = ~nan if valid is None else valid & ~nan
    if arr.dtype not in _NUMPY_TO_TYPE:
        raise NotImplementedError(f"dtype {arr.dtype} is not a fixed-width groupby type")
    return Column.from_numpy(arr, valid, _NUMPY_TO_TYPE[arr.dtype], device)


def _column_to_pandas(c: Column, nullable: bool):
    import pandas as pd
    vals, valid = c.to_numpy()
    t = c.type_id
    if t in _UNIT_OF:
        kind = "M" if t in _TS_TYPES else "m"
        arr = vals.astype(np.int64).view(f"{'datetime64' if kind == 'M' else 'timedelta64'}[{_UNIT_OF[t]}]").copy()
        if valid is not None:
            arr[~valid] = np.datetime64("NaT") if kind == "M" else np.timedelta64("NaT")
        return pd.array(arr)
    if t == TypeId.TIMESTAMP_DAYS:
        arr = vals.astype("datetime64[D]").astype("datetime64[s]")
        if valid is not None:
            arr[~valid] = np.datetime64("NaT")
        return pd.array(arr)
    if t == TypeId.BOOL8:
        vals = vals.astype(bool)
        if valid is None:
            return vals
        return pd.Series(pd.array(vals, dtype="boolean")).where(valid).array
    if valid is None:
        return vals
    if not nullable:
        out = vals.astype(np.float64)
        out[~valid] = np.nan
        return out
    arr = pd.array(vals)
    return pd.Series(arr).where(valid).array
