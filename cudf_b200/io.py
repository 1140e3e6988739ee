"""Parquet input for the engine: the role of cudf's ``read_parquet``
(cpp/src/io/parquet, python/cudf/cudf/io/parquet.py) for the fixed-width
columns the hash groupby takes.

Pages are decoded on the host by Arrow's Parquet reader (multi-threaded C++,
outside the GIL); what this module adds is moving the decoded columns onto
the device and feeding them to the engine:

* ``read_parquet(path, columns)`` -> a device ``DataFrame``;
* ``scan_parquet(path, columns, batch_rows)`` -> device ``DataFrame`` batches:
  a background thread decodes batch i+1 into pinned host buffers while batch
  i is copied to the device on a copy stream and used, so decode, upload and
  aggregation overlap;
* ``groupby_parquet(path, by, aggs)`` -> the groupby of a whole file in
  bounded device memory: each batch is aggregated into partial results (the
  decomposition of the multi-GPU path: MEAN as SUM + COUNT), the partials are
  merged by a second engine call whenever they grow past a bound, and
  finalised at the end.  Files larger than HBM stream through.

Validity bitmaps keep Arrow's bit order (the same as libcudf's); NaN stays a
value (Parquet's nulls are its nulls).
"""
from __future__ import annotations

import queue
import threading
from typing import Dict, Iterator, List, Optional, Sequence, Tuple, Union

import numpy as np
import torch

from .column import Column, pack_mask
from .distributed import engine_local_aggregate, finalize_partials, merge_partials, plan_partials
from .frame import DataFrame
from .interop import arrow_type_id, host_arrays
from .types import Kind, NullPolicy, TypeId

_AGG_KINDS = {"sum": [Kind.SUM], "min": [Kind.MIN], "max": [Kind.MAX], "mean": [Kind.MEAN],
              "count": [Kind.COUNT_VALID], "size": [Kind.COUNT_ALL], "prod": [Kind.PRODUCT],
              "product": [Kind.PRODUCT]}


def parquet_schema(path: str, columns: Optional[Sequence[str]] = None) -> Dict[str, TypeId]:
    """Engine type of every (selected) column; NotImplementedError for a
    column that is not fixed-width."""
    import pyarrow.parquet as pq
    schema = pq.read_schema(path)
    names = list(columns) if columns is not None else schema.names
    return {n: arrow_type_id(schema.field(n).type) for n in names}


def read_parquet(path: str, columns: Optional[Sequence[str]] = None,
                 row_groups: Optional[Sequence[int]] = None, device="cuda") -> DataFrame:
    """Reads a Parquet file (or the given row groups) into a device DataFrame."""
    import pyarrow.parquet as pq
    parquet_schema(path, columns)  # rejects unsupported columns before decoding
    f = pq.ParquetFile(path)
    t = f.read_row_groups(list(row_groups), columns=columns) if row_groups is not None else f.read(columns=columns)
    return DataFrame.from_arrow(t, device)


class _HostBatch:
    """A decoded batch in host memory (pinned when it goes to a GPU): per
    column values, packed validity words (or None) and the engine type."""

    def __init__(self, record_batch, pin: bool):
        self.names = record_batch.schema.names
        self.rows = record_batch.num_rows
        self.cols = []
        for name in self.names:
            vals, valid, tid = host_arrays(record_batch.column(name))
            v = torch.from_numpy(np.ascontiguousarray(vals))
            m = None if valid is None else pack_mask(torch.from_numpy(valid))
            if pin:
                v = v.pin_memory()
                m = None if m is None else m.pin_memory()
            self.cols.append((v, m, tid))


def scan_parquet(path: str, columns: Optional[Sequence[str]] = None, batch_rows: int = 1 << 24,
                 prefetch: int = 2, device="cuda") -> Iterator[DataFrame]:
    """Device DataFrames of about `batch_rows` rows each, in file order.  A
    background thread decodes ahead (up to `prefetch` batches) into pinned
    buffers; each batch's upload runs on a copy stream that the consumer's
    stream waits on."""
    import pyarrow.parquet as pq
    parquet_schema(path, columns)
    f = pq.ParquetFile(path)
    q: "queue.Queue" = queue.Queue(maxsize=max(1, prefetch))
    stop = threading.Event()
    on_gpu = torch.device(device).type == "cuda"

    def producer():
        try:
            for rb in f.iter_batches(batch_size=batch_rows, columns=columns):
                if stop.is_set():
                    break
                q.put(_HostBatch(rb, on_gpu))
            q.put(None)
        except BaseException as e:  # handed to the consumer
            q.put(e)

    th = threading.Thread(target=producer, daemon=True)
    th.start()
    copy = torch.cuda.Stream(device=device) if on_gpu else None
    try:
        while True:
            hb = q.get()
            if hb is None:
                break
            if isinstance(hb, BaseException):
                raise hb
            if not on_gpu:
                yield DataFrame({name: Column(tid, v, m) for name, (v, m, tid) in zip(hb.names, hb.cols)})
                continue
            with torch.cuda.stream(copy):
                cols = {}
                for name, (v, m, tid) in zip(hb.names, hb.cols):
                    dv = v.to(device, non_blocking=True)
                    dm = None if m is None else m.to(device, non_blocking=True)
                    cols[name] = Column(tid, dv, dm)
            ev = torch.cuda.Event()
            ev.record(copy)
            torch.cuda.current_stream(device).wait_event(ev)
            # the pinned buffers stay alive until the copy has run
            hb_keep = hb
            yield DataFrame(cols)
            ev.synchronize()
            del hb_keep
    finally:
        stop.set()
        while th.is_alive():
            try:
                q.get(timeout=0.1)
            except queue.Empty:
                pass
        th.join()


def _spec(aggs: Dict[str, Union[str, Sequence[str]]]) -> List[Tuple[str, List[str]]]:
    out = []
    for col, names in aggs.items():
        names = [names] if isinstance(names, str) else list(names)
        for n in names:
            if n not in _AGG_KINDS:
                raise NotImplementedError(f"aggregation {n!r} is not supported by the streaming groupby")
        out.append((col, names))
    return out


def groupby_parquet(path: str, by: Union[str, Sequence[str]], aggs: Dict[str, Union[str, Sequence[str]]],
                    dropna: bool = True, batch_rows: int = 1 << 24, merge_rows: int = 1 << 25,
                    device="cuda", local=None) -> DataFrame:
    """The groupby of a whole Parquet file, streamed in batches.

    by: key column name(s); aggs: value column -> aggregation name(s) among
    sum, min, max, mean, count, size, prod.  Returns a DataFrame indexed by
    the keys (groups in arbitrary order) with (column, aggregation) labels.
    Partial results are merged by a second groupby whenever they exceed
    `merge_rows` rows, so device memory stays bounded by about one batch plus
    the partials of the distinct groups."""
    by = [by] if isinstance(by, str) else list(by)
    spec = _spec(aggs)
    local = local or engine_local_aggregate
    policy = NullPolicy.EXCLUDE if dropna else NullPolicy.INCLUDE
    columns = list(dict.fromkeys(by + [c for c, _ in spec]))
    schema = parquet_schema(path, columns)
    # requests as the distributed helpers take them: ((data, valid, tid), kinds)
    kinds = [[k for n in names for k in _AGG_KINDS[n]] for _, names in spec]
    proto = [((None, None, schema[c]), ks) for (c, _), ks in zip(spec, kinds)]
    preq = plan_partials(proto)
    acc_keys, acc_vals, acc_rows = None, None, 0

    def concat(a, b):
        return b if a is None else torch.cat([a, b])

    def concat_valid(a, b, na, nb):
        if a is None and b is None:
            return None
        a = torch.ones(na, dtype=torch.bool, device=device) if a is None else a
        b = torch.ones(nb, dtype=torch.bool, device=device) if b is None else b
        return torch.cat([a, b])

    def fold(pkeys, pvals):
        """Adds partial groups to the accumulated ones."""
        nonlocal acc_keys, acc_vals, acc_rows
        n = pkeys[0][0].shape[0]
        if acc_keys is None:
            acc_keys, acc_vals, acc_rows = pkeys, pvals, n
            return
        acc_keys = [(concat(a[0], b[0]), concat_valid(a[1], b[1], acc_rows, n), a[2])
                    for a, b in zip(acc_keys, pkeys)]
        acc_vals = {k: (concat(acc_vals[k][0], pvals[k][0]), concat_valid(acc_vals[k][1], pvals[k][1], acc_rows, n))
                    for k in acc_vals}
        acc_rows += n

    def compact():
        """Merges the accumulated partials (duplicate keys) into one row per group."""
        nonlocal acc_keys, acc_vals, acc_rows
        mk, merged = merge_partials(preq, acc_keys, acc_vals, policy, local)
        acc_keys = mk
        acc_vals = {(r, j): merged[r][p] for r, (_, plist) in enumerate(preq) for j, p in enumerate(plist)}
        acc_rows = mk[0][0].shape[0] if mk else 0

    for df in scan_parquet(path, columns, batch_rows, device=device):
        keys = [(df[c].values(), df[c].valid(), int(df[c].type_id)) for c in by]
        reqs = [((df[c].values(), df[c].valid(), int(df[c].type_id)), plist) for (c, _), (_, plist) in zip(spec, preq)]
        pk, pres = local(keys, reqs, policy)
        fold(pk, {(r, j): pres[r][j] for r in range(len(preq)) for j in range(len(preq[r][1]))})
        if acc_rows > merge_rows:
            compact()
    if acc_keys is None:
        raise ValueError("the file has no rows")
    mk, merged = merge_partials(preq, acc_keys, acc_vals, policy, local)
    results = finalize_partials(proto, merged)
    index = [(name, Column.from_tensor(d, v, t)) for name, (d, v, t) in zip(by, mk)]
    data = {}
    for (col, names), res in zip(spec, results):
        for n, (d, v) in zip(names, res):
            tid = _result_type(schema[col], n)
            data[(col, n)] = Column.from_tensor(d.contiguous(), v, tid)
    return DataFrame(data, index=index, multilevel=True)


_DURATIONS = (TypeId.DURATION_DAYS, TypeId.DURATION_SECONDS, TypeId.DURATION_MILLISECONDS,
              TypeId.DURATION_MICROSECONDS, TypeId.DURATION_NANOSECONDS)


def _result_type(tid: TypeId, name: str) -> int:
    """Result type of an aggregation by name (libcudf's target types)."""
    if name in ("count", "size"):
        return TypeId.INT32
    if name in ("min", "max"):
        return tid
    if name == "mean":
        return tid if tid in _DURATIONS else TypeId.FLOAT64
    if tid in (TypeId.FLOAT32, TypeId.FLOAT64) or tid in _DURATIONS:
        return tid
    return TypeId.INT64
