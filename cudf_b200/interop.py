"""Arrow interop for the engine's columns: the role of cudf's from_arrow /
to_arrow (cpp/src/interop/from_arrow.cu, to_arrow.cu) for the fixed-width
types the hash groupby takes.

Arrow and libcudf share the validity bit order (bit i of the bitmap, LSB
first, is row i), so a validity bitmap only needs its row offset applied and
its bytes widened to the engine's 32-bit words.  Arrow booleans are
bit-packed and become BOOL8 bytes; date32 becomes TIMESTAMP_DAYS, timestamps
and durations keep their unit.  Chunked arrays are concatenated."""
from __future__ import annotations

import numpy as np
import torch

from .column import Column
from .types import NUMPY_DTYPE, TypeId

_UNITS = ["s", "ms", "us", "ns"]
_TS = [TypeId.TIMESTAMP_SECONDS, TypeId.TIMESTAMP_MILLISECONDS, TypeId.TIMESTAMP_MICROSECONDS,
       TypeId.TIMESTAMP_NANOSECONDS]
_DUR = [TypeId.DURATION_SECONDS, TypeId.DURATION_MILLISECONDS, TypeId.DURATION_MICROSECONDS,
        TypeId.DURATION_NANOSECONDS]


def arrow_type_id(t) -> TypeId:
    """libcudf type id of an Arrow fixed-width type."""
    import pyarrow as pa
    simple = {pa.int8(): TypeId.INT8, pa.int16(): TypeId.INT16, pa.int32(): TypeId.INT32,
              pa.int64(): TypeId.INT64, pa.uint8(): TypeId.UINT8, pa.uint16(): TypeId.UINT16,
              pa.uint32(): TypeId.UINT32, pa.uint64(): TypeId.UINT64, pa.float32(): TypeId.FLOAT32,
              pa.float64(): TypeId.FLOAT64, pa.bool_(): TypeId.BOOL8, pa.date32(): TypeId.TIMESTAMP_DAYS}
    if t in simple:
        return simple[t]
    if pa.types.is_timestamp(t) and t.tz is None:
        return _TS[_UNITS.index(t.unit)]
    if pa.types.is_duration(t):
        return _DUR[_UNITS.index(t.unit)]
    raise NotImplementedError(f"Arrow type {t} is not a fixed-width groupby type")


def arrow_type(tid: TypeId):
    import pyarrow as pa
    tid = TypeId(tid)
    simple = {TypeId.INT8: pa.int8(), TypeId.INT16: pa.int16(), TypeId.INT32: pa.int32(),
              TypeId.INT64: pa.int64(), TypeId.UINT8: pa.uint8(), TypeId.UINT16: pa.uint16(),
              TypeId.UINT32: pa.uint32(), TypeId.UINT64: pa.uint64(), TypeId.FLOAT32: pa.float32(),
              TypeId.FLOAT64: pa.float64(), TypeId.BOOL8: pa.bool_(), TypeId.TIMESTAMP_DAYS: pa.date32()}
    if tid in simple:
        return simple[tid]
    if tid in _TS:
        return pa.timestamp(_UNITS[_TS.index(tid)])
    if tid in _DUR:
        return pa.duration(_UNITS[_DUR.index(tid)])
    raise NotImplementedError(str(tid))


def validity_words(bitmap: bytes | None, offset: int, n: int) -> np.ndarray | None:
    """Arrow validity bitmap (LSB-first bytes, row `offset` first) -> the
    engine's uint32 words for rows [0, n), or None when there is no bitmap."""
    if bitmap is None:
        return None
    bits = np.unpackbits(np.frombuffer(bitmap, dtype=np.uint8), bitorder="little")[offset:offset + n]
    words = (n + 31) // 32
    padded = np.zeros(words * 32, dtype=np.uint8)
    padded[:n] = bits
    return np.packbits(padded, bitorder="little").view(np.uint32).copy()


def host_arrays(arr):
    """(values ndarray, valid bool ndarray | None, type id) of an Arrow array
    on the host, with the array's offset applied."""
    import pyarrow as pa
    if isinstance(arr, pa.ChunkedArray):
        arr = arr.combine_chunks() if arr.num_chunks != 1 else arr.chunk(0)
    tid = arrow_type_id(arr.type)
    n = len(arr)
    bufs = arr.buffers()
    valid = None
    if arr.null_count > 0 and bufs[0] is not None:
        valid = np.unpackbits(np.frombuffer(bufs[0], dtype=np.uint8), bitorder="little")[arr.offset:arr.offset + n]
        valid = valid.astype(bool)
    if tid == TypeId.BOOL8:
        vals = np.unpackbits(np.frombuffer(bufs[1], dtype=np.uint8), bitorder="little")[arr.offset:arr.offset + n]
        vals = vals.astype(np.uint8)
    else:
        dt = NUMPY_DTYPE[tid]
        vals = np.frombuffer(bufs[1], dtype=dt)[arr.offset:arr.offset + n].copy()
    return vals, valid, tid


def column_from_arrow(arr, device="cuda") -> Column:
    vals, valid, tid = host_arrays(arr)
    return Column.from_numpy(vals, valid, tid, device)


def column_to_arrow(col: Column):
    import pyarrow as pa
    vals, valid = col.to_numpy()
    t = arrow_type(col.type_id)
    mask = None if valid is None else ~valid
    if col.type_id == TypeId.BOOL8:
        return pa.array(vals.astype(bool), type=t, mask=mask)
    if col.type_id in _TS or col.type_id in _DUR or col.type_id == TypeId.TIMESTAMP_DAYS:
        storage = pa.array(vals, mask=mask)
        return storage.cast(t) if col.type_id != TypeId.TIMESTAMP_DAYS else pa.array(vals.astype(np.int32), mask=mask).cast(t)
    return pa.array(vals, type=t, mask=mask)


def to_device_words(words: np.ndarray | None, device="cuda") -> torch.Tensor | None:
    if words is None:
        return None
    return torch.from_numpy(words.view(np.int32)).to(device)
