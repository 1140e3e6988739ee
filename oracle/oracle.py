"""CPU oracle for the groupby engine -- TEST INFRASTRUCTURE ONLY.

Python face of ``gb_oracle.c`` (a C restatement of libcudf 24.04's hash
groupby semantics; the C file's header lists the reference file:line each rule
follows).  Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg
of ``bench.py`` import this module, and only as the checker or as the timed CPU
baseline; the engine in ``cudf_b200`` never does.

Columns are ``HostColumn(type_id, data: np.ndarray, valid: np.ndarray | None)``;
``valid`` is a bool array (True = valid), packed here into libcudf's LSB-first
32-bit validity words (cpp/include/cudf/utilities/bit.hpp:195-198).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libgb_oracle.so")

# cudf::type_id numbering (cpp/include/cudf/types.hpp:201-233)
INT8, INT16, INT32, INT64, UINT8, UINT16, UINT32, UINT64, FLOAT32, FLOAT64, BOOL8 = range(1, 12)
TIMESTAMP_DAYS, TIMESTAMP_SECONDS, TIMESTAMP_MILLISECONDS, TIMESTAMP_MICROSECONDS, TIMESTAMP_NANOSECONDS = range(12, 17)
DURATION_DAYS, DURATION_SECONDS, DURATION_MILLISECONDS, DURATION_MICROSECONDS, DURATION_NANOSECONDS = range(17, 22)

# cudf::aggregation::Kind numbering (cpp/include/cudf/aggregation.hpp:86-102)
SUM, PRODUCT, MIN, MAX, COUNT_VALID, COUNT_ALL = 0, 1, 2, 3, 4, 5
SUM_OF_SQUARES, MEAN, VARIANCE, STD, ARGMAX, ARGMIN = 8, 9, 11, 12, 15, 16

NP_DTYPE = {
    INT8: np.int8, INT16: np.int16, INT32: np.int32, INT64: np.int64,
    UINT8: np.uint8, UINT16: np.uint16, UINT32: np.uint32, UINT64: np.uint64,
    FLOAT32: np.float32, FLOAT64: np.float64, BOOL8: np.uint8,
    TIMESTAMP_DAYS: np.int32, TIMESTAMP_SECONDS: np.int64, TIMESTAMP_MILLISECONDS: np.int64,
    TIMESTAMP_MICROSECONDS: np.int64, TIMESTAMP_NANOSECONDS: np.int64,
    DURATION_DAYS: np.int32, DURATION_SECONDS: np.int64, DURATION_MILLISECONDS: np.int64,
    DURATION_MICROSECONDS: np.int64, DURATION_NANOSECONDS: np.int64,
}
FLOATS = (FLOAT32, FLOAT64)
DURATIONS = tuple(range(17, 22))


def target_type(type_id: int, kind: int) -> int:
    """Result type id: cpp/include/cudf/detail/aggregation/aggregation.hpp:1168-1290."""
    if kind in (COUNT_VALID, COUNT_ALL, ARGMIN, ARGMAX):
        return INT32
    if kind in (MIN, MAX):
        return type_id
    if kind in (VARIANCE, STD):
        return FLOAT64
    if kind == MEAN:
        return type_id if type_id in DURATIONS else FLOAT64
    if kind in (SUM, PRODUCT, SUM_OF_SQUARES):
        if type_id in FLOATS or type_id in DURATIONS:
            return type_id
        return INT64
    raise ValueError(f"unsupported aggregation kind {kind}")


def pack_mask(valid: Optional[np.ndarray]) -> Optional[np.ndarray]:
    """bool[n] -> uint32 words, bit i of word i//32 set when row i is valid."""
    if valid is None:
        return None
    valid = np.asarray(valid, dtype=bool)
    n = valid.size
    nbytes = ((n + 31) // 32) * 4
    packed = np.packbits(valid, bitorder="little")
    buf = np.zeros(nbytes, dtype=np.uint8)
    buf[: packed.size] = packed
    return buf.view(np.uint32)


def unpack_mask(words: np.ndarray, n: int) -> np.ndarray:
    b = np.unpackbits(np.asarray(words, dtype=np.uint32).view(np.uint8), bitorder="little")
    return b[:n].astype(bool)


@dataclass
class HostColumn:
    """``valid`` (bool per row) or ``packed`` (libcudf validity words) may be
    given; a column built from words unpacks them only if its validity is read
    as bools (key columns)."""
    type_id: int
    data: np.ndarray
    valid: Optional[np.ndarray] = None
    packed: Optional[np.ndarray] = None

    def __post_init__(self):
        self.data = np.ascontiguousarray(self.data, dtype=NP_DTYPE[self.type_id])
        self._words = None
        if self.packed is not None:
            self._words = np.ascontiguousarray(self.packed, dtype=np.uint32)
            assert self._words.size >= (self.data.shape[0] + 31) // 32
            if self.valid is None:
                self.valid = unpack_mask(self._words, self.data.shape[0])
        if self.valid is not None:
            self.valid = np.ascontiguousarray(self.valid, dtype=bool)
            assert self.valid.shape == self.data.shape

    def __len__(self):
        return self.data.shape[0]

    def words(self) -> Optional[np.ndarray]:
        """The validity as packed words, computed once per column."""
        if self._words is None and self.valid is not None:
            self._words = pack_mask(self.valid)
        return self._words


class _Col(ctypes.Structure):
    _fields_ = [("type_id", ctypes.c_int32), ("size", ctypes.c_int64), ("data", ctypes.c_void_p),
                ("mask", ctypes.c_void_p), ("offset", ctypes.c_int64)]


class _Req(ctypes.Structure):
    _fields_ = [("values", _Col), ("num_aggs", ctypes.c_int32), ("kinds", ctypes.c_void_p),
                ("ddof", ctypes.c_void_p)]


_lib = None


def build() -> str:
    """Compile gb_oracle.c with its Makefile (gcc; no GPU needed)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(
                os.path.join(HERE, "gb_oracle.c")):
            build()
        L = ctypes.CDLL(LIB_PATH)
        L.orc_groupby.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                  ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]
        L.orc_groupby.restype = ctypes.c_int
        L.orc_num_groups.argtypes = [ctypes.c_void_p]
        L.orc_num_groups.restype = ctypes.c_int64
        L.orc_group_rows.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.orc_result.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                 ctypes.c_void_p, ctypes.c_void_p]
        L.orc_result.restype = ctypes.c_int
        L.orc_free.argtypes = [ctypes.c_void_p]
        L.orc_valid_agg.argtypes = [ctypes.c_int, ctypes.c_int]
        L.orc_valid_agg.restype = ctypes.c_int
        _lib = L
    return _lib


@dataclass
class OracleResult:
    group_rows: np.ndarray            # first row of each group
    keys: list                        # [(data, valid)] per key column
    results: list                     # results[r][j] = (values, valid, tol)

    @property
    def num_groups(self) -> int:
        return int(self.group_rows.size)


def valid_agg(type_id: int, kind: int) -> bool:
    return bool(lib().orc_valid_agg(type_id, kind))


def groupby(keys: Sequence[HostColumn], requests: Sequence[tuple], include_null_keys: bool = False,
            nthreads: int = 1) -> OracleResult:
    """requests: [(HostColumn values, [kinds], optional [ddof])]."""
    L = lib()
    keep = []
    kcols = (_Col * len(keys))()
    for i, k in enumerate(keys):
        m = k.words()
        keep.append(m)
        kcols[i] = _Col(k.type_id, len(k), k.data.ctypes.data, 0 if m is None else m.ctypes.data, 0)
    reqs = (_Req * max(1, len(requests)))()
    for i, rq in enumerate(requests):
        col, kinds = rq[0], list(rq[1])
        ddof = list(rq[2]) if len(rq) > 2 and rq[2] is not None else [1] * len(kinds)
        m = col.words()
        ka = np.asarray(kinds, dtype=np.int32)
        da = np.asarray(ddof, dtype=np.int32)
        keep += [m, ka, da]
        reqs[i] = _Req(_Col(col.type_id, len(col), col.data.ctypes.data,
                            0 if m is None else m.ctypes.data, 0),
                       len(kinds), ka.ctypes.data, da.ctypes.data)
    h = ctypes.c_void_p()
    rc = L.orc_groupby(kcols, len(keys), int(bool(include_null_keys)), reqs, len(requests),
                       int(nthreads), ctypes.byref(h))
    if rc != 0:
        raise ValueError(f"oracle rejected the request (code {rc})")
    try:
        G = L.orc_num_groups(h)
        rows = np.empty(G, dtype=np.int64)
        if G:
            L.orc_group_rows(h, rows.ctypes.data)
        out_keys = []
        for k in keys:
            d = k.data[rows]
            v = None if k.valid is None else k.valid[rows]
            out_keys.append((d, v))
        results = []
        for i, rq in enumerate(requests):
            col, kinds = rq[0], list(rq[1])
            per = []
            for j, kind in enumerate(kinds):
                raw = np.empty(G, dtype=np.int64)
                valid = np.empty(G, dtype=np.uint8)
                tol = np.empty(G, dtype=np.float64)
                L.orc_result(h, i, j, raw.ctypes.data, valid.ctypes.data, tol.ctypes.data)
                tt = target_type(col.type_id, kind)
                if tt in FLOATS:
                    vals = raw.view(np.float64).astype(NP_DTYPE[tt])
                else:
                    vals = raw.astype(NP_DTYPE[tt])
                per.append((vals, valid.astype(bool), tol))
            results.append(per)
        return OracleResult(rows, out_keys, results)
    finally:
        L.orc_free(h)


def sort_order(key_cols) -> np.ndarray:
    """Row order that sorts groups by key tuple, nulls first, NaN last, for
    comparing two groupby outputs whose group order is arbitrary."""
    arrays = []
    for data, valid in reversed(list(key_cols)):
        d = np.asarray(data)
        if valid is not None:  # the value under a null is arbitrary: sort nulls as 0
            d = np.where(np.asarray(valid, dtype=bool), d, np.zeros((), d.dtype))
        if d.dtype.kind == "f":
            nan = np.isnan(d)
            d = np.where(nan, 0, d)
            d = np.where(d == 0, 0, d)  # -0.0 sorts with +0.0
            arrays.append(d)
            arrays.append(nan)
        else:
            arrays.append(d)
        if valid is not None:
            arrays.append(np.asarray(valid, dtype=bool))
        else:
            arrays.append(np.ones(d.shape[0], dtype=bool))
    return np.lexsort(arrays)
