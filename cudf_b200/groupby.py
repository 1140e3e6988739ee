"""GroupBy / GroupByRequest -- the pylibcudf.groupby interface
(python/cudf/cudf/_lib/pylibcudf/groupby.pyx:22-155) over the engine's C ABI.

    keys = Table([Column.from_tensor(k)])
    gb = GroupBy(keys, NullPolicy.EXCLUDE)
    uniq, results = gb.aggregate([GroupByRequest(Column.from_tensor(v), [agg.sum(), agg.mean()])])

``aggregate`` returns (Table of unique keys, [Table per request]) like
pylibcudf; group order is arbitrary (cpp/include/cudf/groupby.hpp:153-155).
"""
from __future__ import annotations

import ctypes
from typing import List, Optional, Sequence

import torch

from . import _lib
from .aggregation import Aggregation
from .column import Column, Table, mask_from_device, tensor_from_device
from .types import NullPolicy, Sorted


class GroupByRequest:
    """cudf::groupby::aggregation_request: a value column and its aggregations."""

    def __init__(self, values: Column, aggregations: Sequence[Aggregation]):
        self.values = values
        self.aggregations = list(aggregations)


class _ResultOwner:
    """Owns a gb_result; frees its device buffers when the last tensor view dies."""

    def __init__(self, ptr):
        self.ptr = ptr

    def __del__(self):
        try:
            if self.ptr:
                _lib.lib().gb_result_free(self.ptr)
                self.ptr = None
        except Exception:
            pass


def _stream_handle(stream) -> int:
    if stream is None:
        stream = torch.cuda.current_stream()
    return int(stream.cuda_stream) if hasattr(stream, "cuda_stream") else int(stream)


def _out_column(oc: _lib.GbOutColumn, owner) -> Column:
    return Column.from_device_buffers(oc.type_id, oc.data or 0, oc.null_mask or 0, int(oc.size),
                                      int(oc.null_count), owner)


class GroupBy:
    """cudf::groupby::groupby over device key columns.

    Like libcudf it does not copy the keys; it keeps a reference to the Table
    so the tensors outlive the object (cpp/include/cudf/groupby.hpp:111-113).
    """

    def __init__(self, keys: Table, null_handling: NullPolicy = NullPolicy.EXCLUDE,
                 keys_are_sorted: Sorted = Sorted.NO):
        self._keys = keys if isinstance(keys, Table) else Table(keys)
        self.null_handling = NullPolicy(null_handling)
        L = _lib.lib()
        cols = (_lib.GbColumn * len(self._keys))(*[c.gb_view() for c in self._keys])
        h = ctypes.c_void_p()
        _lib.check(L.gb_create(cols, len(self._keys), int(self.null_handling), int(keys_are_sorted),
                               ctypes.byref(h)))
        self._h = h

    def __del__(self):
        try:
            if getattr(self, "_h", None):
                _lib.lib().gb_destroy(self._h)
                self._h = None
        except Exception:
            pass

    def set_tuning(self, block=-1, blocks_per_sm=-1, smem_bytes=-1, smem_fill_pct=-1,
                   smem_max_groups=-1, load_factor_pct=-1, force_mode=-2, groups_hint=-1, profile=-1,
                   scatter=-1, pass2=-1, part_fill_pct=-1, wagg_pct=-1):
        t = _lib.GbTuning(block, blocks_per_sm, smem_bytes, smem_fill_pct, smem_max_groups,
                          load_factor_pct, force_mode, groups_hint, profile, scatter, pass2, part_fill_pct,
                          wagg_pct)
        _lib.check(_lib.lib().gb_set_tuning(self._h, ctypes.byref(t)))
        return self

    def stats(self) -> dict:
        s = _lib.GbStats()
        _lib.check(_lib.lib().gb_get_stats(self._h, ctypes.byref(s)))
        return {"est_groups": s.est_groups, "capacity": s.capacity, "mode": s.mode,
                "retries": s.retries, "kernels": s.kernels, "agg_kernel_ms": s.agg_kernel_ms,
                "compact_ms": s.compact_ms, "scatter_ms": s.scatter_ms, "rule": s.rule}

    def set_profile(self, on: bool = True):
        """Time the aggregation and compaction kernels with CUDA events."""
        return self.set_tuning(profile=1 if on else 0)

    def aggregate(self, requests: List[GroupByRequest], stream=None):
        """Returns (unique keys Table, [results Table per request])."""
        L = _lib.lib()
        n = len(requests)
        reqs = (_lib.GbRequest * max(1, n))()
        keep = []
        for i, r in enumerate(requests):
            aggs = (_lib.GbAgg * max(1, len(r.aggregations)))(
                *[_lib.GbAgg(int(a.kind), int(a.param)) for a in r.aggregations])
            keep.append(aggs)
            reqs[i] = _lib.GbRequest(r.values.gb_view(), len(r.aggregations), aggs)
        out = ctypes.POINTER(_lib.GbResult)()
        _lib.check(L.gb_aggregate(self._h, reqs, n, _stream_handle(stream), None, ctypes.byref(out)))
        owner = _ResultOwner(out)
        res = out.contents
        keys = Table([_out_column(res.keys[k], owner) for k in range(res.num_keys)])
        results = []
        for r in range(res.num_requests):
            cnt = res.num_results[r]
            results.append(Table([_out_column(res.results[r][j], owner) for j in range(cnt)]))
        return keys, results
