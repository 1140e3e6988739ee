"""Batched groupby: many independent groupbys of one schema in one launch.

    bg = BatchGroupBy([(Table([k0]), [GroupByRequest(v0, aggs)]),
                       (Table([k1]), [GroupByRequest(v1, aggs)]), ...],
                      use_graph=True)
    bg.run()                      # one persistent launch (or one graph replay)
    keys, results = bg.result(i)  # views valid until the next run()

Every instance must have the same key types, value types and aggregations
(the schema); columns may differ in length and nullability.  The engine
samples each instance once (in `__init__`) to size its table and outputs, so
later runs must keep the same column shapes.
"""
from __future__ import annotations

import ctypes
from typing import List, Sequence, Tuple

import torch

from . import _lib
from .column import Column, Table, mask_from_device, tensor_from_device
from .groupby import GroupByRequest, _stream_handle
from .types import NullPolicy


class BatchGroupBy:
    def __init__(self, instances: Sequence[Tuple[Table, List[GroupByRequest]]],
                 null_handling: NullPolicy = NullPolicy.EXCLUDE, use_graph: bool = False, stream=None):
        L = _lib.lib()
        self._instances = [(k if isinstance(k, Table) else Table(k), list(r)) for k, r in instances]
        n = len(self._instances)
        if n == 0:
            raise ValueError("a batch needs at least one instance")
        nk = len(self._instances[0][0])
        nr = len(self._instances[0][1])
        self._nk, self._nr = nk, nr
        self._naggs = sum(len(r.aggregations) for r in self._instances[0][1])
        keys = (_lib.GbColumn * (n * nk))()
        reqs = (_lib.GbRequest * max(1, n * nr))()
        self._keep = []
        for i, (kt, rl) in enumerate(self._instances):
            if len(kt) != nk or len(rl) != nr:
                raise ValueError("every instance needs the same number of key columns and requests")
            for k in range(nk):
                keys[i * nk + k] = kt[k].gb_view()
            for r, rq in enumerate(rl):
                aggs = (_lib.GbAgg * max(1, len(rq.aggregations)))(
                    *[_lib.GbAgg(int(a.kind), int(a.param)) for a in rq.aggregations])
                self._keep.append(aggs)
                reqs[i * nr + r] = _lib.GbRequest(rq.values.gb_view(), len(rq.aggregations), aggs)
        h = ctypes.c_void_p()
        _lib.check(L.gb_batch_prepare(n, keys, nk, int(null_handling), reqs, nr, int(bool(use_graph)),
                                      _stream_handle(stream), None, ctypes.byref(h)))
        self._h = h
        self._n = n

    def __len__(self):
        return self._n

    def __del__(self):
        try:
            if getattr(self, "_h", None):
                _lib.lib().gb_batch_destroy(self._h)
                self._h = None
        except Exception:
            pass

    def run(self, stream=None):
        _lib.check(_lib.lib().gb_batch_run(self._h, _stream_handle(stream)))

    def stats(self) -> dict:
        s = _lib.GbBatchStats()
        _lib.check(_lib.lib().gb_batch_get_stats(self._h, ctypes.byref(s)))
        return {f: getattr(s, f) for f, _ in _lib.GbBatchStats._fields_}

    def result(self, i: int):
        """(unique keys Table, [results Table per request]) of instance i."""
        L = _lib.lib()
        ng = ctypes.c_int64()
        ok = (_lib.GbOutColumn * self._nk)()
        orr = (_lib.GbOutColumn * max(1, self._naggs))()
        _lib.check(L.gb_batch_result(self._h, i, ctypes.byref(ng), ok, orr))
        owner = self  # the batch owns the buffers

        def col(oc):
            n = int(oc.size)
            return Column(oc.type_id, tensor_from_device(oc.data or 0, n, oc.type_id, owner),
                          mask_from_device(oc.null_mask or 0, n, owner), size=n,
                          null_count=int(oc.null_count), _owner=owner)

        keys = Table([col(ok[k]) for k in range(self._nk)])
        out, j = [], 0
        for rq in self._instances[i][1]:
            out.append(Table([col(orr[j + a]) for a in range(len(rq.aggregations))]))
            j += len(rq.aggregations)
        return keys, out
