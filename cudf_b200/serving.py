"""Serving loop: continuous batching of groupby queries over device-resident
columns (the C++ loop in csrc/gb_server.cu).

    srv = Server(memory_cap_bytes=150 << 30)
    qid = srv.submit(keys_table, [GroupByRequest(values, aggs)])   # any thread
    info = srv.wait(qid)            # latency, queueing time, group count
    keys, results = srv.result(qid) # views, valid until release()
    srv.release(qid)
"""
from __future__ import annotations

import atexit
import ctypes
import threading
import weakref
from typing import List

from . import _lib
from .column import Column, Table, mask_from_device, tensor_from_device
from .groupby import GroupByRequest
from .types import NullPolicy


# Servers still open at interpreter exit are closed first: their C++ worker
# threads must be joined before the process tears down the CUDA runtime.
_OPEN: "weakref.WeakSet[Server]" = weakref.WeakSet()


@atexit.register
def _close_open_servers():
    for s in list(_OPEN):
        try:
            s.close()
        except Exception:
            pass


class Server:
    def __init__(self, memory_cap_bytes: int = 150 << 30, max_batch_queries: int = 256,
                 max_batch_rows: int = 400 << 20, workers: int = 4, direct_rows: int = 0,
                 direct_groups: int = 0, reserve_bytes: int = 0):
        L = _lib.lib()
        o = _lib.GbServerOptions(memory_cap_bytes, max_batch_queries, max_batch_rows, workers,
                                 direct_rows, direct_groups, reserve_bytes)
        h = ctypes.c_void_p()
        _lib.check(L.gb_server_create(ctypes.byref(o), ctypes.byref(h)))
        self._h = h
        _OPEN.add(self)
        self._mu = threading.Lock()
        self._live = {}  # query id -> (columns kept alive, aggregation counts)

    def close(self):
        if getattr(self, "_h", None):
            _lib.lib().gb_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, keys: Table, requests: List[GroupByRequest],
               null_handling: NullPolicy = NullPolicy.EXCLUDE) -> int:
        kt = keys if isinstance(keys, Table) else Table(keys)
        kc = (_lib.GbColumn * len(kt))(*[c.gb_view() for c in kt])
        reqs = (_lib.GbRequest * max(1, len(requests)))()
        keep = [kt, requests]
        for i, r in enumerate(requests):
            aggs = (_lib.GbAgg * max(1, len(r.aggregations)))(
                *[_lib.GbAgg(int(a.kind), int(a.param)) for a in r.aggregations])
            keep.append(aggs)
            reqs[i] = _lib.GbRequest(r.values.gb_view(), len(r.aggregations), aggs)
        qid = ctypes.c_int64()
        _lib.check(_lib.lib().gb_server_submit(self._h, kc, len(kt), int(null_handling), reqs, len(requests),
                                               ctypes.byref(qid)))
        with self._mu:
            self._live[qid.value] = (keep, len(kt), [len(r.aggregations) for r in requests])
        return qid.value

    def wait(self, qid: int, timeout_s: float = 0.0) -> dict:
        info = _lib.GbQueryInfo()
        _lib.check(_lib.lib().gb_server_wait(self._h, qid, timeout_s, ctypes.byref(info)))
        return {"status": info.status, "latency_s": info.latency_s, "queue_s": info.queue_s,
                "num_groups": info.num_groups}

    def result(self, qid: int):
        with self._mu:
            _, nk, counts = self._live[qid]
        ng = ctypes.c_int64()
        ok = (_lib.GbOutColumn * nk)()
        orr = (_lib.GbOutColumn * max(1, sum(counts)))()
        _lib.check(_lib.lib().gb_server_result(self._h, qid, ctypes.byref(ng), ok, orr))
        owner = self

        def col(oc):
            n = int(oc.size)
            return Column(oc.type_id, tensor_from_device(oc.data or 0, n, oc.type_id, owner),
                          mask_from_device(oc.null_mask or 0, n, owner), size=n,
                          null_count=int(oc.null_count), _owner=owner)

        keys = Table([col(ok[k]) for k in range(nk)])
        out, j = [], 0
        for c in counts:
            out.append(Table([col(orr[j + a]) for a in range(c)]))
            j += c
        return keys, out

    def release(self, qid: int):
        _lib.check(_lib.lib().gb_server_release(self._h, qid))
        with self._mu:
            self._live.pop(qid, None)

    def stats(self) -> dict:
        s = _lib.GbServerStats()
        _lib.check(_lib.lib().gb_server_get_stats(self._h, ctypes.byref(s)))
        return {f: getattr(s, f) for f, _ in _lib.GbServerStats._fields_}
