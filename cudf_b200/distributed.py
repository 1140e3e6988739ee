"""Multi-GPU groupby over row-sharded tables (one process per GPU).

Each rank holds a shard of the rows.  The aggregation decomposes like dask_cudf's
tree/shuffle groupby (python/dask_cudf/dask_cudf/groupby.py:731-766,828):

1. every rank aggregates its shard into partial results (the engine);
2. each partial group is sent to the rank that owns its key (hash of the key
   tuple modulo the world size) with one all-to-all per column
   (torch.distributed over NCCL / NVLink; gloo on CPU);
3. each rank merges the partials it owns with a second groupby
   (SUM of sums and counts, MIN of mins, MAX of maxes, PRODUCT of products);
4. MEAN = merged SUM / merged COUNT_VALID, in double (durations: integer mean).

Every rank returns the groups it owns; the ranks' groups are disjoint and
together are the groupby of the whole table.  Received data lands in local
memory before any kernel reads it; there is no peer-memory load.

The local aggregation is pluggable (`local_aggregate(keys, requests, policy)`
returning (keys, [[(values, valid)]] per request)); the default is the engine.
"""
from __future__ import annotations

from typing import Callable, List, Optional, Sequence, Tuple

import numpy as np
import torch
import torch.distributed as dist

from .types import Kind, NullPolicy, TypeId

# how each aggregation decomposes into partials and merges back
_PARTIALS = {
    Kind.SUM: [Kind.SUM],
    Kind.PRODUCT: [Kind.PRODUCT],
    Kind.MIN: [Kind.MIN],
    Kind.MAX: [Kind.MAX],
    Kind.COUNT_VALID: [Kind.COUNT_VALID],
    Kind.COUNT_ALL: [Kind.COUNT_ALL],
    Kind.SUM_OF_SQUARES: [Kind.SUM_OF_SQUARES],
    Kind.MEAN: [Kind.SUM, Kind.COUNT_VALID],
}
_MERGE = {Kind.SUM: Kind.SUM, Kind.PRODUCT: Kind.PRODUCT, Kind.MIN: Kind.MIN, Kind.MAX: Kind.MAX,
          Kind.COUNT_VALID: Kind.SUM, Kind.COUNT_ALL: Kind.SUM, Kind.SUM_OF_SQUARES: Kind.SUM}
_DURATIONS = {TypeId.DURATION_DAYS, TypeId.DURATION_SECONDS, TypeId.DURATION_MILLISECONDS,
              TypeId.DURATION_MICROSECONDS, TypeId.DURATION_NANOSECONDS}

_GOLD = -7046029254386353131  # 0x9E3779B97F4A7C15 as int64
_M1 = -49064778989728563      # 0xff51afd7ed558ccd
_M2 = -4265267296055464877    # 0xc4ceb9fe1a85ec53


def _lsr(x: torch.Tensor, k: int) -> torch.Tensor:
    """Logical right shift of int64 bits."""
    return (x >> k) & ((1 << (64 - k)) - 1)


def _key_bits(data: torch.Tensor, type_id: int) -> torch.Tensor:
    """int64 bits of a key column with NaN canonical and -0.0 == +0.0, so that
    equal keys (as the engine compares them) land on the same rank."""
    if type_id == TypeId.FLOAT64:
        d = torch.where(torch.isnan(data), torch.full_like(data, float("nan")), data)
        d = torch.where(d == 0, torch.zeros_like(d), d)
        return d.view(torch.int64)
    if type_id == TypeId.FLOAT32:
        d = torch.where(torch.isnan(data), torch.full_like(data, float("nan")), data)
        d = torch.where(d == 0, torch.zeros_like(d), d)
        return d.view(torch.int32).to(torch.int64)
    if type_id == TypeId.BOOL8:
        return (data != 0).to(torch.int64)
    if data.dtype in (torch.uint16, torch.uint32, torch.uint64):
        return data.view({torch.uint16: torch.int16, torch.uint32: torch.int32,
                          torch.uint64: torch.int64}[data.dtype]).to(torch.int64)
    return data.to(torch.int64)


def owner_rank(key_cols: Sequence[Tuple[torch.Tensor, Optional[torch.Tensor], int]], world: int) -> torch.Tensor:
    """Rank that owns each row's key tuple: a 64-bit mix (MurmurHash3 fmix64)
    of the key bits (0 for null, plus a null flag), modulo the world size."""
    n = key_cols[0][0].shape[0]
    h = torch.zeros(n, dtype=torch.int64, device=key_cols[0][0].device)
    for data, valid, tid in key_cols:
        v = _key_bits(data, tid)
        if valid is not None:
            v = torch.where(valid, v, torch.zeros_like(v))
            h = h * _GOLD + valid.to(torch.int64)
        h = h * _GOLD + v
        h = h ^ _lsr(h, 33)
        h = h * _M1
        h = h ^ _lsr(h, 33)
        h = h * _M2
        h = h ^ _lsr(h, 33)
    return torch.remainder(h & 0x7FFFFFFFFFFFFFFF, world)


def _exchange(tensors: List[torch.Tensor], dest: torch.Tensor, world: int, group=None) -> List[torch.Tensor]:
    """Sends row i of every tensor to rank dest[i].  The tensors travel as one
    row-major byte matrix (each row: every tensor's bytes of that row, bool
    as one byte), gathered into destination order once, so the exchange is
    two collectives whatever the number of columns: the per-rank row counts,
    then the payload.  The counts are read on the host (one synchronisation:
    the payload's split sizes)."""
    n = int(dest.shape[0])
    order = torch.argsort(dest, stable=True)
    counts = torch.bincount(dest, minlength=world).to(torch.int64)
    recv_counts = torch.empty_like(counts)
    dist.all_to_all_single(recv_counts, counts, group=group)
    both = torch.stack([counts, recv_counts]).cpu()
    send_splits, recv_splits = both[0].tolist(), both[1].tolist()
    parts, widths = [], []
    for t in tensors:
        u = t.to(torch.uint8) if t.dtype == torch.bool else t
        w = u.element_size() * (int(np.prod(u.shape[1:])) if u.dim() > 1 else 1)
        parts.append(u.contiguous().view(torch.uint8).reshape(n, w) if n else
                     torch.empty((0, w), dtype=torch.uint8, device=dest.device))
        widths.append(w)
    rows = torch.cat(parts, dim=1)[order].contiguous() if parts else torch.empty((n, 0), dtype=torch.uint8,
                                                                                   device=dest.device)
    recv = torch.empty((sum(recv_splits), rows.shape[1]), dtype=torch.uint8, device=rows.device)
    dist.all_to_all_single(recv, rows, recv_splits, send_splits, group=group)
    out, at = [], 0
    for t, w in zip(tensors, widths):
        b = recv[:, at:at + w].contiguous()
        at += w
        if t.dtype == torch.bool:
            out.append(b.reshape(-1) != 0)
        else:
            out.append(b.view(t.dtype).reshape((-1,) + tuple(t.shape[1:])))
    return out


def engine_local_aggregate(keys, requests, null_handling):
    """Local aggregation with the engine.  keys: [(data, valid|None, type_id)];
    requests: [((data, valid|None, type_id), [Kind])].  Returns (keys, results)
    in the same (data, valid) form."""
    from . import aggregation as agg
    from .column import Column, Table
    from .groupby import GroupBy, GroupByRequest
    kt = Table([Column.from_tensor(d, v, t) for d, v, t in keys])
    reqs = [GroupByRequest(Column.from_tensor(d, v, t), [agg.Aggregation(Kind(k)) for k in kinds])
            for (d, v, t), kinds in requests]
    uk, res = GroupBy(kt, null_handling).aggregate(reqs)
    out_keys = [(c.values().clone(), None if c.mask is None else c.valid(), int(c.type_id)) for c in uk.columns]
    out_res = [[(c.values().clone(), None if c.mask is None else c.valid()) for c in t.columns] for t in res]
    return out_keys, out_res


def plan_partials(requests):
    """The partial aggregations each request needs (MEAN -> SUM + COUNT_VALID,
    every other kind itself), without repeats: [(col, [Kind])]."""
    preq = []
    for (col, kinds) in requests:
        plist = []
        for k in kinds:
            k = Kind(k)
            if k not in _PARTIALS:
                raise NotImplementedError(f"{k.name} does not decompose into mergeable partials")
            for p in _PARTIALS[k]:
                if p not in plist:
                    plist.append(p)
        preq.append((col, plist))
    return preq


def _partial_tid(col_tid: int, p: Kind, data: torch.Tensor) -> int:
    """Type id of a partial column (counts merged once are int64 sums)."""
    if p in (Kind.COUNT_VALID, Kind.COUNT_ALL) and data.dtype == torch.int64:
        return TypeId.INT64
    return _partial_type(col_tid, p)


def merge_partials(preq, pkeys, pvals, null_handling, local):
    """Merges partial groups (the same key may appear in several rows) with a
    second groupby: SUM of sums and counts, MIN of mins, MAX of maxes, PRODUCT
    of products.  pkeys: [(data, valid, type_id)]; pvals[(r, j)] = (data,
    valid) of partial j of request r.  Returns (keys, merged) with
    merged[r][kind] = (data, valid) -- again partials, ready to merge again
    or to finalize."""
    mreq = []
    for r, (col, plist) in enumerate(preq):
        for j, p in enumerate(plist):
            d, v = pvals[(r, j)]
            mreq.append(((d, v, _partial_tid(col[2], p, d)), [_MERGE[p]]))
    policy = NullPolicy.INCLUDE if null_handling == NullPolicy.INCLUDE else NullPolicy.EXCLUDE
    mk, mres = local(pkeys, mreq, policy)
    merged, i = [], 0
    for r, (col, plist) in enumerate(preq):
        per = {}
        for p in plist:
            per[p] = mres[i][0]
            i += 1
        merged.append(per)
    return mk, merged


def finalize_partials(requests, merged):
    """Results in request order from merged partials: MEAN = SUM / COUNT in
    double (durations: integer mean), counts as int32, the rest as merged."""
    out = []
    for r, (col, kinds) in enumerate(requests):
        per = []
        for k in kinds:
            k = Kind(k)
            if k == Kind.MEAN:
                s, sv = merged[r][Kind.SUM]
                c, _ = merged[r][Kind.COUNT_VALID]
                c = c.to(torch.int64)
                valid = c > 0
                if col[2] in _DURATIONS:
                    mean = torch.where(valid, torch.div(s.to(torch.int64), c.clamp(min=1), rounding_mode="trunc"),
                                       torch.zeros_like(s, dtype=torch.int64)).to(s.dtype)
                else:
                    mean = torch.where(valid, s.to(torch.float64) / c.clamp(min=1).to(torch.float64),
                                       torch.zeros_like(s, dtype=torch.float64))
                per.append((mean, valid if (sv is not None or col[1] is not None) else None))
            elif k in (Kind.COUNT_VALID, Kind.COUNT_ALL):
                d, _ = merged[r][k]
                per.append((d.to(torch.int32), None))
            else:
                per.append(merged[r][k])
        out.append(per)
    return out


def distributed_groupby(keys, requests, null_handling: NullPolicy = NullPolicy.EXCLUDE, group=None,
                        local_aggregate: Optional[Callable] = None):
    """keys: [(data, valid|None, type_id)] of this rank's shard; requests:
    [((data, valid|None, type_id), [Kind])]; `valid` is a bool per row or
    the packed 32-bit validity words (LSB first) the engine's columns carry.
    Returns (keys, results) of the groups this rank owns,
    results[r][j] = (values, valid|None)."""
    local = local_aggregate or engine_local_aggregate
    world = dist.get_world_size(group)
    # 1. partial aggregation of the shard
    preq = plan_partials(requests)
    pk, pres = local(keys, preq, null_handling)
    # 2. route every partial group to the rank owning its key
    dest = owner_rank([(d, v, t) for d, v, t in pk], world)
    flat, layout = [], []
    for d, v, t in pk:
        layout.append(("key", t, v is not None))
        flat.append(d)
        if v is not None:
            flat.append(v)
    for r, per in enumerate(pres):
        for j, (d, v) in enumerate(per):
            layout.append(("val", (r, j), v is not None))
            flat.append(d)
            if v is not None:
                flat.append(v)
    recv = _exchange(flat, dest.to(torch.int64), world, group)
    it = iter(recv)
    rkeys, rvals = [], {}
    for kind, info, has_valid in layout:
        d = next(it)
        v = next(it) if has_valid else None
        if kind == "key":
            rkeys.append((d, v, info))
        else:
            rvals[info] = (d, v)
    # 3. merge the partials this rank owns; 4. finalize in request order
    mk, merged = merge_partials(preq, rkeys, rvals, null_handling, local)
    return mk, finalize_partials(requests, merged)


def _partial_type(tid: int, p: Kind) -> int:
    if p in (Kind.COUNT_VALID, Kind.COUNT_ALL):
        return TypeId.INT32
    if p in (Kind.MIN, Kind.MAX):
        return tid
    if tid in (TypeId.FLOAT32, TypeId.FLOAT64) or tid in _DURATIONS:
        return tid
    return TypeId.INT64
