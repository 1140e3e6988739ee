"""Per-size-bucket autotuner for the engine's launch parameters.

The engine's kernels have tunables (mode thresholds, shared-memory table size
and fill, global-table load factor, the partition pass's launch shape).  The
best values depend on the call's size: rows and distinct groups.  This module
times candidate settings on synthetic inputs of each (rows, groups) bucket
with CUDA events, keeps the fastest, and installs the result as process-wide
rules (``gb_set_tuning_rules``): a call takes the first rule whose bucket
covers its row count and its estimated group count, after the engine's own
sketch has estimated the groups.

    python -m cudf_b200.autotune --out cudf_b200/tuning_b200.json   # on a B200

Batched launches (``gb_batch_set_tuning``) are tuned the same way: the
aggregation kernel's block size, rows per tile and shared-table budget on a
mix drawn like the batched benchmark, then per instance size bucket the
shared-stage rule (table headroom, or the global table only) that runs a batch
of that bucket fastest.

``cudf_b200`` installs ``tuning_b200.json`` (next to this file) at import
when it exists; ``load(path)`` / ``clear()`` change that at run time.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import time
from typing import Dict, List, Optional, Sequence, Tuple

from . import _lib

TUNING_FILE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuning_b200.json")

# fields of a rule's tuning, with the value meaning "unset" in gb_tuning
_UNSET = {"block": -1, "blocks_per_sm": -1, "smem_bytes": -1, "smem_fill_pct": -1, "smem_max_groups": -1,
          "load_factor_pct": -1, "force_mode": -2, "groups_hint": -1, "profile": -1, "scatter": -1,
          "pass2": -1, "part_fill_pct": -1, "wagg_pct": -1}

# default buckets: row counts x group counts seen by the benchmark shapes
DEFAULT_BUCKETS = [
    (1 << 20, 1 << 10), (1 << 20, 1 << 17), (1 << 20, 1 << 20),
    (1 << 24, 1 << 10), (1 << 24, 1 << 17), (1 << 24, 1 << 20), (1 << 24, 1 << 22), (1 << 24, 1 << 24),
    (1 << 27, 1 << 10), (1 << 27, 1 << 17), (1 << 27, 1 << 20), (1 << 27, 1 << 22), (1 << 27, 1 << 23),
    (1 << 27, 1 << 24), (1 << 27, 1 << 27),
]

# candidate settings per stage of the search (coordinate descent)
_MODES = [{"force_mode": -1}, {"force_mode": 0}, {"force_mode": 1}, {"force_mode": 2}]
_SCATTER = [{"scatter": s} for s in range(9)]
_SMEM = [{"smem_bytes": b, "smem_fill_pct": f} for b in (48 << 10, 96 << 10, 160 << 10) for f in (50, 70)]
_LOAD = [{"load_factor_pct": p} for p in (40, 50, 70)]


def _tuning_struct(t: Dict[str, int]) -> _lib.GbTuning:
    vals = dict(_UNSET)
    vals.update(t)
    return _lib.GbTuning(*[int(vals[name]) for name, _ in _lib.GbTuning._fields_])


def set_rules(rules: Sequence[Dict]) -> None:
    """Installs rules [{"max_rows", "max_groups", "tuning": {field: value}}]
    in order (the first match applies)."""
    arr = (_lib.GbTuningRule * max(1, len(rules)))()
    for i, r in enumerate(rules):
        arr[i] = _lib.GbTuningRule(int(r["max_rows"]), int(r["max_groups"]), int(r.get("key_words", 0)),
                                   _tuning_struct(r.get("tuning", {})))
    _lib.check(_lib.lib().gb_set_tuning_rules(arr, len(rules)))


def clear() -> None:
    _lib.check(_lib.lib().gb_set_tuning_rules(None, 0))


def save(rules: Sequence[Dict], path: str, meta: Optional[Dict] = None) -> None:
    with open(path, "w") as f:
        json.dump({"rules": list(rules), "meta": meta or {}}, f, indent=1)


def load(path: str = TUNING_FILE) -> List[Dict]:
    with open(path) as f:
        d = json.load(f)
    rules = d["rules"]
    set_rules(rules)
    if "batch" in d:
        set_batch_tuning(d["batch"].get("rules", []), d["batch"].get("launch"))
    return rules


# -- batched launches (gb_batch_set_tuning) -------------------------------------
def set_batch_tuning(rules: Sequence[Dict], launch: Optional[Dict] = None) -> None:
    """Installs batch tuning: launch {"block", "tile_rows", "smem_bytes"} and
    per-instance rules [{"max_rows", "max_groups", "smem_slots", "headroom_pct"}]
    (first match applies; -1 / 0 leave a field unset)."""
    arr = (_lib.GbBatchRule * max(1, len(rules)))()
    for i, r in enumerate(rules):
        arr[i] = _lib.GbBatchRule(int(r["max_rows"]), int(r["max_groups"]), int(r.get("smem_slots", -1)),
                                  int(r.get("headroom_pct", 0)))
    lp = None
    if launch:
        lp = ctypes.byref(_lib.GbBatchLaunch(int(launch["block"]), int(launch["tile_rows"]),
                                             int(launch["smem_bytes"])))
    _lib.check(_lib.lib().gb_batch_set_tuning(arr, len(rules), lp))


BATCH_LAUNCH_DEFAULT = {"block": 512, "tile_rows": 65536, "smem_bytes": 160 * 1024}
_BATCH_BLOCKS = [256, 512, 1024]
_BATCH_TILES = [16384, 65536, 262144]
_BATCH_SMEM = [96 * 1024, 160 * 1024, 200 * 1024]
# instance buckets (rows x estimated groups) of the per-instance rules
BATCH_BUCKETS = [(r, g) for r in (16384, 262144, 4194304) for g in (256, 4096, 65536, 1 << 30)]
_BATCH_RULE_CANDS = [{"headroom_pct": 150}, {"headroom_pct": 200}, {"headroom_pct": 400}, {"smem_slots": 0}]


def _batch_workload(sizes, seed: int):
    """Instances with the batched benchmark's schema: int32 keys uniform over
    each instance's cardinality, int64 [0, 1e6] and float64 normal values with
    5% nulls, sum/count/min/max/mean.  sizes: [(rows, cardinality)]."""
    import torch
    from . import aggregation as agg
    from .column import Column, Table, pack_mask
    from .groupby import GroupByRequest
    from .types import TypeId
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    inst = []
    for n, c in sizes:
        k = torch.randint(0, max(1, int(c)), (int(n),), device="cuda", generator=g, dtype=torch.int32)
        v1 = torch.randint(0, 10**6 + 1, (int(n),), device="cuda", generator=g, dtype=torch.int64)
        v2 = torch.randn(int(n), device="cuda", generator=g, dtype=torch.float64)
        m1 = pack_mask(torch.rand(int(n), device="cuda", generator=g) >= 0.05)
        m2 = pack_mask(torch.rand(int(n), device="cuda", generator=g) >= 0.05)
        aggs = [agg.sum(), agg.count(), agg.min(), agg.max(), agg.mean()]
        inst.append((Table([Column(TypeId.INT32, k)]),
                     [GroupByRequest(Column(TypeId.INT64, v1, m1), aggs),
                      GroupByRequest(Column(TypeId.FLOAT64, v2, m2), aggs)]))
    return inst


def _time_batch(inst, steps: int) -> float:
    import torch
    from .batch import BatchGroupBy
    bg = BatchGroupBy(inst, use_graph=True)
    bg.run()
    stream = torch.cuda.current_stream()
    times = []
    for _ in range(steps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        bg.run()
        b.record(stream)
        b.synchronize()
        times.append(a.elapsed_time(b))
    times.sort()
    return times[len(times) // 2]


def tune_batch(instances: int = 512, steps: int = 3, verbose: bool = False) -> Tuple[Dict, Dict]:
    """Launch settings on a mix drawn like the batched benchmark (rows
    log-uniform [1e3, 4e6], cardinality log-uniform [4, 1e5]) by coordinate
    descent over block, tile rows and table budget; then, per instance size
    bucket, the shared-stage rule that runs a batch of that bucket fastest."""
    import numpy as np
    rng = np.random.default_rng(11)
    rows = np.exp(rng.uniform(np.log(1e3), np.log(4e6), instances)).astype(np.int64)
    cards = np.exp(rng.uniform(np.log(4), np.log(1e5), instances)).astype(np.int64)
    mix = _batch_workload(list(zip(rows.tolist(), cards.tolist())), 12)
    log: Dict[str, object] = {}
    set_batch_tuning([], BATCH_LAUNCH_DEFAULT)
    best = dict(BATCH_LAUNCH_DEFAULT)
    best_ms = _time_batch(mix, steps)
    log["launch default"] = best_ms
    for field, cands in (("block", _BATCH_BLOCKS), ("tile_rows", _BATCH_TILES), ("smem_bytes", _BATCH_SMEM)):
        for v in cands:
            t = dict(best)
            t[field] = v
            set_batch_tuning([], t)
            ms = _time_batch(mix, steps)
            log["launch " + json.dumps(t)] = ms
            if ms < best_ms * 0.98:
                best, best_ms = t, ms
    del mix
    rules = []
    for r_hi, g_hi in BATCH_BUCKETS:
        inst = _batch_workload(bucket_sizes(rng, r_hi, g_hi), r_hi ^ g_hi)
        cand_best, cand_ms = None, None
        for cand in [{}] + _BATCH_RULE_CANDS:
            rule = {"max_rows": r_hi, "max_groups": g_hi, **cand}
            set_batch_tuning([rule] if cand else [], best)
            ms = _time_batch(inst, steps)
            log[f"bucket {r_hi}x{g_hi} {json.dumps(cand)}"] = ms
            if cand_ms is None or ms < cand_ms * 0.98:
                cand_best, cand_ms = cand, ms
        if cand_best:
            rules.append({"max_rows": r_hi, "max_groups": g_hi, **cand_best})
        if verbose:
            print(f"batch bucket rows<={r_hi} groups<={g_hi}: {cand_best} {cand_ms:.3f} ms", flush=True)
        del inst
    set_batch_tuning(rules, best)
    if verbose:
        print(f"batch launch: {best} {best_ms:.3f} ms", flush=True)
    return {"launch": best, "rules": rules}, {"launch_ms": best_ms, "trials": log}


def bucket_sizes(rng, r_hi: int, g_hi: int) -> List[Tuple[int, int]]:
    """(rows, groups) of the instances a bucket is tuned on: rows
    log-uniform over the top sixteenth of the bucket's row range (from 4097
    for the smallest), groups log-uniform over the top sixteenth of its group
    range, the open-ended bucket from 65536 to 2^20; never more groups than
    rows."""
    import numpy as np
    lo_r = 4097 if r_hi == 16384 else r_hi // 16
    hi_g = min(g_hi, 1 << 20)
    lo_g = max(2, min(g_hi // 16, 65536))
    sizes = []
    for _ in range(32 if r_hi <= 262144 else 8):
        n = int(np.exp(rng.uniform(np.log(lo_r), np.log(r_hi))))
        g = int(min(n, np.exp(rng.uniform(np.log(lo_g), np.log(hi_g)))))
        sizes.append((n, max(2, g)))
    return sizes


def order_rules(rules: Sequence[Dict]) -> List[Dict]:
    """Smallest buckets first, so the first match is the tightest bucket."""
    return sorted(rules, key=lambda r: (int(r["max_rows"]), int(r["max_groups"])))


# -- the search (needs a GPU) ---------------------------------------------------
def _workload(rows: int, groups: int, seed: int = 0):
    """Synthetic bucket input: int64 keys uniform over `groups` distinct
    values; int64, float64 and float32 values, 10% nulls each; sum, count,
    min, max, mean per value column (the 100M-row benchmark's request)."""
    import torch
    from . import aggregation as agg
    from .column import Column, Table, pack_mask
    from .groupby import GroupByRequest
    from .types import TypeId
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    distinct = torch.randint(-2**62, 2**62, (groups,), device="cuda", generator=g, dtype=torch.int64)
    key = distinct[torch.randint(0, groups, (rows,), device="cuda", generator=g)]
    vals = [torch.randint(-10**9, 10**9, (rows,), device="cuda", generator=g, dtype=torch.int64),
            torch.randn(rows, device="cuda", generator=g, dtype=torch.float64),
            torch.rand(rows, device="cuda", generator=g, dtype=torch.float32)]
    masks = [pack_mask(torch.rand(rows, device="cuda", generator=g) >= 0.1) for _ in range(3)]
    aggs = [agg.sum(), agg.count(), agg.min(), agg.max(), agg.mean()]
    reqs = [GroupByRequest(Column(t, v, m), aggs)
            for t, v, m in zip((TypeId.INT64, TypeId.FLOAT64, TypeId.FLOAT32), vals, masks)]
    return Table([Column(TypeId.INT64, key)]), reqs


def _time(keys, reqs, tuning: Dict[str, int], steps: int) -> float:
    import torch
    from .groupby import GroupBy
    gb = GroupBy(keys)
    if tuning:
        gb.set_tuning(**tuning)
    gb.aggregate(reqs)  # warm (allocator pool, first launches)
    stream = torch.cuda.current_stream()
    times = []
    for _ in range(steps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        gb.aggregate(reqs)
        b.record(stream)
        b.synchronize()
        times.append(a.elapsed_time(b))
    times.sort()
    return times[len(times) // 2]


def tune_bucket(rows: int, groups: int, steps: int = 5, verbose: bool = False) -> Tuple[Dict[str, int], Dict]:
    """Coordinate descent: mode, then (for the chosen mode) the partition
    launch shape or the shared-memory table, then the load factor."""
    keys, reqs = _workload(rows, groups)
    log = {}
    best: Dict[str, int] = {}
    best_ms = _time(keys, reqs, best, steps)
    log["default"] = best_ms
    for stage in (_MODES, _SCATTER, _SMEM, _LOAD):
        if stage is _SCATTER and best.get("force_mode", -1) not in (-1, 2):
            continue
        if stage is _SMEM and best.get("force_mode", -1) not in (-1, 1):
            continue
        for cand in stage:
            t = dict(best)
            t.update(cand)
            try:
                ms = _time(keys, reqs, t, steps)
            except Exception as e:  # a setting the call rejects is skipped
                log[json.dumps(t)] = str(e)
                continue
            log[json.dumps(t)] = ms
            if ms < best_ms * 0.98:
                best, best_ms = t, ms
    if verbose:
        print(f"rows={rows} groups={groups}: {best} {best_ms:.3f} ms", flush=True)
    return best, {"best_ms": best_ms, "trials": log}


def tune(buckets: Sequence[Tuple[int, int]] = DEFAULT_BUCKETS, steps: int = 5, verbose: bool = False):
    clear()
    rules, meta = [], {"when": time.strftime("%Y-%m-%dT%H:%M:%S"), "buckets": {}}
    for rows, groups in buckets:
        t, info = tune_bucket(rows, groups, steps, verbose)
        # tuned on a single 64-bit key: applies to one-word keys only
        rules.append({"max_rows": rows, "max_groups": groups, "key_words": 1, "tuning": t})
        meta["buckets"][f"{rows}x{groups}"] = info
    return order_rules(rules), meta


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--out", default=TUNING_FILE)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--max-rows", type=int, default=1 << 27, help="skip buckets with more rows")
    ap.add_argument("--what", default="all", choices=["all", "single", "batch"],
                    help="tune single-query rules, batched launches, or both (the other part of an "
                         "existing file is kept)")
    args = ap.parse_args()
    import torch
    name = torch.cuda.get_device_name(0)
    old = {}
    if os.path.exists(args.out):
        with open(args.out) as f:
            old = json.load(f)
    rules, meta = old.get("rules", []), old.get("meta", {})
    batch = old.get("batch")
    if args.what in ("all", "single"):
        buckets = [b for b in DEFAULT_BUCKETS if b[0] <= args.max_rows]
        rules, meta = tune(buckets, args.steps, verbose=True)
        meta["device"] = name
    if args.what in ("all", "batch"):
        bt, binfo = tune_batch(steps=max(2, args.steps // 2), verbose=True)
        batch = {**bt, "meta": {"device": name, "when": time.strftime("%Y-%m-%dT%H:%M:%S"), **binfo}}
    with open(args.out, "w") as f:
        json.dump({"rules": list(rules), "meta": meta, **({"batch": batch} if batch else {})}, f, indent=1)
    print(f"wrote {len(rules)} rules{' and batch tuning' if batch else ''} to {args.out}")


if __name__ == "__main__":
    main()
