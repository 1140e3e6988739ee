"""Benchmark of the B200 hash groupby-aggregate engine.

Workload (the 100M-row single groupby): 100,000,000 rows; int64 key drawn
uniformly from 1,000,000 distinct random 64-bit values; v1 int64 uniform in
[-1e9, 1e9], v2 float64 normal(0,1), v3 float32 lognormal(0,1); an independent
10% Bernoulli null mask per value column; SUM/COUNT/MIN/MAX/MEAN on each value
column; seed 1.  Synthetic data, generated on the device.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl engine|reference]

Prints one JSON line (rank 0).  `value` is rows/s of the whole aggregate() call
with inputs resident in HBM (device-timed with CUDA events, max over ranks);
`e2e` is the same call through the public API with pinned host inputs copied
in and results copied out inside the timed region.  `--impl reference` times
the CPU restatement of the reference algorithm (oracle/) on the host cores, one
full pass over the same 100M-row workload per step.  At one GPU the line also
carries `extra`: the Zipf two-key, 1M-row, batched and serving workloads,
measured after the main one (`--no-extra` skips them).  `--check` compares the
last timed call's result with the oracle on the same inputs, group by group,
after the timed region.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_ROWS = 100_000_000
N_DISTINCT = 1_000_000
SEED = 1
NULL_FRAC = 0.10
AGG_NAMES = ["sum", "count", "min", "max", "mean"]
METRIC = "groupby rows/s (100M rows, 1M groups, 3 value cols, sum/count/min/max/mean)"
CPU_SAMPLE_ROWS = N_ROWS

# Kernels whose device time the roofline covers, by engine mode (0 global
# table, 1 shared-memory stage, 2 hash-partitioned two-pass).
KERNELS_BY_MODE = {0: "k_aggregate<false>", 1: "k_aggregate<true>",
                   2: "k_part_scatter_bulk + k_part_aggregate"}
# DRAM bytes (read + write) of those kernels per launch, from an ncu capture
# of a smaller case of the same workload scaled up; the capture command and
# the per-kernel figures are in profiles/.
# Mode 2: (bytes per row, bytes per group); the partitioned copy is written
# and read once, and the dense slots are written once per group.
TRAFFIC_MODEL = {2: (84.93, 75.1)}
TRAFFIC_SOURCE = {2: "ncu dram__bytes_read.sum + dram__bytes_write.sum of both kernels on the 20M-row "
                     "case, scaled by rows (and by groups for the dense-slot writes); "
                     "profiles/k_part_scatter_bulk_k_part_aggregate_20M.md"}


def algorithmic_bytes(n_rows: int, n_groups: int) -> tuple[float, float]:
    """Bytes the groupby must move at least once: every input column and mask
    read once, every output column and mask written once."""
    mask = ((n_rows + 31) // 32) * 4
    inp = n_rows * (8 + 8 + 8 + 4) + 3 * mask
    gmask = ((n_groups + 31) // 32) * 4
    # keys 8; per value col: sum, count(4), min, max, mean(8) + masks for sum/min/max/mean
    out = n_groups * 8 + n_groups * (8 + 4 + 8 + 8 + 8) * 2 + n_groups * (4 + 4 + 4 + 4 + 8) + 3 * 4 * gmask
    return float(inp), float(out)


WORKLOAD = ("groupby 100M rows, int64 key over 1M distinct values, v1 int64, v2 f64, v3 f32, "
            "10% nulls, sum/count/min/max/mean")


def workload_config(rows_per_rank: int, world: int, groups: int) -> dict:
    """The `config` object of both arms (engine and reference)."""
    return {"workload": WORKLOAD, "rows": rows_per_rank * world, "rows_per_rank": rows_per_rank,
            "groups": groups,
            "parallelism": (f"rows sharded over {world} ranks, partial aggregate + NCCL all-to-all by key "
                            f"owner + merge") if world > 1 else "single",
            "l2": "inputs (2.84 GB) larger than L2 (126 MB); no flush needed"}


def make_inputs_host(n: int, seed: int = SEED):
    rng = np.random.default_rng(seed)
    distinct = np.unique(rng.integers(-2**63, 2**63 - 1, N_DISTINCT, dtype=np.int64))
    key = distinct[rng.integers(0, distinct.size, n)]
    v1 = rng.integers(-10**9, 10**9, n, endpoint=True).astype(np.int64)
    v2 = rng.normal(size=n)
    v3 = rng.lognormal(size=n).astype(np.float32)
    masks = [rng.random(n) >= NULL_FRAC for _ in range(3)]
    return key, [v1, v2, v3], masks


def make_inputs_device(n: int, seed: int, device, key_seed=None):
    import torch
    from cudf_b200.column import pack_mask
    rng = np.random.default_rng(seed if key_seed is None else key_seed)
    distinct = torch.from_numpy(np.unique(rng.integers(-2**63, 2**63 - 1, N_DISTINCT, dtype=np.int64))).to(device)
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    idx = torch.randint(0, distinct.numel(), (n,), device=device, generator=g)
    key = distinct[idx]
    del idx
    v1 = torch.randint(-10**9, 10**9 + 1, (n,), device=device, generator=g, dtype=torch.int64)
    v2 = torch.randn(n, device=device, generator=g, dtype=torch.float64)
    v3 = torch.empty(n, device=device, dtype=torch.float32).log_normal_(0.0, 1.0, generator=g)
    masks = [pack_mask(torch.rand(n, device=device, generator=g) >= NULL_FRAC) for _ in range(3)]
    return key, [v1, v2, v3], masks


class ClockSampler:
    """SM clocks and throttle reasons during the timed region, read through NVML
    (the library nvidia-smi uses) from a background thread every 50 ms.  An
    nvidia-smi subprocess polling the driver stalls CUDA API calls for tens of
    milliseconds, which would show up in the timed region; in-process NVML
    queries cost microseconds once each kind has been made once."""

    REASONS = {"hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40,
               "sw_power_cap": 0x4}

    def __init__(self, index: int, period: float = 0.05):
        self.index = index
        self.period = period
        self.samples = []
        self.max_mhz = None
        self._stop = threading.Event()
        self.ok = False

    def __enter__(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            vis = os.environ.get("CUDA_VISIBLE_DEVICES")
            idx = self.index
            if vis:
                try:
                    idx = int(vis.split(",")[self.index])
                except ValueError:
                    idx = self.index
            self.h = pynvml.nvmlDeviceGetHandleByIndex(idx)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
            # the first query of each kind costs milliseconds inside the
            # driver: make them here, before the timed region starts
            pynvml.nvmlDeviceGetClockInfo(self.h, pynvml.NVML_CLOCK_SM)
            pynvml.nvmlDeviceGetCurrentClocksEventReasons(self.h)
            self.ok = True
            self.t = threading.Thread(target=self._run, daemon=True)
            self.t.start()
        except Exception:
            self.ok = False
        return self

    def _run(self):
        while not self._stop.is_set():
            try:
                mhz = self.nv.nvmlDeviceGetClockInfo(self.h, self.nv.NVML_CLOCK_SM)
                rs = self.nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                self.samples.append((mhz, rs))
            except Exception:
                pass
            self._stop.wait(self.period)

    def __exit__(self, *a):
        self._stop.set()
        if self.ok:
            self.t.join(timeout=2)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["unsampled"]}
        reasons = set()
        for _, rs in self.samples:
            for name, bit in self.REASONS.items():
                if rs & bit:
                    reasons.add(name)
        return {"sm_mhz": float(np.median([m for m, _ in self.samples])), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(reasons), "samples": len(self.samples), "source": "nvml"}


def dist_setup():
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def _oracle_inputs(key, vals, masks):
    from oracle import oracle as O
    kinds = [O.SUM, O.COUNT_VALID, O.MIN, O.MAX, O.MEAN]
    kc = O.HostColumn(O.INT64, key)
    reqs = [(O.HostColumn(O.INT64, vals[0], masks[0]), kinds),
            (O.HostColumn(O.FLOAT64, vals[1], masks[1]), kinds),
            (O.HostColumn(O.FLOAT32, vals[2], masks[2]), kinds)]
    return [kc], reqs


def cpu_reference(n_rows: int, threads: int, steps: int = 1, warmup: int = 1):
    """The oracle (CPU restatement of the reference algorithm) over n_rows rows of
    the workload's distributions, `warmup` untimed and `steps` timed full passes.
    Returns (rows/s over the timed passes, seconds per pass, groups)."""
    from oracle import oracle as O
    key, vals, masks = make_inputs_host(n_rows)
    keys, reqs = _oracle_inputs(key, vals, masks)
    r = None
    for _ in range(warmup):
        r = O.groupby(keys, reqs, nthreads=threads)
    t = time.perf_counter()
    for _ in range(steps):
        r = O.groupby(keys, reqs, nthreads=threads)
    dt = (time.perf_counter() - t) / max(1, steps)
    return n_rows / dt, dt, r.num_groups


def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    n = args.rows
    v, sec, groups = cpu_reference(n, threads, steps=max(1, args.steps), warmup=args.warmup)
    line = {"metric": METRIC, "value": v, "unit": "rows/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": sec * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int64/f64/f32", "data": "synthetic",
            "impl": "reference",
            "config": workload_config(n, 1, groups),
            "cpu_baseline": {"value": v, "unit": "rows/s", "cores": threads, "kind": "port",
                             "sample": f"every step one full pass over {n} rows with the workload's "
                                       f"distributions (numpy seed 1, 1M distinct keys), oracle/gb_oracle.c "
                                       f"(rows hash-partitioned by key, partitions aggregated in parallel) "
                                       f"with {threads} threads"},
            "e2e": {"value": v, "unit": "rows/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def check_with_oracle(host_keys, host_reqs, include_null_keys, uk, res):
    """Compares an engine result with the oracle on the same host inputs, group by
    group after sorting by key: integer results bit-exact, float SUM/MEAN within
    the oracle's per-group bound.  Raises AssertionError on a mismatch."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import parity
    from oracle import oracle as O
    o = O.groupby(host_keys, host_reqs, include_null_keys=include_null_keys, nthreads=os.cpu_count() or 1)
    parity.compare(o, parity.gpu_pairs(uk), [parity.gpu_pairs(t) for t in res],
                   [list(kinds) for _, kinds in host_reqs], None)
    return o.num_groups


def run_engine(args):
    import torch
    world, rank, local = dist_setup()
    import cudf_b200 as cb
    from cudf_b200 import aggregation as agg
    from cudf_b200.types import TypeId

    dev = torch.device("cuda", local if world > 1 else 0)
    torch.cuda.set_device(dev)
    n = args.rows
    # every rank: its own rows drawn over the same 1M distinct keys
    key, vals, masks = make_inputs_device(n, SEED + rank, dev, key_seed=SEED)
    torch.cuda.synchronize()
    aggs = [agg.sum(), agg.count(), agg.min(), agg.max(), agg.mean()]
    kcol = cb.Column(TypeId.INT64, key)
    vcols = [cb.Column(TypeId.INT64, vals[0], masks[0]), cb.Column(TypeId.FLOAT64, vals[1], masks[1]),
             cb.Column(TypeId.FLOAT32, vals[2], masks[2])]
    gb = cb.GroupBy(cb.Table([kcol]))
    gb.set_tuning(**json.loads(args.tuning)) if args.tuning else None
    gb.set_profile(True)
    reqs = [cb.GroupByRequest(c, aggs) for c in vcols]
    stream = torch.cuda.current_stream()

    if world > 1:
        from cudf_b200.distributed import distributed_groupby
        from cudf_b200.types import Kind
        kinds = [Kind.SUM, Kind.COUNT_VALID, Kind.MIN, Kind.MAX, Kind.MEAN]
        dkeys = [(key, None, TypeId.INT64)]
        # the packed validity words go to the engine as they are
        dreqs = [((vals[0], masks[0], TypeId.INT64), kinds),
                 ((vals[1], masks[1], TypeId.FLOAT64), kinds),
                 ((vals[2], masks[2], TypeId.FLOAT32), kinds)]

        class _Res:
            def __init__(self, k):
                self.k = k

            def num_rows(self):
                return int(self.k[0][0].shape[0])

        def step():
            mk, mres = distributed_groupby(dkeys, dreqs)
            return _Res(mk), mres
    else:
        def step():
            return gb.aggregate(reqs)

    for _ in range(args.warmup):
        out = step()
    del out
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    kernel_ms, scatter_ms = [], []
    last_stats = {}
    groups = 0
    launches = 0
    with ClockSampler(dev.index) as clk:
        torch.cuda.synchronize()
        start.record(stream)
        for _ in range(args.steps):
            uk, res = step()
            st = gb.stats()
            kernel_ms.append(st["agg_kernel_ms"])
            scatter_ms.append(st["scatter_ms"])
            last_stats = st
            launches += st["kernels"]
            groups = uk.num_rows()
        if world > 1:
            t = torch.tensor([groups], device=dev, dtype=torch.int64)
            torch.distributed.all_reduce(t)
            groups = int(t.item())
        end.record(stream)
        torch.cuda.synchronize()
    ms = start.elapsed_time(end) / args.steps
    if world > 1:
        t = torch.tensor([ms], device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t.item())
    checked = None
    if args.check and world == 1:
        # outside the timed region: the last timed call's groups against the
        # oracle on the same inputs
        t0 = time.perf_counter()
        hk, hr = _oracle_inputs(key.cpu().numpy(), [v.cpu().numpy() for v in vals],
                                [cb.column.unpack_mask(m, n).cpu().numpy() for m in masks])
        g = check_with_oracle(hk, hr, False, uk, res)
        checked = {"groups": g, "result": "match", "seconds": round(time.perf_counter() - t0, 1)}
        del hk, hr
    del uk, res

    # ---- e2e through the public API from pinned host buffers ----
    hkey = key.cpu().pin_memory()
    hvals = [v.cpu().pin_memory() for v in vals]
    hmasks = [m.cpu().pin_memory() for m in masks]
    # two device copies of the inputs: while one step aggregates from one,
    # the next step's inputs stream into the other on a copy stream
    bufs = []
    for _ in range(2):
        dkey = torch.empty_like(key)
        dvals = [torch.empty_like(v) for v in vals]
        dmasks = [torch.empty_like(m) for m in masks]
        ek = cb.Column(TypeId.INT64, dkey)
        ev = [cb.Column(TypeId.INT64, dvals[0], dmasks[0]), cb.Column(TypeId.FLOAT64, dvals[1], dmasks[1]),
              cb.Column(TypeId.FLOAT32, dvals[2], dmasks[2])]
        bufs.append(([dkey, *dvals, *dmasks], ek, [cb.GroupByRequest(c, aggs) for c in ev]))
    del key, vals, masks, kcol, vcols, reqs, gb
    hosts = [hkey, *hvals, *hmasks]
    h2d = sum(t.numel() * t.element_size() for t in hosts)
    d2h = 0
    staging = cb.HostStaging()  # pinned result buffers, reused every step
    copy_stream = torch.cuda.Stream()

    def upload(b, s):
        with torch.cuda.stream(s):
            for d, h in zip(bufs[b][0], hosts):
                d.copy_(h, non_blocking=True)

    def compute(b):
        nonlocal d2h
        if world > 1:
            # the whole multi-GPU call: partial aggregate, exchange, merge
            from cudf_b200.distributed import distributed_groupby
            from cudf_b200.types import Kind
            kinds = [Kind.SUM, Kind.COUNT_VALID, Kind.MIN, Kind.MAX, Kind.MEAN]
            t = bufs[b][0]
            types = (TypeId.INT64, TypeId.FLOAT64, TypeId.FLOAT32)
            mk, mres = distributed_groupby(
                [(t[0], None, TypeId.INT64)],
                [((t[1 + i], t[4 + i], types[i]), kinds) for i in range(3)])
            outs = [d for d, _, _ in mk] + [x for per in mres for pair in per for x in pair if x is not None]
        else:
            uk2, res2 = cb.GroupBy(cb.Table([bufs[b][1]])).aggregate(bufs[b][2], stream=stream)
            outs = [c.values() for c in uk2.columns] + [c.values() for t in res2 for c in t.columns]
            outs += [c.mask for t in res2 for c in t.columns if c.mask is not None]
        host = staging.to_host(outs, stream)
        d2h = sum(h.nbytes for h in host)
        return host

    def e2e_sequential(steps):
        for _ in range(steps):
            upload(0, stream)
            compute(0)

    def e2e_pipelined(steps):
        copied = [torch.cuda.Event(), torch.cuda.Event()]
        used = [torch.cuda.Event(), torch.cuda.Event()]
        copy_stream.wait_stream(stream)
        upload(0, copy_stream)
        copied[0].record(copy_stream)
        for i in range(steps):
            cur, nxt = i % 2, (i + 1) % 2
            if i + 1 < steps:
                if i >= 1:
                    copy_stream.wait_event(used[nxt])
                upload(nxt, copy_stream)
                copied[nxt].record(copy_stream)
            stream.wait_event(copied[cur])
            compute(cur)
            used[cur].record(stream)

    def timed(fn, steps):
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fn(steps)
        b.record(stream)
        torch.cuda.synchronize()
        t = a.elapsed_time(b) / steps
        if world > 1:
            tt = torch.tensor([t], device=dev)
            torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.MAX)
            t = float(tt.item())
        return t

    e2e_sequential(1)  # warm
    e_steps = max(2, min(args.steps, 4))
    e_seq_ms = timed(e2e_sequential, e_steps)
    e_ms = timed(e2e_pipelined, e_steps)

    if rank == 0:
        peaks = {}
        try:
            peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        except Exception:
            pass
        peak = float(peaks.get("hbm_gbs", 6650.0))
        peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
        inp, outb = algorithmic_bytes(n, groups)
        kmean = float(np.mean(kernel_ms)) if kernel_ms else float("nan")
        smean = float(np.mean(scatter_ms)) if scatter_ms else 0.0
        # every input read once plus every output written once, over the
        # device time of the dominant kernels of one call
        achieved = (inp + outb) / (kmean * 1e-3) / 1e9
        mode = last_stats.get("mode", -1)
        kname = KERNELS_BY_MODE.get(mode, "unknown")
        tm = TRAFFIC_MODEL.get(mode)
        traffic = None if tm is None else tm[0] * n + tm[1] * groups / world
        value = world * n / (ms * 1e-3)
        line = {
            "metric": METRIC, "value": value, "unit": "rows/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int64/f64/f32", "data": "synthetic",
            "config": workload_config(n, world, groups),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "kernel": kname,
                         "kernel_ms": kmean, "kernel_ms_steps": [round(x, 3) for x in kernel_ms],
                         "kernel_split_ms": {"partition_scatter": smean,
                                                                 "partition_aggregate": kmean - smean}
                         if mode == 2 else None,
                         "algorithmic_bytes": inp + outb, "input_bytes": inp, "output_bytes": outb,
                         "peak_source": peak_src,
                         "traffic_source": TRAFFIC_SOURCE.get(mode),
                         "whole_call_frac": (inp + outb) / (ms * 1e-3) / 1e9 / peak},
            "e2e": {"value": world * n / (e_ms * 1e-3), "unit": "rows/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "ms_per_step": e_ms,
                    "how": "pinned host inputs copied in and all results copied back every step; the next "
                           "step's upload overlaps this step's aggregate (two device input buffers)",
                    "sequential_value": world * n / (e_seq_ms * 1e-3)},
            "gpu_launches": launches,
            "engine": last_stats,
            "clocks": clk.summary(),
        }
        if checked is not None:
            line["check"] = checked
        if not args.no_cpu_baseline and world == 1:
            threads = os.cpu_count() or 1
            v, _, _ = cpu_reference(args.cpu_sample, threads)
            line["cpu_baseline"] = {"value": v, "unit": "rows/s", "cores": threads, "kind": "port",
                                    "sample": f"one full pass over {args.cpu_sample} rows with the workload's "
                                              f"distributions (numpy seed 1, 1M distinct keys) through "
                                              f"oracle/gb_oracle.c, {threads} threads"}
        if not args.no_extra and world == 1:
            bufs.clear()
            hosts.clear()
            torch.cuda.empty_cache()
            line["extra"] = run_extras(args)
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return 0


def run_batch(args):
    """4096 independent groupbys (rows log-uniform in [1e3, 4e6], int32 keys of
    cardinality log-uniform in [4, 1e5], int64 values in [0, 1e6] and float64
    normal values with 5% nulls; sum/count/min/max/mean; seed 3): one batched,
    graph-replayed launch against one plain aggregate() call per instance."""
    import torch
    import cudf_b200 as cb
    from cudf_b200 import aggregation as agg
    from cudf_b200.column import pack_mask
    from cudf_b200.types import TypeId
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    rng = np.random.default_rng(3)
    ninst = args.instances
    rows = np.exp(rng.uniform(np.log(1e3), np.log(4e6), ninst)).astype(np.int64)
    cards = np.exp(rng.uniform(np.log(4), np.log(1e5), ninst)).astype(np.int64)
    g = torch.Generator(device=dev)
    g.manual_seed(3)
    inst = []
    for n, c in zip(rows.tolist(), cards.tolist()):
        k = torch.randint(0, int(c), (n,), device=dev, generator=g, dtype=torch.int32)
        v1 = torch.randint(0, 10**6 + 1, (n,), device=dev, generator=g, dtype=torch.int64)
        v2 = torch.randn(n, device=dev, generator=g, dtype=torch.float64)
        m1 = pack_mask(torch.rand(n, device=dev, generator=g) >= 0.05)
        m2 = pack_mask(torch.rand(n, device=dev, generator=g) >= 0.05)
        inst.append((cb.Table([cb.Column(TypeId.INT32, k)]),
                     [cb.GroupByRequest(cb.Column(TypeId.INT64, v1, m1), [agg.sum(), agg.count(), agg.min(), agg.max(), agg.mean()]),
                      cb.GroupByRequest(cb.Column(TypeId.FLOAT64, v2, m2), [agg.sum(), agg.count(), agg.min(), agg.max(), agg.mean()])]))
    torch.cuda.synchronize()
    total_rows = int(rows.sum())
    stream = torch.cuda.current_stream()
    # plain: one aggregate() per instance
    def plain_pass():
        for kt, rq in inst:
            uk, res = cb.GroupBy(kt).aggregate(rq)
    plain_pass()  # warm
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    plain_pass()
    b.record(stream)
    torch.cuda.synchronize()
    plain_ms = a.elapsed_time(b)
    # batched + graph replay
    t0 = time.perf_counter()
    bg = cb.BatchGroupBy(inst, use_graph=True)
    torch.cuda.synchronize()
    prepare_ms = (time.perf_counter() - t0) * 1e3
    for _ in range(args.warmup):
        bg.run()
    torch.cuda.synchronize()
    a.record(stream)
    for _ in range(args.steps):
        bg.run()
    b.record(stream)
    torch.cuda.synchronize()
    batch_ms = a.elapsed_time(b) / args.steps
    st = bg.stats()
    line = {"metric": f"batched groupby instances/s ({ninst} instances, {total_rows} rows)",
            "value": ninst / (batch_ms * 1e-3), "unit": "instances/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": batch_ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int32/int64/f64", "data": "synthetic",
            "config": {"workload": "4096 groupbys, rows log-uniform [1e3,4e6], int32 keys with cardinality "
                                   "log-uniform [4,1e5], int64+f64 values, 5% nulls, sum/count/min/max/mean",
                       "instances": ninst, "rows": total_rows},
            "plain": {"ms_per_pass": plain_ms, "instances_per_s": ninst / (plain_ms * 1e-3),
                      "rows_per_s": total_rows / (plain_ms * 1e-3)},
            "batched": {"ms_per_pass": batch_ms, "rows_per_s": total_rows / (batch_ms * 1e-3),
                        "prepare_ms": prepare_ms, **st},
            "speedup_vs_plain": plain_ms / batch_ms}
    return line


def run_serve(args):
    """Serving stream: Poisson arrivals at --rate queries/s for --duration s;
    each query a groupby over int64 keys (cardinality log-uniform [10, 1e6]),
    rows log-uniform [1e4, 2e7], int64 and float64 values with 10% nulls,
    sum/count/mean; admission capped at 150 GB; seed 4.  Queries read prefixes of
    a pool of device-resident tables.  The batched server (continuous batching)
    is compared with plain one-aggregate()-per-query serving in arrival order."""
    import threading
    import torch
    import cudf_b200 as cb
    from cudf_b200 import aggregation as agg
    from cudf_b200.column import pack_mask
    from cudf_b200.types import TypeId
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    rng = np.random.default_rng(4)
    pool_n = 20_000_000
    pool = []
    g = torch.Generator(device=dev)
    g.manual_seed(4)
    cards = np.exp(np.linspace(np.log(10), np.log(1e6), args.pool)).astype(np.int64)
    for c in cards.tolist():
        k = torch.randint(0, int(c), (pool_n,), device=dev, generator=g, dtype=torch.int64) * 7919
        v1 = torch.randint(-10**9, 10**9 + 1, (pool_n,), device=dev, generator=g, dtype=torch.int64)
        v2 = torch.randn(pool_n, device=dev, generator=g, dtype=torch.float64)
        m1 = pack_mask(torch.rand(pool_n, device=dev, generator=g) >= 0.1)
        m2 = pack_mask(torch.rand(pool_n, device=dev, generator=g) >= 0.1)
        pool.append((k, v1, v2, m1, m2))
    torch.cuda.synchronize()

    def one_stream(rate):
        nq = int(rng.poisson(rate * args.duration))
        arrivals = np.sort(rng.uniform(0, args.duration, nq))
        which = rng.integers(0, args.pool, nq)
        rows = np.exp(rng.uniform(np.log(1e4), np.log(2e7), nq)).astype(np.int64)

        def query(i):
            k, v1, v2, m1, m2 = pool[which[i]]
            n = int(rows[i])
            kt = cb.Table([cb.Column(TypeId.INT64, k, size=n)])
            aggs = [agg.sum(), agg.count(), agg.mean()]
            return kt, [cb.GroupByRequest(cb.Column(TypeId.INT64, v1, m1, size=n), aggs),
                        cb.GroupByRequest(cb.Column(TypeId.FLOAT64, v2, m2, size=n), aggs)]

        qs = [query(i) for i in range(nq)]
        # plain single-query latency (no queueing): a sample of queries run alone
        for i in range(5):
            cb.GroupBy(qs[i][0]).aggregate(qs[i][1])
        alone = []
        for i in range(min(nq, 200)):
            t = time.perf_counter()
            cb.GroupBy(qs[i][0]).aggregate(qs[i][1])
            alone.append(time.perf_counter() - t)
        alone_p50 = float(np.median(alone))

        def plain():
            lat = []
            t0 = time.perf_counter()
            for i in range(nq):
                now = time.perf_counter() - t0
                if now < arrivals[i]:
                    time.sleep(arrivals[i] - now)
                cb.GroupBy(qs[i][0]).aggregate(qs[i][1])
                lat.append(time.perf_counter() - t0 - arrivals[i])
            span = time.perf_counter() - t0
            return {"queries_per_s": nq / span, "p50_s": float(np.percentile(lat, 50)),
                    "p99_s": float(np.percentile(lat, 99)), "completed": nq}

        def batched():
            srv = cb.Server(memory_cap_bytes=150 << 30, workers=args.workers, direct_rows=args.direct_rows)
            ids = [None] * nq
            done = threading.Event()

            def collector():
                for i in range(nq):
                    while ids[i] is None:
                        time.sleep(1e-4)
                    srv.wait(ids[i], timeout_s=600)
                    srv.release(ids[i])
                done.set()

            th = threading.Thread(target=collector)
            th.start()
            try:
                t0 = time.perf_counter()
                for i in range(nq):
                    now = time.perf_counter() - t0
                    if now < arrivals[i]:
                        time.sleep(arrivals[i] - now)
                    ids[i] = srv.submit(*qs[i])
                th.join()
                return srv.stats()
            finally:
                srv.close()

        b = batched()
        p = plain()
        line = {"metric": f"served groupby queries/s (Poisson {rate}/s for {args.duration}s)",
                "value": b["queries_per_s"], "unit": "queries/s", "n_gpus": 1, "steps": 1, "warmup": 0,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64/f64",
                "data": "synthetic",
                "config": {"workload": "serving stream: int64 keys (cardinality log-uniform [10,1e6]), rows "
                                       "log-uniform [1e4,2e7], int64+f64 values 10% nulls, sum/count/mean, "
                                       "admission cap 150 GB", "queries": nq, "rate": rate,
                           "duration_s": args.duration, "pool_tables": args.pool, "workers": args.workers,
                           "mean_rows": float(rows.mean())},
                "batched": b, "plain": p, "plain_single_query_latency_s": alone_p50,
                "qps_ratio_vs_plain": b["queries_per_s"] / p["queries_per_s"],
                "p99_over_plain_single": b["p99_s"] / alone_p50}
        return line

    rates = [float(r) for r in args.rates.split(",")] if args.rates else [args.rate]
    lines = [one_stream(r) for r in rates]
    line = lines[0]
    if len(lines) > 1:
        # offered-rate curve: where the plain loop saturates and what the
        # server delivers there
        line["curve"] = [{"offered_qps": r, "batched_qps": l["batched"]["queries_per_s"],
                          "plain_qps": l["plain"]["queries_per_s"], "qps_ratio_vs_plain": l["qps_ratio_vs_plain"],
                          "batched_p99_s": l["batched"]["p99_s"], "plain_p99_s": l["plain"]["p99_s"],
                          "p99_over_plain_single": l["p99_over_plain_single"], "queries": l["config"]["queries"]}
                         for r, l in zip(rates, lines)]
    return line


def zipf_inputs_device(n: int, dev):
    """Zipf two-key workload on the device (seed 2): k1 int32, k2 int64,
    packed key masks (5% nulls each), v_int int64 [0, 1e6], v_f f64 [0, 1)."""
    import torch
    from cudf_b200.column import pack_mask
    g = torch.Generator(device=dev)
    g.manual_seed(2)
    p = _zipf_pairs(n, dev, g)
    k1 = (p // 1000).to(torch.int32)
    k2 = p % 1000
    del p
    km = [pack_mask(torch.rand(n, device=dev, generator=g) >= 0.05) for _ in range(2)]
    vi = torch.randint(0, 10**6 + 1, (n,), device=dev, generator=g, dtype=torch.int64)
    vf = torch.rand(n, device=dev, generator=g, dtype=torch.float64)
    return k1, k2, km, vi, vf


def small_inputs_device(n: int, dev):
    """1M-row workload on the device (seed 0): int32 key over 1000 values,
    v1 int64 [0, 1e6], v2 f64 [0, 1), no nulls."""
    import torch
    g = torch.Generator(device=dev)
    g.manual_seed(0)
    k = torch.randint(0, 1000, (n,), device=dev, generator=g, dtype=torch.int32)
    v1 = torch.randint(0, 10**6 + 1, (n,), device=dev, generator=g, dtype=torch.int64)
    v2 = torch.rand(n, device=dev, generator=g, dtype=torch.float64)
    return k, v1, v2


def _flat(cols):
    out = []
    for c in cols:
        out.extend(c if isinstance(c, (list, tuple)) else [c])
    return out


def config_oracle_inputs(workload, host, n):
    """Oracle columns for the zipf/small workloads from host copies of the
    device inputs (in the order of `_flat`)."""
    from oracle import oracle as O
    if workload == "zipf":
        k1, k2, m1, m2, vi, vf = [t.numpy() for t in host]
        kinds = [O.SUM, O.COUNT_VALID, O.MAX]
        keys = [O.HostColumn(O.INT32, k1, packed=m1.view(np.uint32)),
                O.HostColumn(O.INT64, k2, packed=m2.view(np.uint32))]
        return keys, [(O.HostColumn(O.INT64, vi), kinds), (O.HostColumn(O.FLOAT64, vf), kinds)], True
    k, v1, v2 = [t.numpy() for t in host]
    return ([O.HostColumn(O.INT32, k)],
            [(O.HostColumn(O.INT64, v1), [O.SUM, O.COUNT_VALID, O.MIN, O.MAX]),
             (O.HostColumn(O.FLOAT64, v2), [O.MEAN])], False)


def _zipf_pairs(n, dev, g, s=1.1, support=50_000_000):
    """Pair indices with P(p) proportional to (p+1)^-s on [0, support), by the
    continuous inverse CDF of that power law (seeded torch generator)."""
    import torch
    u = torch.rand(n, device=dev, generator=g, dtype=torch.float64)
    a = 1.0 - s
    top = (support + 1.0) ** a
    x = (1.0 - u * (1.0 - top)) ** (1.0 / a) - 1.0
    return x.floor().clamp_(0, support - 1).to(torch.int64)


def run_config(args):
    """The other single-GPU shapes of the benchmark, one aggregate() per step:
      zipf  -- 100M rows; (k1 int32, k2 int64) = divmod(p, 1000) with p Zipf(1.1)
               on [0, 50M); 5% nulls in each key column, null keys included
               (INCLUDE); v_int int64 uniform [0, 1e6], v_f f64 uniform [0, 1);
               SUM, COUNT, MAX of each; seed 2.
      small -- 1M rows; int32 key uniform over 1000 values; v1 int64 uniform
               [0, 1e6], v2 f64 uniform [0, 1); v1 sum/count/min/max, v2 mean;
               no nulls; seed 0.
    Inputs are generated on the device; `value` is rows/s of the aggregate()
    call; cpu_baseline runs the oracle on the same distributions."""
    import torch
    import cudf_b200 as cb
    from cudf_b200 import aggregation as agg
    from cudf_b200.column import pack_mask
    from cudf_b200.types import NullPolicy, TypeId
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    if args.workload == "zipf":
        n = args.rows if args.rows != N_ROWS else 100_000_000
        cols = zipf_inputs_device(n, dev)
        k1, k2, km, vi, vf = cols
        keys = cb.Table([cb.Column(TypeId.INT32, k1, km[0]), cb.Column(TypeId.INT64, k2, km[1])])
        aggs = [agg.sum(), agg.count(), agg.max()]
        reqs = [cb.GroupByRequest(cb.Column(TypeId.INT64, vi), aggs), cb.GroupByRequest(cb.Column(TypeId.FLOAT64, vf), aggs)]
        policy = NullPolicy.INCLUDE
        workload = ("groupby 100M rows, (int32, int64) keys = divmod(Zipf(1.1) on [0,50M), 1000), 5% key nulls, "
                    "INCLUDE, int64 + f64 values, sum/count/max")
        inp = n * (4 + 8 + 8 + 8) + 2 * ((n + 31) // 32) * 4
        out_per_group, out_masks = 4 + 8 + 8 + 4 + 8 + 8 + 4 + 8, 2
    else:
        n = args.rows if args.rows != N_ROWS else 1_000_000
        cols = small_inputs_device(n, dev)
        k, v1, v2 = cols
        keys = cb.Table([cb.Column(TypeId.INT32, k)])
        reqs = [cb.GroupByRequest(cb.Column(TypeId.INT64, v1), [agg.sum(), agg.count(), agg.min(), agg.max()]),
                cb.GroupByRequest(cb.Column(TypeId.FLOAT64, v2), [agg.mean()])]
        policy = NullPolicy.EXCLUDE
        workload = "groupby 1M rows, int32 key over 1000 values, v1 int64 sum/count/min/max, v2 f64 mean"
        inp = n * (4 + 8 + 8)
        out_per_group, out_masks = 4 + 8 + 4 + 8 + 8 + 8, 0
    torch.cuda.synchronize()
    gb = cb.GroupBy(keys, policy)
    gb.set_profile(True)
    for _ in range(args.warmup):
        gb.aggregate(reqs)
    stream = torch.cuda.current_stream()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    kms = []
    with ClockSampler(0) as clk:
        a.record(stream)
        for _ in range(args.steps):
            uk, res = gb.aggregate(reqs)
            kms.append(gb.stats()["agg_kernel_ms"])
        b.record(stream)
        torch.cuda.synchronize()
    ms = a.elapsed_time(b) / args.steps
    st = gb.stats()
    groups = uk.num_rows()
    checked = None
    if args.check:
        t0 = time.perf_counter()
        hk, hr, inc = config_oracle_inputs(args.workload, [c.cpu() for c in _flat(cols)], n)
        g = check_with_oracle(hk, hr, inc, uk, res)
        checked = {"groups": g, "result": "match", "seconds": round(time.perf_counter() - t0, 1)}
        del hk, hr
    algo = inp + groups * out_per_group + out_masks * ((groups + 31) // 32) * 4
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    kmean = float(np.mean(kms))
    line = {"metric": f"groupby rows/s ({args.workload})", "value": n / (ms * 1e-3), "unit": "rows/s",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32/int64/f64",
            "data": "synthetic", "config": {"workload": workload, "rows": n, "groups": groups},
            "roofline": {"bound": "hbm", "achieved": algo / (kmean * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": algo / (kmean * 1e-3) / 1e9 / peak, "traffic": None,
                         "kernel": KERNELS_BY_MODE.get(st["mode"]), "kernel_ms": kmean,
                         "algorithmic_bytes": algo, "input_bytes": inp,
                         "whole_call_frac": algo / (ms * 1e-3) / 1e9 / peak},
            "engine": st, "clocks": clk.summary()}
    if checked is not None:
        line["check"] = checked
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = _cpu_config(args.workload, min(n, args.cpu_sample))
    return line


def _cpu_config(workload, n):
    """The oracle on n rows of the same distributions (numpy generator)."""
    from oracle import oracle as O
    threads = os.cpu_count() or 1
    rng = np.random.default_rng(2 if workload == "zipf" else 0)
    if workload == "zipf":
        u = rng.random(n)
        a = 1.0 - 1.1
        p = np.clip(np.floor((1.0 - u * (1.0 - (50_000_001.0) ** a)) ** (1.0 / a) - 1.0), 0, 49_999_999).astype(np.int64)
        keys = [O.HostColumn(O.INT32, (p // 1000).astype(np.int32), rng.random(n) >= 0.05),
                O.HostColumn(O.INT64, p % 1000, rng.random(n) >= 0.05)]
        kinds = [O.SUM, O.COUNT_VALID, O.MAX]
        reqs = [(O.HostColumn(O.INT64, rng.integers(0, 10**6, n, endpoint=True)), kinds),
                (O.HostColumn(O.FLOAT64, rng.random(n)), kinds)]
        inc = True
    else:
        keys = [O.HostColumn(O.INT32, rng.integers(0, 1000, n).astype(np.int32))]
        reqs = [(O.HostColumn(O.INT64, rng.integers(0, 10**6, n, endpoint=True)), [O.SUM, O.COUNT_VALID, O.MIN, O.MAX]),
                (O.HostColumn(O.FLOAT64, rng.random(n)), [O.MEAN])]
        inc = False
    O.groupby(keys, reqs, include_null_keys=inc, nthreads=threads)
    t = time.perf_counter()
    O.groupby(keys, reqs, include_null_keys=inc, nthreads=threads)
    v = n / (time.perf_counter() - t)
    return {"value": v, "unit": "rows/s", "cores": threads, "kind": "port",
            "sample": f"{n} rows with the workload's distributions through oracle/gb_oracle.c, {threads} threads"}


def run_extras(args) -> dict:
    """The other workloads, each measured once after the main one (shorter runs
    than their own --workload lines; each entry says what it ran)."""
    import copy
    import torch
    out = {}

    def one(name, fn, **kw):
        a = copy.copy(args)
        for k, v in kw.items():
            setattr(a, k, v)
        try:
            r = fn(a)
        except Exception as e:  # one failing workload leaves the others
            r = {"error": f"{type(e).__name__}: {e}"}
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
        return r

    z = one("zipf", run_config, workload="zipf", rows=N_ROWS, steps=5, warmup=2, no_cpu_baseline=True)
    out["zipf"] = {k: z.get(k) for k in ("metric", "value", "unit", "ms_per_step", "config", "roofline", "error")
                   if k in z}
    sm = one("small", run_config, workload="small", rows=N_ROWS, steps=50, warmup=5, no_cpu_baseline=True)
    out["small"] = {k: sm.get(k) for k in ("metric", "value", "unit", "ms_per_step", "config", "error") if k in sm}
    b = one("batch", run_batch, steps=3, warmup=2)
    out["batch"] = {k: b.get(k) for k in ("metric", "value", "unit", "ms_per_step", "config", "plain",
                                          "speedup_vs_plain", "error") if k in b}
    sv = one("serve", run_serve, duration=args.serve_duration)
    out["serve"] = {k: sv.get(k) for k in ("metric", "value", "unit", "config", "batched", "plain",
                                           "plain_single_query_latency_s", "qps_ratio_vs_plain",
                                           "p99_over_plain_single", "error") if k in sv}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--rows", type=int, default=N_ROWS)
    ap.add_argument("--tuning", default="")
    ap.add_argument("--cpu-sample", type=int, default=CPU_SAMPLE_ROWS)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="single", choices=["single", "batch", "serve", "zipf", "small"])
    ap.add_argument("--instances", type=int, default=4096)
    ap.add_argument("--rate", type=float, default=2000.0)
    ap.add_argument("--rates", default="", help="serve: comma-separated offered rates (a curve); first is the line's")
    ap.add_argument("--duration", type=float, default=5.0)
    ap.add_argument("--pool", type=int, default=16)
    ap.add_argument("--workers", type=int, default=4)
    ap.add_argument("--direct-rows", type=int, default=0,
                    help="serve: queries with at least this many rows run alone (0: server default)")
    ap.add_argument("--check", action="store_true",
                    help="compare the last timed result with the oracle on the same inputs")
    ap.add_argument("--no-extra", action="store_true", help="skip the other workloads in the main line")
    ap.add_argument("--serve-duration", type=float, default=5.0,
                    help="length of the serving stream measured in the main line's extra")
    args = ap.parse_args()
    if args.impl == "engine" and args.workload in ("batch", "serve", "zipf", "small"):
        fn = {"batch": run_batch, "serve": run_serve}.get(args.workload, run_config)
        print(json.dumps(fn(args)), flush=True)
        return 0
    if args.impl == "reference":
        return run_reference(args)
    return run_engine(args)


if __name__ == "__main__":
    sys.exit(main())
