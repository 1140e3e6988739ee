"""Multi-rank groupby (partial aggregate -> all-to-all by key owner -> merge)
on CPU with the gloo backend, world size 2.  The local aggregation is the
oracle here (no GPU in this environment); the exchange, routing and merge
logic is the production code in cudf_b200/distributed.py.  The union of the
ranks' groups must equal the single-process groupby of the whole table, with
every group owned by exactly one rank."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from oracle import oracle as O

KINDS = [O.SUM, O.COUNT_VALID, O.COUNT_ALL, O.MIN, O.MAX, O.MEAN]


def _table(n, seed):
    rng = np.random.default_rng(seed)
    k1 = rng.integers(0, 500, n).astype(np.int64)
    k2 = rng.integers(0, 3, n).astype(np.int32)
    kv2 = rng.random(n) > 0.05
    v1 = rng.integers(-10**9, 10**9, n).astype(np.int64)
    v2 = rng.normal(size=n)
    m1, m2 = rng.random(n) > 0.1, rng.random(n) > 0.1
    return k1, k2, kv2, v1, v2, m1, m2


def oracle_local_aggregate(keys, requests, null_handling):
    """Local aggregation on CPU tensors through the oracle (test stand-in)."""
    hk = [O.HostColumn(int(t), d.numpy(), None if v is None else v.numpy()) for d, v, t in keys]
    hr = [(O.HostColumn(int(t), d.numpy(), None if v is None else v.numpy()), [int(k) for k in kinds])
          for (d, v, t), kinds in requests]
    r = O.groupby(hk, hr, include_null_keys=int(null_handling) == 1)
    out_keys = [(torch.from_numpy(np.ascontiguousarray(d)), None if v is None else torch.from_numpy(v.copy()), int(k.type_id))
                for (d, v), k in zip(r.keys, hk)]
    out_res = []
    for (col, kinds), per in zip(hr, r.results):
        row = []
        for kind, (vals, valid, _) in zip(kinds, per):
            has_mask = col.valid is not None and kind not in (O.COUNT_VALID, O.COUNT_ALL)
            row.append((torch.from_numpy(np.ascontiguousarray(vals)), torch.from_numpy(valid.copy()) if has_mask else None))
        out_res.append(row)
    return out_keys, out_res


def _worker(rank, world, port, n, include, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from cudf_b200.distributed import distributed_groupby
        from cudf_b200.types import NullPolicy
        k1, k2, kv2, v1, v2, m1, m2 = _table(n, 1234)
        lo, hi = n * rank // world, n * (rank + 1) // world
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a[lo:hi]))
        keys = [(t(k1), None, O.INT64), (t(k2), t(kv2), O.INT32)]
        reqs = [((t(v1), t(m1), O.INT64), KINDS), ((t(v2), t(m2), O.FLOAT64), KINDS)]
        mk, mres = distributed_groupby(keys, reqs, NullPolicy.INCLUDE if include else NullPolicy.EXCLUDE,
                                       local_aggregate=oracle_local_aggregate)
        payload = ([(d.numpy(), None if v is None else v.numpy()) for d, v, _ in mk],
                   [[(d.numpy(), None if v is None else v.numpy()) for d, v in per] for per in mres])
        got = [None] * world
        dist.all_gather_object(got, payload)
        if rank == 0:
            q.put(got)
    finally:
        dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


@pytest.mark.parametrize("include", [False, True])
def test_two_rank_groupby_equals_single_process(include):
    n, world = 40_000, 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, n, include, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = q.get(timeout=240)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # single-process reference
    k1, k2, kv2, v1, v2, m1, m2 = _table(n, 1234)
    ref = O.groupby([O.HostColumn(O.INT64, k1), O.HostColumn(O.INT32, k2, kv2)],
                    [(O.HostColumn(O.INT64, v1, m1), KINDS), (O.HostColumn(O.FLOAT64, v2, m2), KINDS)],
                    include_null_keys=include)
    # concatenate the ranks' groups; every group owned by one rank only
    keys = []
    for kc in range(2):
        d = np.concatenate([g[0][kc][0] for g in got])
        vs = [g[0][kc][1] for g in got]
        v = None if vs[0] is None else np.concatenate(vs)
        keys.append((d, v))
    G = ref.num_groups
    assert keys[0][0].shape[0] == G, "a group is missing or owned by two ranks"
    oo, go = O.sort_order(ref.keys), O.sort_order(keys)
    for (rd, rv), (gd, gv) in zip(ref.keys, keys):
        rvv = np.ones(G, bool) if rv is None else rv[oo]
        gvv = np.ones(G, bool) if gv is None else gv[go]
        assert np.array_equal(rvv, gvv)
        assert np.array_equal(rd[oo][rvv], gd[go][gvv])
    for r in range(2):
        for j, kind in enumerate(KINDS):
            rv, rval, tol = ref.results[r][j]
            gd = np.concatenate([g[1][r][j][0] for g in got])[go]
            gvs = [g[1][r][j][1] for g in got]
            gv = np.ones(G, bool) if gvs[0] is None else np.concatenate(gvs)[go]
            rv, rval, tol = rv[oo], rval[oo], tol[oo]
            assert np.array_equal(rval, gv), f"request {r} kind {kind}: validity"
            if rv.dtype.kind == "f":
                assert np.all(np.abs(rv[rval] - gd[gv]) <= 2 * tol[rval] + 1e-12), f"request {r} kind {kind}"
            else:
                assert np.array_equal(rv[rval], gd[gv].astype(rv.dtype)), f"request {r} kind {kind}"


def test_owner_rank_is_consistent_and_balanced():
    from cudf_b200.distributed import owner_rank
    rng = np.random.default_rng(3)
    k = torch.from_numpy(rng.integers(-2**62, 2**62, 100_000))
    f = torch.tensor([0.0, -0.0, float("nan"), -float("nan"), 1.5], dtype=torch.float64)
    a = owner_rank([(k, None, O.INT64)], 4)
    b = owner_rank([(k.clone(), None, O.INT64)], 4)
    assert torch.equal(a, b)
    counts = torch.bincount(a, minlength=4).numpy()
    assert counts.min() > 0.9 * counts.mean()
    fr = owner_rank([(f, None, O.FLOAT64)], 8)
    assert fr[0] == fr[1] and fr[2] == fr[3]  # -0.0 == +0.0, all NaNs one key


def _exchange_worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from cudf_b200.distributed import _exchange
        rng = np.random.default_rng(100 + rank)
        n = 0 if rank == 1 else 37  # rank 1 sends nothing
        dest = torch.from_numpy(rng.integers(0, world, n).astype(np.int64))
        cols = [torch.from_numpy(rng.integers(-2**62, 2**62, n).astype(np.int64)),
                torch.from_numpy(rng.random(n).astype(np.float32)),
                torch.from_numpy(rng.random(n) > 0.5),
                torch.from_numpy(rng.integers(0, 100, (n, 3)).astype(np.int16))]
        got = _exchange(cols, dest, world)
        sent = [(dest.numpy(), [c.numpy() for c in cols])]
        everything = [None] * world
        dist.all_gather_object(everything, (rank, sent, [g.numpy() for g in got]))
        if rank == 0:
            q.put(everything)
    finally:
        dist.destroy_process_group()


def test_exchange_packs_every_column_into_one_payload():
    """Rows reach the rank named by `dest` with every column intact (int64,
    float32, bool, a 2-D int16 block), in the senders' rank order and each
    sender's row order; a rank with no rows takes part."""
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_exchange_worker, args=(r, world, port, q)) for r in range(world)]
    for p in ps:
        p.start()
    everything = q.get(timeout=120)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    by_rank = {r: (sent, got) for r, sent, got in everything}
    for dst in range(world):
        expect = [[] for _ in range(4)]
        for src in range(world):
            d, cols = by_rank[src][0][0]
            for i, c in enumerate(cols):
                expect[i].append(c[d == dst])
        got = by_rank[dst][1]
        for i in range(4):
            e = np.concatenate(expect[i]) if expect[i] else np.zeros(0)
            assert got[i].dtype == e.dtype and got[i].shape == e.shape
            assert np.array_equal(got[i], e)


def test_packed_validity_words_are_taken_as_the_mask():
    from cudf_b200.column import Column, pack_mask
    valid = torch.from_numpy(np.random.default_rng(3).random(70) > 0.3)
    data = torch.arange(70, dtype=torch.int64)
    a = Column.from_tensor(data, valid)
    b = Column.from_tensor(data, pack_mask(valid))
    assert torch.equal(a.mask, b.mask)
    assert torch.equal(b.valid(), valid)
