"""Serving loop: queries submitted from several threads while others run are
admitted under the memory cap, batched, and each result equals the same query
run alone (gb_aggregate) and the CPU oracle."""
import threading

import numpy as np
import pytest
import torch

from oracle import oracle as O
from parity import compare, gpu_pairs

pytestmark = pytest.mark.gpu


def _cb():
    import cudf_b200 as cb
    from cudf_b200 import aggregation as agg
    return cb, agg


def _queries(seed, count):
    cb, agg = _cb()
    rng = np.random.default_rng(seed)
    qs = []
    for i in range(count):
        n = int(np.exp(rng.uniform(np.log(1000), np.log(300_000))))
        card = max(2, int(np.exp(rng.uniform(np.log(10), np.log(100_000)))))
        k = (rng.integers(0, card, n) * 1_000_003).astype(np.int64)
        v1 = rng.integers(-10**6, 10**6, n).astype(np.int64)
        v2 = rng.normal(size=n)
        m1, m2 = rng.random(n) > 0.1, rng.random(n) > 0.1
        qs.append((k, v1, v2, m1, m2))
    return qs


KINDS = [O.SUM, O.COUNT_VALID, O.MEAN]


def _dev(q):
    cb, agg = _cb()
    k, v1, v2, m1, m2 = q
    kt = cb.Table([cb.Column.from_numpy(k)])
    reqs = [cb.GroupByRequest(cb.Column.from_numpy(v1, m1), [agg.sum(), agg.count(), agg.mean()]),
            cb.GroupByRequest(cb.Column.from_numpy(v2, m2), [agg.sum(), agg.count(), agg.mean()])]
    return kt, reqs


def _check(q, uk, res):
    k, v1, v2, m1, m2 = q
    o = O.groupby([O.HostColumn(O.INT64, k)],
                  [(O.HostColumn(O.INT64, v1, m1), KINDS), (O.HostColumn(O.FLOAT64, v2, m2), KINDS)])
    compare(o, gpu_pairs(uk), [gpu_pairs(t) for t in res], [KINDS, KINDS], None)


def test_served_results_equal_alone_results():
    cb, _ = _cb()
    qs = _queries(41, 24)
    dev = [_dev(q) for q in qs]
    torch.cuda.synchronize()
    srv = cb.Server(workers=2, max_batch_queries=8)
    ids = [None] * len(qs)

    def submitter(lo, hi):
        for i in range(lo, hi):
            ids[i] = srv.submit(*dev[i])

    th = [threading.Thread(target=submitter, args=(i * 8, (i + 1) * 8)) for i in range(3)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    for i, q in enumerate(qs):
        info = srv.wait(ids[i], timeout_s=120)
        assert info["status"] == 2
        uk, res = srv.result(ids[i])
        _check(q, uk, res)  # in the mix == oracle
        alone_k, alone_r = cb.GroupBy(dev[i][0]).aggregate(dev[i][1])
        _check(q, alone_k, alone_r)  # alone == oracle, so both agree within the bound
        assert uk.num_rows() == alone_k.num_rows() == info["num_groups"]
        srv.release(ids[i])
    st = srv.stats()
    assert st["completed"] == len(qs) and st["failed"] == 0
    assert st["batches"] >= 1 and st["p99_s"] >= st["p50_s"] > 0
    srv.close()


def test_admission_cap_serialises_but_completes():
    cb, _ = _cb()
    qs = _queries(42, 6)
    dev = [_dev(q) for q in qs]
    srv = cb.Server(memory_cap_bytes=1 << 16, workers=1)  # every query exceeds the cap alone
    ids = [srv.submit(*d) for d in dev]
    for i, q in enumerate(qs):
        assert srv.wait(ids[i], timeout_s=120)["status"] == 2
        uk, res = srv.result(ids[i])
        _check(q, uk, res)
        srv.release(ids[i])
    st = srv.stats()
    assert st["completed"] == len(qs)
    srv.close()


def test_invalid_query_is_rejected_at_submit():
    cb, agg = _cb()
    srv = cb.Server()
    k = cb.Table([cb.Column.from_numpy(np.arange(4, dtype=np.int64))])
    ts = cb.Column.from_numpy(np.arange(4, dtype=np.int64), None, O.TIMESTAMP_SECONDS)
    with pytest.raises(ValueError, match="Invalid type/aggregation"):
        srv.submit(k, [cb.GroupByRequest(ts, [agg.sum()])])
    with pytest.raises(ValueError):
        srv.wait(12345, timeout_s=0.1)
    srv.close()


def test_large_queries_run_alone_and_match():
    cb, _ = _cb()
    rng = np.random.default_rng(43)
    qs = []
    for n, card in ((5_000_000, 200_000), (4_500_000, 3_000_000), (200_000, 50)):
        k = rng.integers(0, card, n).astype(np.int64)
        qs.append((k, rng.integers(-10**6, 10**6, n).astype(np.int64), rng.normal(size=n),
                   rng.random(n) > 0.1, rng.random(n) > 0.1))
    dev = [_dev(q) for q in qs]
    srv = cb.Server(workers=2)
    ids = [srv.submit(*d) for d in dev]
    for i, q in enumerate(qs):
        assert srv.wait(ids[i], timeout_s=300)["status"] == 2
        uk, res = srv.result(ids[i])
        _check(q, uk, res)
        srv.release(ids[i])
    assert srv.stats()["direct_runs"] >= 1
    srv.close()


def test_admission_by_free_device_memory_holds_then_completes():
    """A reserve that leaves less free device memory than one query needs:
    admission waits on free memory (one query at a time runs), yet every
    query completes with the oracle's result."""
    cb, _ = _cb()
    qs = _queries(44, 6)
    dev = [_dev(q) for q in qs]
    torch.cuda.synchronize()
    free, _ = torch.cuda.mem_get_info()
    srv = cb.Server(workers=2, reserve_bytes=free)  # nothing is left above the reserve
    ids = [srv.submit(*d) for d in dev]
    for i, q in enumerate(qs):
        assert srv.wait(ids[i], timeout_s=120)["status"] == 2
        uk, res = srv.result(ids[i])
        _check(q, uk, res)
        srv.release(ids[i])
    st = srv.stats()
    assert st["completed"] == len(qs) and st["failed"] == 0
    # a query waits while an earlier one is admitted and unreleased
    assert st["held_for_memory"] >= 1 and 0 < st["min_free_bytes"] <= free
    srv.close()
