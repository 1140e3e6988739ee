"""Batched groupby (many instances, one launch; optional CUDA-graph replay)
against the CPU oracle, instance by instance."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from parity import compare, gpu_pairs, host_cols

pytestmark = pytest.mark.gpu


def _cb():
    import cudf_b200 as cb
    from cudf_b200 import aggregation as agg
    return cb, agg


def _instances(seed, count, max_rows=200_000, max_card=50_000, two_keys=False):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(np.exp(rng.uniform(np.log(1), np.log(max_rows))))
        if i == 0:
            n = 0
        if i == 1:
            n = 1
        card = max(1, int(np.exp(rng.uniform(np.log(1), np.log(max_card)))))
        k = rng.integers(0, card, n).astype(np.int32)
        kv = None
        if i == 2:
            kv = np.zeros(n, bool)  # every key null: no group under EXCLUDE
        v1 = rng.integers(0, 10**6, n).astype(np.int64)
        v2 = rng.normal(size=n)
        m1 = rng.random(n) > 0.05 if i % 3 else None
        m2 = rng.random(n) > 0.05
        keys = [(O.INT32, k, kv)]
        if two_keys:
            keys.append((O.INT64, rng.integers(0, 3, n).astype(np.int64), rng.random(n) > 0.05))
        out.append((keys, [(O.INT64, v1, m1), (O.FLOAT64, v2, m2)]))
    return out


def _run(instances, use_graph, include_nulls, replays=2):
    cb, agg = _cb()
    aggs = lambda: [agg.sum(), agg.count(), agg.min(), agg.max(), agg.mean()]
    dev = []
    for keys, vals in instances:
        kt = cb.Table([cb.Column.from_numpy(d, v, t) for t, d, v in keys])
        rq = [cb.GroupByRequest(cb.Column.from_numpy(d, v, t), aggs()) for t, d, v in vals]
        dev.append((kt, rq))
    bg = cb.BatchGroupBy(dev, cb.NullPolicy.INCLUDE if include_nulls else cb.NullPolicy.EXCLUDE,
                         use_graph=use_graph)
    kinds = [O.SUM, O.COUNT_VALID, O.MIN, O.MAX, O.MEAN]
    for rep in range(replays):
        bg.run()
        torch.cuda.synchronize()
        for i, (keys, vals) in enumerate(instances):
            uk, res = bg.result(i)
            o = O.groupby([O.HostColumn(t, d, v) for t, d, v in keys],
                          [(O.HostColumn(t, d, v), kinds) for t, d, v in vals], include_null_keys=include_nulls)
            compare(o, gpu_pairs(uk), [gpu_pairs(t) for t in res], [kinds, kinds], None)
    return bg


@pytest.mark.parametrize("use_graph", [False, True])
def test_batch_matches_oracle(use_graph):
    bg = _run(_instances(7, 40), use_graph, False)
    st = bg.stats()
    assert st["instances"] == 40 and st["kernels_per_run"] >= 4


def test_batch_two_word_keys_include_nulls():
    _run(_instances(8, 12, max_rows=50_000, max_card=2_000, two_keys=True), True, True)


@pytest.fixture
def default_batch_tuning():
    """Batches prepared inside the test use the built-in launch and no rules
    (the shipped tuning file may set others); the shipped tuning is put back."""
    from cudf_b200 import autotune
    autotune.set_batch_tuning([], autotune.BATCH_LAUNCH_DEFAULT)
    yield autotune
    autotune.set_batch_tuning([], autotune.BATCH_LAUNCH_DEFAULT)
    autotune.load()


def test_batch_low_cardinality_uses_shared_tables(default_batch_tuning):
    rng = np.random.default_rng(9)
    inst = []
    for card in (1, 2, 4, 8, 100):
        n = 300_000
        inst.append(([(O.INT32, rng.integers(0, card, n).astype(np.int32), None)],
                     [(O.INT64, rng.integers(-5, 5, n).astype(np.int64), None),
                      (O.FLOAT64, rng.random(n), rng.random(n) > 0.5)]))
    bg = _run(inst, True, False, replays=1)
    assert bg.stats()["smem_instances"] == len(inst)


def test_batch_rejects_mixed_schemas():
    cb, agg = _cb()
    a = cb.Table([cb.Column.from_numpy(np.arange(10, dtype=np.int32))])
    b = cb.Table([cb.Column.from_numpy(np.arange(10, dtype=np.int64))])
    v = cb.Column.from_numpy(np.arange(10, dtype=np.int64))
    with pytest.raises(ValueError):
        cb.BatchGroupBy([(a, [cb.GroupByRequest(v, [agg.sum()])]), (b, [cb.GroupByRequest(v, [agg.sum()])])])


@pytest.mark.parametrize("launch", [{"block": 256, "tile_rows": 4096, "smem_bytes": 96 * 1024},
                                    {"block": 1024, "tile_rows": 262144, "smem_bytes": 200 * 1024}])
def test_batch_tuned_launch_and_rules_match_oracle(default_batch_tuning, launch):
    """Other block sizes and tile lengths, and per-instance rules that send
    one size bucket to the global table and give another more headroom."""
    autotune = default_batch_tuning
    rules = [{"max_rows": 20_000, "max_groups": 1 << 30, "smem_slots": 0},
             {"max_rows": 1 << 30, "max_groups": 2_000, "headroom_pct": 400}]
    autotune.set_batch_tuning(rules, launch)
    bg = _run(_instances(10, 24), True, False, replays=1)
    st = bg.stats()
    assert st["block"] == launch["block"] and st["tile_rows"] == launch["tile_rows"]
    assert st["ruled_instances"] >= 1
