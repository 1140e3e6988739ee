"""Engine vs CPU oracle on seeded random inputs: every supported value type and
aggregation, nulls, null_policy INCLUDE/EXCLUDE, multi-column keys, both
aggregation modes, table-overflow retries and sliced (offset) columns."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from parity import run_both

pytestmark = pytest.mark.gpu


# pass-2 settings: sorted chunks (512x4, 256x8), per-row updates (1024x1 and
# 512x2 rows) with the
# warp-combining kernel for heavy partitions only (default), for every
# partition, and for split partitions only
PASS2 = [{"pass2": 0}, {"pass2": 1}, {"pass2": 3}, {"pass2": 4}, {"pass2": 1, "wagg_pct": 0}, {"pass2": 1, "wagg_pct": 100000}]
PASS2_ROW = [{"pass2": 0}, {"pass2": 1}, {"pass2": 4}, {"pass2": 1, "wagg_pct": 0}]


def _cb():
    import cudf_b200 as cb
    from cudf_b200 import aggregation as agg
    return cb, agg


def _rand(rng, type_id, n, lo=-1000, hi=1000):
    dt = O.NP_DTYPE[type_id]
    if type_id in (O.FLOAT32, O.FLOAT64):
        return (rng.normal(size=n) * 100).astype(dt)
    if type_id == O.BOOL8:
        return rng.integers(0, 2, n).astype(np.uint8)
    info = np.iinfo(dt)
    return rng.integers(max(lo, info.min), min(hi, info.max), n, endpoint=True).astype(dt)


ALL_AGGS = ["sum", "min", "max", "count_valid", "count_all", "mean", "sum_of_squares", "variance",
            "std", "argmin", "argmax"]


def _aggs_for(agg, type_id, names):
    m = {"sum": agg.sum(), "min": agg.min(), "max": agg.max(), "count_valid": agg.count(),
         "count_all": agg.count(agg.NullPolicy.INCLUDE) if hasattr(agg, "NullPolicy") else None,
         "mean": agg.mean(), "sum_of_squares": agg.sum_of_squares(), "variance": agg.variance(),
         "std": agg.std(), "argmin": agg.argmin(), "argmax": agg.argmax(), "product": agg.product()}
    from cudf_b200.types import NullPolicy
    m["count_all"] = agg.count(NullPolicy.INCLUDE)
    return [m[x] for x in names if O.valid_agg(type_id, int(m[x].kind))]


@pytest.mark.parametrize("type_id", [O.INT8, O.INT16, O.INT32, O.INT64, O.UINT8, O.UINT16, O.UINT32,
                                     O.UINT64, O.FLOAT32, O.FLOAT64, O.BOOL8, O.TIMESTAMP_DAYS,
                                     O.TIMESTAMP_NANOSECONDS, O.DURATION_DAYS, O.DURATION_SECONDS])
@pytest.mark.parametrize("mode", [0, 1])
def test_value_types_all_aggs(type_id, mode):
    cb, agg = _cb()
    rng = np.random.default_rng(100 + type_id)
    n = 200_000
    key = rng.integers(0, 3000, n).astype(np.int32)
    vals = _rand(rng, type_id, n)
    valid = rng.random(n) > 0.15
    aggs = _aggs_for(agg, type_id, ALL_AGGS)
    run_both([cb.Column.from_numpy(key)], [(cb.Column.from_numpy(vals, valid, type_id), aggs)],
             tuning={"force_mode": mode})


@pytest.mark.parametrize("mode", [0, 1])
def test_product_small_values(mode):
    cb, agg = _cb()
    rng = np.random.default_rng(3)
    n = 50_000
    key = rng.integers(0, 20000, n).astype(np.int64)
    v = rng.integers(-3, 4, n).astype(np.int64)
    f = rng.uniform(0.5, 1.5, n)
    run_both([cb.Column.from_numpy(key)],
             [(cb.Column.from_numpy(v, rng.random(n) > 0.1), [agg.product()]),
              (cb.Column.from_numpy(f), [agg.product()])], tuning={"force_mode": mode})


@pytest.mark.parametrize("policy", [False, True])
@pytest.mark.parametrize("mode", [0, 1])
def test_multi_column_nullable_keys(policy, mode):
    cb, agg = _cb()
    rng = np.random.default_rng(11)
    n = 300_000
    k1 = rng.integers(0, 300, n).astype(np.int32)
    k2 = rng.integers(0, 40, n).astype(np.int64)
    kv1, kv2 = rng.random(n) > 0.05, rng.random(n) > 0.05
    v = rng.integers(0, 10**6, n).astype(np.int64)
    f = rng.random(n)
    run_both([cb.Column.from_numpy(k1, kv1), cb.Column.from_numpy(k2, kv2)],
             [(cb.Column.from_numpy(v), [agg.sum(), agg.count(), agg.max()]),
              (cb.Column.from_numpy(f, rng.random(n) > 0.3), [agg.sum(), agg.mean(), agg.min()])],
             include_null_keys=policy, tuning={"force_mode": mode})


@pytest.mark.parametrize("ktype", [O.INT8, O.INT16, O.UINT32, O.FLOAT32, O.FLOAT64, O.BOOL8, O.UINT64])
def test_key_types(ktype):
    cb, agg = _cb()
    rng = np.random.default_rng(ktype)
    n = 100_000
    if ktype in (O.FLOAT32, O.FLOAT64):
        base = rng.integers(-50, 50, n).astype(O.NP_DTYPE[ktype]) / 4
        base[rng.random(n) < 0.02] = np.nan
        base[rng.random(n) < 0.02] = -0.0
        k = base
    else:
        k = _rand(rng, ktype, n, 0, 200)
    v = rng.integers(0, 100, n).astype(np.int32)
    run_both([cb.Column.from_numpy(k, None, ktype)], [(cb.Column.from_numpy(v), [agg.sum(), agg.count()])])


def test_three_keys_two_words():
    cb, agg = _cb()
    rng = np.random.default_rng(5)
    n = 200_000
    ks = [rng.integers(0, 7, n).astype(np.int64), rng.integers(0, 9, n).astype(np.int32),
          rng.integers(0, 5, n).astype(np.int16)]
    v = rng.normal(size=n)
    run_both([cb.Column.from_numpy(k) for k in ks], [(cb.Column.from_numpy(v), [agg.sum(), agg.variance(0)])])


@pytest.mark.parametrize("mode", [0, 1, 2])
def test_all_ones_key_uses_special_slot(mode):
    cb, agg = _cb()
    n = 10_000
    k = np.full(n, -1, dtype=np.int64)
    k[::3] = 5
    v = np.arange(n, dtype=np.int64)
    run_both([cb.Column.from_numpy(k)], [(cb.Column.from_numpy(v), [agg.sum(), agg.min(), agg.count()])],
             tuning={"force_mode": mode})


def test_overflow_retry_with_tiny_hint():
    cb, agg = _cb()
    rng = np.random.default_rng(9)
    n = 400_000
    k = rng.integers(0, 10**12, n).astype(np.int64)
    v = rng.integers(-5, 5, n).astype(np.int64)
    gb, *_ = run_both([cb.Column.from_numpy(k)], [(cb.Column.from_numpy(v), [agg.sum(), agg.count()])],
                      tuning={"groups_hint": 10, "force_mode": 0})
    assert gb.stats()["retries"] >= 1


def test_sliced_columns_with_offset():
    cb, agg = _cb()
    rng = np.random.default_rng(21)
    n = 100_003
    k = rng.integers(0, 500, n).astype(np.int32)
    v = rng.integers(0, 100, n).astype(np.int64)
    vv = rng.random(n) > 0.2
    kc = cb.Column.from_numpy(k)
    vc = cb.Column.from_numpy(v, vv)
    off, m = 37, 90_001
    kcs = cb.Column(kc.type_id, kc.data, kc.mask, size=m, offset=off)
    vcs = cb.Column(vc.type_id, vc.data, vc.mask, size=m, offset=off)
    run_both([kcs], [(vcs, [agg.sum(), agg.count(), agg.mean(), agg.argmax()])])


def test_nan_values_min_max_terminate():
    cb, agg = _cb()
    k = np.array([1, 1, 2, 2, 2, 3], dtype=np.int32)
    v = np.array([np.nan, np.nan, 1.0, np.nan, -2.0, np.inf])
    run_both([cb.Column.from_numpy(k)], [(cb.Column.from_numpy(v), [agg.min(), agg.max(), agg.argmin(), agg.argmax()])])


def test_mismatched_sizes_raise_logic_error():
    cb, agg = _cb()
    gb = cb.GroupBy(cb.Table([cb.Column.from_numpy(np.arange(3, dtype=np.int32))]))
    with pytest.raises(ValueError, match="Size mismatch"):
        gb.aggregate([cb.GroupByRequest(cb.Column.from_numpy(np.arange(5, dtype=np.int32)), [agg.count()])])


def test_invalid_type_aggregation_raises():
    cb, agg = _cb()
    gb = cb.GroupBy(cb.Table([cb.Column.from_numpy(np.arange(3, dtype=np.int32))]))
    ts = cb.Column.from_numpy(np.arange(3, dtype=np.int64), None, O.TIMESTAMP_SECONDS)
    with pytest.raises(ValueError, match="Invalid type/aggregation"):
        gb.aggregate([cb.GroupByRequest(ts, [agg.sum()])])


def test_results_same_on_a_non_default_stream():
    """cpp/tests/streams/groupby_test.cpp:25-67: all work on the given stream."""
    cb, agg = _cb()
    rng = np.random.default_rng(2)
    n = 100_000
    k = cb.Column.from_numpy(rng.integers(0, 100, n).astype(np.int32))
    v = cb.Column.from_numpy(rng.integers(0, 100, n).astype(np.int64))
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        gb = cb.GroupBy(cb.Table([k]))
        uk, res = gb.aggregate([cb.GroupByRequest(v, [agg.sum()])], stream=s)
    s.synchronize()
    total = int(res[0].columns[0].values().sum().item())
    assert total == int(v.values().sum().item())


@pytest.mark.parametrize("n,card,nulls", [(1_000_000, 1000, 0.0), (2_000_000, 1_000_000, 0.1)])
def test_config_shapes_medium(n, card, nulls):
    """The 1M-row pandas configuration and a 2M-row slice of the 100M-row one."""
    cb, agg = _cb()
    rng = np.random.default_rng(0)
    if card == 1000:
        key = rng.integers(0, 1000, n).astype(np.int32)
    else:
        distinct = np.unique(rng.integers(-2**63, 2**63 - 1, card, dtype=np.int64))
        key = distinct[rng.integers(0, distinct.size, n)]
    v1 = rng.integers(-10**9, 10**9, n).astype(np.int64)
    v2 = rng.normal(size=n)
    v3 = rng.lognormal(size=n).astype(np.float32)
    masks = [rng.random(n) >= nulls if nulls else None for _ in range(3)]
    aggs = [agg.sum(), agg.count(), agg.min(), agg.max(), agg.mean()]
    run_both([cb.Column.from_numpy(key)],
             [(cb.Column.from_numpy(v1, masks[0]), aggs), (cb.Column.from_numpy(v2, masks[1]), aggs),
              (cb.Column.from_numpy(v3, masks[2]), aggs)])


@pytest.mark.parametrize("scatter", [0, 1, 2, 3, 4, 5, 6, 7, 8])
@pytest.mark.parametrize("nulls", [False, True])
@pytest.mark.parametrize("two_word", [False, True])
def test_partitioned_mode(nulls, two_word, scatter):
    cb, agg = _cb()
    rng = np.random.default_rng(31)
    n = 3_000_000
    card = 200_000
    distinct = np.unique(rng.integers(-2**63, 2**63 - 1, card, dtype=np.int64))
    key = distinct[rng.integers(0, distinct.size, n)]
    v1 = rng.integers(-10**9, 10**9, n).astype(np.int64)
    v2 = rng.normal(size=n)
    v3 = rng.lognormal(size=n).astype(np.float32)
    ms = [rng.random(n) > 0.1 if nulls else None for _ in range(3)]
    keys = [cb.Column.from_numpy(key)]
    if two_word:
        keys.append(cb.Column.from_numpy(rng.integers(0, 3, n).astype(np.int16), rng.random(n) > 0.05))
    aggs = [agg.sum(), agg.count(), agg.min(), agg.max(), agg.mean()]
    gb, *_ = run_both(keys, [(cb.Column.from_numpy(v1, ms[0]), aggs), (cb.Column.from_numpy(v2, ms[1]), aggs),
                             (cb.Column.from_numpy(v3, ms[2]), aggs + [agg.count(cb.NullPolicy.INCLUDE)])],
                      include_null_keys=two_word, tuning={"force_mode": 2, "scatter": scatter})
    assert gb.stats()["mode"] == 2


@pytest.mark.parametrize("pass2", PASS2)
@pytest.mark.parametrize("nulls", [False, True])
@pytest.mark.parametrize("two_word", [False, True])
def test_partitioned_pass2_variants(nulls, two_word, pass2):
    """Pass 2 as chunks sorted by slot (512x4 and 256x8 rows per chunk) and as
    per-row shared reductions, on every value type of the benchmark."""
    cb, agg = _cb()
    rng = np.random.default_rng(39)
    n = 2_500_000
    distinct = np.unique(rng.integers(-2**63, 2**63 - 1, 300_000, dtype=np.int64))
    key = distinct[rng.integers(0, distinct.size, n)]
    v1 = rng.integers(-10**9, 10**9, n).astype(np.int64)
    v2 = rng.normal(size=n)
    v3 = rng.lognormal(size=n).astype(np.float32)
    v4 = rng.integers(-1000, 1000, n).astype(np.int32)
    ms = [rng.random(n) > 0.1 if nulls else None for _ in range(4)]
    keys = [cb.Column.from_numpy(key)]
    if two_word:
        keys.append(cb.Column.from_numpy(rng.integers(0, 3, n).astype(np.int16), rng.random(n) > 0.05))
    aggs = [agg.sum(), agg.count(), agg.min(), agg.max(), agg.mean()]
    gb, *_ = run_both(keys, [(cb.Column.from_numpy(v1, ms[0]), aggs), (cb.Column.from_numpy(v2, ms[1]), aggs),
                             (cb.Column.from_numpy(v3, ms[2]), aggs + [agg.count(cb.NullPolicy.INCLUDE)]),
                             (cb.Column.from_numpy(v4, ms[3]), aggs + [agg.sum_of_squares()])],
                      include_null_keys=two_word, tuning={"force_mode": 2, **pass2})
    assert gb.stats()["mode"] == 2


def test_partitioned_mode_is_chosen_for_many_groups():
    cb, agg = _cb()
    rng = np.random.default_rng(32)
    n = 4_000_000
    key = rng.integers(0, 2**40, n).astype(np.int64)
    v = rng.integers(0, 100, n).astype(np.int64)
    gb, *_ = run_both([cb.Column.from_numpy(key)], [(cb.Column.from_numpy(v), [agg.sum(), agg.max()])])
    assert gb.stats()["mode"] == 2


@pytest.mark.parametrize("pass2", PASS2)
@pytest.mark.parametrize("scatter", [0, 1, 7, 8])
def test_partitioned_spill_when_groups_underestimated(scatter, pass2):
    cb, agg = _cb()
    rng = np.random.default_rng(33)
    n = 1_500_000
    key = rng.integers(0, 300_000, n).astype(np.int64)
    key[::97] = -1  # all-ones key words: the special slot
    v = rng.integers(-5, 5, n).astype(np.int64)
    f = rng.random(n).astype(np.float32)
    run_both([cb.Column.from_numpy(key)], [(cb.Column.from_numpy(v), [agg.sum(), agg.count(), agg.min()]),
                                           (cb.Column.from_numpy(f, rng.random(n) > 0.2), [agg.mean(), agg.max()])],
             tuning={"force_mode": 2, "groups_hint": 1000, "scatter": scatter, **pass2})


@pytest.mark.parametrize("pass2", PASS2)
@pytest.mark.parametrize("scatter", [0, 1, 7, 8])
def test_partitioned_all_ones_key_heavy(scatter, pass2):
    """40% of the rows carry the all-ones key: one partition aggregates them in
    its dedicated shared slot, merged into the global table's slot at flush."""
    cb, agg = _cb()
    rng = np.random.default_rng(35)
    n = 2_000_000
    key = rng.integers(0, 200_000, n).astype(np.int64)
    key[rng.random(n) < 0.4] = -1
    v = rng.integers(-10**6, 10**6, n).astype(np.int64)
    d = rng.normal(size=n)
    gb, *_ = run_both([cb.Column.from_numpy(key)],
                      [(cb.Column.from_numpy(v, rng.random(n) > 0.1), [agg.sum(), agg.count(), agg.min(), agg.max()]),
                       (cb.Column.from_numpy(d, rng.random(n) > 0.1), [agg.mean(), agg.min(), agg.max()])],
                      tuning={"force_mode": 2, "scatter": scatter, **pass2})
    assert gb.stats()["mode"] == 2


@pytest.mark.parametrize("pass2", PASS2)
def test_partitioned_skew_splits_heavy_partitions(pass2):
    """Zipf(1.3) keys: a few keys hold a large share of the rows; their
    partitions are cut into row ranges whose tables merge globally."""
    cb, agg = _cb()
    rng = np.random.default_rng(34)
    n = 2_000_000
    key = (rng.zipf(1.3, n) % 1_000_003).astype(np.int64)
    v = rng.integers(0, 1000, n).astype(np.int64)
    gb, *_ = run_both([cb.Column.from_numpy(key)], [(cb.Column.from_numpy(v), [agg.sum(), agg.count(), agg.max()])],
                      tuning={"force_mode": 2, **pass2})
    assert gb.stats()["mode"] == 2


@pytest.mark.parametrize("pass2", PASS2)
@pytest.mark.parametrize("hot_frac", [0.5, 0.95])
def test_partitioned_hot_key_warp_combined_updates(hot_frac, pass2):
    """One key holds most rows: its partition is split and each warp combines
    the hot key's values before one shared update, for every value type and
    accumulator the partitioned path takes."""
    cb, agg = _cb()
    rng = np.random.default_rng(37)
    n = 3_000_000
    key = rng.integers(0, 400_000, n).astype(np.int64)
    key[rng.random(n) < hot_frac] = 12345
    cols = [
        (rng.integers(-100, 100, n).astype(np.int8), None),
        (rng.integers(-30000, 30000, n).astype(np.int16), rng.random(n) > 0.1),
        (rng.integers(-2**31, 2**31 - 1, n).astype(np.int32), None),
        (rng.integers(0, 2**63, n, dtype=np.uint64), rng.random(n) > 0.3),
        (rng.normal(size=n).astype(np.float32), rng.random(n) > 0.1),
        (rng.normal(size=n), None),
        (rng.integers(0, 2, n).astype(np.uint8), None),
    ]
    types = [None, None, None, None, None, None, cb.TypeId.BOOL8]
    aggs = [agg.sum(), agg.min(), agg.max(), agg.count(), agg.mean(), agg.sum_of_squares()]
    reqs = []
    for (v, m), t in zip(cols, types):
        reqs.append((cb.Column.from_numpy(v, m, t) if t is not None else cb.Column.from_numpy(v, m), aggs))
    gb, *_ = run_both([cb.Column.from_numpy(key)], reqs[:4], tuning={"force_mode": 2, **pass2})
    assert gb.stats()["mode"] == 2
    gb, *_ = run_both([cb.Column.from_numpy(key)], reqs[4:], tuning={"force_mode": 2, **pass2})
    assert gb.stats()["mode"] == 2


@pytest.mark.parametrize("pass2", PASS2_ROW)
@pytest.mark.parametrize("include", [False, True])
def test_zipf_pairs_two_word_keys(include, pass2):
    """The shape of the high-cardinality benchmark at 4M rows: (int32, int64)
    keys = divmod(p, 1000) with p Zipf-skewed, 5% nulls per key column."""
    cb, agg = _cb()
    rng = np.random.default_rng(36)
    n = 4_000_000
    u = rng.random(n)
    a = 1.0 - 1.1
    p = np.clip(np.floor((1.0 - u * (1.0 - 2_000_001.0 ** a)) ** (1.0 / a) - 1.0), 0, 1_999_999).astype(np.int64)
    k1 = cb.Column.from_numpy((p // 1000).astype(np.int32), rng.random(n) >= 0.05)
    k2 = cb.Column.from_numpy(p % 1000, rng.random(n) >= 0.05)
    vi = rng.integers(0, 10**6, n, endpoint=True).astype(np.int64)
    vf = rng.random(n)
    aggs = [agg.sum(), agg.count(), agg.max()]
    gb, *_ = run_both([k1, k2], [(cb.Column.from_numpy(vi), aggs), (cb.Column.from_numpy(vf), aggs)],
                      include_null_keys=include, tuning={**pass2})
    assert gb.stats()["mode"] == 2


@pytest.mark.parametrize("scatter", [7, 8])
def test_two_word_keys_many_partitions(scatter):
    """(int32, int64) keys with nulls over ~3M groups: 2048 partitions, too
    many for the bulk pass's 4096-row tiles with two-word keys, so it runs on
    3072-row tiles (scatter 7) or 2048-row tiles with two CTAs per SM (8)."""
    cb, agg = _cb()
    rng = np.random.default_rng(52)
    n = 6_000_000
    p = rng.integers(0, 3_000_000, n)
    k1 = cb.Column.from_numpy((p // 1000).astype(np.int32), rng.random(n) >= 0.05)
    k2 = cb.Column.from_numpy(p % 1000 * 7919, rng.random(n) >= 0.05)
    vi = rng.integers(-10**9, 10**9, n).astype(np.int64)
    vf = rng.normal(size=n)
    aggs = [agg.sum(), agg.count(), agg.min(), agg.max()]
    gb, *_ = run_both([k1, k2], [(cb.Column.from_numpy(vi), aggs), (cb.Column.from_numpy(vf), aggs)],
                      include_null_keys=True, tuning={"force_mode": 2, "scatter": scatter})
    assert gb.stats()["mode"] == 2


def test_distributed_groupby_single_rank_with_engine():
    """The multi-GPU path with the engine as local aggregation (world size 1 on
    one GPU: partial aggregate, self-exchange, merge)."""
    import os
    import torch.distributed as dist
    from cudf_b200.distributed import distributed_groupby
    from cudf_b200.types import Kind, NullPolicy
    if not dist.is_initialized():
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        os.environ.setdefault("MASTER_PORT", "29561")
        dist.init_process_group("gloo", rank=0, world_size=1)
    rng = np.random.default_rng(77)
    n = 200_000
    k = rng.integers(0, 5000, n).astype(np.int64)
    v = rng.integers(-10**6, 10**6, n).astype(np.int64)
    f = rng.normal(size=n)
    m = rng.random(n) > 0.1
    kinds = [Kind.SUM, Kind.COUNT_VALID, Kind.MIN, Kind.MAX, Kind.MEAN]
    dev = torch.device("cuda")
    mk, mres = distributed_groupby([(torch.from_numpy(k).to(dev), None, O.INT64)],
                                   [((torch.from_numpy(v).to(dev), torch.from_numpy(m).to(dev), O.INT64), kinds),
                                    ((torch.from_numpy(f).to(dev), None, O.FLOAT64), kinds)], NullPolicy.EXCLUDE)
    o = O.groupby([O.HostColumn(O.INT64, k)], [(O.HostColumn(O.INT64, v, m), [int(x) for x in kinds]),
                                               (O.HostColumn(O.FLOAT64, f), [int(x) for x in kinds])])
    from parity import compare
    gk = [(mk[0][0].cpu().numpy(), None)]
    gr = [[(d.cpu().numpy(), None if vv is None else vv.cpu().numpy()) for d, vv in per] for per in mres]
    compare(o, gk, gr, [[int(x) for x in kinds]] * 2, None)


def test_concurrent_calls_on_separate_streams():
    """Four host threads, each with its own stream, run groupbys of different
    modes (and so different shared-memory sizes for the same kernels) at the
    same time; every result equals the same call made alone."""
    import threading
    cb, agg = _cb()
    rng = np.random.default_rng(38)
    shapes = [(1_500_000, 300_000), (200_000, 50), (2_500_000, 1_000_000), (800_000, 5_000)]
    inputs = []
    for n, card in shapes:
        k = rng.integers(0, card, n).astype(np.int64) * 7919
        v = rng.integers(-10**9, 10**9, n).astype(np.int64)
        inputs.append((cb.Column.from_numpy(k), cb.Column.from_numpy(v, rng.random(n) > 0.1)))
    aggs = [agg.sum(), agg.count(), agg.min(), agg.max()]

    def run(i, out):
        k, v = inputs[i]
        s = torch.cuda.Stream()
        with torch.cuda.stream(s):
            for _ in range(3):
                uk, res = cb.GroupBy(cb.Table([k])).aggregate([cb.GroupByRequest(v, aggs)], stream=s)
            s.synchronize()
        out[i] = (uk, res)

    alone = [None] * 4
    for i in range(4):
        run(i, alone)
    mixed = [None] * 4
    th = [threading.Thread(target=run, args=(i, mixed)) for i in range(4)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    for i in range(4):
        (ka, ra), (km, rm) = alone[i], mixed[i]
        a_keys, a_vals = ka[0].to_numpy()[0], [c.to_numpy() for c in ra[0].columns]
        m_keys, m_vals = km[0].to_numpy()[0], [c.to_numpy() for c in rm[0].columns]
        oa, om = np.argsort(a_keys), np.argsort(m_keys)
        assert np.array_equal(a_keys[oa], m_keys[om])
        for (av, avv), (mv, mvv) in zip(a_vals, m_vals):
            assert np.array_equal(av[oa], mv[om])
            if avv is not None:
                assert np.array_equal(avv[oa], mvv[om])


def test_tuning_rules_pick_settings_by_size_bucket():
    """A rule for small calls forces the global table; a larger call falls in
    the next rule; a handle's own setting wins over the rules."""
    from cudf_b200 import autotune
    cb, agg = _cb()
    rng = np.random.default_rng(39)
    try:
        autotune.set_rules([{"max_rows": 300_000, "max_groups": 1 << 30, "tuning": {"force_mode": 0}},
                            {"max_rows": 1 << 40, "max_groups": 1 << 30, "tuning": {"force_mode": 1}}])
        for n, want_mode, want_rule in ((200_000, 0, 0), (1_500_000, 1, 1)):
            k = rng.integers(0, 3000, n).astype(np.int64)
            v = rng.integers(-10**6, 10**6, n).astype(np.int64)
            gb, *_ = run_both([cb.Column.from_numpy(k)], [(cb.Column.from_numpy(v), [agg.sum(), agg.max()])])
            st = gb.stats()
            assert st["mode"] == want_mode and st["rule"] == want_rule
        k = rng.integers(0, 3000, 200_000).astype(np.int64)
        gb, *_ = run_both([cb.Column.from_numpy(k)], [(cb.Column.from_numpy(k), [agg.sum()])],
                          tuning={"force_mode": 1})
        assert gb.stats()["mode"] == 1
    finally:
        autotune.clear()
        import os
        if os.path.exists(autotune.TUNING_FILE):
            autotune.load()  # the shipped rules, for the tests that follow


@pytest.mark.parametrize("policy", [False, True])
def test_shared_stage_row_ranges_match_both_kernels(policy):
    """Low cardinality: the row-range kernel (closed-form plans, warp-combined
    updates) and the per-row shared-stage kernel (taken when the caller sizes
    the table) both equal the oracle, on sliced columns with nullable keys."""
    cb, agg = _cb()
    rng = np.random.default_rng(40)
    n = 1_200_000
    off = 37
    k1 = rng.integers(0, 4, n + off).astype(np.int32)           # a few hot keys
    k2 = rng.integers(0, 60, n + off).astype(np.int64)
    kv = rng.random(n + off) > 0.05
    cols = [(rng.integers(-2**40, 2**40, n + off).astype(np.int64), rng.random(n + off) > 0.1),
            (rng.normal(size=n + off).astype(np.float32), rng.random(n + off) > 0.1),
            (rng.integers(0, 2**16, n + off).astype(np.uint16), None)]

    def sliced(arr, valid, tid=None):
        c = cb.Column.from_numpy(arr, valid, tid) if tid is not None else cb.Column.from_numpy(arr, valid)
        return cb.Column(c.type_id, c.data, c.mask, size=n, offset=off)

    keys = [sliced(k1, kv), sliced(k2, None)]
    aggs = [agg.sum(), agg.min(), agg.max(), agg.count(), agg.mean(), agg.sum_of_squares()]
    reqs = [(sliced(v, m), aggs) for v, m in cols]
    gb, *_ = run_both(keys, reqs, include_null_keys=policy)
    assert gb.stats()["mode"] == 1
    gb, *_ = run_both(keys, reqs, include_null_keys=policy, tuning={"smem_bytes": 200_000, "smem_fill_pct": 70})
    assert gb.stats()["mode"] == 1


@pytest.mark.parametrize("pass2", PASS2_ROW)
def test_partitioned_many_partitions_wide_slots(pass2):
    """Wide slots (eight value columns) leave ~1000 slots per shared table, so
    3.5M groups need 8192 partitions; every group and value must still match."""
    cb, agg = _cb()
    rng = np.random.default_rng(41)
    n = 4_000_000
    key = rng.integers(0, 3_500_000, n).astype(np.int64) * 1_000_003
    reqs = []
    for i in range(8):
        v = rng.integers(-10**9, 10**9, n).astype(np.int64)
        reqs.append((cb.Column.from_numpy(v, rng.random(n) > 0.1 if i % 2 else None),
                     [agg.sum(), agg.min(), agg.max()]))
    gb, *_ = run_both([cb.Column.from_numpy(key)], reqs, tuning={**pass2})
    assert gb.stats()["mode"] == 2
