"""Parity at the full sizes the benchmark times.

The engine runs on exactly the inputs `bench.py` generates for its two 100M-row
workloads, and every group is compared with the CPU oracle on host copies of
the same inputs, after sorting both by key (libcudf's own harness sorts the
same way, cpp/tests/groupby/groupby_test_util.cpp:88-91): keys, counts and
integer SUM/MIN/MAX bit for bit, floating SUM/MEAN within the oracle's
per-group bound 2*n*eps*sum|x| (eps of the accumulator type), floating MIN/MAX
exactly.

  * 100M rows, int64 key over 1M distinct values, three value columns with 10%
    nulls each, SUM/COUNT/MIN/MAX/MEAN: about 97k rows per partition of the
    partitioned path (1024 partitions), the regime the benchmark runs in.
  * 100M rows, (int32, int64) key pairs Zipf(1.1) over the full 50M-pair
    support, 5% nulls per key column under INCLUDE, SUM/COUNT/MAX: millions
    of groups with a few very heavy keys (split work items).
"""
import os

import numpy as np
import pytest
import torch

import bench
import parity
from oracle import oracle as O

pytestmark = pytest.mark.gpu

THREADS = os.cpu_count() or 1


def _engine(keys, reqs, policy):
    import cudf_b200 as cb
    gb = cb.GroupBy(cb.Table(keys), policy)
    gb.set_profile(True)
    uk, res = gb.aggregate(reqs)
    torch.cuda.synchronize()
    return gb, uk, res


def test_fullsize_100M_rows_1M_groups():
    import cudf_b200 as cb
    from cudf_b200 import aggregation as agg
    from cudf_b200.types import NullPolicy, TypeId
    dev = torch.device("cuda", 0)
    n = bench.N_ROWS
    key, vals, masks = bench.make_inputs_device(n, bench.SEED, dev, key_seed=bench.SEED)
    aggs = [agg.sum(), agg.count(), agg.min(), agg.max(), agg.mean()]
    types = (TypeId.INT64, TypeId.FLOAT64, TypeId.FLOAT32)
    reqs = [cb.GroupByRequest(cb.Column(t, v, m), aggs) for t, v, m in zip(types, vals, masks)]
    gb, uk, res = _engine([cb.Column(TypeId.INT64, key)], reqs, NullPolicy.EXCLUDE)
    st = gb.stats()
    assert st["mode"] == 2, f"expected the partitioned path at this size, got {st}"
    hk, hr = bench._oracle_inputs(key.cpu().numpy(), [v.cpu().numpy() for v in vals],
                                  [cb.column.unpack_mask(m, n).cpu().numpy() for m in masks])
    del key, vals, masks
    g = bench.check_with_oracle(hk, hr, False, uk, res)
    assert g == bench.N_DISTINCT


def test_fullsize_zipf_pairs_100M_rows_include_nulls():
    import cudf_b200 as cb
    from cudf_b200 import aggregation as agg
    from cudf_b200.types import NullPolicy, TypeId
    dev = torch.device("cuda", 0)
    n = 100_000_000
    cols = bench.zipf_inputs_device(n, dev)
    k1, k2, km, vi, vf = cols
    aggs = [agg.sum(), agg.count(), agg.max()]
    keys = [cb.Column(TypeId.INT32, k1, km[0]), cb.Column(TypeId.INT64, k2, km[1])]
    reqs = [cb.GroupByRequest(cb.Column(TypeId.INT64, vi), aggs),
            cb.GroupByRequest(cb.Column(TypeId.FLOAT64, vf), aggs)]
    gb, uk, res = _engine(keys, reqs, NullPolicy.INCLUDE)
    hk, hr, inc = bench.config_oracle_inputs("zipf", [c.cpu() for c in bench._flat(cols)], n)
    del cols, k1, k2, km, vi, vf
    g = bench.check_with_oracle(hk, hr, inc, uk, res)
    # Zipf(1.1) over 50M pairs with 5% nulls per key column leaves millions
    # of groups, four of them made of null keys
    assert g > 1_000_000
    kv = [np.asarray(v) for _, v in parity.gpu_pairs(uk)]
    assert not kv[0].all() and not kv[1].all()
