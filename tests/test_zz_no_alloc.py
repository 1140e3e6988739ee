"""gb_aggregate_noalloc: the groupby entry point that allocates nothing.

Callers whose device memory belongs to another allocator, or that must not
call cudaMalloc/cudaFree (they synchronise the device), use this entry point:
its hash table lives in a fixed file-scope device array and it writes into
output buffers the caller allocated.  These tests call it through the C ABI,
twice in a row on different inputs, and check each result against the
regular entry point (gb_aggregate) on the same inputs -- integers bit for bit,
floating sums and means within twice the oracle's per-group bound (each result
lies within the bound of the exact sum).  The file sorts last so that a run
that stops at the first failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

MAX_GROUPS = 20_000


def _inputs(seed, n, card):
    rng = np.random.default_rng(seed)
    key = rng.integers(0, card, n).astype(np.int64) * 7919 - 3
    v1 = rng.integers(-10**9, 10**9, n).astype(np.int64)
    v2 = rng.normal(size=n)
    m1 = rng.random(n) > 0.1
    m2 = rng.random(n) > 0.2
    return key, v1, v2, m1, m2


def _kinds():
    return [O.SUM, O.COUNT_VALID, O.MIN, O.MAX, O.MEAN], [O.SUM, O.MEAN, O.MAX, O.COUNT_ALL]


def _noalloc(cb, L, _lib, torch, kc, vc1, vc2):
    k1, k2 = _kinds()
    reqs = (_lib.GbRequest * 2)()
    aggs1 = (_lib.GbAgg * len(k1))(*[_lib.GbAgg(k, 0) for k in k1])
    aggs2 = (_lib.GbAgg * len(k2))(*[_lib.GbAgg(k, 0) for k in k2])
    reqs[0] = _lib.GbRequest(vc1.gb_view(), len(k1), aggs1)
    reqs[1] = _lib.GbRequest(vc2.gb_view(), len(k2), aggs2)
    keys = (_lib.GbColumn * 1)(kc.gb_view())
    # caller-allocated outputs: data for MAX_GROUPS rows, masks for nullable results
    words = (MAX_GROUPS + 31) // 32
    out_types = [O.target_type(O.INT64, k) for k in k1] + [O.target_type(O.FLOAT64, k) for k in k2]
    widths = {O.INT32: 4, O.INT64: 8, O.FLOAT64: 8}
    bufs, masks = [], []
    for t in out_types:
        bufs.append(torch.empty(MAX_GROUPS * widths[t], dtype=torch.uint8, device="cuda"))
        masks.append(torch.empty(words, dtype=torch.int32, device="cuda"))
    kbuf = torch.empty(MAX_GROUPS * 8, dtype=torch.uint8, device="cuda")
    okeys = (_lib.GbOutColumn * 1)(_lib.GbOutColumn(0, 0, kbuf.data_ptr(), 0, 0))
    ores = (_lib.GbOutColumn * len(out_types))(
        *[_lib.GbOutColumn(0, 0, b.data_ptr(), m.data_ptr(), 0) for b, m in zip(bufs, masks)])
    ng = ctypes.c_int64(-1)
    stream = torch.cuda.current_stream().cuda_stream
    rc = L.gb_aggregate_noalloc(keys, 1, 0, reqs, 2, MAX_GROUPS, okeys, ores, ctypes.byref(ng), stream)
    assert rc == 0, L.gb_last_error()
    torch.cuda.synchronize()
    G = ng.value
    keys_np = kbuf[: G * 8].view(torch.int64).cpu().numpy()
    res = []
    for j, t in enumerate(out_types):
        np_t = {O.INT32: torch.int32, O.INT64: torch.int64, O.FLOAT64: torch.float64}[t]
        vals = bufs[j][: G * widths[t]].view(np_t).cpu().numpy()
        if ores[j].null_mask:
            valid = O.unpack_mask(masks[j].cpu().numpy().view(np.uint32), G)
        else:
            valid = np.ones(G, bool)
        assert ores[j].type_id == t and ores[j].size == G
        assert ores[j].null_count == int((~valid).sum())
        res.append((vals, valid))
    return keys_np, res


def _regular(cb, agg, kc, vc1, vc2):
    gb = cb.GroupBy(cb.Table([kc]))
    uk, res = gb.aggregate([
        cb.GroupByRequest(vc1, [agg.sum(), agg.count(), agg.min(), agg.max(), agg.mean()]),
        cb.GroupByRequest(vc2, [agg.sum(), agg.mean(), agg.max(), agg.count(cb.NullPolicy.INCLUDE)]),
    ])
    keys_np = uk.columns[0].to_numpy()[0]
    out = []
    for t in res:
        for c in t.columns:
            d, v = c.to_numpy()
            out.append((d, np.ones(d.shape[0], bool) if v is None else v))
    return keys_np, out


@pytest.mark.parametrize("dummy", [0])
def test_noalloc_matches_regular_entry_point_on_two_calls(dummy):
    import torch

    import cudf_b200 as cb
    from cudf_b200 import _lib
    from cudf_b200 import aggregation as agg
    L = _lib.lib()
    k1, k2 = _kinds()
    for call, (seed, n, card) in enumerate([(101, 300_000, 15_000), (202, 120_000, 4_000)]):
        key, v1, v2, m1, m2 = _inputs(seed, n, card)
        kc = cb.Column.from_numpy(key)
        vc1 = cb.Column.from_numpy(v1, m1)
        vc2 = cb.Column.from_numpy(v2, m2)
        nk, nres = _noalloc(cb, L, _lib, torch, kc, vc1, vc2)
        rk, rres = _regular(cb, agg, kc, vc1, vc2)
        assert nk.shape[0] == rk.shape[0] > 0, f"call {call}: group counts differ"
        no, ro = np.argsort(nk), np.argsort(rk)
        assert np.array_equal(nk[no], rk[ro]), f"call {call}: keys differ"
        # floating tolerance: the oracle's per-group bound, doubled
        orc = O.groupby([O.HostColumn(O.INT64, key)],
                        [(O.HostColumn(O.INT64, v1, m1), k1), (O.HostColumn(O.FLOAT64, v2, m2), k2)])
        oo = np.argsort(orc.keys[0][0])
        tols = [t for per in orc.results for (_, _, t) in per]
        for j, ((a, av), (b, bv)) in enumerate(zip(nres, rres)):
            a, av, b, bv = a[no], av[no], b[ro], bv[ro]
            assert np.array_equal(av, bv), f"call {call} output {j}: validity differs"
            if a.dtype.kind == "f":
                tol = 2 * tols[j][oo]
                assert np.all(np.abs(a[av] - b[bv]) <= tol[av]), f"call {call} output {j}: beyond tolerance"
            else:
                assert np.array_equal(a[av], b[bv]), f"call {call} output {j}: differs"


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch

    import cudf_b200 as cb
    from cudf_b200 import _lib
    L = _lib.lib()
    kc = cb.Column.from_numpy(np.arange(1000, dtype=np.int64))
    keys = (_lib.GbColumn * 1)(kc.gb_view())
    buf = torch.empty(8 * 1000, dtype=torch.uint8, device="cuda")
    okeys = (_lib.GbOutColumn * 1)(_lib.GbOutColumn(0, 0, buf.data_ptr(), 0, 0))
    ng = ctypes.c_int64(-1)
    # a table for 10^8 groups cannot fit the fixed scratch array
    rc = L.gb_aggregate_noalloc(keys, 1, 0, None, 0, 100_000_000, okeys, None, ctypes.byref(ng), 0)
    assert rc == _lib.GB_ERR_LOGIC
    assert b"needs" in L.gb_last_error()
    # more groups (1000) than the caller's max_groups (100)
    rc = L.gb_aggregate_noalloc(keys, 1, 0, None, 0, 100, okeys, None, ctypes.byref(ng), 0)
    assert rc == _lib.GB_ERR_LOGIC
    assert b"max_groups" in L.gb_last_error()
