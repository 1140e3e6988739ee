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


# ---- generic driver: any keys / requests through gb_aggregate_noalloc ----

def _noalloc_any(L, _lib, torch, key_cols, reqs, policy, max_groups):
    """reqs: [(Column, [kinds], [ddof])]; returns ([(keys, valid)], [(values, valid)])."""
    keys = (_lib.GbColumn * len(key_cols))(*[c.gb_view() for c in key_cols])
    creqs = (_lib.GbRequest * max(1, len(reqs)))()
    keep, out_types = [], []
    for i, (col, kinds, ddof) in enumerate(reqs):
        aggs = (_lib.GbAgg * len(kinds))(*[_lib.GbAgg(k, d) for k, d in zip(kinds, ddof)])
        keep.append(aggs)
        creqs[i] = _lib.GbRequest(col.gb_view(), len(kinds), aggs)
        out_types += [O.target_type(int(col.type_id), k) for k in kinds]
    rows = max(1, max_groups)
    words = (rows + 31) // 32

    def out(t):
        b = torch.empty(rows * np.dtype(O.NP_DTYPE[t]).itemsize, dtype=torch.uint8, device="cuda")
        m = torch.empty(words, dtype=torch.int32, device="cuda")
        return b, m
    kb = [out(int(c.type_id)) for c in key_cols]
    rb = [out(t) for t in out_types]
    okeys = (_lib.GbOutColumn * len(key_cols))(*[_lib.GbOutColumn(0, 0, b.data_ptr(), m.data_ptr(), 0) for b, m in kb])
    ores = (_lib.GbOutColumn * max(1, len(out_types)))(
        *[_lib.GbOutColumn(0, 0, b.data_ptr(), m.data_ptr(), 0) for b, m in rb])
    ng = ctypes.c_int64(-1)
    stream = torch.cuda.current_stream().cuda_stream
    rc = L.gb_aggregate_noalloc(keys, len(key_cols), int(policy), creqs, len(reqs), max_groups, okeys, ores,
                                ctypes.byref(ng), stream)
    assert rc == 0, L.gb_last_error()
    torch.cuda.synchronize()
    G = ng.value

    def read(oc, bm, t):
        b, m = bm
        w = np.dtype(O.NP_DTYPE[t]).itemsize
        vals = b[: G * w].cpu().numpy().view(O.NP_DTYPE[t]) if G else np.zeros(0, O.NP_DTYPE[t])
        valid = O.unpack_mask(m.cpu().numpy().view(np.uint32), G) if oc.null_mask else None
        assert oc.size == G and oc.type_id == t
        assert oc.null_count == (0 if valid is None else int((~valid).sum()))
        return vals, valid
    ko = [read(okeys[i], kb[i], int(c.type_id)) for i, c in enumerate(key_cols)]
    ro = [read(ores[j], rb[j], t) for j, t in enumerate(out_types)]
    return G, ko, ro


def _compare_with_regular(cb, G, ko, ro, key_cols, reqs, policy, tol_of):
    from cudf_b200 import aggregation as agg
    from cudf_b200.types import Kind
    gb = cb.GroupBy(cb.Table(key_cols), policy)
    uk, res = gb.aggregate([cb.GroupByRequest(c, [agg.Aggregation(Kind(k), d) for k, d in zip(kinds, ddof)])
                            for c, kinds, ddof in reqs])
    rk = [c.to_numpy() for c in uk.columns]
    rr = [c.to_numpy() for t in res for c in t.columns]
    assert G == rk[0][0].shape[0]
    no, ro_ = O.sort_order(ko), O.sort_order(rk)
    for (a, av), (b, bv) in zip(ko, rk):
        av = np.ones(G, bool) if av is None else av[no]
        bv = np.ones(G, bool) if bv is None else bv[ro_]
        assert np.array_equal(av, bv)
        assert np.array_equal(a[no][av], b[ro_][bv])
    for j, ((a, av), (b, bv)) in enumerate(zip(ro, rr)):
        a, b = a[no], b[ro_]
        av = np.ones(G, bool) if av is None else av[no]
        bv = np.ones(G, bool) if bv is None else bv[ro_]
        assert np.array_equal(av, bv), f"output {j}: validity differs"
        if a.dtype.kind == "f":
            t = tol_of(j)[av]
            d = np.abs(a[av].astype(np.float64) - b[bv].astype(np.float64))
            assert np.all((d <= t) | (np.isnan(a[av]) & np.isnan(b[bv]))), f"output {j}: beyond tolerance"
        else:
            assert np.array_equal(a[av], b[bv]), f"output {j}: differs"


@pytest.mark.parametrize("policy", [0, 1], ids=["exclude", "include"])
def test_noalloc_nullable_two_column_keys_and_variance_on_a_sliced_column(policy):
    """Two nullable key columns (two packed key words, the output key masks and
    their clearing), INCLUDE and EXCLUDE, and VARIANCE/STD (the second pass on
    the static table) over a value column read at a row offset."""
    import torch

    import cudf_b200 as cb
    from cudf_b200 import _lib
    L = _lib.lib()
    rng = np.random.default_rng(5)
    n, off = 200_000, 37
    k1 = rng.integers(0, 60, n).astype(np.int32)
    k2 = rng.integers(-5, 40, n).astype(np.int64) * 1_000_003
    kv1, kv2 = rng.random(n) > 0.07, rng.random(n) > 0.05
    v = rng.normal(size=n + off)
    vv = rng.random(n + off) > 0.1
    vi = rng.integers(-1000, 1000, n).astype(np.int64)
    key_cols = [cb.Column.from_numpy(k1, kv1), cb.Column.from_numpy(k2, kv2)]
    full = cb.Column.from_numpy(v, vv)
    sliced = cb.Column(full.type_id, full.data, full.mask, size=n, offset=off)
    kinds_f = [O.VARIANCE, O.STD, O.SUM, O.MEAN, O.COUNT_VALID]
    ddof_f = [1, 0, 0, 0, 0]
    kinds_i = [O.MIN, O.MAX, O.SUM, O.COUNT_ALL]
    reqs = [(sliced, kinds_f, ddof_f), (cb.Column.from_numpy(vi), kinds_i, [0] * 4)]
    for call in range(2):
        G, ko, ro = _noalloc_any(L, _lib, torch, key_cols, reqs, policy, 20_000)
        assert G > 0
        orc = O.groupby([O.HostColumn(O.INT32, k1, kv1), O.HostColumn(O.INT64, k2, kv2)],
                        [(O.HostColumn(O.FLOAT64, v[off:], vv[off:]), kinds_f, ddof_f),
                         (O.HostColumn(O.INT64, vi), kinds_i)], include_null_keys=bool(policy))
        assert orc.num_groups == G
        oo = O.sort_order(orc.keys)
        # each engine result lies within the oracle's bound of the exact value
        tols = [2 * t[oo] for per in orc.results for (_, _, t) in per]
        _compare_with_regular(cb, G, ko, ro, key_cols, reqs, policy, lambda j: tols[j])


def test_noalloc_empty_input():
    import torch

    import cudf_b200 as cb
    from cudf_b200 import _lib
    L = _lib.lib()
    kc = cb.Column.from_numpy(np.zeros(0, np.int64))
    vc = cb.Column.from_numpy(np.zeros(0, np.float64), np.zeros(0, bool))
    G, ko, ro = _noalloc_any(L, _lib, torch, [kc], [(vc, [O.SUM, O.COUNT_VALID, O.MEAN], [0, 0, 0])], 0, 16)
    assert G == 0
    assert all(v.shape[0] == 0 for v, _ in ko + ro)


def _cudart():
    lib = ctypes.CDLL("libcudart.so.12")
    lib.cudaDeviceGetDefaultMemPool.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int]
    lib.cudaMemPoolGetAttribute.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
    lib.cudaMemPoolSetAttribute.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
    return lib


def test_noalloc_second_call_allocates_nothing():
    """After a first call (which looks up the scratch array's address), a second
    call leaves device memory untouched: the free memory the driver reports,
    the stream-ordered pool the engine's regular path allocates from (current
    and high-water use), and torch's caching allocator are all unchanged."""
    import torch

    import cudf_b200 as cb
    from cudf_b200 import _lib
    L = _lib.lib()
    key, v1, v2, m1, m2 = _inputs(303, 250_000, 9_000)
    kc, vc1, vc2 = cb.Column.from_numpy(key), cb.Column.from_numpy(v1, m1), cb.Column.from_numpy(v2, m2)
    k1, k2 = _kinds()
    reqs = [(vc1, k1, [0] * len(k1)), (vc2, k2, [0] * len(k2))]
    _noalloc_any(L, _lib, torch, [kc], reqs, 0, MAX_GROUPS)  # warm: address lookup, module load
    # the outputs of the measured call are allocated before the measurement
    keys = (_lib.GbColumn * 1)(kc.gb_view())
    creqs = (_lib.GbRequest * 2)()
    keep = []
    outs = []
    for i, (col, kinds, ddof) in enumerate(reqs):
        aggs = (_lib.GbAgg * len(kinds))(*[_lib.GbAgg(k, d) for k, d in zip(kinds, ddof)])
        keep.append(aggs)
        creqs[i] = _lib.GbRequest(col.gb_view(), len(kinds), aggs)
        outs += [torch.empty(MAX_GROUPS * 8, dtype=torch.uint8, device="cuda") for _ in kinds]
    masks = [torch.empty((MAX_GROUPS + 31) // 32, dtype=torch.int32, device="cuda") for _ in outs]
    kbuf = torch.empty(MAX_GROUPS * 8, dtype=torch.uint8, device="cuda")
    okeys = (_lib.GbOutColumn * 1)(_lib.GbOutColumn(0, 0, kbuf.data_ptr(), 0, 0))
    ores = (_lib.GbOutColumn * len(outs))(*[_lib.GbOutColumn(0, 0, b.data_ptr(), m.data_ptr(), 0)
                                            for b, m in zip(outs, masks)])
    ng = ctypes.c_int64(-1)
    rt = _cudart()
    pool = ctypes.c_void_p()
    assert rt.cudaDeviceGetDefaultMemPool(ctypes.byref(pool), torch.cuda.current_device()) == 0
    used, high, reserved = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
    zero = ctypes.c_uint64(0)
    torch.cuda.synchronize()
    assert rt.cudaMemPoolSetAttribute(pool, 8, ctypes.byref(zero)) == 0  # reset the high-water mark
    rt.cudaMemPoolGetAttribute(pool, 7, ctypes.byref(used))
    rt.cudaMemPoolGetAttribute(pool, 5, ctypes.byref(reserved))
    free0, _ = torch.cuda.mem_get_info()
    torch_alloc0 = torch.cuda.memory_allocated()
    torch_reserved0 = torch.cuda.memory_reserved()
    used0, reserved0 = used.value, reserved.value
    rc = L.gb_aggregate_noalloc(keys, 1, 0, creqs, 2, MAX_GROUPS, okeys, ores, ctypes.byref(ng),
                                torch.cuda.current_stream().cuda_stream)
    assert rc == 0, L.gb_last_error()
    torch.cuda.synchronize()
    rt.cudaMemPoolGetAttribute(pool, 7, ctypes.byref(used))
    rt.cudaMemPoolGetAttribute(pool, 8, ctypes.byref(high))
    rt.cudaMemPoolGetAttribute(pool, 5, ctypes.byref(reserved))
    free1, _ = torch.cuda.mem_get_info()
    assert ng.value > 0
    assert used.value == used0 and high.value <= used0, (used0, used.value, high.value)
    assert reserved.value == reserved0
    assert free1 == free0, (free0, free1)
    assert torch.cuda.memory_allocated() == torch_alloc0
    assert torch.cuda.memory_reserved() == torch_reserved0
