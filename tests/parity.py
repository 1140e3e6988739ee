"""Compares an engine result with the CPU oracle on the same inputs: both are
sorted by key (libcudf's own tests do the same, cpp/tests/groupby/
groupby_test_util.cpp:88-91), integer results must match bit for bit and
floating SUM/MEAN/VAR/STD must lie within the oracle's per-group bound
(2*n*eps*sum|x| for sums, eps of the accumulator type)."""
import numpy as np
import torch

from oracle import oracle as O


def host_cols(cols):
    return [O.HostColumn(int(c.type_id), *c.to_numpy()) for c in cols]


def gpu_pairs(table):
    return [c.to_numpy() for c in table.columns]


def _eq_values(a, b):
    if a.dtype.kind == "f":
        return (a == b) | (np.isnan(a) & np.isnan(b))
    return a == b


def compare(oracle_res, gpu_keys, gpu_results, kinds_per_req, value_types):
    """oracle_res: oracle.OracleResult; gpu_keys: [(data, valid)]; gpu_results:
    [[(data, valid)]] per request."""
    G = oracle_res.num_groups
    assert all(k[0].shape[0] == G for k in gpu_keys), \
        f"group count {gpu_keys[0][0].shape[0]} != oracle {G}"
    og = O.sort_order(oracle_res.keys)
    gg = O.sort_order(gpu_keys)
    for (od, ov), (gd, gv) in zip(oracle_res.keys, gpu_keys):
        od, gd = np.asarray(od)[og], np.asarray(gd)[gg]
        ov = np.ones(G, bool) if ov is None else np.asarray(ov)[og]
        gv = np.ones(G, bool) if gv is None else np.asarray(gv)[gg]
        assert np.array_equal(ov, gv), "key validity differs"
        if od.dtype != gd.dtype and od.dtype.kind != "f":
            gd = gd.astype(od.dtype)
        ok = _eq_values(od[ov], gd[ov])
        assert ok.all(), f"keys differ at {np.nonzero(~ok)[0][:5]}"
    for r, kinds in enumerate(kinds_per_req):
        for j, kind in enumerate(kinds):
            ovals, ovalid, otol = oracle_res.results[r][j]
            gvals, gvalid = gpu_results[r][j]
            ovals, ovalid, otol = ovals[og], ovalid[og], otol[og]
            gvals = np.asarray(gvals)[gg]
            gvalid = np.ones(G, bool) if gvalid is None else np.asarray(gvalid)[gg]
            assert np.array_equal(ovalid, gvalid), \
                f"request {r} agg {kind}: validity differs at {np.nonzero(ovalid != gvalid)[0][:5]}"
            a, b, t = ovals[ovalid], gvals[ovalid], otol[ovalid]
            if kind in (O.ARGMIN, O.ARGMAX):
                assert np.array_equal(a, b.astype(a.dtype)), f"request {r} {kind}: arg index differs"
                continue
            if a.dtype.kind == "f":
                a64, b64 = a.astype(np.float64), b.astype(np.float64)
                both_nan = np.isnan(a64) & np.isnan(b64)
                exact = kind in (O.MIN, O.MAX)
                if exact:
                    ok = (a64 == b64) | both_nan
                else:
                    ok = (np.abs(a64 - b64) <= t) | both_nan | (a64 == b64)
                bad = np.nonzero(~ok)[0]
                assert ok.all(), (f"request {r} kind {kind}: {len(bad)} groups off, e.g. oracle "
                                  f"{a64[bad[:3]]} gpu {b64[bad[:3]]} tol {t[bad[:3]]}")
            else:
                if b.dtype != a.dtype:
                    b = b.astype(a.dtype)
                ok = a == b
                bad = np.nonzero(~ok)[0]
                assert ok.all(), f"request {r} kind {kind}: {len(bad)} groups differ, e.g. {a[bad[:3]]} vs {b[bad[:3]]}"


def run_both(keys_dev, reqs_dev, include_null_keys=False, tuning=None, nthreads=8):
    """keys_dev: [Column]; reqs_dev: [(Column, [Aggregation])]."""
    import cudf_b200 as cb
    gb = cb.GroupBy(cb.Table(keys_dev), cb.NullPolicy.INCLUDE if include_null_keys else cb.NullPolicy.EXCLUDE)
    if tuning:
        gb.set_tuning(**tuning)
    uk, res = gb.aggregate([cb.GroupByRequest(c, aggs) for c, aggs in reqs_dev])
    torch.cuda.synchronize()
    o = O.groupby(host_cols(keys_dev),
                  [(host_cols([c])[0], [int(a.kind) for a in aggs], [int(a.param) for a in aggs])
                   for c, aggs in reqs_dev],
                  include_null_keys=include_null_keys, nthreads=nthreads)
    compare(o, gpu_pairs(uk), [gpu_pairs(t) for t in res],
            [[int(a.kind) for a in aggs] for _, aggs in reqs_dev], None)
    return gb, uk, res, o
