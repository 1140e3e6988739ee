"""Expands tests/golden/golden_vectors.json into concrete cases and checks a
groupby result against them, the way libcudf's test_single_agg does: sort the
result by key, then compare keys and values
(cpp/tests/groupby/groupby_test_util.cpp:33-97)."""
import json
import math
import os

import numpy as np

from oracle import oracle as O

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "golden_vectors.json")

TYPE_IDS = {
    "INT8": O.INT8, "INT16": O.INT16, "INT32": O.INT32, "INT64": O.INT64,
    "UINT8": O.UINT8, "UINT16": O.UINT16, "UINT32": O.UINT32, "UINT64": O.UINT64,
    "FLOAT32": O.FLOAT32, "FLOAT64": O.FLOAT64, "BOOL8": O.BOOL8,
    "TIMESTAMP_DAYS": O.TIMESTAMP_DAYS, "TIMESTAMP_SECONDS": O.TIMESTAMP_SECONDS,
    "TIMESTAMP_MILLISECONDS": O.TIMESTAMP_MILLISECONDS,
    "TIMESTAMP_MICROSECONDS": O.TIMESTAMP_MICROSECONDS,
    "TIMESTAMP_NANOSECONDS": O.TIMESTAMP_NANOSECONDS,
    "DURATION_DAYS": O.DURATION_DAYS, "DURATION_SECONDS": O.DURATION_SECONDS,
    "DURATION_MILLISECONDS": O.DURATION_MILLISECONDS,
    "DURATION_MICROSECONDS": O.DURATION_MICROSECONDS,
    "DURATION_NANOSECONDS": O.DURATION_NANOSECONDS,
}
AGG_IDS = {"SUM": O.SUM, "PRODUCT": O.PRODUCT, "MIN": O.MIN, "MAX": O.MAX,
           "COUNT_VALID": O.COUNT_VALID, "COUNT_ALL": O.COUNT_ALL, "MEAN": O.MEAN,
           "SUM_OF_SQUARES": O.SUM_OF_SQUARES, "VARIANCE": O.VARIANCE, "STD": O.STD,
           "ARGMIN": O.ARGMIN, "ARGMAX": O.ARGMAX}


def _num(x):
    if isinstance(x, str):
        return {"nan": math.nan, "inf": math.inf, "-inf": -math.inf}[x]
    return x


def _column(type_name, values, valid):
    tid = TYPE_IDS[type_name]
    vals = [_num(v) for v in values]
    if tid == O.BOOL8:
        data = np.array([1 if v else 0 for v in vals], dtype=np.uint8)
    else:
        data = np.array(vals, dtype=O.NP_DTYPE[tid]) if vals else np.zeros(0, O.NP_DTYPE[tid])
    return O.HostColumn(tid, data, None if valid is None else np.array(valid, dtype=bool))


def expand():
    """Yield (case_id, case, keys HostColumn, values HostColumn, kinds)."""
    with open(GOLDEN) as f:
        cases = json.load(f)["cases"]
    for c in cases:
        for kt in c["key_types"]:
            for vt in c["value_types"]:
                # bool values only take part where the typed suite includes them
                k = _column(kt, c["keys"], c["key_valid"])
                v = _column(vt, c["vals"], c["val_valid"])
                kinds = [AGG_IDS[a] for a in c["aggs"]]
                yield f"{c['name']}[{kt}-{vt}]", c, k, v, kinds


def expected_values(case, value_type_id, agg_name, kind):
    exp = case["expect"][agg_name]
    tt = O.target_type(value_type_id, kind)
    valid = np.array([e is not None for e in exp], dtype=bool)
    vals = [0 if e is None else _num(e) for e in exp]
    if tt == O.BOOL8:
        arr = np.array([1 if v else 0 for v in vals], dtype=np.uint8)
    else:
        arr = np.array(vals, dtype=O.NP_DTYPE[tt]) if vals else np.zeros(0, O.NP_DTYPE[tt])
    return arr, valid


def check(case, key_col, value_col, kinds, out_keys, out_results, tol_results=None):
    """out_keys: (data, valid|None) of the single key column; out_results: list of
    (values, valid|None) per aggregation, in request order."""
    exp_keys = _column(_type_name(key_col.type_id), case["expect_keys"],
                       case["expect_key_valid"])
    order = O.sort_order([out_keys])
    kd, kv = out_keys
    kd = np.asarray(kd)[order]
    kv = np.ones(kd.shape[0], bool) if kv is None else np.asarray(kv, bool)[order]
    ev = np.ones(len(exp_keys), bool) if exp_keys.valid is None else exp_keys.valid
    assert kd.shape[0] == len(exp_keys), f"{case['name']}: {kd.shape[0]} groups, expected {len(exp_keys)}"
    assert np.array_equal(kv, ev), f"{case['name']}: key validity {kv} != {ev}"
    assert np.array_equal(kd[kv], exp_keys.data[ev]), f"{case['name']}: keys {kd} != {exp_keys.data}"
    for j, (name, kind) in enumerate(zip(case["aggs"], kinds)):
        vals, valid = out_results[j]
        vals = np.asarray(vals)[order]
        valid = np.ones(vals.shape[0], bool) if valid is None else np.asarray(valid, bool)[order]
        evals, evalid = expected_values(case, value_col.type_id, name, kind)
        assert np.array_equal(valid, evalid), f"{case['name']} {name}: validity {valid} != {evalid}"
        a, b = vals[evalid], evals[evalid]
        if a.dtype.kind == "f":
            ok = np.isclose(a, b, rtol=1e-12, atol=0) | (np.isnan(a) & np.isnan(b))
            assert ok.all(), f"{case['name']} {name}: {a} != {b}"
        else:
            if value_col.type_id == O.BOOL8 and kind in (O.MIN, O.MAX):
                a, b = a != 0, b != 0
            assert np.array_equal(a, b), f"{case['name']} {name}: {a} != {b}"


def _type_name(tid):
    for k, v in TYPE_IDS.items():
        if v == tid:
            return k
    raise KeyError(tid)
