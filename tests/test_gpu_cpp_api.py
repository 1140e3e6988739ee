"""libcudf's own known answers (cpp/tests/groupby/*.cpp), run through the
engine's libcudf-shaped C++ API (include/cudf_b200/groupby.hpp) by a compiled
C++ program: column_views over device buffers, make_*_aggregation factories,
cudf::groupby::groupby(keys, null_policy).aggregate(requests, stream, mr) on a
non-default stream, owning result columns, cudf::logic_error on invalid input.
"""
import subprocess

import numpy as np
import pytest

import golden_harness as GH
from oracle import oracle as O

CASES = list(GH.expand())


def _hex(col):
    w = col.data.dtype.itemsize
    u = np.ascontiguousarray(col.data).view({1: np.uint8, 2: np.uint16, 4: np.uint32, 8: np.uint64}[w])
    return " ".join(format(int(x), "x") for x in u)


def _valid(col):
    return "-" if col.valid is None else " ".join("1" if v else "0" for v in col.valid)


def _column(tokens):
    tid, n = int(tokens[0]), int(tokens[1])
    dt = np.dtype(O.NP_DTYPE[tid])
    u = np.array([int(t, 16) for t in tokens[2:2 + n]], dtype=np.uint64)
    raw = u.astype({1: np.uint8, 2: np.uint16, 4: np.uint32, 8: np.uint64}[dt.itemsize])
    return raw.view(dt)


def _validity(tokens):
    return None if tokens == ["-"] else np.array([t == "1" for t in tokens], dtype=bool)


def _run(cases):
    from cudf_b200 import build as B
    exe = B.build_cpp_tests()
    lines = []
    for cid, case, keys, vals, kinds in cases:
        lines += [f"case {cid}", f"policy {int(case['include_null_keys'])}",
                  f"key {keys.type_id} {len(keys)} {_hex(keys)}", f"keyvalid {_valid(keys)}",
                  f"val {vals.type_id} {len(vals)} {_hex(vals)}", f"valvalid {_valid(vals)}",
                  "aggs " + " ".join(str(k) for k in kinds), "run"]
    r = subprocess.run([exe], input="\n".join(lines) + "\n", capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    out, cur, mr = {}, None, None
    for ln in r.stdout.splitlines():
        t = ln.split()
        if not t:
            continue
        if t[0] == "case":
            cur = {"results": {}, "error": None}
            out[t[1]] = cur
        elif t[0] == "error":
            cur["error"] = t[1]
        elif t[0] == "groups":
            cur["groups"] = int(t[1])
        elif t[0] == "key":
            cur["key"] = _column(t[1:])
        elif t[0] == "keyvalid":
            cur["keyvalid"] = _validity(t[1:])
        elif t[0] == "result":
            cur["results"][int(t[1])] = [_column(t[2:]), None]
        elif t[0] == "resultvalid":
            cur["results"][max(cur["results"])][1] = _validity(t[1:])
        elif t[0] == "mr":
            mr = (int(t[1]), int(t[2]))
    return out, mr


@pytest.mark.gpu
def test_cpp_api_matches_reference_golden_vectors():
    out, mr = _run(CASES)
    assert len(out) == len(CASES)
    for cid, case, keys, vals, kinds in CASES:
        got = out[cid]
        if case["error"]:
            assert got["error"] == "logic", f"{cid}: expected cudf::logic_error, got {got}"
            continue
        assert got["error"] is None, f"{cid}: {got['error']}"
        results = [tuple(got["results"][j]) for j in range(len(kinds))]
        GH.check(case, keys, vals, kinds, (got["key"], got["keyvalid"]), results)
    # the last case ran once more through a counting device_memory_resource:
    # results were allocated through it and all of it was given back
    allocations, live = mr
    assert allocations > 0 and live == 0, mr
