"""libcudf's own known answers (cpp/tests/groupby/*.cpp), run through the
engine's C ABI on the GPU."""
import numpy as np
import pytest

import golden_harness as GH

CASES = list(GH.expand())


@pytest.mark.gpu
@pytest.mark.parametrize("cid,case,keys,vals,kinds", CASES, ids=[c[0] for c in CASES])
def test_engine_matches_reference_golden_vectors(cid, case, keys, vals, kinds):
    import cudf_b200 as cb
    from cudf_b200 import aggregation as agg
    from cudf_b200.types import Kind
    kc = cb.Column.from_numpy(keys.data, keys.valid, keys.type_id)
    vc = cb.Column.from_numpy(vals.data, vals.valid, vals.type_id)
    aggs = [agg.Aggregation(Kind(k)) for k in kinds]
    policy = cb.NullPolicy.INCLUDE if case["include_null_keys"] else cb.NullPolicy.EXCLUDE
    gb = cb.GroupBy(cb.Table([kc]), policy)
    if case["error"]:
        with pytest.raises(ValueError):
            gb.aggregate([cb.GroupByRequest(vc, aggs)])
        return
    uk, res = gb.aggregate([cb.GroupByRequest(vc, aggs)])
    out = [c.to_numpy() for c in res[0].columns]
    GH.check(case, keys, vals, kinds, uk.columns[0].to_numpy(), out)
