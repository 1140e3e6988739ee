"""Tuning rules through the C ABI (host-only calls, no GPU): install, order,
save/load, and rejection of invalid settings."""
import json

import pytest

from cudf_b200 import _lib, autotune


def test_rules_install_and_clear(tmp_path):
    rules = [{"max_rows": 1 << 24, "max_groups": 1 << 20, "tuning": {"force_mode": 2, "scatter": 3}},
             {"max_rows": 1 << 20, "max_groups": 1 << 10, "tuning": {"force_mode": 1, "smem_bytes": 49152}}]
    ordered = autotune.order_rules(rules)
    assert [r["max_rows"] for r in ordered] == [1 << 20, 1 << 24]
    autotune.set_rules(ordered)
    p = tmp_path / "t.json"
    autotune.save(ordered, str(p), {"device": "test"})
    assert json.load(open(p))["rules"] == ordered
    assert autotune.load(str(p)) == ordered
    autotune.clear()


def test_invalid_rule_is_rejected():
    with pytest.raises(ValueError):
        autotune.set_rules([{"max_rows": 10, "max_groups": 10, "tuning": {"scatter": 9}}])
    with pytest.raises(ValueError):
        autotune.set_rules([{"max_rows": 10, "max_groups": 10, "tuning": {"force_mode": 5}}])
    autotune.clear()


def test_tuning_struct_defaults_are_unset():
    t = autotune._tuning_struct({"scatter": 2})
    assert t.scatter == 2 and t.force_mode == -2 and t.block == -1 and t.smem_bytes == -1


def test_batch_tuning_install_and_reject():
    autotune.set_batch_tuning([{"max_rows": 1 << 20, "max_groups": 1 << 10, "headroom_pct": 300},
                               {"max_rows": 1 << 30, "max_groups": 1 << 30, "smem_slots": 0}],
                              {"block": 256, "tile_rows": 16384, "smem_bytes": 96 * 1024})
    with pytest.raises(ValueError):
        autotune.set_batch_tuning([], {"block": 300, "tile_rows": 16384, "smem_bytes": 0})
    with pytest.raises(ValueError):
        autotune.set_batch_tuning([], {"block": 512, "tile_rows": 10, "smem_bytes": 0})
    autotune.set_batch_tuning([], autotune.BATCH_LAUNCH_DEFAULT)


def test_batch_bucket_sizes_stay_inside_their_bucket():
    import numpy as np
    rng = np.random.default_rng(0)
    bounds = sorted({g for _, g in autotune.BATCH_BUCKETS})
    for r_hi, g_hi in autotune.BATCH_BUCKETS:
        sizes = autotune.bucket_sizes(rng, r_hi, g_hi)
        assert sizes
        g_lo = max([b for b in bounds if b < g_hi], default=1)
        for n, g in sizes:
            assert 1 <= n <= r_hi and 2 <= g <= n
            # groups from the bucket's own range unless the rows cap them
            assert g <= g_hi and (g > g_lo // 16 or g == max(2, n))
