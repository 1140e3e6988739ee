"""The C-ABI library loads and exports every symbol include/*.h declares; its
host-side type rules agree with the oracle (CPU only, no kernels launched)."""
import glob
import os
import re

import pytest

from cudf_b200 import _lib
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        names |= set(re.findall(r"GB_API\s+[\w\s\*]+?\b(gb_\w+)\s*\(", text))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    syms = declared_symbols()
    assert "gb_aggregate" in syms and "gb_create" in syms
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing, f"declared but not exported: {missing}"


def test_every_export_has_a_binding_signature():
    for s in declared_symbols():
        assert s in _lib.SIGNATURES, f"{s} has no ctypes signature in cudf_b200/_lib.py"


@pytest.mark.parametrize("type_id", list(range(1, 22)))
def test_type_rules_match_oracle(type_id):
    L = _lib.lib()
    for kind in (O.SUM, O.PRODUCT, O.MIN, O.MAX, O.COUNT_VALID, O.COUNT_ALL, O.SUM_OF_SQUARES,
                 O.MEAN, O.VARIANCE, O.STD, O.ARGMAX, O.ARGMIN, 6, 7, 13, 14):
        ok = bool(L.gb_is_valid_aggregation(type_id, kind))
        assert ok == O.valid_agg(type_id, kind), (type_id, kind)
        if ok:
            assert L.gb_target_type(type_id, kind) == O.target_type(type_id, kind)


def test_invalid_arguments_are_reported_not_thrown():
    import ctypes
    L = _lib.lib()
    h = ctypes.c_void_p()
    rc = L.gb_create(None, 0, 0, 0, ctypes.byref(h))
    assert rc == _lib.GB_ERR_LOGIC
    assert b"key column" in L.gb_last_error()
    col = _lib.GbColumn(3, 4, 0, 0, 0)
    rc = L.gb_create(ctypes.byref(col), 1, 7, 0, ctypes.byref(h))
    assert rc == _lib.GB_ERR_LOGIC


def test_cpp_api_header_compiles_standalone():
    """include/cudf_b200/groupby.hpp (libcudf's groupby API shapes over the C
    ABI) compiles on its own with warnings as errors, and a caller written
    against libcudf's signatures type-checks against it."""
    import subprocess
    import tempfile
    src = r'''
#include <cudf_b200/groupby.hpp>
int use(cudf::table_view const& keys, cudf::column_view const& vals) {
  cudf::groupby::groupby gb(keys, cudf::null_policy::INCLUDE, cudf::sorted::NO);
  std::vector<cudf::groupby::aggregation_request> reqs(1);
  reqs[0].values = vals;
  reqs[0].aggregations.push_back(cudf::make_sum_aggregation<cudf::groupby_aggregation>());
  reqs[0].aggregations.push_back(cudf::make_mean_aggregation<cudf::groupby_aggregation>());
  reqs[0].aggregations.push_back(cudf::make_count_aggregation<cudf::groupby_aggregation>(cudf::null_policy::INCLUDE));
  auto [uk, res] = gb.aggregate(reqs, cudf::get_default_stream(), rmm::mr::get_current_device_resource());
  return uk->num_rows() + static_cast<int>(res[0].results.size());
}
'''
    with tempfile.TemporaryDirectory() as d:
        f = os.path.join(d, "use.cpp")
        open(f, "w").write(src)
        r = subprocess.run(["g++", "-std=c++17", "-Wall", "-Wextra", "-Werror", "-fsyntax-only",
                            "-I", os.path.join(ROOT, "include"), "-I", "/usr/local/cuda/include", f],
                           capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_tuning_fields_are_range_checked_on_the_host():
    """gb_set_tuning accepts every documented pass-2 variant (0-4) and rejects
    the next value; the handle holds column views only, so no device is needed."""
    import ctypes
    L = _lib.lib()
    h = ctypes.c_void_p()
    col = _lib.GbColumn(4, 8, 0, 0, 0)
    assert L.gb_create(ctypes.byref(col), 1, 0, 0, ctypes.byref(h)) == _lib.GB_OK
    try:
        def tuning(pass2):
            return _lib.GbTuning(-1, -1, -1, -1, -1, -1, -2, -1, -1, -1, pass2, -1, -1)
        for p in range(5):
            assert L.gb_set_tuning(h, ctypes.byref(tuning(p))) == _lib.GB_OK, p
        assert L.gb_set_tuning(h, ctypes.byref(tuning(5))) == _lib.GB_ERR_LOGIC
        assert b"pass2" in L.gb_last_error()
    finally:
        L.gb_destroy(h)
