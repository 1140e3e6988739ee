"""Writes golden_vectors.json: the known-answer groupby cases of libcudf 24.04's
own gtest suite for the hash path, transcribed from the test sources (which
cannot be built or run here: libcudf needs network access to configure).

Each case names the reference test (file:line).  Expected outputs are listed
sorted by key (nulls first), as ``test_single_agg`` compares them after sorting
(cpp/tests/groupby/groupby_test_util.cpp:33-97).  ``None`` marks a null.

Run: python tests/golden/make_golden.py  (rewrites golden_vectors.json)
"""
import json
import os

N = None
# value types of the typed suites (cpp/tests/groupby/sum_tests.cpp:30-36 etc.)
SUM_TYPES = ["INT8", "INT16", "INT32", "INT64", "FLOAT32", "FLOAT64",
             "DURATION_DAYS", "DURATION_SECONDS", "DURATION_MILLISECONDS",
             "DURATION_MICROSECONDS", "DURATION_NANOSECONDS"]
MINMAX_TYPES = ["INT8", "INT16", "INT32", "INT64", "UINT8", "UINT16", "UINT32", "UINT64",
                "FLOAT32", "FLOAT64", "BOOL8",
                "TIMESTAMP_DAYS", "TIMESTAMP_SECONDS", "TIMESTAMP_MILLISECONDS",
                "TIMESTAMP_MICROSECONDS", "TIMESTAMP_NANOSECONDS",
                "DURATION_DAYS", "DURATION_SECONDS", "DURATION_MILLISECONDS",
                "DURATION_MICROSECONDS", "DURATION_NANOSECONDS"]
KEY_TYPES = ["INT8", "INT16", "INT32", "INT64", "FLOAT32", "FLOAT64"]

K10 = [1, 2, 3, 1, 2, 2, 1, 3, 3, 2]
V10 = [0, 1, 2, 3, 4, 5, 6, 7, 8, 9]
K11 = [1, 2, 3, 1, 2, 2, 1, 3, 3, 2, 4]
K11_VALID = [1, 1, 1, 1, 1, 1, 1, 0, 1, 1, 1]
V11 = [0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 4]
V11_VALID = [0, 1, 1, 1, 1, 0, 1, 1, 1, 1, 0]


def case(name, cite, keys, vals, aggs, expect_keys, expect, *, value_types=("INT32",),
         key_types=("INT32",), key_valid=None, val_valid=None, include_null_keys=False,
         expect_key_valid=None, error=None, bool_values_ok=True):
    return dict(name=name, cite=cite, keys=keys, key_valid=key_valid, vals=vals,
                val_valid=val_valid, aggs=aggs, include_null_keys=include_null_keys,
                expect_keys=expect_keys, expect_key_valid=expect_key_valid, expect=expect,
                value_types=list(value_types), key_types=list(key_types), error=error)


CASES = [
    # ---- SUM (cpp/tests/groupby/sum_tests.cpp) ----
    case("sum_basic", "cpp/tests/groupby/sum_tests.cpp:38-54", K10, V10, ["SUM"],
         [1, 2, 3], {"SUM": [9, 19, 17]}, value_types=SUM_TYPES),
    case("sum_empty_cols", "cpp/tests/groupby/sum_tests.cpp:56-72", [], [], ["SUM"], [],
         {"SUM": []}, value_types=SUM_TYPES),
    case("sum_zero_valid_keys", "cpp/tests/groupby/sum_tests.cpp:74-90", [1, 2, 3], [3, 4, 5],
         ["SUM"], [], {"SUM": []}, key_valid=[0, 0, 0], value_types=SUM_TYPES),
    case("sum_zero_valid_values", "cpp/tests/groupby/sum_tests.cpp:92-108", [1, 1, 1], [3, 4, 5],
         ["SUM"], [1], {"SUM": [N]}, val_valid=[0, 0, 0], value_types=SUM_TYPES),
    case("sum_null_keys_and_values", "cpp/tests/groupby/sum_tests.cpp:110-131", K11, V11, ["SUM"],
         [1, 2, 3, 4], {"SUM": [9, 14, 10, N]}, key_valid=K11_VALID, val_valid=V11_VALID,
         value_types=SUM_TYPES),
    case("sum_overflow_integer", "cpp/tests/groupby/sum_tests.cpp:154-171", [0, 0],
         [-2147483648, -2147483648], ["SUM"], [0], {"SUM": [-4294967296]}),
    # ---- MEAN (cpp/tests/groupby/mean_tests.cpp); durations stay durations (integer mean) ----
    case("mean_basic", "cpp/tests/groupby/mean_tests.cpp:48-66", K10, V10, ["MEAN"], [1, 2, 3],
         {"MEAN": [3.0, 19.0 / 4, 17.0 / 3]},
         value_types=["INT8", "INT16", "INT32", "INT64", "FLOAT32", "FLOAT64"]),
    case("mean_basic_duration", "cpp/tests/groupby/mean_tests.cpp:48-66", K10, V10, ["MEAN"],
         [1, 2, 3], {"MEAN": [3, 4, 5]},
         value_types=["DURATION_DAYS", "DURATION_SECONDS", "DURATION_MILLISECONDS",
                      "DURATION_MICROSECONDS", "DURATION_NANOSECONDS"]),
    case("mean_empty_cols", "cpp/tests/groupby/mean_tests.cpp:68-81", [], [], ["MEAN"], [],
         {"MEAN": []}, value_types=SUM_TYPES),
    case("mean_zero_valid_keys", "cpp/tests/groupby/mean_tests.cpp:83-96", [1, 2, 3], [3, 4, 5],
         ["MEAN"], [], {"MEAN": []}, key_valid=[0, 0, 0], value_types=SUM_TYPES),
    case("mean_zero_valid_values", "cpp/tests/groupby/mean_tests.cpp:98-111", [1, 1, 1], [3, 4, 5],
         ["MEAN"], [1], {"MEAN": [N]}, val_valid=[0, 0, 0], value_types=SUM_TYPES),
    case("mean_null_keys_and_values", "cpp/tests/groupby/mean_tests.cpp:113-137", K11, V11,
         ["MEAN"], [1, 2, 3, 4], {"MEAN": [4.5, 14.0 / 3, 5.0, N]}, key_valid=K11_VALID,
         val_valid=V11_VALID, value_types=["INT8", "INT16", "INT32", "INT64", "FLOAT32", "FLOAT64"]),
    # ---- COUNT (cpp/tests/groupby/count_tests.cpp); COUNT_ALL = count(null_policy::INCLUDE) ----
    case("count_basic", "cpp/tests/groupby/count_tests.cpp:32-51", K10, V10,
         ["COUNT_VALID", "COUNT_ALL"], [1, 2, 3], {"COUNT_VALID": [3, 4, 3], "COUNT_ALL": [3, 4, 3]},
         value_types=MINMAX_TYPES),
    case("count_empty_cols", "cpp/tests/groupby/count_tests.cpp:53-69", [], [], ["COUNT_VALID"], [],
         {"COUNT_VALID": []}, value_types=MINMAX_TYPES),
    case("count_zero_valid_keys", "cpp/tests/groupby/count_tests.cpp:71-90", [1, 2, 3], [3, 4, 5],
         ["COUNT_VALID", "COUNT_ALL"], [], {"COUNT_VALID": [], "COUNT_ALL": []},
         key_valid=[0, 0, 0], value_types=MINMAX_TYPES),
    case("count_zero_valid_values", "cpp/tests/groupby/count_tests.cpp:92-112", [1, 1, 1],
         [3, 4, 5], ["COUNT_VALID", "COUNT_ALL"], [1], {"COUNT_VALID": [0], "COUNT_ALL": [3]},
         val_valid=[0, 0, 0], value_types=MINMAX_TYPES),
    case("count_null_keys_and_values", "cpp/tests/groupby/count_tests.cpp:114-142", K11, V11,
         ["COUNT_VALID", "COUNT_ALL"], [1, 2, 3, 4],
         {"COUNT_VALID": [2, 3, 2, 0], "COUNT_ALL": [3, 4, 2, 1]}, key_valid=K11_VALID,
         val_valid=V11_VALID, value_types=MINMAX_TYPES),
    # ---- MIN (cpp/tests/groupby/min_tests.cpp) ----
    case("min_basic", "cpp/tests/groupby/min_tests.cpp:37-53", K10, V10, ["MIN"], [1, 2, 3],
         {"MIN": [0, 1, 2]}, value_types=MINMAX_TYPES),
    case("min_empty_cols", "cpp/tests/groupby/min_tests.cpp:55-71", [], [], ["MIN"], [],
         {"MIN": []}, value_types=MINMAX_TYPES),
    case("min_zero_valid_keys", "cpp/tests/groupby/min_tests.cpp:73-89", [1, 2, 3], [3, 4, 5],
         ["MIN"], [], {"MIN": []}, key_valid=[0, 0, 0], value_types=MINMAX_TYPES),
    case("min_zero_valid_values", "cpp/tests/groupby/min_tests.cpp:91-107", [1, 1, 1], [3, 4, 5],
         ["MIN"], [1], {"MIN": [N]}, val_valid=[0, 0, 0], value_types=MINMAX_TYPES),
    case("min_null_keys_and_values", "cpp/tests/groupby/min_tests.cpp:109-131", K11, V11, ["MIN"],
         [1, 2, 3, 4], {"MIN": [3, 1, 2, N]}, key_valid=K11_VALID, val_valid=V11_VALID,
         value_types=MINMAX_TYPES),
    case("min_values_with_infinity", "cpp/tests/groupby/min_tests.cpp:503-522", [1, 2, 1, 2],
         [1.0, 1.0, "-inf", 2.0], ["MIN"], [1, 2], {"MIN": ["-inf", 1.0]},
         value_types=["FLOAT32", "FLOAT64"]),
    case("min_values_with_nan", "cpp/tests/groupby/min_tests.cpp:524-547", [1, 1], ["nan", "nan"],
         ["MIN"], [1], {"MIN": ["nan"]}, value_types=["FLOAT32", "FLOAT64"]),
    # ---- MAX (cpp/tests/groupby/max_tests.cpp) ----
    case("max_basic", "cpp/tests/groupby/max_tests.cpp:37-53", K10, V10, ["MAX"], [1, 2, 3],
         {"MAX": [6, 9, 8]}, value_types=MINMAX_TYPES),
    case("max_empty_cols", "cpp/tests/groupby/max_tests.cpp:55-71", [], [], ["MAX"], [],
         {"MAX": []}, value_types=MINMAX_TYPES),
    case("max_zero_valid_keys", "cpp/tests/groupby/max_tests.cpp:73-89", [1, 2, 3], [3, 4, 5],
         ["MAX"], [], {"MAX": []}, key_valid=[0, 0, 0], value_types=MINMAX_TYPES),
    case("max_zero_valid_values", "cpp/tests/groupby/max_tests.cpp:91-107", [1, 1, 1], [3, 4, 5],
         ["MAX"], [1], {"MAX": [N]}, val_valid=[0, 0, 0], value_types=MINMAX_TYPES),
    case("max_null_keys_and_values", "cpp/tests/groupby/max_tests.cpp:109-131", K11, V11, ["MAX"],
         [1, 2, 3, 4], {"MAX": [3, 5, 8, N]}, key_valid=K11_VALID,
         val_valid=[1, 1, 1, 1, 1, 1, 0, 1, 1, 0, 0], value_types=MINMAX_TYPES),
    case("max_values_with_infinity", "cpp/tests/groupby/max_tests.cpp:507-526", [1, 2, 1, 2],
         [1.0, 1.0, "inf", 2.0], ["MAX"], [1, 2], {"MAX": ["inf", 2.0]},
         value_types=["FLOAT32", "FLOAT64"]),
    case("max_values_with_nan", "cpp/tests/groupby/max_tests.cpp:528-551", [1, 1], ["nan", "nan"],
         ["MAX"], [1], {"MAX": ["nan"]}, value_types=["FLOAT32", "FLOAT64"]),
    # ---- keys (cpp/tests/groupby/keys_tests.cpp) ----
    case("keys_basic", "cpp/tests/groupby/keys_tests.cpp:37-53", K10, V10, ["COUNT_VALID"],
         [1, 2, 3], {"COUNT_VALID": [3, 4, 3]}, key_types=KEY_TYPES),
    case("keys_zero_valid_keys", "cpp/tests/groupby/keys_tests.cpp:55-71", [1, 2, 3], [3, 4, 5],
         ["COUNT_VALID"], [], {"COUNT_VALID": []}, key_valid=[0, 0, 0], key_types=KEY_TYPES),
    case("keys_some_null_keys", "cpp/tests/groupby/keys_tests.cpp:73-92", K11, V11,
         ["COUNT_VALID"], [1, 2, 3, 4], {"COUNT_VALID": [3, 4, 2, 1]}, key_valid=K11_VALID,
         key_types=KEY_TYPES),
    case("keys_include_null_keys", "cpp/tests/groupby/keys_tests.cpp:94-120", K11, V11, ["SUM"],
         [3, 1, 2, 3, 4], {"SUM": [7, 9, 19, 10, 4]}, key_valid=K11_VALID,
         include_null_keys=True, expect_key_valid=[0, 1, 1, 1, 1], key_types=KEY_TYPES),
    case("keys_mismatch_num_rows", "cpp/tests/groupby/keys_tests.cpp:227-243", [1, 2, 3],
         [0, 1, 2, 3, 4], ["COUNT_VALID"], [], {}, key_types=KEY_TYPES, error="logic_error"),
    # ---- result cache (cpp/tests/groupby/keys_tests.cpp:367-421): duplicates in request order ----
    case("cache_duplicate_aggregations", "cpp/tests/groupby/keys_tests.cpp:367-390", K10, V10,
         ["SUM", "SUM"], [1, 2, 3], {"SUM": [9, 19, 17]}),
]


def main():
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden_vectors.json")
    with open(out, "w") as f:
        json.dump({"source": "libcudf 24.04 cpp/tests/groupby (transcribed)", "cases": CASES}, f,
                  indent=1)
    print(f"wrote {len(CASES)} cases to {out}")


if __name__ == "__main__":
    main()
