// gb_plan.h -- the groupby "plan": how key columns pack into hash-table key
// words, which accumulators every table slot carries, and how the outputs are
// finalised.  Shared by host planning code and the device kernels.
#pragma once
#include <stdint.h>

namespace gb {

// libcudf type ids (cpp/include/cudf/types.hpp:201-233)
enum TypeId : int32_t {
  T_EMPTY = 0, T_INT8, T_INT16, T_INT32, T_INT64, T_UINT8, T_UINT16, T_UINT32, T_UINT64,
  T_FLOAT32, T_FLOAT64, T_BOOL8, T_TS_D, T_TS_S, T_TS_MS, T_TS_US, T_TS_NS,
  T_DUR_D, T_DUR_S, T_DUR_MS, T_DUR_US, T_DUR_NS
};

// libcudf aggregation kinds (cpp/include/cudf/aggregation.hpp:86-102)
enum AggKind : int32_t {
  K_SUM = 0, K_PRODUCT = 1, K_MIN = 2, K_MAX = 3, K_COUNT_VALID = 4, K_COUNT_ALL = 5,
  K_SUM_OF_SQUARES = 8, K_MEAN = 9, K_VARIANCE = 11, K_STD = 12, K_ARGMAX = 15, K_ARGMIN = 16
};

// Value categories of a column element.
enum Cat : uint8_t { CAT_SIGNED = 0, CAT_UNSIGNED = 1, CAT_F32 = 2, CAT_F64 = 3, CAT_BOOL = 4 };

// Accumulator operations held in a table slot.  MIN/MAX keep values in an
// order-preserving unsigned encoding so that one unsigned atomic min/max works
// for every type (floats: sign-magnitude flip; NaN placed so that it loses to
// every number, which makes MIN/MAX skip NaN unless a group holds only NaN).
enum Op : uint8_t {
  OP_NULLS = 0,     // u32 count of null values of one column
  OP_SUM_I64,       // i64 wrapping sum (integral and bool sources)
  OP_SUM_I32,       // i32 wrapping sum (32-bit durations keep their type)
  OP_SUM_F32,       // f32 sum
  OP_SUM_F64,       // f64 sum
  OP_MIN_U32,       // ordered u32 min
  OP_MAX_U32,
  OP_MIN_U64,       // ordered u64 min
  OP_MAX_U64,
  OP_SQ_I64,        // i64 wrapping sum of squares
  OP_SQ_F32,
  OP_SQ_F64,
  OP_PROD_I64,      // i64 wrapping product (CAS loop)
  OP_PROD_F32,
  OP_PROD_F64,
  OP_ARGMIN_P32,    // u64 (ordered value << 32 | row) for <=32-bit values
  OP_ARGMAX_P32,    // u64 (ordered value << 32 | ~row)
  OP_ARGMIN_R64,    // u64 row index, CAS loop comparing (value,row) through the column
  OP_ARGMAX_R64,
  OP_M2_F64,        // second pass: sum of (x-mean)^2/(n-ddof)
  OP_COUNT
};

constexpr int kMaxKeyCols = 16;
constexpr int kMaxValCols = 32;
constexpr int kMaxAccs = 96;
constexpr int kMaxOutputs = 96;

struct KeyCol {
  const void* data;
  const uint32_t* mask;   // LSB-first validity words, or null
  int64_t offset;         // row offset applied to data and mask
  int32_t type_id;
  uint8_t width;          // bytes
  uint8_t cat;
  uint8_t word;           // key word holding the value bits
  uint8_t shift;          // bit offset of the value inside that word
  uint8_t null_word;      // word/bit of the null flag (INCLUDE + nullable only)
  uint8_t null_shift;
  uint8_t has_null_bit;
  uint8_t pad;
};

struct ValCol {
  const void* data;
  const uint32_t* mask;
  int64_t offset;
  int32_t type_id;
  uint8_t width;
  uint8_t cat;
  int16_t nulls_off;      // slot byte offset of OP_NULLS, or -1
  int16_t sum_off;        // slot byte offset of the SUM accumulator (MEAN/VAR use it), or -1
  int16_t m2_off;         // slot byte offset of OP_M2_F64, or -1
  int16_t acc_begin;      // accumulators [acc_begin, acc_end) of the first pass
  int16_t acc_end;
  int32_t ddof;           // VARIANCE/STD ddof (one per column; requests with another ddof get a copy)
  const uint8_t* bits;    // partitioned rows: validity byte per row (bit `bit`), else null
  int32_t bit;
  // the column's accumulators in closed form, for kernels that skip the
  // per-accumulator interpreter: offsets (-1 when absent) and the sum op
  int16_t min_off;
  int16_t max_off;
  int16_t sq_off;
  uint8_t sum_op;         // OP_SUM_* or 0
  uint8_t basic;          // 1 when every accumulator is a SUM, MIN, MAX or sum of squares
};

struct Acc {
  uint8_t op;
  uint8_t col;
  uint16_t off;           // byte offset in the slot
};

// One output column of the result.
struct OutSpec {
  int32_t kind;           // aggregation kind
  int32_t col;            // value column
  int32_t out_type;       // target type id
  int16_t acc_off;        // accumulator this output reads (-1 if none)
  uint8_t out_width;
  uint8_t nullable;       // output gets a null mask
  int32_t ddof;
};

struct Plan {
  int32_t num_keys;
  int32_t num_vals;
  int32_t num_accs;
  int32_t num_outs;
  int32_t key_words;      // 1 or 2 (64 or 128 packed key bits)
  int32_t include_nulls;  // null_policy::INCLUDE
  int32_t any_key_nullable;
  int32_t slot_bytes;     // stride of one slot (multiple of 16)
  int32_t rows_off;       // u32 rows-in-group counter
  int32_t need_second_pass;
  int32_t has_arg;        // ARGMIN/ARGMAX present (needs original row indices)
  int64_t num_rows;
  const uint64_t* packed_keys;  // partitioned rows: key words per row (key_words each), else null
  KeyCol keys[kMaxKeyCols];
  ValCol vals[kMaxValCols];
  Acc accs[kMaxAccs];
  OutSpec outs[kMaxOutputs];
};

}  // namespace gb
