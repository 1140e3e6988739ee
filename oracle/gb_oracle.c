/*
 * gb_oracle.c -- CPU restatement of libcudf's hash groupby-aggregate semantics.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the correctness oracle for the
 * B200 engine in cudf_b200/.  Only tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py may load it; the engine never calls it.
 *
 * What it restates (paths relative to the libcudf source tree, tag 24.04):
 *  - group membership: rows whose key tuples compare equal form one group;
 *    nulls compare equal (null_equality::EQUAL) and, for floating keys, all
 *    NaNs are one key and -0.0 == +0.0
 *      cpp/src/groupby/hash/groupby.cu:557,614-618
 *      cpp/include/cudf/hashing/detail/murmurhash3_x86_32.cuh:66-68
 *      cpp/include/cudf/table/experimental/row_operators.cuh:1828
 *  - null_policy::EXCLUDE drops every row with a null in any key column
 *    (bitmask_and of the key masks), INCLUDE keeps them as their own group
 *      cpp/src/groupby/hash/groupby.cu:482-485
 *  - per-aggregation updates skip null values; identities and target types
 *      cpp/include/cudf/detail/aggregation/aggregation.cuh:116-434
 *      cpp/include/cudf/detail/aggregation/aggregation.hpp:1168-1290
 *  - MEAN = SUM / COUNT_VALID computed in double, null when COUNT_VALID == 0
 *      cpp/src/groupby/hash/groupby.cu:137-147,287-306
 *      cpp/src/binaryop/compiled/binary_ops.cuh:97-121
 *  - VARIANCE/STD second pass: sum over rows of (x-mean)^2/(n-ddof), null
 *    when n-ddof <= 0; STD = sqrt(VARIANCE)
 *      cpp/src/groupby/hash/multi_pass_kernels.cuh:79-94
 *      cpp/src/groupby/hash/groupby.cu:308-348
 *  - result columns are nullable iff the value column has a null mask
 *    (COUNT_* never null; VARIANCE/STD always nullable)
 *      cpp/src/groupby/hash/groupby.cu:424-454
 *
 * Integer SUM / SUM_OF_SQUARES / PRODUCT wrap in two's complement exactly like
 * the 64-bit atomics of cpp/include/cudf/detail/utilities/device_atomics.cuh:
 * 195-205.  Floating SUM is a Neumaier-compensated FP64 sum (the reference's
 * atomic order is not fixed, so the engine is compared against this within
 * 2*n*eps*sum|x|, with eps of the accumulator type).  Floating MIN/MAX skip
 * NaN unless every valid value of the group is NaN (the reference's CAS loop
 * leaves this order-dependent; cpp/tests/groupby/min_tests.cpp:524-547 only
 * pins that it terminates).
 *
 * One thread reports groups in first-appearance order; several threads report
 * them partition by partition (see groupby_parallel).  The reference's order
 * is arbitrary (cpp/include/cudf/groupby.hpp:153-155); callers sort by key.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "gb_oracle.h"

/* ---- libcudf type ids and aggregation kinds (cpp/include/cudf/types.hpp:201-233,
 *      cpp/include/cudf/aggregation.hpp:86-102) ---- */
enum {
  T_INT8 = 1, T_INT16, T_INT32, T_INT64, T_UINT8, T_UINT16, T_UINT32, T_UINT64,
  T_FLOAT32, T_FLOAT64, T_BOOL8, T_TS_D, T_TS_S, T_TS_MS, T_TS_US, T_TS_NS,
  T_DUR_D, T_DUR_S, T_DUR_MS, T_DUR_US, T_DUR_NS
};
enum {
  A_SUM = 0, A_PRODUCT = 1, A_MIN = 2, A_MAX = 3, A_COUNT_VALID = 4, A_COUNT_ALL = 5,
  A_SUM_OF_SQUARES = 8, A_MEAN = 9, A_VARIANCE = 11, A_STD = 12, A_ARGMAX = 15, A_ARGMIN = 16
};

typedef enum { C_SIGNED, C_UNSIGNED, C_FLOAT } category;

static int type_width(int t)
{
  switch (t) {
    case T_INT8: case T_UINT8: case T_BOOL8: return 1;
    case T_INT16: case T_UINT16: return 2;
    case T_INT32: case T_UINT32: case T_FLOAT32: case T_TS_D: case T_DUR_D: return 4;
    case T_INT64: case T_UINT64: case T_FLOAT64: case T_TS_S: case T_TS_MS: case T_TS_US:
    case T_TS_NS: case T_DUR_S: case T_DUR_MS: case T_DUR_US: case T_DUR_NS: return 8;
    default: return 0;
  }
}
static category type_cat(int t)
{
  if (t == T_FLOAT32 || t == T_FLOAT64) return C_FLOAT;
  if (t >= T_UINT8 && t <= T_UINT64) return C_UNSIGNED;
  return C_SIGNED;
}
static int is_timestamp(int t) { return t >= T_TS_D && t <= T_TS_NS; }
static int is_duration(int t) { return t >= T_DUR_D && t <= T_DUR_NS; }

/* Valid (type, aggregation) pairs of the hash path:
 * cpp/include/cudf/detail/aggregation/aggregation.hpp:1168-1290 (target types)
 * and cpp/src/groupby/hash/groupby.cu:73-84 (hash_aggregations). */
int orc_valid_agg(int t, int k)
{
  if (type_width(t) == 0) return 0;
  int numeric = !is_timestamp(t) && !is_duration(t);
  switch (k) {
    case A_MIN: case A_MAX: case A_COUNT_VALID: case A_COUNT_ALL:
    case A_ARGMIN: case A_ARGMAX: return 1;
    case A_SUM: return numeric || is_duration(t);
    case A_MEAN: return numeric || is_duration(t);
    case A_PRODUCT: case A_SUM_OF_SQUARES: return numeric;
    case A_VARIANCE: case A_STD: return numeric;
    default: return 0;
  }
}

static inline int bit_is_set(const uint32_t* m, int64_t i)
{
  return (m[i >> 5] >> (i & 31)) & 1u;
}
static inline int col_valid(const orc_column* c, int64_t row)
{
  return c->mask == NULL || bit_is_set(c->mask, row + c->offset);
}
static inline int64_t load_signed(const orc_column* c, int64_t row)
{
  const char* p = (const char*)c->data + (row + c->offset) * (int64_t)type_width(c->type_id);
  switch (type_width(c->type_id)) {
    case 1: return c->type_id == T_BOOL8 ? (int64_t)(*(const int8_t*)p != 0) : (int64_t)*(const int8_t*)p;
    case 2: return *(const int16_t*)p;
    case 4: return *(const int32_t*)p;
    default: return *(const int64_t*)p;
  }
}
static inline uint64_t load_unsigned(const orc_column* c, int64_t row)
{
  const char* p = (const char*)c->data + (row + c->offset) * (int64_t)type_width(c->type_id);
  switch (type_width(c->type_id)) {
    case 1: return *(const uint8_t*)p;
    case 2: return *(const uint16_t*)p;
    case 4: return *(const uint32_t*)p;
    default: return *(const uint64_t*)p;
  }
}
static inline double load_float(const orc_column* c, int64_t row)
{
  const char* p = (const char*)c->data + (row + c->offset) * (int64_t)type_width(c->type_id);
  return c->type_id == T_FLOAT32 ? (double)*(const float*)p : *(const double*)p;
}

/* Key word of one key column: normalised bits, so that equal keys have equal
 * words (NaN canonical, -0.0 -> +0.0, bool -> 0/1). */
static inline uint64_t key_word(const orc_column* c, int64_t row)
{
  const char* p = (const char*)c->data + (row + c->offset) * (int64_t)type_width(c->type_id);
  if (c->type_id == T_FLOAT32) {
    float f = *(const float*)p;
    if (isnan(f)) f = NAN;
    if (f == 0.0f) f = 0.0f;
    uint32_t u; memcpy(&u, &f, 4); return u;
  }
  if (c->type_id == T_FLOAT64) {
    double d = *(const double*)p;
    if (isnan(d)) d = NAN;
    if (d == 0.0) d = 0.0;
    uint64_t u; memcpy(&u, &d, 8); return u;
  }
  if (c->type_id == T_BOOL8) return *(const uint8_t*)p != 0;
  return load_unsigned(c, row);
}

/* ---------------------------------------------------------------------- */
/* per-request accumulators                                                 */
typedef struct {
  category cat;
  int type_id;
  int need_sum, need_prod, need_min, need_max, need_sq, need_arg, need_var;
  int64_t* n_all;
  int64_t* n_valid;
  uint64_t* isum; double* fsum; double* fcomp; double* fabs_sum;
  uint64_t* iprod; long double* fprod;
  int64_t* imin; int64_t* imax; uint64_t* umin; uint64_t* umax;
  double* fmin; double* fmax; uint8_t* fmin_seen; uint8_t* fmax_seen;
  uint64_t* isq; double* fsq; double* fsq_comp;
  int64_t* argmin; int64_t* argmax;
  long double* m2;
} acc_t;

struct orc_handle {
  int nkeys;
  int nkw;               /* key words per group = nkeys + 1 (null bits) */
  int include_nulls;
  int nreq;
  const orc_column* keys;
  const orc_request* reqs;
  int64_t ngroups, gcap;
  uint64_t* gkeys;       /* ngroups * nkw */
  int64_t* first_row;
  int64_t tcap;          /* hash table capacity (power of two) */
  int64_t* slots;        /* group id or -1 */
  acc_t* acc;
};

static uint64_t mix64(uint64_t z)
{ /* splitmix64 finaliser (Steele, Lea, Flood 2014) */
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
static uint64_t hash_words(const uint64_t* w, int n)
{
  uint64_t h = 0x243F6A8885A308D3ull;
  for (int i = 0; i < n; ++i) h = mix64(h ^ (w[i] + 0x9E3779B97F4A7C15ull * (uint64_t)(i + 1)));
  return h;
}

static void* xcalloc(int64_t n, size_t sz)
{
  void* p = calloc((size_t)(n > 0 ? n : 1), sz);
  if (!p) abort();
  return p;
}
static void* xrealloc(void* p, int64_t n, size_t sz)
{
  void* q = realloc(p, (size_t)(n > 0 ? n : 1) * sz);
  if (!q) abort();
  return q;
}

#define GROW(ptr, T, newcap, oldcap, initval)                                    \
  do {                                                                           \
    if (ptr) {                                                                   \
      ptr = (T*)xrealloc(ptr, newcap, sizeof(T));                                \
      for (int64_t _i = oldcap; _i < newcap; ++_i) ptr[_i] = (T)(initval);       \
    }                                                                            \
  } while (0)

static void acc_alloc(acc_t* a, int64_t cap)
{
  a->n_all = xcalloc(cap, 8);
  a->n_valid = xcalloc(cap, 8);
  if (a->need_sum || a->need_var) {
    if (a->cat == C_FLOAT) { a->fsum = xcalloc(cap, 8); a->fcomp = xcalloc(cap, 8); a->fabs_sum = xcalloc(cap, 8); }
    else a->isum = xcalloc(cap, 8);
  }
  if (a->need_prod) {
    if (a->cat == C_FLOAT) { a->fprod = xcalloc(cap, sizeof(long double)); for (int64_t i = 0; i < cap; ++i) a->fprod[i] = 1.0L; }
    else { a->iprod = xcalloc(cap, 8); for (int64_t i = 0; i < cap; ++i) a->iprod[i] = 1; }
  }
  if (a->need_min) {
    if (a->cat == C_FLOAT) { a->fmin = xcalloc(cap, 8); a->fmin_seen = xcalloc(cap, 1); }
    else if (a->cat == C_UNSIGNED) { a->umin = xcalloc(cap, 8); for (int64_t i = 0; i < cap; ++i) a->umin[i] = UINT64_MAX; }
    else { a->imin = xcalloc(cap, 8); for (int64_t i = 0; i < cap; ++i) a->imin[i] = INT64_MAX; }
  }
  if (a->need_max) {
    if (a->cat == C_FLOAT) { a->fmax = xcalloc(cap, 8); a->fmax_seen = xcalloc(cap, 1); }
    else if (a->cat == C_UNSIGNED) a->umax = xcalloc(cap, 8);
    else { a->imax = xcalloc(cap, 8); for (int64_t i = 0; i < cap; ++i) a->imax[i] = INT64_MIN; }
  }
  if (a->need_sq) {
    if (a->cat == C_FLOAT) { a->fsq = xcalloc(cap, 8); a->fsq_comp = xcalloc(cap, 8); }
    else a->isq = xcalloc(cap, 8);
  }
  if (a->need_arg) {
    a->argmin = xcalloc(cap, 8); a->argmax = xcalloc(cap, 8);
    for (int64_t i = 0; i < cap; ++i) a->argmin[i] = a->argmax[i] = -1;
  }
  if (a->need_var) a->m2 = xcalloc(cap, sizeof(long double));
}

static void acc_grow(acc_t* a, int64_t old, int64_t cap)
{
  GROW(a->n_all, int64_t, cap, old, 0);
  GROW(a->n_valid, int64_t, cap, old, 0);
  GROW(a->isum, uint64_t, cap, old, 0);
  GROW(a->fsum, double, cap, old, 0);
  GROW(a->fcomp, double, cap, old, 0);
  GROW(a->fabs_sum, double, cap, old, 0);
  GROW(a->iprod, uint64_t, cap, old, 1);
  GROW(a->fprod, long double, cap, old, 1.0L);
  GROW(a->imin, int64_t, cap, old, INT64_MAX);
  GROW(a->imax, int64_t, cap, old, INT64_MIN);
  GROW(a->umin, uint64_t, cap, old, UINT64_MAX);
  GROW(a->umax, uint64_t, cap, old, 0);
  GROW(a->fmin, double, cap, old, 0);
  GROW(a->fmax, double, cap, old, 0);
  GROW(a->fmin_seen, uint8_t, cap, old, 0);
  GROW(a->fmax_seen, uint8_t, cap, old, 0);
  GROW(a->isq, uint64_t, cap, old, 0);
  GROW(a->fsq, double, cap, old, 0);
  GROW(a->fsq_comp, double, cap, old, 0);
  GROW(a->argmin, int64_t, cap, old, -1);
  GROW(a->argmax, int64_t, cap, old, -1);
  GROW(a->m2, long double, cap, old, 0.0L);
}

static void acc_free(acc_t* a)
{
  void* ps[] = {a->n_all, a->n_valid, a->isum, a->fsum, a->fcomp, a->fabs_sum, a->iprod, a->fprod,
                a->imin, a->imax, a->umin, a->umax, a->fmin, a->fmax, a->fmin_seen, a->fmax_seen,
                a->isq, a->fsq, a->fsq_comp, a->argmin, a->argmax, a->m2};
  for (size_t i = 0; i < sizeof(ps) / sizeof(ps[0]); ++i) free(ps[i]);
}

static inline void neumaier(double* s, double* c, double x)
{ /* Neumaier's improved Kahan summation (Neumaier 1974) */
  double t = *s + x;
  if (fabs(*s) >= fabs(x)) *c += (*s - t) + x; else *c += (x - t) + *s;
  *s = t;
}

static orc_handle* handle_new(const orc_column* keys, int nkeys, int include_nulls,
                              const orc_request* reqs, int nreq)
{
  orc_handle* h = xcalloc(1, sizeof(orc_handle));
  h->nkeys = nkeys; h->nkw = nkeys + 1; h->include_nulls = include_nulls;
  h->keys = keys; h->reqs = reqs; h->nreq = nreq;
  h->gcap = 1024;
  h->gkeys = xcalloc(h->gcap * h->nkw, 8);
  h->first_row = xcalloc(h->gcap, 8);
  h->tcap = 2048;
  h->slots = xcalloc(h->tcap, 8);
  for (int64_t i = 0; i < h->tcap; ++i) h->slots[i] = -1;
  h->acc = xcalloc(nreq > 0 ? nreq : 1, sizeof(acc_t));
  for (int r = 0; r < nreq; ++r) {
    acc_t* a = &h->acc[r];
    a->type_id = reqs[r].values.type_id;
    a->cat = type_cat(a->type_id);
    for (int j = 0; j < reqs[r].num_aggs; ++j) {
      switch (reqs[r].kinds[j]) {
        case A_SUM: case A_MEAN: a->need_sum = 1; break;
        case A_PRODUCT: a->need_prod = 1; break;
        case A_MIN: a->need_min = 1; break;
        case A_MAX: a->need_max = 1; break;
        case A_SUM_OF_SQUARES: a->need_sq = 1; break;
        case A_ARGMIN: case A_ARGMAX: a->need_arg = 1; break;
        case A_VARIANCE: case A_STD: a->need_var = 1; a->need_sum = 1; break;
        default: break;
      }
    }
    acc_alloc(a, h->gcap);
  }
  return h;
}

static void handle_free(orc_handle* h)
{
  if (!h) return;
  for (int r = 0; r < h->nreq; ++r) acc_free(&h->acc[r]);
  free(h->acc); free(h->gkeys); free(h->first_row); free(h->slots); free(h);
}

static void rehash(orc_handle* h)
{
  int64_t ncap = h->tcap * 2;
  int64_t* ns = xcalloc(ncap, 8);
  for (int64_t i = 0; i < ncap; ++i) ns[i] = -1;
  for (int64_t g = 0; g < h->ngroups; ++g) {
    uint64_t s = hash_words(&h->gkeys[g * h->nkw], h->nkw) & (uint64_t)(ncap - 1);
    while (ns[s] >= 0) s = (s + 1) & (uint64_t)(ncap - 1);
    ns[s] = g;
  }
  free(h->slots); h->slots = ns; h->tcap = ncap;
}

/* find-or-insert the group of a normalised key tuple */
static int64_t find_or_insert(orc_handle* h, const uint64_t* kw, int64_t row)
{
  uint64_t s = hash_words(kw, h->nkw) & (uint64_t)(h->tcap - 1);
  for (;;) {
    int64_t g = h->slots[s];
    if (g < 0) break;
    if (memcmp(&h->gkeys[g * h->nkw], kw, 8 * (size_t)h->nkw) == 0) return g;
    s = (s + 1) & (uint64_t)(h->tcap - 1);
  }
  int64_t g = h->ngroups++;
  if (g >= h->gcap) {
    int64_t nc = h->gcap * 2;
    h->gkeys = xrealloc(h->gkeys, nc * h->nkw, 8);
    h->first_row = xrealloc(h->first_row, nc, 8);
    for (int r = 0; r < h->nreq; ++r) acc_grow(&h->acc[r], h->gcap, nc);
    h->gcap = nc;
  }
  memcpy(&h->gkeys[g * h->nkw], kw, 8 * (size_t)h->nkw);
  h->first_row[g] = row;
  h->slots[s] = g;
  if (2 * h->ngroups > h->tcap) rehash(h);
  return g;
}

/* Returns 0 and fills kw when the row takes part, 1 when EXCLUDE drops it. */
static inline int row_key(const orc_handle* h, int64_t row, uint64_t* kw)
{
  uint64_t nulls = 0;
  for (int k = 0; k < h->nkeys; ++k) {
    const orc_column* c = &h->keys[k];
    if (!col_valid(c, row)) {
      if (!h->include_nulls) return 1;
      nulls |= 1ull << (k & 63);
      kw[k] = 0;
    } else {
      kw[k] = key_word(c, row);
    }
  }
  kw[h->nkeys] = nulls;
  return 0;
}

static void update_row(acc_t* a, const orc_column* v, int64_t g, int64_t row)
{
  a->n_all[g]++;
  if (!col_valid(v, row)) return;
  a->n_valid[g]++;
  if (a->cat == C_FLOAT) {
    double x = load_float(v, row);
    if (a->fsum) { neumaier(&a->fsum[g], &a->fcomp[g], x); a->fabs_sum[g] += fabs(x); }
    if (a->fprod) a->fprod[g] *= (long double)x;
    if (a->fmin && !isnan(x)) {
      if (!a->fmin_seen[g] || x < a->fmin[g]) a->fmin[g] = x;
      a->fmin_seen[g] = 1;
    }
    if (a->fmax && !isnan(x)) {
      if (!a->fmax_seen[g] || x > a->fmax[g]) a->fmax[g] = x;
      a->fmax_seen[g] = 1;
    }
    if (a->fsq) neumaier(&a->fsq[g], &a->fsq_comp[g], x * x);
    if (a->argmin) {
      /* first row among ties; NaN never wins against a number */
      if (a->argmin[g] < 0) a->argmin[g] = row;
      else { double b = load_float(v, a->argmin[g]); if (x < b || (isnan(b) && !isnan(x))) a->argmin[g] = row; }
      if (a->argmax[g] < 0) a->argmax[g] = row;
      else { double b = load_float(v, a->argmax[g]); if (x > b || (isnan(b) && !isnan(x))) a->argmax[g] = row; }
    }
  } else if (a->cat == C_UNSIGNED) {
    uint64_t x = load_unsigned(v, row);
    if (a->isum) a->isum[g] += x;
    if (a->iprod) a->iprod[g] *= x;
    if (a->umin && x < a->umin[g]) a->umin[g] = x;
    if (a->umax && x > a->umax[g]) a->umax[g] = x;
    if (a->isq) a->isq[g] += x * x;
    if (a->argmin) {
      if (a->argmin[g] < 0 || x < load_unsigned(v, a->argmin[g])) a->argmin[g] = row;
      if (a->argmax[g] < 0 || x > load_unsigned(v, a->argmax[g])) a->argmax[g] = row;
    }
  } else {
    int64_t x = load_signed(v, row);
    if (a->isum) a->isum[g] += (uint64_t)x;
    if (a->iprod) a->iprod[g] *= (uint64_t)x;
    if (a->imin && x < a->imin[g]) a->imin[g] = x;
    if (a->imax && x > a->imax[g]) a->imax[g] = x;
    if (a->isq) a->isq[g] += (uint64_t)x * (uint64_t)x;
    if (a->argmin) {
      if (a->argmin[g] < 0 || x < load_signed(v, a->argmin[g])) a->argmin[g] = row;
      if (a->argmax[g] < 0 || x > load_signed(v, a->argmax[g])) a->argmax[g] = row;
    }
  }
}

/* Aggregates rows idx[0..cnt) (or rows lo..lo+cnt when idx is NULL) in order. */
static void aggregate_rows(orc_handle* h, const int64_t* idx, int64_t lo, int64_t cnt)
{
  uint64_t kw[65];
  for (int64_t i = 0; i < cnt; ++i) {
    const int64_t row = idx ? idx[i] : lo + i;
    if (row_key(h, row, kw)) continue;
    int64_t g = find_or_insert(h, kw, row);
    for (int r = 0; r < h->nreq; ++r) update_row(&h->acc[r], &h->reqs[r].values, g, row);
  }
}

/* mean of group g in double, as the second pass sees it (sum of the target type / count) */
static double group_mean(const acc_t* a, int64_t g)
{
  double s;
  if (a->cat == C_FLOAT) s = a->type_id == T_FLOAT32 ? (double)(float)(a->fsum[g] + a->fcomp[g]) : a->fsum[g] + a->fcomp[g];
  else s = (double)(int64_t)a->isum[g];
  return s / (double)a->n_valid[g];
}

static void second_pass_var(orc_handle* h, const int64_t* idx, int64_t lo, int64_t cnt)
{
  uint64_t kw[65];
  int any = 0;
  for (int r = 0; r < h->nreq; ++r) any |= h->acc[r].need_var;
  if (!any) return;
  for (int64_t i = 0; i < cnt; ++i) {
    const int64_t row = idx ? idx[i] : lo + i;
    if (row_key(h, row, kw)) continue;
    uint64_t s = hash_words(kw, h->nkw) & (uint64_t)(h->tcap - 1);
    int64_t g;
    for (;;) {
      g = h->slots[s];
      if (memcmp(&h->gkeys[g * h->nkw], kw, 8 * (size_t)h->nkw) == 0) break;
      s = (s + 1) & (uint64_t)(h->tcap - 1);
    }
    for (int r = 0; r < h->nreq; ++r) {
      acc_t* a = &h->acc[r];
      const orc_column* v = &h->reqs[r].values;
      if (!a->need_var || !col_valid(v, row)) continue;
      double x = a->cat == C_FLOAT ? load_float(v, row)
               : a->cat == C_UNSIGNED ? (double)load_unsigned(v, row) : (double)load_signed(v, row);
      long double d = (long double)x - (long double)group_mean(a, g);
      a->m2[g] += d * d;
    }
  }
}

/* ---- parallel path -------------------------------------------------------
 * Rows are hash-partitioned by their normalised key tuple, so every group lives
 * in exactly one partition; each partition is then aggregated on its own in
 * increasing row order.  A group therefore sees its rows in the same order as
 * in the single-threaded path (identical float sums, first rows and argmin/
 * argmax ties), and the partitions' groups are concatenated.  Only the order of
 * the groups differs, which the reference leaves arbitrary. */
#define ORC_PART_BITS 10
#define ORC_NPART (1 << ORC_PART_BITS)
#define ORC_SKIP 0xFFFFu

typedef struct {
  orc_handle* proto;       /* keys, requests, policy */
  int nthreads;
  int64_t n;
  uint16_t* pid;           /* partition of each row, ORC_SKIP when dropped */
  int64_t* counts;         /* [nthreads][ORC_NPART], then running offsets */
  int64_t* idx;            /* rows grouped by partition */
  int64_t part_start[ORC_NPART + 1];
  orc_handle* parts[ORC_NPART];
  int next;                /* next partition to aggregate (atomic) */
} par_t;

typedef struct { par_t* p; int t; } par_job;

static void* par_count(void* arg)
{
  par_job* j = (par_job*)arg;
  par_t* p = j->p;
  orc_handle* h = p->proto;
  const int64_t lo = p->n * j->t / p->nthreads, hi = p->n * (j->t + 1) / p->nthreads;
  int64_t* cnt = p->counts + (int64_t)j->t * ORC_NPART;
  uint64_t kw[65];
  for (int64_t row = lo; row < hi; ++row) {
    if (row_key(h, row, kw)) { p->pid[row] = ORC_SKIP; continue; }
    const unsigned q = (unsigned)(hash_words(kw, h->nkw) >> (64 - ORC_PART_BITS));
    p->pid[row] = (uint16_t)q;
    cnt[q]++;
  }
  return NULL;
}

static void* par_scatter(void* arg)
{
  par_job* j = (par_job*)arg;
  par_t* p = j->p;
  const int64_t lo = p->n * j->t / p->nthreads, hi = p->n * (j->t + 1) / p->nthreads;
  int64_t* off = p->counts + (int64_t)j->t * ORC_NPART;
  for (int64_t row = lo; row < hi; ++row) {
    const unsigned q = p->pid[row];
    if (q != ORC_SKIP) p->idx[off[q]++] = row;
  }
  return NULL;
}

static void* par_aggregate(void* arg)
{
  par_job* j = (par_job*)arg;
  par_t* p = j->p;
  orc_handle* pr = p->proto;
  for (;;) {
    const int q = __atomic_fetch_add(&p->next, 1, __ATOMIC_RELAXED);
    if (q >= ORC_NPART) break;
    const int64_t b = p->part_start[q], cnt = p->part_start[q + 1] - b;
    orc_handle* h = handle_new(pr->keys, pr->nkeys, pr->include_nulls, pr->reqs, pr->nreq);
    aggregate_rows(h, p->idx + b, 0, cnt);
    second_pass_var(h, p->idx + b, 0, cnt);
    p->parts[q] = h;
  }
  return NULL;
}

static void run_threads(par_t* p, void* (*fn)(void*))
{
  pthread_t th[256];
  par_job jobs[256];
  for (int t = 0; t < p->nthreads; ++t) {
    jobs[t].p = p;
    jobs[t].t = t;
    pthread_create(&th[t], NULL, fn, &jobs[t]);
  }
  for (int t = 0; t < p->nthreads; ++t) pthread_join(th[t], NULL);
}

/* Appends the accumulators of groups [0, n) of s at position at of d
 * (d's arrays are allocated for at least at + n groups). */
#define CAT(field, T)                                                                  \
  do {                                                                                 \
    if (d->field) memcpy(d->field + at, s->field, (size_t)n * sizeof(T));              \
  } while (0)
static void acc_append(acc_t* d, const acc_t* s, int64_t at, int64_t n)
{
  CAT(n_all, int64_t); CAT(n_valid, int64_t); CAT(isum, uint64_t); CAT(fsum, double);
  CAT(fcomp, double); CAT(fabs_sum, double); CAT(iprod, uint64_t); CAT(fprod, long double);
  CAT(imin, int64_t); CAT(imax, int64_t); CAT(umin, uint64_t); CAT(umax, uint64_t);
  CAT(fmin, double); CAT(fmax, double); CAT(fmin_seen, uint8_t); CAT(fmax_seen, uint8_t);
  CAT(isq, uint64_t); CAT(fsq, double); CAT(fsq_comp, double); CAT(argmin, int64_t);
  CAT(argmax, int64_t); CAT(m2, long double);
}
#undef CAT

static orc_handle* groupby_parallel(const orc_column* keys, int nkeys, int include_null_keys,
                                    const orc_request* reqs, int nreq, int nthreads, int64_t n)
{
  par_t* p = xcalloc(1, sizeof(par_t));
  p->proto = handle_new(keys, nkeys, include_null_keys, reqs, nreq);
  p->nthreads = nthreads;
  p->n = n;
  p->pid = xcalloc(n, sizeof(uint16_t));
  p->counts = xcalloc((int64_t)nthreads * ORC_NPART, sizeof(int64_t));
  run_threads(p, par_count);
  /* partition-major offsets: partition q's rows from thread 0, then 1, ... */
  int64_t total = 0;
  for (int q = 0; q < ORC_NPART; ++q) {
    p->part_start[q] = total;
    for (int t = 0; t < nthreads; ++t) {
      int64_t c = p->counts[(int64_t)t * ORC_NPART + q];
      p->counts[(int64_t)t * ORC_NPART + q] = total;
      total += c;
    }
  }
  p->part_start[ORC_NPART] = total;
  p->idx = xcalloc(total, sizeof(int64_t));
  run_threads(p, par_scatter);
  free(p->pid);
  p->pid = NULL;
  run_threads(p, par_aggregate);
  free(p->idx);
  free(p->counts);
  /* concatenate the partitions' groups */
  int64_t G = 0;
  for (int q = 0; q < ORC_NPART; ++q) G += p->parts[q]->ngroups;
  orc_handle* h = p->proto;
  if (G > h->gcap) {
    h->gkeys = xrealloc(h->gkeys, G * h->nkw, 8);
    h->first_row = xrealloc(h->first_row, G, 8);
    for (int r = 0; r < nreq; ++r) acc_grow(&h->acc[r], h->gcap, G);
    h->gcap = G;
  }
  int64_t at = 0;
  for (int q = 0; q < ORC_NPART; ++q) {
    orc_handle* s = p->parts[q];
    const int64_t m = s->ngroups;
    if (m) {
      memcpy(h->gkeys + at * h->nkw, s->gkeys, (size_t)(m * h->nkw) * 8);
      memcpy(h->first_row + at, s->first_row, (size_t)m * 8);
      for (int r = 0; r < nreq; ++r) acc_append(&h->acc[r], &s->acc[r], at, m);
    }
    at += m;
    handle_free(s);
  }
  h->ngroups = G;
  free(p);
  return h;
}

int orc_groupby(const orc_column* keys, int nkeys, int include_null_keys,
                const orc_request* reqs, int nreq, int nthreads, orc_handle** out)
{
  *out = NULL;
  if (nkeys < 1 || nkeys > 64) return -1;
  int64_t n = keys[0].size;
  for (int k = 0; k < nkeys; ++k) {
    if (keys[k].size != n || type_width(keys[k].type_id) == 0) return -2;
  }
  for (int r = 0; r < nreq; ++r) {
    if (reqs[r].values.size != n) return -3;
    for (int j = 0; j < reqs[r].num_aggs; ++j)
      if (!orc_valid_agg(reqs[r].values.type_id, reqs[r].kinds[j])) return -4;
  }
  if (nthreads < 1) nthreads = 1;
  if (n < 65536) nthreads = 1;
  if (nthreads > 256) nthreads = 256;
  if (nthreads > 1) {
    *out = groupby_parallel(keys, nkeys, include_null_keys, reqs, nreq, nthreads, n);
    return 0;
  }
  orc_handle* h = handle_new(keys, nkeys, include_null_keys, reqs, nreq);
  aggregate_rows(h, NULL, 0, n);
  second_pass_var(h, NULL, 0, n);
  *out = h;
  return 0;
}

int64_t orc_num_groups(const orc_handle* h) { return h->ngroups; }

void orc_group_rows(const orc_handle* h, int64_t* out)
{
  memcpy(out, h->first_row, 8 * (size_t)h->ngroups);
}

static double f_eps(int t) { return t == T_FLOAT32 ? 1.1920928955078125e-07 : 2.220446049250313e-16; }

static int64_t wrap_to_width(uint64_t v, int t)
{
  switch (type_width(t)) {
    case 4: return (int64_t)(int32_t)(uint32_t)v;
    default: return (int64_t)v;
  }
}

/* Result of aggregation j of request r.  Integer targets are written as int64
 * (unsigned MIN/MAX as their uint64 bits), floating targets as double.  valid
 * gets 1/0 per group; tol (optional) the admissible absolute error per group
 * (0 for results that must match exactly). */
int orc_result(const orc_handle* h, int r, int j, void* out_v, uint8_t* valid, double* tol)
{
  if (r < 0 || r >= h->nreq || j < 0 || j >= h->reqs[r].num_aggs) return -1;
  const acc_t* a = &h->acc[r];
  const orc_request* rq = &h->reqs[r];
  int k = rq->kinds[j];
  int has_nulls = rq->values.mask != NULL;
  int ddof = rq->ddof ? rq->ddof[j] : 1;
  int64_t* oi = (int64_t*)out_v;
  double* of = (double*)out_v;
  int t = a->type_id;
  for (int64_t g = 0; g < h->ngroups; ++g) {
    int64_t nv = a->n_valid[g];
    int ok = nv > 0 || !has_nulls;
    double e = 0.0;
    switch (k) {
      case A_COUNT_VALID: oi[g] = nv; ok = 1; break;
      case A_COUNT_ALL: oi[g] = a->n_all[g]; ok = 1; break;
      case A_SUM:
        if (a->cat == C_FLOAT) {
          of[g] = a->fsum[g] + a->fcomp[g];
          if (t == T_FLOAT32) of[g] = (double)(float)of[g];
          e = 2.0 * (double)nv * f_eps(t) * a->fabs_sum[g] + fabs(of[g]) * f_eps(t);
        } else {
          oi[g] = is_duration(t) ? wrap_to_width(a->isum[g], t) : (int64_t)a->isum[g];
        }
        break;
      case A_PRODUCT:
        if (a->cat == C_FLOAT) { of[g] = (double)a->fprod[g]; e = fabs(of[g]) * 2.0 * (double)(nv + 1) * f_eps(t); }
        else oi[g] = (int64_t)a->iprod[g];
        break;
      case A_SUM_OF_SQUARES:
        if (a->cat == C_FLOAT) { of[g] = a->fsq[g] + a->fsq_comp[g]; e = 2.0 * (double)nv * f_eps(t) * of[g] + fabs(of[g]) * f_eps(t); }
        else oi[g] = (int64_t)a->isq[g];
        break;
      case A_MIN:
        if (a->cat == C_FLOAT) of[g] = a->fmin_seen[g] ? a->fmin[g] : NAN;
        else if (a->cat == C_UNSIGNED) oi[g] = (int64_t)a->umin[g];
        else oi[g] = a->imin[g];
        break;
      case A_MAX:
        if (a->cat == C_FLOAT) of[g] = a->fmax_seen[g] ? a->fmax[g] : NAN;
        else if (a->cat == C_UNSIGNED) oi[g] = (int64_t)a->umax[g];
        else oi[g] = a->imax[g];
        break;
      case A_MEAN:
        if (nv == 0) { if (is_duration(t)) oi[g] = 0; else of[g] = 0.0; break; }
        if (is_duration(t)) { oi[g] = wrap_to_width(a->isum[g], t) / nv; break; }
        if (a->cat == C_FLOAT) {
          double s = a->fsum[g] + a->fcomp[g];
          if (t == T_FLOAT32) s = (double)(float)s;
          of[g] = s / (double)nv;
          e = (2.0 * (double)nv * f_eps(t) * a->fabs_sum[g] + fabs(s) * f_eps(t)) / (double)nv + fabs(of[g]) * 4.4e-16;
        } else {
          of[g] = (double)(int64_t)a->isum[g] / (double)nv;
        }
        break;
      case A_VARIANCE: case A_STD: {
        ok = (nv - ddof) > 0;
        double var = ok ? (double)(a->m2[g] / (long double)(nv - ddof)) : 0.0;
        of[g] = k == A_STD ? sqrt(var) : var;
        /* the engine's mean and per-row terms round in double (and its SUM in
         * the value type); bound relative to the magnitude of the terms */
        double scale = (a->cat == C_FLOAT ? a->fabs_sum[g] : fabs((double)(int64_t)a->isum[g])) / (nv > 0 ? nv : 1);
        e = 64.0 * (double)(nv + 1) * f_eps(a->cat == C_FLOAT ? t : T_FLOAT64) * (fabs(var) + scale * scale);
        if (k == A_STD) e = var > 0 ? fmin(sqrt(e), e / (2.0 * sqrt(var))) : sqrt(e);
        break;
      }
      case A_ARGMIN: oi[g] = a->argmin[g]; ok = a->argmin[g] >= 0; break;
      case A_ARGMAX: oi[g] = a->argmax[g]; ok = a->argmax[g] >= 0; break;
      default: return -2;
    }
    if (k == A_ARGMIN || k == A_ARGMAX) ok = ok || !has_nulls;
    if (valid) valid[g] = (uint8_t)ok;
    if (tol) tol[g] = e;
  }
  return 0;
}

void orc_free(orc_handle* h) { handle_free(h); }
