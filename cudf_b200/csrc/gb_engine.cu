// gb_engine.cu -- host orchestration of the hash groupby: planning, table
// sizing from a key sample, launches, overflow retry and compaction.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <set>
#include <string>
#include <tuple>
#include <vector>

#include "gb_engine.h"
#include "gb_kernels.cuh"
#include "gb_partition.cuh"
#include "gb_scatter.h"
#include "gb_sorted.h"

namespace gb {

// ---------------------------------------------------------------------------
// type system (cpp/include/cudf/detail/aggregation/aggregation.hpp:1168-1290)
int type_width(int t)
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
static bool is_ts(int t) { return t >= T_TS_D && t <= T_TS_NS; }
static bool is_dur(int t) { return t >= T_DUR_D && t <= T_DUR_NS; }
static uint8_t type_cat(int t)
{
  if (t == T_FLOAT32) return CAT_F32;
  if (t == T_FLOAT64) return CAT_F64;
  if (t == T_BOOL8) return CAT_BOOL;
  if (t >= T_UINT8 && t <= T_UINT64) return CAT_UNSIGNED;
  return CAT_SIGNED;
}

bool valid_agg(int t, int k)
{
  if (type_width(t) == 0) return false;
  bool numeric = !is_ts(t) && !is_dur(t);
  switch (k) {
    case K_MIN: case K_MAX: case K_COUNT_VALID: case K_COUNT_ALL: case K_ARGMIN: case K_ARGMAX: return true;
    case K_SUM: case K_MEAN: return numeric || is_dur(t);
    case K_PRODUCT: case K_SUM_OF_SQUARES: case K_VARIANCE: case K_STD: return numeric;
    default: return false;
  }
}

int target_type(int t, int k)
{
  switch (k) {
    case K_COUNT_VALID: case K_COUNT_ALL: case K_ARGMIN: case K_ARGMAX: return T_INT32;
    case K_MIN: case K_MAX: return t;
    case K_VARIANCE: case K_STD: return T_FLOAT64;
    case K_MEAN: return is_dur(t) ? t : T_FLOAT64;
    case K_SUM: case K_PRODUCT: case K_SUM_OF_SQUARES:
      return (t == T_FLOAT32 || t == T_FLOAT64 || is_dur(t)) ? t : T_INT64;
    default: return T_EMPTY;
  }
}

// ---------------------------------------------------------------------------
static void ck(cudaError_t e, const char* what)
{
  if (e == cudaSuccess) return;
  cudaGetLastError();
  throw Error(e == cudaErrorMemoryAllocation ? ERR_ALLOC : ERR_CUDA,
              std::string(what) + ": " + cudaGetErrorString(e));
}

static void* default_alloc(void*, size_t bytes, void* stream)
{
  static std::once_flag once;
  std::call_once(once, [] {
    // keep freed blocks cached in the pool: repeated calls then allocate in O(1)
    int dev = 0;
    cudaGetDevice(&dev);
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
      uint64_t thr = UINT64_MAX;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
  });
  void* p = nullptr;
  if (bytes == 0) bytes = 16;
  cudaError_t e = cudaMallocAsync(&p, bytes, (cudaStream_t)stream);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return p;
}
static void default_free(void*, void* p, size_t, void* stream)
{
  if (p) cudaFreeAsync(p, (cudaStream_t)stream);
}
Allocator default_allocator() { return Allocator{default_alloc, default_free, nullptr}; }

// Scratch buffers of one call, returned to the allocator on scope exit.
struct Scratch {
  Allocator A;
  cudaStream_t s;
  struct Buf { void* p; size_t n; };
  std::vector<Buf> bufs;
  Scratch(const Allocator& a, cudaStream_t st) : A(a), s(st) {}
  void* get(size_t n)
  {
    void* p = A.allocate(A.ctx, n, (void*)s);
    if (!p) throw Error(ERR_ALLOC, "device allocation of " + std::to_string(n) + " bytes failed");
    bufs.push_back({p, n});
    // kernels read scratch arrays with 16-byte vector loads and bulk copies
    if ((uintptr_t)p & 15) throw Error(ERR_LOGIC, "the allocator returned a block that is not 16-byte aligned");
    return p;
  }
  void put(void* p)
  {
    for (size_t i = 0; i < bufs.size(); ++i)
      if (bufs[i].p == p) {
        A.deallocate(A.ctx, p, bufs[i].n, (void*)s);
        bufs.erase(bufs.begin() + i);
        return;
      }
  }
  ~Scratch()
  {
    for (auto& b : bufs) A.deallocate(A.ctx, b.p, b.n, (void*)s);
  }
};

void Result::release()
{
  auto fr = [&](void* p, size_t n) {
    if (p && alloc.deallocate) alloc.deallocate(alloc.ctx, p, n, (void*)stream);
  };
  for (auto& c : keys) { fr(c.data, c.data_bytes); fr(c.mask, c.mask_bytes); }
  for (auto& r : results)
    for (auto& c : r) { fr(c.data, c.data_bytes); fr(c.mask, c.mask_bytes); }
  keys.clear();
  results.clear();
}

struct DevInfo {
  int sms = 148;
  int smem_optin = 227 * 1024;
};
static DevInfo dev_info()
{
  static std::mutex mu;
  static DevInfo cache[64];
  static bool have[64] = {};
  int dev = 0;
  ck(cudaGetDevice(&dev), "cudaGetDevice");
  std::lock_guard<std::mutex> g(mu);
  if (dev < 64 && !have[dev]) {
    cudaDeviceGetAttribute(&cache[dev].sms, cudaDevAttrMultiProcessorCount, dev);
    cudaDeviceGetAttribute(&cache[dev].smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    have[dev] = true;
  }
  return cache[dev < 64 ? dev : 0];
}

static uint64_t next_pow2(uint64_t x)
{
  uint64_t p = 1;
  while (p < x) p <<= 1;
  return p;
}

// ---------------------------------------------------------------------------
// planning
void build_plan(const std::vector<Column>& keys, int null_policy, const std::vector<Request>& reqs,
                Plan& P, std::vector<int>& out_types)
{
  std::memset(&P, 0, sizeof(P));
  if (keys.empty()) throw Error(ERR_LOGIC, "groupby needs at least one key column");
  if (keys.size() > (size_t)kMaxKeyCols) throw Error(ERR_UNSUPPORTED, "too many key columns");
  int64_t n = keys[0].size;
  for (auto& k : keys) {
    if (k.size != n) throw Error(ERR_LOGIC, "Size mismatch between key columns.");
    if (type_width(k.type_id) == 0) throw Error(ERR_UNSUPPORTED, "unsupported key column type");
  }
  // cpp/src/groupby/groupby.cu:208-212
  for (auto& r : reqs)
    if (r.values.size != n) throw Error(ERR_LOGIC, "Size mismatch between request values and groupby keys.");
  // cpp/src/groupby/groupby.cu:174-190
  for (auto& r : reqs)
    for (auto& a : r.aggs)
      if (!valid_agg(r.values.type_id, a.kind)) throw Error(ERR_LOGIC, "Invalid type/aggregation combination.");
  if (n >= (int64_t)0xFFFFFFF0ll) throw Error(ERR_UNSUPPORTED, "more than 2^32-16 rows in one groupby");

  P.num_rows = n;
  P.include_nulls = null_policy == 1;
  P.num_keys = (int)keys.size();
  // key packing, first-fit decreasing: value bits never straddle a word, null
  // flags (INCLUDE only) are single bits; word 0 holds 64 bits, word 1 at most
  // 63 so that its top bit stays clear (the empty-slot marker of 2-word keys)
  struct Item { int bits, key; bool null_flag; };
  std::vector<Item> items;
  for (int k = 0; k < P.num_keys; ++k) {
    KeyCol& c = P.keys[k];
    c.data = keys[k].data;
    c.mask = keys[k].mask;
    c.offset = keys[k].offset;
    c.type_id = keys[k].type_id;
    c.width = (uint8_t)type_width(c.type_id);
    c.cat = type_cat(c.type_id);
    if (c.mask) P.any_key_nullable = 1;
    items.push_back({8 * c.width, k, false});
    if (c.mask && P.include_nulls) {
      items.push_back({1, k, true});
      c.has_null_bit = 1;
    }
  }
  std::stable_sort(items.begin(), items.end(), [](const Item& a, const Item& b) { return a.bits > b.bits; });
  int used[2] = {0, 0};
  const int room[2] = {64, 63};
  int words = 1;
  for (auto& it : items) {
    int w = 0;
    while (w < 2 && used[w] + it.bits > room[w]) ++w;
    if (w == 2) throw Error(ERR_UNSUPPORTED, "key rows wider than 127 packed bits are not supported");
    KeyCol& c = P.keys[it.key];
    if (it.null_flag) { c.null_word = (uint8_t)w; c.null_shift = (uint8_t)used[w]; }
    else { c.word = (uint8_t)w; c.shift = (uint8_t)used[w]; }
    used[w] += it.bits;
    words = std::max(words, w + 1);
  }
  P.key_words = words;

  // value columns: one entry per distinct (column view, ddof of VAR/STD)
  struct VKey { Column c; int ddof; };
  std::vector<VKey> vk;
  std::vector<std::vector<int>> need(0);
  auto find_col = [&](const Column& c, int ddof) {
    for (size_t i = 0; i < vk.size(); ++i)
      if (vk[i].c.data == c.data && vk[i].c.mask == c.mask && vk[i].c.offset == c.offset &&
          vk[i].c.type_id == c.type_id && vk[i].ddof == ddof)
        return (int)i;
    vk.push_back({c, ddof});
    return (int)vk.size() - 1;
  };
  // per request/agg: column index
  std::vector<std::vector<int>> colof(reqs.size());
  for (size_t r = 0; r < reqs.size(); ++r)
    for (auto& a : reqs[r].aggs) {
      bool var = a.kind == K_VARIANCE || a.kind == K_STD;
      colof[r].push_back(find_col(reqs[r].values, var ? a.ddof : -1));
    }
  if (vk.size() > (size_t)kMaxValCols) throw Error(ERR_UNSUPPORTED, "too many distinct value columns");
  P.num_vals = (int)vk.size();

  // which accumulator ops each column needs
  std::vector<std::vector<uint8_t>> ops(vk.size());
  std::vector<bool> need_nulls(vk.size(), false), need_m2(vk.size(), false);
  auto add = [&](int v, uint8_t op) {
    if (std::find(ops[v].begin(), ops[v].end(), op) == ops[v].end()) ops[v].push_back(op);
  };
  for (size_t r = 0; r < reqs.size(); ++r)
    for (size_t j = 0; j < reqs[r].aggs.size(); ++j) {
      int v = colof[r][j];
      const Column& c = vk[v].c;
      int t = c.type_id, w = type_width(t);
      uint8_t cat = type_cat(t);
      bool fl = cat == CAT_F32 || cat == CAT_F64;
      int k = reqs[r].aggs[j].kind;
      if (c.mask && k != K_COUNT_ALL) need_nulls[v] = true;
      auto sum_op = [&]() -> uint8_t {
        if (cat == CAT_F32) return OP_SUM_F32;
        if (cat == CAT_F64) return OP_SUM_F64;
        if (is_dur(t) && w == 4) return OP_SUM_I32;
        return OP_SUM_I64;
      };
      switch (k) {
        case K_SUM: case K_MEAN: add(v, sum_op()); break;
        case K_VARIANCE: case K_STD: add(v, sum_op()); need_m2[v] = true; break;
        case K_MIN: add(v, w == 8 ? OP_MIN_U64 : OP_MIN_U32); break;
        case K_MAX: add(v, w == 8 ? OP_MAX_U64 : OP_MAX_U32); break;
        case K_SUM_OF_SQUARES: add(v, cat == CAT_F32 ? OP_SQ_F32 : cat == CAT_F64 ? OP_SQ_F64 : OP_SQ_I64); break;
        case K_PRODUCT: add(v, cat == CAT_F32 ? OP_PROD_F32 : cat == CAT_F64 ? OP_PROD_F64 : OP_PROD_I64); break;
        case K_ARGMIN: add(v, w == 8 ? OP_ARGMIN_R64 : OP_ARGMIN_P32); P.has_arg = 1; break;
        case K_ARGMAX: add(v, w == 8 ? OP_ARGMAX_R64 : OP_ARGMAX_P32); P.has_arg = 1; break;
        default: break;
      }
      (void)fl;
    }

  // slot layout: key words | rows u32 | null counters u32 | 4-byte accs | 8-byte accs
  auto op_size = [](uint8_t op) {
    switch (op) {
      case OP_SUM_I32: case OP_SUM_F32: case OP_MIN_U32: case OP_MAX_U32: case OP_SQ_F32:
      case OP_PROD_F32: return 4;
      default: return 8;
    }
  };
  int off = 8 * P.key_words;
  P.rows_off = off;
  off += 4;
  for (size_t v = 0; v < vk.size(); ++v) {
    ValCol& c = P.vals[v];
    c.data = vk[v].c.data;
    c.mask = vk[v].c.mask;
    c.offset = vk[v].c.offset;
    c.type_id = vk[v].c.type_id;
    c.width = (uint8_t)type_width(c.type_id);
    c.cat = type_cat(c.type_id);
    c.ddof = vk[v].ddof < 0 ? 1 : vk[v].ddof;
    c.nulls_off = -1;
    c.sum_off = -1;
    c.m2_off = -1;
    if (need_nulls[v]) { c.nulls_off = (int16_t)off; off += 4; }
  }
  // accumulators grouped per column, 4-byte ones first within the slot
  std::vector<std::pair<int, int>> acc_off;  // (col, op) -> offset resolved below
  int na = 0;
  for (int pass = 0; pass < 2; ++pass) {
    if (pass == 1) off = (off + 7) & ~7;
    for (size_t v = 0; v < vk.size(); ++v)
      for (uint8_t op : ops[v]) {
        if ((op_size(op) == 4) != (pass == 0)) continue;
        if (na >= kMaxAccs) throw Error(ERR_UNSUPPORTED, "too many aggregations in one call");
        P.accs[na].op = op;
        P.accs[na].col = (uint8_t)v;
        P.accs[na].off = (uint16_t)off;
        off += op_size(op);
        ++na;
      }
  }
  for (size_t v = 0; v < vk.size(); ++v)
    if (need_m2[v]) {
      P.vals[v].m2_off = (int16_t)off;
      off += 8;
      P.need_second_pass = 1;
    }
  P.num_accs = na;
  // stride: an odd multiple of 8 bytes (16 for two-word keys, whose 128-bit
  // CAS needs 16-byte alignment) so that one field of 32 different slots
  // falls into many shared-memory banks
  {
    int unit = P.key_words == 2 ? 16 : 8;
    int q = (off + unit - 1) / unit;
    if ((q & 1) == 0) ++q;
    P.slot_bytes = q * unit;
  }
  if (P.slot_bytes > kMaxSlotBytes) throw Error(ERR_UNSUPPORTED, "too many aggregations in one call");
  // reorder accs by column so each column owns a contiguous range
  std::stable_sort(P.accs, P.accs + na, [](const Acc& a, const Acc& b) { return a.col < b.col; });
  for (size_t v = 0; v < vk.size(); ++v) {
    ValCol& c = P.vals[v];
    c.acc_begin = c.acc_end = 0;
    c.min_off = c.max_off = c.sq_off = -1;
    c.sum_op = 0;
    c.basic = 1;
    bool first = true;
    for (int a = 0; a < na; ++a)
      if (P.accs[a].col == v) {
        if (first) { c.acc_begin = (int16_t)a; first = false; }
        c.acc_end = (int16_t)(a + 1);
        uint8_t op = P.accs[a].op;
        int16_t o = (int16_t)P.accs[a].off;
        if (op == OP_SUM_I64 || op == OP_SUM_I32 || op == OP_SUM_F32 || op == OP_SUM_F64) { c.sum_off = o; c.sum_op = op; }
        else if (op == OP_MIN_U32 || op == OP_MIN_U64) c.min_off = o;
        else if (op == OP_MAX_U32 || op == OP_MAX_U64) c.max_off = o;
        else if (op == OP_SQ_I64 || op == OP_SQ_F32 || op == OP_SQ_F64) c.sq_off = o;
        else c.basic = 0;
      }
  }
  auto acc_for = [&](int v, uint8_t op) -> int16_t {
    for (int a = 0; a < na; ++a)
      if (P.accs[a].col == v && P.accs[a].op == op) return (int16_t)P.accs[a].off;
    return -1;
  };

  // outputs in request order
  out_types.clear();
  int no = 0;
  for (size_t r = 0; r < reqs.size(); ++r)
    for (size_t j = 0; j < reqs[r].aggs.size(); ++j) {
      if (no >= kMaxOutputs) throw Error(ERR_UNSUPPORTED, "too many aggregations in one call");
      int v = colof[r][j];
      const ValCol& c = P.vals[v];
      OutSpec& o = P.outs[no++];
      o.kind = reqs[r].aggs[j].kind;
      o.col = v;
      o.out_type = target_type(c.type_id, o.kind);
      o.out_width = (uint8_t)type_width(o.out_type);
      o.ddof = reqs[r].aggs[j].ddof;
      bool has_nulls = c.mask != nullptr;
      int w = c.width;
      switch (o.kind) {
        case K_COUNT_VALID: case K_COUNT_ALL: o.nullable = 0; o.acc_off = -1; break;
        case K_SUM: case K_MEAN: o.nullable = has_nulls; o.acc_off = c.sum_off; break;
        case K_VARIANCE: case K_STD: o.nullable = 1; o.acc_off = c.m2_off; break;
        case K_MIN: o.nullable = has_nulls; o.acc_off = acc_for(v, w == 8 ? OP_MIN_U64 : OP_MIN_U32); break;
        case K_MAX: o.nullable = has_nulls; o.acc_off = acc_for(v, w == 8 ? OP_MAX_U64 : OP_MAX_U32); break;
        case K_SUM_OF_SQUARES: o.nullable = has_nulls;
          o.acc_off = acc_for(v, c.cat == CAT_F32 ? OP_SQ_F32 : c.cat == CAT_F64 ? OP_SQ_F64 : OP_SQ_I64); break;
        case K_PRODUCT: o.nullable = has_nulls;
          o.acc_off = acc_for(v, c.cat == CAT_F32 ? OP_PROD_F32 : c.cat == CAT_F64 ? OP_PROD_F64 : OP_PROD_I64); break;
        case K_ARGMIN: o.nullable = has_nulls; o.acc_off = acc_for(v, w == 8 ? OP_ARGMIN_R64 : OP_ARGMIN_P32); break;
        case K_ARGMAX: o.nullable = has_nulls; o.acc_off = acc_for(v, w == 8 ? OP_ARGMAX_R64 : OP_ARGMAX_P32); break;
        default: break;
      }
      out_types.push_back(o.out_type);
    }
  P.num_outs = no;
}

static void build_template(const Plan& P, SlotTemplate& t)
{
  std::memset(&t, 0, sizeof(t));
  uint8_t* b = (uint8_t*)&t.w[0];
  std::memset(b, 0xFF, 8 * P.key_words);
  for (int a = 0; a < P.num_accs; ++a) {
    uint8_t* p = b + P.accs[a].off;
    switch (P.accs[a].op) {
      case OP_MIN_U32: std::memset(p, 0xFF, 4); break;
      case OP_MIN_U64: case OP_ARGMIN_P32: case OP_ARGMIN_R64: case OP_ARGMAX_R64: std::memset(p, 0xFF, 8); break;
      case OP_PROD_I64: { int64_t one = 1; std::memcpy(p, &one, 8); break; }
      case OP_PROD_F32: { float one = 1.0f; std::memcpy(p, &one, 4); break; }
      case OP_PROD_F64: { double one = 1.0; std::memcpy(p, &one, 8); break; }
      default: break;
    }
  }
}

void allow_max_smem(const void* kernel)
{
  static std::mutex mu;
  static std::set<std::pair<int, const void*>> done;
  int dev = 0;
  ck(cudaGetDevice(&dev), "cudaGetDevice");
  std::lock_guard<std::mutex> lk(mu);
  if (done.count({dev, kernel})) return;
  int optin = 0;
  ck(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev), "smem attr");
  cudaFuncAttributes fa;
  ck(cudaFuncGetAttributes(&fa, kernel), "func attr");
  ck(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes),
     "smem attr");
  done.insert({dev, kernel});
}

// ---------------------------------------------------------------------------
namespace {
thread_local uint32_t* t_pinned = nullptr;
thread_local cudaEvent_t t_ev[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
cudaEvent_t* events()
{
  if (!t_ev[0])
    for (auto& e : t_ev) ck(cudaEventCreate(&e), "cudaEventCreate");
  return t_ev;
}
// Per-thread pinned host words: [0, 1024) counters read back by the host,
// [1024, 1024 + 2^kHllBits + 2^kBucketBits) the key sketch.
constexpr size_t kPinnedWords = 1024 + (size_t(1) << kHllBits) + (size_t(1) << kBucketBits);
uint32_t* pinned()
{
  if (!t_pinned) ck(cudaMallocHost((void**)&t_pinned, kPinnedWords * 4), "cudaMallocHost");
  return t_pinned;
}
// Pinned staging of the partitioned path's region table (starts, ends,
// cursors: 3 x 8 bytes for up to 8192 partitions), per host thread.  A call
// finishes with a stream synchronisation, so the copy out of it is done before
// the thread's next call writes it again.
thread_local int64_t* t_regions = nullptr;
constexpr size_t kRegionWords = 3 * 8192;
int64_t* pinned_regions()
{
  if (!t_regions) ck(cudaMallocHost((void**)&t_regions, kRegionWords * 8), "cudaMallocHost");
  return t_regions;
}

// HyperLogLog cardinality from 2^kHllBits registers (Flajolet et al. 2007):
// E = alpha_m m^2 / sum 2^-M[j], with linear counting m ln(m/V) while E is
// below 2.5 m and V registers are still zero.  64-bit hashes need no
// large-range correction.
double hll_estimate(const std::vector<uint32_t>& regs)
{
  const double m = (double)regs.size();
  double z = 0;
  int zeros = 0;
  for (uint32_t r : regs) {
    z += std::ldexp(1.0, -(int)r);
    zeros += r == 0;
  }
  const double alpha = 0.7213 / (1.0 + 1.079 / m);
  double e = alpha * m * m / z;
  if (e <= 2.5 * m && zeros > 0) e = m * std::log(m / zeros);
  return e;
}


OutColumn make_out(const Allocator& A, cudaStream_t s, int type_id, int64_t rows, bool nullable)
{
  OutColumn c;
  c.type_id = type_id;
  c.size = rows;
  c.data_bytes = (size_t)std::max<int64_t>(rows, 1) * type_width(type_id);
  c.data = A.allocate(A.ctx, c.data_bytes, (void*)s);
  if (!c.data) throw Error(ERR_ALLOC, "device allocation of an output column failed");
  if (nullable) {
    c.mask_bytes = (size_t)((std::max<int64_t>(rows, 1) + 511) / 512) * 64;
    c.mask = (uint32_t*)A.allocate(A.ctx, c.mask_bytes, (void*)s);
    if (!c.mask) throw Error(ERR_ALLOC, "device allocation of an output mask failed");
    ck(cudaMemsetAsync(c.mask, 0, c.mask_bytes, s), "memset mask");
  }
  return c;
}
}  // namespace

int grid_for(const void* kernel, int block, size_t smem, int bps_cap)
{
  DevInfo d = dev_info();
  // the occupancy of a (kernel, block, shared memory) launch does not change
  // once allow_max_smem has raised the kernel's limit: ask the runtime once
  // per device and launch shape
  static std::mutex mu;
  static std::map<std::tuple<int, const void*, int, size_t>, int> memo;
  int dev = 0;
  ck(cudaGetDevice(&dev), "cudaGetDevice");
  const auto key = std::make_tuple(dev, kernel, block, smem);
  int bps = 0;
  {
    std::lock_guard<std::mutex> lk(mu);
    auto it = memo.find(key);
    if (it != memo.end()) bps = it->second;
  }
  if (bps == 0) {
    ck(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, kernel, block, smem), "occupancy");
    if (bps < 1) bps = 1;
    std::lock_guard<std::mutex> lk(mu);
    memo[key] = bps;
  }
  if (bps < 1) bps = 1;
  if (bps_cap > 0) bps = std::min(bps, bps_cap);
  return d.sms * bps;
}

namespace {
std::mutex g_rules_mu;
std::vector<TuningRule> g_rules;
}  // namespace

void set_tuning_rules(const std::vector<TuningRule>& rules)
{
  std::lock_guard<std::mutex> lk(g_rules_mu);
  g_rules = rules;
}

int apply_tuning_rules(Options& o, int64_t rows, int64_t groups, int key_words, uint32_t* applied)
{
  std::lock_guard<std::mutex> lk(g_rules_mu);
  if (applied) *applied = 0;
  for (size_t i = 0; i < g_rules.size(); ++i) {
    const TuningRule& r = g_rules[i];
    if (rows > r.max_rows || groups > r.max_groups || (r.key_words && r.key_words != key_words)) continue;
    const uint32_t m = r.mask & ~o.set_mask;
    if (applied) *applied = m;
    if (m & OPT_BLOCK) o.block = r.opt.block;
    if (m & OPT_BPS) o.blocks_per_sm = r.opt.blocks_per_sm;
    if (m & OPT_SMEM) o.smem_bytes = r.opt.smem_bytes;
    if (m & OPT_FILL) o.smem_fill = r.opt.smem_fill;
    if (m & OPT_SMEM_MAX) o.smem_max_groups = r.opt.smem_max_groups;
    if (m & OPT_LOAD) o.load_factor = r.opt.load_factor;
    if (m & OPT_MODE) o.force_mode = r.opt.force_mode;
    if (m & OPT_SCATTER) o.scatter = r.opt.scatter;
    if (m & OPT_PASS2) o.pass2 = r.opt.pass2;
    if (m & OPT_PART_FILL) o.part_fill = r.opt.part_fill;
    if (m & OPT_WAGG) o.wagg_pct = r.opt.wagg_pct;
    return (int)i;
  }
  return -1;
}

Result aggregate(const std::vector<Column>& keys, int null_policy, const std::vector<Request>& reqs,
                 cudaStream_t stream, const Allocator& alloc, const Options& opt_in, Stats* stats)
{
  Options opt = opt_in;  // tuning rules may adjust it once the group estimate is known
  Plan P;
  std::vector<int> out_types;
  build_plan(keys, null_policy, reqs, P, out_types);
  Stats st;
  Result R;
  R.alloc = alloc;
  R.stream = stream;
  const int64_t n = P.num_rows;
  static const bool trace = std::getenv("GB_TRACE") != nullptr;
  auto t0 = std::chrono::steady_clock::now();
  auto mark = [&](const char* what) {
    if (!trace) return;
    auto t = std::chrono::steady_clock::now();
    std::fprintf(stderr, "[gb] %-28s %9.3f ms\n", what, std::chrono::duration<double, std::milli>(t - t0).count());
  };

  // cpp/src/groupby/groupby.cu:216 -- empty input gives empty outputs
  if (n == 0) {
    for (auto& k : keys) R.keys.push_back(make_out(alloc, stream, k.type_id, 0, k.mask != nullptr));
    int j = 0;
    for (auto& r : reqs) {
      std::vector<OutColumn> cols;
      for (size_t a = 0; a < r.aggs.size(); ++a, ++j)
        cols.push_back(make_out(alloc, stream, out_types[j], 0, P.outs[j].nullable));
      R.results.push_back(cols);
    }
    if (stats) *stats = st;
    return R;
  }

  Scratch S(alloc, stream);
  mark("begin");
  unsigned int* counters = (unsigned int*)S.get(4096);
  ck(cudaMemsetAsync(counters, 0, 4096, stream), "memset counters");
  mark("counters");
  uint32_t* host = pinned();
  DevInfo dev = dev_info();
  SlotTemplate tmpl;
  build_template(P, tmpl);

  // ---- group-count estimate from a key sample ----
  int64_t est;
  std::vector<uint32_t> buckets;
  bool exact_buckets = false;  // buckets hold exact row counts (full-pass sketch)
  int64_t nsamp = 0;
  if (opt.groups_hint >= 0) {
    est = std::max<int64_t>(1, opt.groups_hint);
  } else if (n <= 65536) {
    est = n;
  } else {
    // full pass over the keys: exact rows per hash bucket (partition region
    // sizes) and a HyperLogLog estimate of the number of distinct keys
    unsigned int* hll = (unsigned int*)S.get((sizeof(unsigned int) << kHllBits) + (sizeof(unsigned int) << kBucketBits));
    unsigned int* bk = hll + (1 << kHllBits);
    ck(cudaMemsetAsync(hll, 0, (sizeof(unsigned int) << kHllBits) + (sizeof(unsigned int) << kBucketBits), stream),
       "memset sketch");
    {
      const size_t sm = sketch_smem();
      allow_max_smem((const void*)k_sketch);
      // at least 16Ki rows per CTA: each CTA clears and merges 80 KB of
      // shared counters, which dominates on small inputs
      int grid = grid_for((const void*)k_sketch, 512, sm, 0);
      grid = (int)std::min<int64_t>(grid, (n + 16383) / 16384);
      k_sketch<<<grid, 512, sm, stream>>>(P, hll, bk);
    }
    st.kernels += 1;
    ck(cudaGetLastError(), "sketch launch");
    mark("sketch launched");
    uint32_t* hs = host + 1024;  // registers then buckets, adjacent on the device too
    ck(cudaMemcpyAsync(hs, hll, ((size_t(1) << kHllBits) + (size_t(1) << kBucketBits)) * 4, cudaMemcpyDeviceToHost,
                       stream), "sketch d2h");
    ck(cudaStreamSynchronize(stream), "sketch sync");
    std::vector<uint32_t> regs(hs, hs + (size_t(1) << kHllBits));
    buckets.assign(hs + (size_t(1) << kHllBits), hs + (size_t(1) << kHllBits) + (size_t(1) << kBucketBits));
    S.put(hll);
    exact_buckets = true;
    int64_t valid_rows = 0;
    for (auto b : buckets) valid_rows += b;
    est = (int64_t)std::llround(hll_estimate(regs));
    est = std::min<int64_t>(std::max<int64_t>(est, valid_rows > 0 ? 1 : 0), valid_rows);
    est = std::max<int64_t>(est, 1);
    nsamp = valid_rows;
  }
  st.est_groups = est;
  uint32_t rule_fields = 0;
  st.rule = apply_tuning_rules(opt, n, est, P.key_words, &rule_fields);
  // Many heavy hitters (a long-tailed key distribution, e.g. Zipf): besides
  // the few partitions well above the average size, most partitions hold keys
  // with hundreds of rows, whose lanes would queue on one shared address, so
  // every partition combines the rows of one slot per warp first.  The sign is
  // in the exact bucket counts: at least 32 buckets above four times the mean
  // of the non-empty ones (uniform keys have none; one hot key makes one).
  if (exact_buckets && !((opt.set_mask | rule_fields) & OPT_WAGG)) {
    int64_t rows_in = 0, nonempty = 0;
    for (auto b : buckets) {
      rows_in += b;
      nonempty += b > 0;
    }
    const double mean = nonempty ? (double)rows_in / (double)nonempty : 0.0;
    int heavy = 0;
    for (auto b : buckets) heavy += (double)b > 4.0 * mean;
    if (heavy >= 32) opt.wagg_pct = 0;
  }
  mark("estimate");

  // ---- mode ----
  auto smem_cap_for = [&](int budget) {
    int sb = std::min(budget, dev.smem_optin - 4096);
    int c = 0;
    if (sb > 0 && P.slot_bytes <= sb) {
      c = 1;
      while ((int64_t)c * 2 * P.slot_bytes <= sb) c *= 2;
    }
    return c;
  };
  int scap = smem_cap_for(opt.smem_bytes);
  int sfill = std::max(1, (int)(scap * opt.smem_fill));
  // groups that outgrow the configured shared-stage table but fit a larger
  // one (up to ~200 KB at fill 0.7) get the larger one, unless the caller
  // sized the table
  if (!(opt.set_mask & (OPT_SMEM | OPT_FILL))) {
    const int big = smem_cap_for(200 * 1024);
    if (est > sfill && est <= (int64_t)(0.7 * big)) {
      scap = big;
      sfill = std::max(1, (int)(0.7 * big));
    }
  }
  int64_t smem_max = opt.smem_max_groups >= 0 ? opt.smem_max_groups : (int64_t)sfill;
  // partitioned pass 2.  Per-row variant: as many slots as fit ~220 KB (any
  // count), one more for the all-ones key.  Sorted-chunk variants: the slots
  // that fit beside the chunk's sorted stage and the two per-slot count arrays.
  bool any_val_null = false;
  for (int v = 0; v < P.num_vals; ++v) any_val_null |= P.vals[v].mask != nullptr;
  const bool p2_sorted = opt.pass2 != 1 && opt.pass2 != 4;
  const int p2_rows = part_sorted_rows(opt.pass2, P.num_vals);  // rows per sorted chunk
  int scap2;
  if (p2_sorted) {
    const size_t budget = (size_t)std::min(227 * 1024, dev.smem_optin) - 4096;
    const size_t fixed = part_sorted_smem(P, 0, p2_rows, any_val_null);
    const size_t per_slot = (size_t)P.slot_bytes + 8;
    scap2 = budget > fixed + 256 + 2 * per_slot ? (int)((budget - fixed - 256) / per_slot) - 1 : 0;
    while (scap2 > 0 && part_sorted_smem(P, scap2, p2_rows, any_val_null) > budget) --scap2;
    scap2 = std::min(scap2, 65000);  // slot indices are 16-bit in the sorted stage
  } else {
    scap2 = std::max(0, std::min(220 * 1024, dev.smem_optin - 8192) / P.slot_bytes - 1);
  }
  const int sfill2 = std::max(1, (int)(scap2 * 0.8));
  bool part_ok = !P.has_arg && !P.need_second_pass && P.num_vals <= 8 && scap2 >= 256;
  for (int v = 0; v < P.num_vals; ++v) part_ok = part_ok && P.vals[v].basic;
  for (int a = 0; a < P.num_accs; ++a) {
    uint8_t op = P.accs[a].op;
    if (op >= OP_PROD_I64 && op <= OP_PROD_F64) part_ok = false;
  }
  // partitions: enough for ~70% table fill, at most 8192 (the scatter's
  // per-tile partition arrays take 16 B each in shared memory); beyond
  // ~85% of that capacity the shared tables would spill most groups and
  // the global table is faster
  constexpr int kMaxParts = 8192;
  int nparts = 0;
  if (part_ok) {
    double per = scap2 * opt.part_fill;
    nparts = (int)std::min<uint64_t>(kMaxParts, std::max<uint64_t>(2, next_pow2((uint64_t)std::ceil(est / per))));
  }
  const bool part_fits = (double)est <= 0.85 * (double)kMaxParts * sfill2;
  int mode;
  if (opt.force_mode >= 0) mode = opt.force_mode;
  else if (scap >= 64 && est <= smem_max) mode = 1;
  else if (part_ok && part_fits && n >= (1 << 20) && est > smem_max) mode = 2;
  else mode = 0;
  if (mode == 1 && scap < 16) mode = 0;
  if (mode == 2 && !part_ok) mode = 0;

  // region sizes of the partitioned path: exact rows per partition from the
  // full-pass sketch (else the sample's share with slack)
  std::vector<int64_t> pbase, pend, prows;
  if (mode == 2) {
    if (buckets.empty()) {  // no sketch (hint given or small input): uniform regions
      buckets.assign((size_t)1 << kBucketBits, 1);
      nsamp = (int64_t)buckets.size();
      exact_buckets = false;
    }
    int lg = 0;
    while ((1 << lg) < nparts) ++lg;
    int per_bucket = kBucketBits - lg;
    pbase.resize(nparts);
    pend.resize(nparts);
    prows.resize(nparts);
    int64_t total = 0, maxload = 0;
    double samp = 0;
    for (auto b : buckets) samp += b;
    for (int p = 0; p < nparts; ++p) {
      double c = 0;
      for (int b = p << per_bucket; b < ((p + 1) << per_bucket); ++b) c += buckets[b];
      int64_t capp;
      if (exact_buckets) {
        capp = (int64_t)c;
        prows[p] = capp;
      } else {
        int64_t expect = (int64_t)std::ceil((double)n * c / std::max(1.0, samp));
        capp = std::max<int64_t>((int64_t)(1.3 * expect), (int64_t)(1.15 * n / nparts)) + 2048;
        capp = std::min<int64_t>(capp, n);
        prows[p] = expect;
        maxload = std::max<int64_t>(maxload, expect);
      }
      pbase[p] = total;
      total += (capp + 31) & ~31ll;
      pend[p] = total;
    }
    // heavy skew seen only through a sample: one partition could hold far
    // more than its share (exact counts split heavy partitions instead)
    if (!exact_buckets && opt.force_mode != 2 && maxload > 4 * (n / nparts) + 4096) mode = (scap >= 64) ? 1 : 0;
  }
  st.mode = mode;

  uint64_t cap = next_pow2((uint64_t)std::max<double>(1024.0, std::ceil((double)est / opt.load_factor)));
  cap = std::min<uint64_t>(cap, next_pow2((uint64_t)(2 * n + 2)));
  cap = std::max<uint64_t>(cap, 1024);

  uint8_t* T = nullptr;
  TableRef G{};
  uint8_t* dense = nullptr;
  int64_t dense_n = 0;
  int64_t dense_cap = 0;
  bool done = false;
  // one read-back for the whole call (see Options::sync_checks)
  const bool deferred = !opt.sync_checks;
  bool prof_part = false, prof_agg = false;

  if (mode == 2) {
    // ---- pass 1: scatter rows into hash partitions ----
    int64_t total = pend.back();
    // region starts, ends and cursors (= starts): one pinned staging copy
    // into one device block
    int64_t* d_base = (int64_t*)S.get(3 * sizeof(int64_t) * nparts);
    int64_t* d_end = d_base + nparts;
    unsigned long long* d_cur = (unsigned long long*)(d_end + nparts);
    {
      if ((size_t)3 * nparts > kRegionWords) throw Error(ERR_LOGIC, "internal error: too many partitions");
      int64_t* st3 = pinned_regions();
      std::memcpy(st3, pbase.data(), 8 * nparts);
      std::memcpy(st3 + nparts, pend.data(), 8 * nparts);
      std::memcpy(st3 + 2 * nparts, pbase.data(), 8 * nparts);
      ck(cudaMemcpyAsync(d_base, st3, 24 * (size_t)nparts, cudaMemcpyHostToDevice, stream), "h2d");
    }
    PartArgs A;
    std::memset(&A, 0, sizeof(A));
    A.nparts = nparts;
    int lg = 0;
    while ((1 << lg) < nparts) ++lg;
    A.shift = 64 - lg;
    A.base = d_base;
    A.end = d_end;
    A.cursor = d_cur;
    A.keys = (uint64_t*)S.get((size_t)total * 8 * P.key_words);
    bool any_null = false;
    for (int v = 0; v < P.num_vals; ++v) {
      A.vals[v] = S.get((size_t)total * P.vals[v].width);
      any_null |= P.vals[v].mask != nullptr;
    }
    A.bits = any_null ? (uint8_t*)S.get((size_t)total) : nullptr;
    A.counters = counters;
    mark("partition scratch");
    if (opt.profile) ck(cudaEventRecord(events()[0], stream), "event");
    {
      auto launch = [&](auto kern, int nt, int rpt) {
        size_t psmem = part_scatter_smem(P.key_words, nt * rpt, nparts);
        allow_max_smem((const void*)kern);
        int grid = grid_for((const void*)kern, nt, psmem, 0);
        kern<<<grid, nt, psmem, stream>>>(P, A);
      };
      const bool kw1 = P.key_words == 1;
      // 7 (the default): tiles staged by bulk copies when every column allows
      // it; 8: the same with 2048-row tiles, two CTAs per SM
      std::vector<uint8_t> spec(part_scatter_spec_bytes());
      const size_t bsm = opt.scatter >= 7
                           ? part_scatter_bulk_plan(P, nparts, dev.smem_optin, spec.data(), opt.scatter == 8)
                           : 0;
      if (bsm) launch_part_scatter_bulk(P, A, spec.data(), bsm, stream);
      else switch (opt.scatter) {
        case 1: kw1 ? launch(k_part_scatter<1, 16, 256, 3>, 256, 16) : launch(k_part_scatter<2, 16, 256, 3>, 256, 16); break;
        case 2: kw1 ? launch(k_part_scatter<1, 16, 512, 2>, 512, 16) : launch(k_part_scatter<2, 16, 512, 2>, 512, 16); break;
        case 3: kw1 ? launch(k_part_scatter<1, 8, 1024, 1>, 1024, 8) : launch(k_part_scatter<2, 8, 1024, 1>, 1024, 8); break;
        case 4: kw1 ? launch(k_part_scatter<1, 8, 512, 3>, 512, 8) : launch(k_part_scatter<2, 8, 512, 3>, 512, 8); break;
        case 5: kw1 ? launch(k_part_scatter<1, 4, 1024, 2, false>, 1024, 4) : launch(k_part_scatter<2, 4, 1024, 2, false>, 1024, 4); break;
        case 6: kw1 ? launch(k_part_scatter<1, 8, 256, 4>, 256, 8) : launch(k_part_scatter<2, 8, 256, 4>, 256, 8); break;
        default: kw1 ? launch(k_part_scatter<1, 8, 512, 3, false>, 512, 8) : launch(k_part_scatter<2, 8, 512, 2, false>, 512, 8); break;
      }
    }
    ++st.kernels;
    ck(cudaGetLastError(), "partition launch");
    if (opt.profile) ck(cudaEventRecord(events()[4], stream), "event");

    // ---- pass 2: per-partition shared-memory aggregation ----
    Plan P2 = P;
    P2.packed_keys = A.keys;
    for (int v = 0; v < P.num_vals; ++v) {
      P2.vals[v].data = A.vals[v];
      P2.vals[v].mask = nullptr;
      P2.vals[v].offset = 0;
      P2.vals[v].bits = A.bits;
      P2.vals[v].bit = v;
    }
    // pass-2 work: one item per partition, except that a partition holding
    // far more rows than the average (a heavy key) is cut into row ranges
    // handled by several CTAs, each merging its table into the global table
    std::vector<PartItem> items;
    int64_t nsplit = 0;
    int nwagg = 0;  // leading items taken by the warp-combining launch
    {
      int64_t nrows = 0;
      for (auto r : prows) nrows += r;
      // a work item is at most a partition's average share, and small
      // enough that few partitions still spread over every SM
      // (a multiple of 64 rows: pass 2 reads rows in pairs from even starts)
      const int64_t chunk = std::max<int64_t>(
        32768, std::min<int64_t>(nrows / std::max(1, nparts), nrows / (4 * (int64_t)dev.sms))) & ~(int64_t)63;
      for (int p = 0; p < nparts; ++p) {
        const int64_t r = prows[p];
        if (exact_buckets && r > 2 * chunk) {
          ++nsplit;
          for (int64_t b = 0; b < r; b += chunk)
            items.push_back(PartItem{p, 1, pbase[p] + b, pbase[p] + std::min(r, b + chunk)});
        }
      }
      // whole partitions with well over the average rows hold heavy keys:
      // they follow the split items into the warp-combining launch
      const double heavy = opt.wagg_pct / 100.0 * ((double)nrows / std::max(1, nparts));
      for (int pass = 0; pass < 2; ++pass) {
        for (int p = 0; p < nparts; ++p) {
          const int64_t r = prows[p];
          if (exact_buckets && r > 2 * chunk) continue;
          if ((pass == 0) == ((double)r > heavy || opt.wagg_pct == 0)) items.push_back(PartItem{p, 0, pbase[p], pend[p]});
        }
        if (pass == 0) nwagg = (int)items.size();
      }
      // CTAs claim items in order: largest first within each launch, so the
      // launch does not end waiting on one long item taken last
      auto rows_of = [&](const PartItem& it) { return it.merge ? it.end - it.begin : prows[it.part]; };
      auto larger = [&](const PartItem& x, const PartItem& y) { return rows_of(x) > rows_of(y); };
      std::stable_sort(items.begin(), items.begin() + nwagg, larger);
      std::stable_sort(items.begin() + nwagg, items.end(), larger);
    }
    PartItem* d_items = (PartItem*)S.get(sizeof(PartItem) * items.size());
    ck(cudaMemcpyAsync(d_items, items.data(), sizeof(PartItem) * items.size(), cudaMemcpyHostToDevice, stream), "h2d");
    // groups expected to miss their partition's shared table, plus those of
    // split partitions, go to the global spill table
    const double expect_spill = std::max(0.0, (double)est - 0.85 * (double)nparts * sfill2);
    uint64_t spill_cap = next_pow2((uint64_t)std::max<double>(65536.0, 2.0 * expect_spill + 2.0 * (double)nsplit * scap2));
    // spill list: room for the rows of the groups expected to spill
    uint32_t spill_list = (uint32_t)std::min<uint64_t>(
      1ull << 31, next_pow2((uint64_t)std::max<double>(262144.0, 4.0 * expect_spill)));
    int64_t dcap = (int64_t)(est * 1.5) + (int64_t)nparts * 256 + 4096;
    dense_cap = dcap;
    for (int attempt = 0;; ++attempt) {
      T = (uint8_t*)S.get((size_t)(spill_cap + 1) * P.slot_bytes);
      dense = (uint8_t*)S.get((size_t)dcap * P.slot_bytes);
      A.spill_rows = (int64_t*)S.get((size_t)spill_list * sizeof(int64_t));
      A.spill_cap = spill_list;
      k_init_slots<<<dev.sms * 4, 256, 0, stream>>>(T, (int64_t)spill_cap + 1, P.slot_bytes, tmpl);
      ck(cudaMemsetAsync(counters, 0, 16, stream), "memset");
      // [6] dense overflow, [8..9] work, [10..11] dense count, [12] spill list length, [13] list overflow
      ck(cudaMemsetAsync(counters + 6, 0, 8 * 4, stream), "memset");
      G = TableRef{T, spill_cap - 1, P.slot_bytes, P.key_words, counters};
      DenseRef D{dense, dcap, (unsigned long long*)(counters + 10), counters + 6};
      // shared table plus the all-ones key's slot (sorted variants: plus the
      // count arrays and the chunk's sorted stage)
      size_t sm2 = p2_sorted ? part_sorted_smem(P, scap2, p2_rows, any_val_null)
                             : (size_t)(scap2 + 1) * P.slot_bytes;
      // items of split (heavy) partitions first, with rows of one slot
      // combined per warp before their shared update; then the rest
      auto launch2 = [&](auto kern, int nt, int first, int count, unsigned int* work) {
        if (count <= 0) return;
        PartArgs Ai = A;
        Ai.items = d_items + first;
        Ai.nitems = count;
        Ai.work = work;
        allow_max_smem((const void*)kern);
        int grid = grid_for((const void*)kern, nt, sm2, 0);
        grid = std::min(grid, count);
        kern<<<grid, nt, sm2, stream>>>(P2, Ai, G, D, scap2, sfill2, tmpl);
        ++st.kernels;
      };
      auto launch_s = [&](int first, int count, unsigned int* work, bool wagg) {
        if (count <= 0) return;
        PartArgs Ai = A;
        Ai.items = d_items + first;
        Ai.nitems = count;
        Ai.work = work;
        launch_part_sorted(opt.pass2, P2, Ai, G, D, scap2, sfill2, tmpl, sm2, wagg, stream);
        ++st.kernels;
      };
      const bool few = P.num_vals <= 4;
      const int nrest = (int)items.size() - nwagg;
      if (p2_sorted) {
        launch_s(0, nwagg, counters + 8, true);
        launch_s(nwagg, nrest, counters + 9, false);
      } else if (opt.pass2 == 4 && few) {  // 512 threads x 2 rows
        if (P.key_words == 1) {
          launch2(k_part_aggregate<1, 2, 512, 4, true>, 512, 0, nwagg, counters + 8);
          launch2(k_part_aggregate<1, 2, 512, 4, false>, 512, nwagg, nrest, counters + 9);
        } else {
          launch2(k_part_aggregate<2, 2, 512, 4, true>, 512, 0, nwagg, counters + 8);
          launch2(k_part_aggregate<2, 2, 512, 4, false>, 512, nwagg, nrest, counters + 9);
        }
      } else if (P.key_words == 1) {
        if (few) {
          launch2(k_part_aggregate<1, 1, 1024, 4, true>, 1024, 0, nwagg, counters + 8);
          launch2(k_part_aggregate<1, 1, 1024, 4, false>, 1024, nwagg, nrest, counters + 9);
        } else {
          launch2(k_part_aggregate<1, 1, 1024, 8, true>, 1024, 0, nwagg, counters + 8);
          launch2(k_part_aggregate<1, 1, 1024, 8, false>, 1024, nwagg, nrest, counters + 9);
        }
      } else {
        if (few) {
          launch2(k_part_aggregate<2, 1, 1024, 4, true>, 1024, 0, nwagg, counters + 8);
          launch2(k_part_aggregate<2, 1, 1024, 4, false>, 1024, nwagg, nrest, counters + 9);
        } else {
          launch2(k_part_aggregate<2, 1, 1024, 8, true>, 1024, 0, nwagg, counters + 8);
          launch2(k_part_aggregate<2, 1, 1024, 8, false>, 1024, nwagg, nrest, counters + 9);
        }
      }
      if (opt.profile) ck(cudaEventRecord(events()[1], stream), "event");
      // rows listed as not fitting their partition's table (none when the
      // sample sized the partitions well): one grid-stride launch that reads
      // the list length on the device
      k_part_spill<false><<<dev.sms * 2, 256, 0, stream>>>(P2, G, A);
      k_finish_count<<<1, 1, 0, stream>>>(P, G);
      st.kernels += 3;
      ck(cudaGetLastError(), "partition aggregate launch");
      if (deferred) {
        // counts and flags stay on the device until the compaction is done
        mark("partition passes launched");
        done = true;
        dense_n = -1;
        cap = spill_cap;
        prof_part = opt.profile;
        break;
      }
      ck(cudaMemcpyAsync(host, counters, 64, cudaMemcpyDeviceToHost, stream), "d2h");
      ck(cudaStreamSynchronize(stream), "partition sync");
      if (opt.profile && attempt == 0) {
        float ms = 0, ms1 = 0;
        ck(cudaEventElapsedTime(&ms, events()[0], events()[1]), "event time");
        ck(cudaEventElapsedTime(&ms1, events()[0], events()[4]), "event time");
        st.agg_kernel_ms += ms;
        st.scatter_ms = ms1;
      }
      mark("partition passes (synced)");
      if (host[14]) throw Error(ERR_CUDA, "partition pass: a bulk copy did not complete in time");
      if (host[5]) break;  // a region overflowed: fall back to the global table
      if (host[1] == 0 && host[6] == 0 && host[13] == 0) {
        done = true;
        dense_n = (int64_t)(host[10] | ((uint64_t)host[11] << 32));
        cap = spill_cap;
        break;
      }
      if (attempt >= 6) throw Error(ERR_CUDA, "hash table overflow");
      if (host[1]) spill_cap *= 8;
      if (host[6]) dcap *= 2;
      if (host[13]) {
        spill_list = (uint32_t)std::min<uint64_t>((uint64_t)spill_list * 8, 1ull << 31);
        spill_cap = std::max<uint64_t>(spill_cap, next_pow2((uint64_t)host[12] * 2));
      }
      S.put(T);
      S.put(dense);
      S.put(A.spill_rows);
      ++st.retries;
    }
    if (!done) {
      mode = 0;
      st.mode = 0;
      ++st.retries;
      S.put(T);
      S.put(dense);
      S.put(A.spill_rows);
      dense = nullptr;
    }
  }

  // shared stage through the row-range kernel: plans whose columns all have
  // closed-form updates and whose groups fit one CTA's ~220 KB table
  bool raw_stage = mode == 1 && part_ok && opt.block >= 512 && !(opt.set_mask & (OPT_SMEM | OPT_FILL)) &&
                   est <= (int64_t)(0.7 * sfill2);
  std::vector<PartItem> raw_items;
  PartItem* d_raw_items = nullptr;
  int64_t* d_raw_spill = nullptr;
  const uint32_t raw_spill_cap = 1u << 16;
  if (!done && raw_stage) {
    // one row range per CTA for small inputs (each range pays a table reset
    // and a merge), four per SM for large ones
    const int64_t per_cta = (n + dev.sms - 1) / dev.sms;
    const int64_t chunk = per_cta < 4 * 32768 ? per_cta : std::max<int64_t>(32768, (n + 4 * dev.sms - 1) / (4 * dev.sms));
    for (int64_t b = 0; b < n; b += chunk) raw_items.push_back(PartItem{0, 1, b, std::min(n, b + chunk)});
    d_raw_items = (PartItem*)S.get(sizeof(PartItem) * raw_items.size());
    ck(cudaMemcpyAsync(d_raw_items, raw_items.data(), sizeof(PartItem) * raw_items.size(), cudaMemcpyHostToDevice,
                       stream), "h2d");
    d_raw_spill = (int64_t*)S.get(sizeof(int64_t) * raw_spill_cap);
  }

  if (!done) {
    for (int attempt = 0;; ++attempt) {
      size_t tbytes = (size_t)(cap + 1) * P.slot_bytes;
      T = (uint8_t*)S.get(tbytes);
      k_init_slots<<<dev.sms * 8, 256, 0, stream>>>(T, (int64_t)cap + 1, P.slot_bytes, tmpl);
      ck(cudaMemsetAsync(counters, 0, 16, stream), "memset counters");
      G = TableRef{T, cap - 1, P.slot_bytes, P.key_words, counters};
      int block = std::min(opt.block, 512);
      if (opt.profile) ck(cudaEventRecord(events()[0], stream), "event");
      if (raw_stage) {
        ck(cudaMemsetAsync(counters + 8, 0, 6 * 4, stream), "memset");  // [8] work, [12..13] spill list
        PartArgs A;
        std::memset(&A, 0, sizeof(A));
        A.counters = counters;
        A.items = d_raw_items;
        A.nitems = (int)raw_items.size();
        A.work = counters + 8;
        A.spill_rows = d_raw_spill;
        A.spill_cap = raw_spill_cap;
        DenseRef D{nullptr, 0, (unsigned long long*)(counters + 10), counters + 6};
        const size_t sm2 = (size_t)(scap2 + 1) * P.slot_bytes;
        auto launch_raw = [&](auto kern) {
          allow_max_smem((const void*)kern);
          int grid = grid_for((const void*)kern, 1024, sm2, 0);
          grid = std::min(grid, A.nitems);
          kern<<<grid, 1024, sm2, stream>>>(P, A, G, D, scap2, sfill2, tmpl);
        };
        const bool few = P.num_vals <= 4;
        if (P.key_words == 1) few ? launch_raw(k_part_aggregate<1, 1, 1024, 4, true, true>)
                                  : launch_raw(k_part_aggregate<1, 1, 1024, 8, true, true>);
        else few ? launch_raw(k_part_aggregate<2, 1, 1024, 4, true, true>)
                 : launch_raw(k_part_aggregate<2, 1, 1024, 8, true, true>);
        k_part_spill<true><<<dev.sms * 2, 256, 0, stream>>>(P, G, A);
        st.kernels += 2;
      } else if (mode == 1) {
        size_t sm = (size_t)scap * P.slot_bytes;
        allow_max_smem((const void*)k_aggregate<true>);
        int grid = grid_for((const void*)k_aggregate<true>, block, sm, opt.blocks_per_sm);
        grid = (int)std::min<int64_t>(grid, (n + block - 1) / block);
        k_aggregate<true><<<grid, block, sm, stream>>>(P, G, scap, sfill, tmpl);
      } else {
        int grid = grid_for((const void*)k_aggregate<false>, block, 0, opt.blocks_per_sm);
        grid = (int)std::min<int64_t>(grid, (n + block - 1) / block);
        k_aggregate<false><<<grid, block, 0, stream>>>(P, G, 1, 0, tmpl);
      }
      if (opt.profile) ck(cudaEventRecord(events()[1], stream), "event");
      k_finish_count<<<1, 1, 0, stream>>>(P, G);
      st.kernels += 3;
      ck(cudaGetLastError(), "aggregate launch");
      if (deferred) {
        prof_agg = opt.profile;
        break;
      }
      ck(cudaMemcpyAsync(host, counters, 64, cudaMemcpyDeviceToHost, stream), "count d2h");
      ck(cudaStreamSynchronize(stream), "aggregate sync");
      if (raw_stage && host[13]) {
        // more groups than the tables held: redo through the per-row kernel
        raw_stage = false;
        host[1] = 1;
      }
      if (opt.profile) {
        float ms = 0;
        ck(cudaEventElapsedTime(&ms, events()[0], events()[1]), "event time");
        st.agg_kernel_ms += ms;
      }
      if (host[1] == 0) break;
      // table overflow: the kernel stopped inserting; redo with a larger table
      if (attempt >= 6) throw Error(ERR_CUDA, "hash table overflow");
      S.put(T);
      cap *= 4;
      ++st.retries;
    }
  }
  st.capacity = (int64_t)cap;
  mark("aggregate done");
  mark("outputs");
  // deferred: outputs are sized for every slot that could hold a group
  int64_t G_n = deferred ? -1 : (int64_t)host[0] + dense_n;
  const int64_t out_rows = deferred ? (dense ? dense_cap : 0) + (int64_t)cap + 1 : G_n;
  R.num_groups = G_n;

  if (P.need_second_pass) {
    int grid = grid_for((const void*)k_var_pass, 256, 0, 0);
    k_var_pass<<<grid, 256, 0, stream>>>(P, G);
    ++st.kernels;
    ck(cudaGetLastError(), "variance pass launch");
  }

  // ---- outputs ----
  try {
    OutPtrs O;
    std::memset(&O, 0, sizeof(O));
    for (int k = 0; k < P.num_keys; ++k) {
      R.keys.push_back(make_out(alloc, stream, keys[k].type_id, out_rows, keys[k].mask != nullptr));
      O.key_data[k] = R.keys.back().data;
      O.key_mask[k] = R.keys.back().mask;
    }
    {
      int j = 0;
      for (auto& r : reqs) {
        std::vector<OutColumn> cols;
        for (size_t a = 0; a < r.aggs.size(); ++a, ++j) {
          cols.push_back(make_out(alloc, stream, out_types[j], out_rows, P.outs[j].nullable));
          O.out_data[j] = cols.back().data;
          O.out_mask[j] = cols.back().mask;
        }
        R.results.push_back(cols);
      }
    }
    // position and null counters of the compaction, apart from the
    // aggregation's counts and flags in counters[0, 16)
    unsigned int* ccount = counters + 256;
    uint32_t* chost = host + 256;
    O.counters = ccount;
    ck(cudaMemsetAsync(ccount, 0, 512, stream), "memset");
    if (opt.profile) ck(cudaEventRecord(events()[2], stream), "event");
    const int64_t limit = deferred ? out_rows : G_n;
    if (deferred && dense) {
      int grid = (int)std::min<int64_t>((dense_cap + 255) / 256, (int64_t)dev.sms * 8);
      k_compact<<<grid, 256, 0, stream>>>(P, dense, dense_cap, P.slot_bytes, limit, 1, O,
                                          (const unsigned long long*)(counters + 10));
      ++st.kernels;
    } else if (dense_n > 0) {
      int grid = (int)std::min<int64_t>((dense_n + 255) / 256, (int64_t)dev.sms * 8);
      k_compact<<<grid, 256, 0, stream>>>(P, dense, dense_n, P.slot_bytes, limit, 1, O);
      ++st.kernels;
    }
    if (deferred || G_n > dense_n) {
      int64_t nslots = (int64_t)cap + 1;
      int grid = (int)std::min<int64_t>((nslots + 255) / 256, (int64_t)dev.sms * 8);
      k_compact<<<grid, 256, 0, stream>>>(P, T, nslots, P.slot_bytes, limit, 0, O);
      ++st.kernels;
    }
    if (opt.profile) ck(cudaEventRecord(events()[3], stream), "event");
    ck(cudaGetLastError(), "compact launch");
    if (deferred) ck(cudaMemcpyAsync(host, counters, 64, cudaMemcpyDeviceToHost, stream), "counts d2h");
    ck(cudaMemcpyAsync(chost, ccount, 4 * (4 + P.num_keys + P.num_outs), cudaMemcpyDeviceToHost, stream),
       "null counts d2h");
    ck(cudaStreamSynchronize(stream), "compact sync");
    mark("compaction (synced)");
    if (deferred) {
      if (host[14]) throw Error(ERR_CUDA, "partition pass: a bulk copy did not complete in time");
      // an overflow anywhere (a table, a region, the dense slots, a spill
      // list): redo the call with checks after every stage
      const bool again = host[1] || chost[1] || (mode == 2 && (host[5] || host[6] || host[13])) ||
                         (raw_stage && host[13]);
      if (again) {
        R.release();
        Options o2 = opt_in;
        o2.sync_checks = 1;
        return aggregate(keys, null_policy, reqs, stream, alloc, o2, stats);
      }
      const int64_t dn = mode == 2 ? (int64_t)(host[10] | ((uint64_t)host[11] << 32)) : 0;
      G_n = (int64_t)chost[2];
      if (G_n != (int64_t)host[0] + dn)
        throw Error(ERR_CUDA, "internal error: compaction wrote " + std::to_string(G_n) + " groups of " +
                                  std::to_string((int64_t)host[0] + dn));
      R.num_groups = G_n;
      for (auto& c : R.keys) c.size = G_n;
      for (auto& cols : R.results)
        for (auto& c : cols) c.size = G_n;
      if (prof_part || prof_agg) {
        float ms = 0, ms1 = 0;
        ck(cudaEventElapsedTime(&ms, events()[0], events()[1]), "event time");
        st.agg_kernel_ms += ms;
        if (prof_part) {
          ck(cudaEventElapsedTime(&ms1, events()[0], events()[4]), "event time");
          st.scatter_ms = ms1;
        }
      }
    } else if (chost[1]) {
      throw Error(ERR_CUDA, "internal error: compaction found more groups than were counted");
    }
    if (opt.profile) {
      float ms = 0;
      ck(cudaEventElapsedTime(&ms, events()[2], events()[3]), "event time");
      st.compact_ms = ms;
    }
    for (int k = 0; k < P.num_keys; ++k) R.keys[k].null_count = chost[4 + k];
    int j = 0;
    for (auto& cols : R.results)
      for (auto& c : cols) c.null_count = chost[4 + P.num_keys + j++];
  } catch (...) {
    R.release();
    throw;
  }
  if (stats) *stats = st;
  return R;
}

}  // namespace gb

namespace gb {

// Global-table aggregation whose hash table and counters live in `scratch`
// (caller-owned device memory) and whose results go to caller-owned columns:
// the path makes no device or pinned-host allocation.  Counters are read back
// with pageable copies.  Returns the number of groups.
int64_t aggregate_into_scratch(const std::vector<Column>& keys, int null_policy,
                               const std::vector<Request>& reqs, cudaStream_t stream, void* scratch,
                               size_t scratch_bytes, int64_t max_groups,
                               std::vector<OutColumn>& out_keys, std::vector<OutColumn>& out_results)
{
  Plan P;
  std::vector<int> out_types;
  build_plan(keys, null_policy, reqs, P, out_types);
  if (max_groups < 0) throw Error(ERR_LOGIC, "max_groups must be >= 0");
  if (out_keys.size() != (size_t)P.num_keys || out_results.size() != (size_t)P.num_outs)
    throw Error(ERR_LOGIC, "output column count does not match the keys and requests");
  for (int k = 0; k < P.num_keys; ++k) {
    OutColumn& o = out_keys[k];
    o.type_id = keys[k].type_id;
    if (max_groups > 0 && !o.data) throw Error(ERR_LOGIC, "output key column without a data buffer");
    if (keys[k].mask && max_groups > 0 && !o.mask) throw Error(ERR_LOGIC, "nullable output key column without a mask buffer");
    if (!keys[k].mask) o.mask = nullptr;
  }
  for (int j = 0; j < P.num_outs; ++j) {
    OutColumn& o = out_results[j];
    o.type_id = out_types[j];
    if (max_groups > 0 && !o.data) throw Error(ERR_LOGIC, "output result column without a data buffer");
    if (P.outs[j].nullable && max_groups > 0 && !o.mask) throw Error(ERR_LOGIC, "nullable output result column without a mask buffer");
    if (!P.outs[j].nullable) o.mask = nullptr;
  }
  const int64_t n = P.num_rows;
  const uint64_t cap = next_pow2((uint64_t)std::max<int64_t>(64, 2 * max_groups));
  const size_t need = 4096 + (size_t)(cap + 1) * P.slot_bytes;
  if (need > scratch_bytes)
    throw Error(ERR_LOGIC, "max_groups " + std::to_string(max_groups) + " with this plan's " +
                               std::to_string(P.slot_bytes) + "-byte slots needs " + std::to_string(need) +
                               " bytes of table; the allocation-free entry point has " +
                               std::to_string(scratch_bytes));
  unsigned int* counters = (unsigned int*)scratch;
  uint8_t* T = (uint8_t*)scratch + 4096;
  ck(cudaMemsetAsync(counters, 0, 4096, stream), "memset counters");
  for (int k = 0; k < P.num_keys; ++k)
    if (out_keys[k].mask && max_groups > 0)
      ck(cudaMemsetAsync(out_keys[k].mask, 0, (size_t)((max_groups + 31) / 32) * 4, stream), "memset mask");
  for (int j = 0; j < P.num_outs; ++j)
    if (out_results[j].mask && max_groups > 0)
      ck(cudaMemsetAsync(out_results[j].mask, 0, (size_t)((max_groups + 31) / 32) * 4, stream), "memset mask");
  uint32_t host[4 + kMaxKeyCols + kMaxOutputs];
  std::memset(host, 0, sizeof(host));
  if (n > 0) {
    DevInfo dev = dev_info();
    SlotTemplate tmpl;
    build_template(P, tmpl);
    k_init_slots<<<dev.sms * 4, 256, 0, stream>>>(T, (int64_t)cap + 1, P.slot_bytes, tmpl);
    TableRef G{T, cap - 1, P.slot_bytes, P.key_words, counters};
    int grid = grid_for((const void*)k_aggregate<false>, 512, 0, 0);
    grid = (int)std::min<int64_t>(grid, (n + 511) / 512);
    k_aggregate<false><<<grid, 512, 0, stream>>>(P, G, 1, 0, tmpl);
    k_finish_count<<<1, 1, 0, stream>>>(P, G);
    ck(cudaGetLastError(), "aggregate launch");
    ck(cudaMemcpyAsync(host, counters, 8, cudaMemcpyDeviceToHost, stream), "count d2h");
    ck(cudaStreamSynchronize(stream), "aggregate sync");
    if (host[1]) throw Error(ERR_LOGIC, "more groups than max_groups (table full)");
    if ((int64_t)host[0] > max_groups)
      throw Error(ERR_LOGIC, "more groups (" + std::to_string(host[0]) + ") than max_groups (" +
                                 std::to_string(max_groups) + ")");
    const int64_t G_n = host[0];
    if (P.need_second_pass) {
      int g2 = grid_for((const void*)k_var_pass, 256, 0, 0);
      k_var_pass<<<g2, 256, 0, stream>>>(P, G);
    }
    OutPtrs O;
    std::memset(&O, 0, sizeof(O));
    for (int k = 0; k < P.num_keys; ++k) {
      O.key_data[k] = out_keys[k].data;
      O.key_mask[k] = out_keys[k].mask;
    }
    for (int j = 0; j < P.num_outs; ++j) {
      O.out_data[j] = out_results[j].data;
      O.out_mask[j] = out_results[j].mask;
    }
    O.counters = counters;
    ck(cudaMemsetAsync(counters, 0, 512, stream), "memset");
    if (G_n > 0) {
      int64_t nslots = (int64_t)cap + 1;
      int g3 = (int)std::min<int64_t>((nslots + 255) / 256, (int64_t)dev.sms * 8);
      k_compact<<<g3, 256, 0, stream>>>(P, T, nslots, P.slot_bytes, G_n, 0, O);
    }
    ck(cudaGetLastError(), "compact launch");
    ck(cudaMemcpyAsync(host, counters, 4 * (4 + P.num_keys + P.num_outs), cudaMemcpyDeviceToHost, stream),
       "null counts d2h");
    ck(cudaStreamSynchronize(stream), "compact sync");
    if (host[1]) throw Error(ERR_CUDA, "internal error: compaction found more groups than were counted");
    host[0] = (uint32_t)G_n;
  } else {
    ck(cudaStreamSynchronize(stream), "sync");
  }
  const int64_t groups = n > 0 ? (int64_t)host[0] : 0;
  for (int k = 0; k < P.num_keys; ++k) {
    out_keys[k].size = groups;
    out_keys[k].null_count = n > 0 ? host[4 + k] : 0;
  }
  for (int j = 0; j < P.num_outs; ++j) {
    out_results[j].size = groups;
    out_results[j].null_count = n > 0 ? host[4 + P.num_keys + j] : 0;
  }
  return groups;
}

}  // namespace gb
