// gb_sorted.cuh -- pass 2 of the partitioned path, sorted-chunk variant.
//
// The shared-memory table holds one partition's groups.  Rows are taken in
// chunks of R*NT; each chunk is counting-sorted by table slot in shared memory,
// so that the rows of one slot sit next to each other, and each run of equal
// slots is then reduced in registers by ONE thread and written back to its slot
// with plain shared loads and stores:
//
//   P1  keys (loaded a chunk ahead, 128-bit vector loads, two rows a load)
//       are placed in the table; rank within the slot = native u32 shared
//       atomicAdd on the chunk's per-slot count (warp-aggregated for items of
//       heavy partitions, where one key fills whole warps)
//   P2  exclusive scan of the counts -> start of every slot's run
//   P3  each row's values, validity byte and slot are stored at their sorted
//       position (values loaded with 128-bit vector loads while P1/P2 ran)
//   P4  thread t owns the runs that start in positions [t*R, t*R+R): it reduces
//       each in registers and updates the slot with plain ld/st.shared (it is
//       the slot's only writer in this chunk).  A run longer than L is cut at
//       the thread ranges instead; its pieces are combined across the lanes of
//       a warp with shuffles and the warp's sum goes in with one shared
//       reduction per field.
//
// Against per-row shared reductions (compare-and-swap loops for 64-bit and
// floating-point fields on this architecture, ~15 instructions each) the
// per-row cost becomes one register operation per field, and the per-slot
// write-back is amortised over the run.
#pragma once
#include "gb_partition.cuh"
#include "gb_sorted.h"

namespace gb {

// Slot index of a key in the shared table (any slot count; multiply-shift
// start slot), inserting it if absent.  Returns scap for the all-ones key of a
// one-word table, -1 when the key does not fit (table at its fill limit or 64
// probes).
__device__ __forceinline__ int smem_index(uint8_t* smem, int stride, uint32_t scap, int sfill,
                                          unsigned int* s_used, int words, uint64_t w0, uint64_t w1,
                                          uint64_t h)
{
  uint32_t i = (uint32_t)(((uint64_t)(uint32_t)h * scap) >> 32);
  if (words == 1) {
    if (w0 == kEmpty) return (int)scap;
    for (int p = 0; p < 64; ++p) {
      unsigned long long* kp = (unsigned long long*)(smem + (size_t)i * stride);
      const uint64_t cur = *(volatile unsigned long long*)kp;
      if (cur == w0) return (int)i;
      if (cur == kEmpty) {
        if (*(volatile unsigned int*)s_used >= (unsigned)sfill) return -1;
        const uint64_t old = atomicCAS(kp, kEmpty, w0);
        if (old == kEmpty) {
          atomicAdd(s_used, 1u);
          return (int)i;
        }
        if (old == w0) return (int)i;
      }
      i = i + 1 == scap ? 0 : i + 1;
    }
    return -1;
  }
  const unsigned __int128 want = ((unsigned __int128)w1 << 64) | w0;
  const unsigned __int128 empty = ~(unsigned __int128)0;
  for (int p = 0; p < 64; ++p) {
    unsigned __int128* kp = (unsigned __int128*)(smem + (size_t)i * stride);
    const ulonglong2 cur = vload2(kp);
    if (cur.x == w0 && cur.y == w1 && w0 != kEmpty) return (int)i;
    if ((cur.y >> 63) || cur.x == kEmpty) {
      if ((cur.y >> 63) && *(volatile unsigned int*)s_used >= (unsigned)sfill) return -1;
      const unsigned __int128 old = atomicCAS(kp, empty, want);
      if (old == empty) {
        atomicAdd(s_used, 1u);
        return (int)i;
      }
      if (old == want) return (int)i;
    }
    i = i + 1 == scap ? 0 : i + 1;
  }
  return -1;
}

// Two rows (r, r+1; r even) of a column of width W: 16-, 8-, 4- or 2-byte load.
template <int W>
__device__ __forceinline__ void load_pair(const void* base, int64_t r, uint64_t& x0, uint64_t& x1)
{
  if (W == 8) {
    const ulonglong2 v = __ldg((const ulonglong2*)((const unsigned long long*)base + r));
    x0 = v.x;
    x1 = v.y;
  } else if (W == 4) {
    const uint2 v = __ldg((const uint2*)((const uint32_t*)base + r));
    x0 = v.x;
    x1 = v.y;
  } else if (W == 2) {
    const uint32_t v = __ldg((const uint32_t*)((const uint16_t*)base + r));
    x0 = v & 0xFFFFu;
    x1 = v >> 16;
  } else {
    const uint32_t v = __ldg((const uint16_t*)((const uint8_t*)base + r));
    x0 = v & 0xFFu;
    x1 = v >> 8;
  }
}
__device__ __forceinline__ void load_pair_w(const void* base, int64_t r, int w, uint64_t& x0, uint64_t& x1)
{
  switch (w) {
    case 8: load_pair<8>(base, r, x0, x1); break;
    case 4: load_pair<4>(base, r, x0, x1); break;
    case 2: load_pair<2>(base, r, x0, x1); break;
    default: load_pair<1>(base, r, x0, x1); break;
  }
}

// Register accumulators of one run of one column.
template <int CAT, int W>
struct RunAcc {
  using S = typename std::conditional<CAT == CAT_F64, double, typename std::conditional<CAT == CAT_F32, float, uint64_t>::type>::type;
  S sum, sq;
  // floats: native min/max started from NaN (fmin/fmax skip NaN, and a run
  // of NaNs only stays NaN, which is the slot encoding's rule too); integers:
  // min/max of the value (signed or unsigned), from the type's extremes
  S mn, mx;
  uint32_t nvalid;
  __device__ __forceinline__ void init()
  {
    nvalid = 0;
    if (CAT == CAT_F64 || CAT == CAT_F32) {
      sum = 0;
      sq = 0;
      mn = (S)__int_as_float(0x7FC00000);
      mx = mn;
    } else {
      sum = 0;
      sq = 0;
      if (CAT == CAT_SIGNED) {
        mn = (S)0x7FFFFFFFFFFFFFFFull;
        mx = (S)0x8000000000000000ull;
      } else {
        mn = (S)~0ull;
        mx = 0;
      }
    }
  }
  // x: staged bits of a valid element
  __device__ __forceinline__ void add(uint64_t x)
  {
    ++nvalid;
    if (CAT == CAT_F64) {
      const double d = __longlong_as_double((long long)x);
      sum += d;
      sq += d * d;
      mn = fmin(mn, d);
      mx = fmax(mx, d);
    } else if (CAT == CAT_F32) {
      const float f = __uint_as_float((uint32_t)x);
      sum += f;
      sq += f * f;
      mn = fminf(mn, f);
      mx = fmaxf(mx, f);
    } else {
      int64_t iv;
      if (CAT == CAT_SIGNED) iv = W == 8 ? (int64_t)x : W == 4 ? (int64_t)(int32_t)x : W == 2 ? (int64_t)(int16_t)x
                                                                                     : (int64_t)(int8_t)x;
      else if (CAT == CAT_BOOL) iv = x != 0;
      else iv = (int64_t)x;
      sum += (uint64_t)iv;
      sq += (uint64_t)iv * (uint64_t)iv;
      if (CAT == CAT_SIGNED) {
        mn = (uint64_t)min((long long)mn, (long long)iv);
        mx = (uint64_t)max((long long)mx, (long long)iv);
      } else {
        mn = min((unsigned long long)mn, (unsigned long long)iv);
        mx = max((unsigned long long)mx, (unsigned long long)iv);
      }
    }
  }
  // order-preserving encodings of the slot's MIN/MAX fields; a run without
  // valid values gives the field's identity (all ones for MIN, zero for MAX:
  // the register extremes of a narrow signed type would truncate to real
  // encodings)
  __device__ __forceinline__ uint64_t enc_min() const
  {
    if (nvalid == 0) return W == 8 ? ~0ull : 0xFFFFFFFFull;
    if (CAT == CAT_F64) return ord64_f(mn, true);
    if (CAT == CAT_F32) return ord32_f(mn, true);
    if (CAT == CAT_SIGNED) return W == 8 ? ((uint64_t)mn ^ 0x8000000000000000ull) : ((uint32_t)(int32_t)(int64_t)mn ^ 0x80000000u);
    return W == 8 ? (uint64_t)mn : (uint32_t)mn;
  }
  __device__ __forceinline__ uint64_t enc_max() const
  {
    if (nvalid == 0) return 0;
    if (CAT == CAT_F64) return ord64_f(mx, false);
    if (CAT == CAT_F32) return ord32_f(mx, false);
    if (CAT == CAT_SIGNED) return W == 8 ? ((uint64_t)mx ^ 0x8000000000000000ull) : ((uint32_t)(int32_t)(int64_t)mx ^ 0x80000000u);
    return W == 8 ? (uint64_t)mx : (uint32_t)mx;
  }
};

// MIN/MAX fields are 8 bytes for 8-byte columns (and f64), 4 otherwise.
template <int CAT, int W>
__device__ __forceinline__ constexpr bool wide_minmax() { return W == 8; }

// Plain update of a slot by its only writer in this chunk.
template <int CAT, int W>
__device__ __forceinline__ void flush_plain(uint8_t* slot, const ValCol& c, const RunAcc<CAT, W>& a, uint32_t nulls)
{
  if (nulls && c.nulls_off >= 0) *(uint32_t*)(slot + c.nulls_off) += nulls;
  if (a.nvalid == 0) return;
  if (c.sum_off >= 0) {
    if (CAT == CAT_F64) *(double*)(slot + c.sum_off) += (double)a.sum;
    else if (CAT == CAT_F32) *(float*)(slot + c.sum_off) += (float)a.sum;
    else if (c.sum_op == OP_SUM_I32) *(uint32_t*)(slot + c.sum_off) += (uint32_t)(uint64_t)a.sum;
    else *(uint64_t*)(slot + c.sum_off) += (uint64_t)a.sum;
  }
  if (c.sq_off >= 0) {
    if (CAT == CAT_F64) *(double*)(slot + c.sq_off) += (double)a.sq;
    else if (CAT == CAT_F32) *(float*)(slot + c.sq_off) += (float)a.sq;
    else *(uint64_t*)(slot + c.sq_off) += (uint64_t)a.sq;
  }
  if (wide_minmax<CAT, W>()) {
    if (c.min_off >= 0) {
      uint64_t* p = (uint64_t*)(slot + c.min_off);
      const uint64_t e = a.enc_min();
      if (e < *p) *p = e;
    }
    if (c.max_off >= 0) {
      uint64_t* p = (uint64_t*)(slot + c.max_off);
      const uint64_t e = a.enc_max();
      if (e > *p) *p = e;
    }
  } else {
    if (c.min_off >= 0) {
      uint32_t* p = (uint32_t*)(slot + c.min_off);
      const uint32_t e = (uint32_t)a.enc_min();
      if (e < *p) *p = e;
    }
    if (c.max_off >= 0) {
      uint32_t* p = (uint32_t*)(slot + c.max_off);
      const uint32_t e = (uint32_t)a.enc_max();
      if (e > *p) *p = e;
    }
  }
}

// Shared reductions of a piece of a long run (several threads update the slot).
template <int CAT, int W>
__device__ __forceinline__ void flush_atomic(uint32_t sa, const ValCol& c, uint64_t sum, uint64_t sq, uint64_t emn,
                                             uint64_t emx, uint32_t nvalid)
{
  if (nvalid == 0) return;
  if (c.sum_off >= 0) {
    if (CAT == CAT_F64) sred_add_f64(sa + c.sum_off, __longlong_as_double((long long)sum));
    else if (CAT == CAT_F32) sred_add_f32(sa + c.sum_off, __uint_as_float((uint32_t)sum));
    else if (c.sum_op == OP_SUM_I32) sred_add_u32(sa + c.sum_off, (uint32_t)sum);
    else sred_add_u64(sa + c.sum_off, sum);
  }
  if (c.sq_off >= 0) {
    if (CAT == CAT_F64) sred_add_f64(sa + c.sq_off, __longlong_as_double((long long)sq));
    else if (CAT == CAT_F32) sred_add_f32(sa + c.sq_off, __uint_as_float((uint32_t)sq));
    else sred_add_u64(sa + c.sq_off, sq);
  }
  if (wide_minmax<CAT, W>()) {
    if (c.min_off >= 0) sred_min_u64(sa + c.min_off, emn);
    if (c.max_off >= 0) sred_max_u64(sa + c.max_off, emx);
  } else {
    if (c.min_off >= 0) sred_min_u32(sa + c.min_off, (uint32_t)emn);
    if (c.max_off >= 0) sred_max_u32(sa + c.max_off, (uint32_t)emx);
  }
}

// Bits of a register sum for shuffling (floats as their bit patterns).
template <int CAT, int W>
__device__ __forceinline__ uint64_t sum_bits(typename RunAcc<CAT, W>::S s)
{
  if (CAT == CAT_F64) return (uint64_t)__double_as_longlong((double)s);
  if (CAT == CAT_F32) return __float_as_uint((float)s);
  return (uint64_t)s;
}

// Where sorted position p of a chunk of R*NT rows is stored in the stage
// arrays: thread-major (p % R) * NT + p / R, so that when thread t walks its
// positions t*R .. t*R+R-1 the lanes of a warp touch consecutive elements
// (no bank conflicts) instead of elements R apart.
template <int R, int NT>
__device__ __forceinline__ int stage_at(int p)
{
  return (p & (R - 1)) * NT + (p / R);
}

// The runs of thread t's positions [a, b) in the sorted chunk.  `cur` holds
// the start of every slot's run (cur[s+1] is where run s ends).  Calls
// fn(pos, len, slot, piece): a light run (at most L rows) whose start lies in
// [a, b) is visited whole (piece = false; this thread is its only writer);
// a heavy run is visited as its part inside [a, b) (piece = true).
template <int R, int NT, typename F>
__device__ __forceinline__ void for_runs(const uint16_t* sslot, const uint32_t* cur, int a, int b, int L, F fn)
{
  int p = a;
  if (p < b) {
    const int s = sslot[stage_at<R, NT>(p)];
    const int rs = (int)cur[s], re = (int)cur[s + 1];
    if (rs < a) {
      if (re - rs > L) {
        const int e = min(b, re);
        fn(p, e - p, s, true);
      }
      p = re;  // a light run is its starting thread's
    }
  }
  while (p < b) {
    const int s = sslot[stage_at<R, NT>(p)];
    const int re = (int)cur[s + 1];
    if (re - p <= L) {
      fn(p, re - p, s, false);
      p = re;
    } else {
      const int e = min(b, re);
      fn(p, e - p, s, true);
      p = e;
    }
  }
}

// P4 for one value column of type (CAT, W).
template <int CAT, int W, int R, int NT>
__device__ __forceinline__ void sorted_column(const ValCol& c, int v, uint8_t* table, uint32_t tbase, int stride,
                                              const uint16_t* sslot, const uint8_t* sbits, const uint8_t* stage,
                                              const uint32_t* cur, int a, int b, int L)
{
  using Acc = RunAcc<CAT, W>;
  constexpr int SW = W == 8 ? 8 : 4;
  // pieces of heavy runs: at most one starting before a (the first) and one
  // starting inside [a, b) (the last); their partials go through the warp
  uint64_t hsum = 0, hsq = 0, hmn = 0, hmx = 0;
  uint32_t hn = 0, hnull = 0;
  int hslot = -1;
  uint64_t tsum = 0, tsq = 0, tmn = 0, tmx = 0;
  uint32_t tn = 0, tnull = 0;
  int tslot = -1;
  for_runs<R, NT>(sslot, cur, a, b, L, [&](int pos, int len, int s, bool piece) {
    Acc acc;
    acc.init();
    uint32_t nulls = 0;
    for (int p = pos; p < pos + len; ++p) {
      const int q = stage_at<R, NT>(p);
      const bool valid = sbits == nullptr || ((sbits[q] >> v) & 1);
      const uint64_t x = SW == 8 ? ((const uint64_t*)stage)[q] : ((const uint32_t*)stage)[q];
      if (valid) acc.add(x);
      else ++nulls;
    }
    if (!piece) {
      flush_plain<CAT, W>(table + (size_t)s * stride, c, acc, nulls);
    } else if (pos == a && (int)cur[s] < a) {
      hslot = s;
      hsum = sum_bits<CAT, W>(acc.sum);
      hsq = sum_bits<CAT, W>(acc.sq);
      hmn = acc.enc_min();
      hmx = acc.enc_max();
      hn = acc.nvalid;
      hnull = nulls;
    } else {
      tslot = s;
      tsum = sum_bits<CAT, W>(acc.sum);
      tsq = sum_bits<CAT, W>(acc.sq);
      tmn = acc.enc_min();
      tmx = acc.enc_max();
      tn = acc.nvalid;
      tnull = nulls;
    }
  });
  // heavy pieces: lanes holding pieces of one run combine them, the group's
  // lowest lane applies the result (two rounds: first pieces, last pieces)
  const int lane = threadIdx.x & 31;
  const unsigned full = 0xFFFFFFFFu;
#pragma unroll
  for (int round = 0; round < 2; ++round) {
    const int s = round == 0 ? hslot : tslot;
    if (!__any_sync(full, s >= 0)) continue;
    uint64_t sum = round == 0 ? hsum : tsum, sq = round == 0 ? hsq : tsq;
    uint64_t mn = round == 0 ? hmn : tmn, mx = round == 0 ? hmx : tmx;
    uint32_t n = round == 0 ? hn : tn, nul = round == 0 ? hnull : tnull;
    const unsigned grp = __match_any_sync(full, s >= 0 ? (unsigned)s : (0x10000u | (unsigned)lane));
    const bool lead = lane == __ffs(grp) - 1;
    auto add64 = [](uint64_t p, uint64_t q) { return p + q; };
    if (CAT == CAT_F64) {
      sum = (uint64_t)__double_as_longlong(grp_reduce(grp, __longlong_as_double((long long)sum), [](double p, double q) { return p + q; }));
      sq = (uint64_t)__double_as_longlong(grp_reduce(grp, __longlong_as_double((long long)sq), [](double p, double q) { return p + q; }));
    } else if (CAT == CAT_F32) {
      sum = __float_as_uint(grp_reduce(grp, __uint_as_float((uint32_t)sum), [](float p, float q) { return p + q; }));
      sq = __float_as_uint(grp_reduce(grp, __uint_as_float((uint32_t)sq), [](float p, float q) { return p + q; }));
    } else {
      sum = grp_reduce(grp, sum, add64);
      sq = grp_reduce(grp, sq, add64);
    }
    mn = grp_reduce(grp, mn, [](uint64_t p, uint64_t q) { return p < q ? p : q; });
    mx = grp_reduce(grp, mx, [](uint64_t p, uint64_t q) { return p > q ? p : q; });
    n = grp_reduce(grp, n, [](uint32_t p, uint32_t q) { return p + q; });
    nul = grp_reduce(grp, nul, [](uint32_t p, uint32_t q) { return p + q; });
    if (s >= 0 && lead) {
      const uint32_t sa = tbase + (uint32_t)s * (uint32_t)stride;
      if (nul && c.nulls_off >= 0) sred_add_u32(sa + c.nulls_off, nul);
      flush_atomic<CAT, W>(sa, c, sum, sq, mn, mx, n);
    }
  }
}

// Pass 2 over sorted chunks.  P2 is the plan with value columns redirected to
// the partitioned arrays (offset 0, `bits` validity) and packed_keys set, as
// for k_part_aggregate; WAGG ranks rows of one slot per warp with one atomic
// (items of heavy partitions).  Rows of a work item are read two at a time
// with vector loads: item starts are even and regions are padded to 32 rows.
template <int KW, int R, int NT, int MAXV, bool WAGG>
__global__ void __launch_bounds__(NT, 1) k_part_sorted(const __grid_constant__ Plan P2,
                                                       const __grid_constant__ PartArgs A, TableRef G,
                                                       DenseRef D, int scap, int sfill, int L,
                                                       const __grid_constant__ SlotTemplate tmpl)
{
  static_assert(R % 2 == 0, "rows are loaded in pairs");
  static_assert((R & (R - 1)) == 0, "rows per thread: a power of two (stage_at)");
  constexpr int C = R * NT;
  constexpr int64_t STEP = C;
  extern __shared__ __align__(16) uint8_t smem[];
  using ScanT = cub::BlockScan<unsigned, NT>;
  __shared__ typename ScanT::TempStorage scan_tmp;
  __shared__ int s_part;
  __shared__ unsigned int s_used, s_spill, s_new, s_total;
  __shared__ unsigned long long s_base;
  if (threadIdx.x == 0) s_new = 0;
  const int stride = G.stride;
  const int nw = stride / 8;
  const bool have_bits = A.bits != nullptr;
  const int nv = P2.num_vals;
  const int nslots = scap + (KW == 1);
  auto a16 = [](size_t x) { return (x + 15) & ~(size_t)15; };
  size_t off = a16((size_t)nslots * stride);
  uint32_t* cnt0 = (uint32_t*)(smem + off);
  off += a16((size_t)(nslots + 1) * 4);
  uint32_t* cnt1 = (uint32_t*)(smem + off);
  off += a16((size_t)(nslots + 1) * 4);
  uint16_t* sslot = (uint16_t*)(smem + off);
  off += a16((size_t)C * 2);
  uint8_t* sbits = have_bits ? smem + off : nullptr;
  if (have_bits) off += a16((size_t)C);
  uint8_t* stage0 = smem + off;
  const uint32_t tbase = (uint32_t)__cvta_generic_to_shared(smem);
  const int lane = threadIdx.x & 31;
  const int per = (nslots + 1 + NT - 1) / NT;  // count entries per thread in the scan
  // L2 prefetch line of this thread (two chunks ahead), as in k_part_aggregate
  const uint8_t* pf_base = nullptr;
  int pf_w = 0, pf_off = 0;
  {
    int line = threadIdx.x;
    auto take = [&](const void* base, int w) {
      const int lines = (int)((STEP * w + 127) / 128);
      if (pf_base == nullptr && line >= 0 && line < lines) {
        pf_base = (const uint8_t*)base;
        pf_w = w;
        pf_off = line * 128;
      }
      line -= lines;
    };
    take(P2.packed_keys, 8 * KW);
    for (int v = 0; v < nv; ++v) take(P2.vals[v].data, P2.vals[v].width);
    if (have_bits) take(A.bits, 1);
  }
  for (;;) {
    // both count arrays start the item at zero (p2_claim's barrier orders
    // this before the first chunk's counting)
    for (int i = threadIdx.x; i <= nslots; i += NT) {
      cnt0[i] = 0;
      cnt1[i] = 0;
    }
    const int it = p2_claim<NT>(A, smem, nslots, nw, tmpl, &s_part, &s_used, &s_spill);
    if (it >= A.nitems) break;
    const PartItem item = A.items[it];
    const int64_t b0 = item.begin;
    const int64_t e = min(item.end, min((int64_t)A.cursor[item.part], A.end[item.part]));
    // this thread's rows of a chunk at r0: r0 + 2*(threadIdx.x + NT*q) + {0, 1}
    auto row_of = [&](int64_t r0, int j) { return r0 + 2 * ((int64_t)threadIdx.x + (int64_t)NT * (j >> 1)) + (j & 1); };
    auto load_keys = [&](int64_t r0, uint64_t (&k0)[R], uint64_t (&k1)[R], uint32_t (&vb)[R]) {
#pragma unroll
      for (int j = 0; j < R; j += 2) {
        const int64_t r = row_of(r0, j);
        k0[j] = k0[j + 1] = kEmpty;
        k1[j] = k1[j + 1] = 0;
        vb[j] = vb[j + 1] = 0xFFFFFFFFu;
        if (r < e) {
          if (KW == 1) {
            const ulonglong2 kk = __ldg((const ulonglong2*)(P2.packed_keys + r));
            k0[j] = kk.x;
            k0[j + 1] = kk.y;
          } else {
            const ulonglong2 ka = __ldg((const ulonglong2*)(P2.packed_keys + 2 * r));
            const ulonglong2 kb = __ldg((const ulonglong2*)(P2.packed_keys + 2 * r + 2));
            k0[j] = ka.x;
            k1[j] = ka.y;
            k0[j + 1] = kb.x;
            k1[j + 1] = kb.y;
          }
          if (have_bits) {
            const uint32_t bb = __ldg((const uint16_t*)(A.bits + r));
            vb[j] = bb & 0xFFu;
            vb[j + 1] = bb >> 8;
          }
        }
      }
    };
    uint64_t k0[R], k1[R];
    uint32_t vb[R];
    load_keys(b0, k0, k1, vb);
    int chunk = 0;
    for (int64_t r0 = b0; r0 < e; r0 += STEP, ++chunk) {
      uint32_t* cur = (chunk & 1) ? cnt1 : cnt0;
      uint32_t* nxt = (chunk & 1) ? cnt0 : cnt1;
      if (pf_base) {
        const int64_t at = (r0 + 2 * STEP) * pf_w + pf_off;
        if (at < e * pf_w) prefetch_l2(pf_base + at);
      }
      // this chunk's values, in flight while its keys are placed
      uint64_t xv[R][MAXV];
#pragma unroll
      for (int j = 0; j < R; j += 2) {
        const int64_t r = row_of(r0, j);
#pragma unroll
        for (int v = 0; v < MAXV; ++v) {
          xv[j][v] = 0;
          xv[j + 1][v] = 0;
          if (v < nv && r < e) load_pair_w(P2.vals[v].data, r, P2.vals[v].width, xv[j][v], xv[j + 1][v]);
        }
      }
      // P1: slot and rank of every row
      int slot[R];
      uint32_t rank[R];
#pragma unroll
      for (int j = 0; j < R; ++j) {
        const int64_t r = row_of(r0, j);
        slot[j] = -1;
        rank[j] = 0;
        if (r < e) {
          const uint64_t h = hash_key(k0[j], k1[j], KW);
          slot[j] = smem_index(smem, stride, (uint32_t)scap, sfill, &s_used, KW, k0[j], k1[j], h);
          if (slot[j] < 0) {
            // listed for the global table; one list reservation per warp
            s_spill = 1;
            const unsigned mates = __activemask();
            const int leader = __ffs(mates) - 1;
            unsigned at = 0;
            if (lane == leader) at = atomicAdd(A.counters + 12, (unsigned)__popc(mates));
            at = __shfl_sync(mates, at, leader) + __popc(mates & ((1u << lane) - 1));
            if (at < A.spill_cap) A.spill_rows[at] = r;
            else atomicOr(A.counters + 13, 1u);
          }
        }
        if (WAGG) {
          const unsigned grp =
            __match_any_sync(0xFFFFFFFFu, slot[j] >= 0 ? (unsigned)slot[j] : (0x10000u | (unsigned)lane));
          const int ld = __ffs(grp) - 1;
          uint32_t base = 0;
          if (slot[j] >= 0 && lane == ld) base = atomicAdd(&cur[slot[j]], (unsigned)__popc(grp));
          base = __shfl_sync(0xFFFFFFFFu, base, ld);
          rank[j] = base + __popc(grp & ((1u << lane) - 1));
        } else if (slot[j] >= 0) {
          rank[j] = atomicAdd(&cur[slot[j]], 1u);
        }
      }
      uint32_t cvb[R];
#pragma unroll
      for (int j = 0; j < R; ++j) cvb[j] = vb[j];
      // the next chunk's keys, in flight through P2-P4
      load_keys(r0 + STEP, k0, k1, vb);
      __syncthreads();
      // P2: run starts in place of the counts; the next chunk's counts zeroed
      {
        const int q0 = threadIdx.x * per, q1 = min(q0 + per, nslots + 1);
        unsigned mine = 0;
        for (int q = q0; q < q1; ++q) mine += cur[q];
        unsigned pre, total;
        ScanT(scan_tmp).ExclusiveSum(mine, pre, total);
        for (int q = q0; q < q1; ++q) {
          const unsigned c = cur[q];
          cur[q] = pre;
          pre += c;
          nxt[q] = 0;
        }
        if (threadIdx.x == 0) s_total = total;
      }
      __syncthreads();
      // P3: slot, validity byte and values at the sorted position
#pragma unroll
      for (int j = 0; j < R; ++j) {
        if (slot[j] < 0) continue;
        const int pos = stage_at<R, NT>((int)(cur[slot[j]] + rank[j]));
        sslot[pos] = (uint16_t)slot[j];
        if (have_bits) sbits[pos] = (uint8_t)cvb[j];
        uint8_t* st = stage0;
#pragma unroll
        for (int v = 0; v < MAXV; ++v) {
          if (v >= nv) break;
          if (P2.vals[v].width == 8) {
            ((uint64_t*)st)[pos] = xv[j][v];
            st += (size_t)C * 8;
          } else {
            ((uint32_t*)st)[pos] = (uint32_t)xv[j][v];
            st += (size_t)C * 4;
          }
        }
      }
      __syncthreads();
      // P4: rows per slot, then every column, run by run
      const int a = threadIdx.x * R, b = min(a + R, (int)s_total);
      for_runs<R, NT>(sslot, cur, a, b, L, [&](int pos, int len, int s, bool piece) {
        (void)pos;
        if (!piece) *(uint32_t*)(smem + (size_t)s * stride + P2.rows_off) += (uint32_t)len;
        else sred_add_u32(tbase + (uint32_t)s * (uint32_t)stride + P2.rows_off, (uint32_t)len);
      });
      {
        const uint8_t* st = stage0;
#pragma unroll 1
        for (int v = 0; v < MAXV; ++v) {
          if (v >= nv) break;
          const ValCol& c = P2.vals[v];
#define GB_SORTED_COL(CAT_, W_) \
  sorted_column<CAT_, W_, R, NT>(c, v, smem, tbase, stride, sslot, sbits, st, cur, a, b, L)
          switch ((c.cat << 4) | c.width) {
            case (CAT_F64 << 4) | 8: GB_SORTED_COL(CAT_F64, 8); break;
            case (CAT_F32 << 4) | 4: GB_SORTED_COL(CAT_F32, 4); break;
            case (CAT_SIGNED << 4) | 8: GB_SORTED_COL(CAT_SIGNED, 8); break;
            case (CAT_SIGNED << 4) | 4: GB_SORTED_COL(CAT_SIGNED, 4); break;
            case (CAT_SIGNED << 4) | 2: GB_SORTED_COL(CAT_SIGNED, 2); break;
            case (CAT_SIGNED << 4) | 1: GB_SORTED_COL(CAT_SIGNED, 1); break;
            case (CAT_UNSIGNED << 4) | 8: GB_SORTED_COL(CAT_UNSIGNED, 8); break;
            case (CAT_UNSIGNED << 4) | 4: GB_SORTED_COL(CAT_UNSIGNED, 4); break;
            case (CAT_UNSIGNED << 4) | 2: GB_SORTED_COL(CAT_UNSIGNED, 2); break;
            case (CAT_UNSIGNED << 4) | 1: GB_SORTED_COL(CAT_UNSIGNED, 1); break;
            default: GB_SORTED_COL(CAT_BOOL, 1); break;
          }
#undef GB_SORTED_COL
          st += (size_t)C * (c.width == 8 ? 8 : 4);
        }
      }
    }
    __syncthreads();
    p2_flush<NT, ScanT>(P2, G, D, smem, scap, s_spill != 0 || item.merge, scan_tmp, &s_base, &s_new);
    __syncthreads();
  }
  if (threadIdx.x == 0 && s_new) atomicAdd(G.counters, s_new);
}

}  // namespace gb
