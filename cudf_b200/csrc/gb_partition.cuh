// gb_partition.cuh -- hash-partitioned aggregation for high group counts.
//
// When the groups do not fit one CTA's shared memory, per-row global atomics
// into an L2/HBM table are bound by the L2 atomic rate (~0.15-0.19 G/s per
// SM-free table op on B200), far below HBM bandwidth.  This path trades one
// extra write+read of the rows for atomics that stay in shared memory:
//
//   k_part_scatter    pass 1: pack each row's key, take the top bits of its
//                     hash as partition id, and scatter key words, value bits
//                     and a validity byte into that partition's region.  One
//                     global atomic per (tile, partition) reserves space.
//   k_part_aggregate  pass 2: one CTA at a time owns a partition and
//                     aggregates it in a shared-memory table; its groups are
//                     then copied out as dense slots (or merged into a global
//                     spill table when the partition did not fit).
#pragma once
#include <cub/block/block_scan.cuh>

#include "gb_kernels.cuh"

namespace gb {

struct PartArgs {
  int32_t nparts;
  int32_t shift;                 // partition = hash >> shift
  const int64_t* base;           // [nparts] first row of each region
  const int64_t* end;            // [nparts] one past the last row of each region
  unsigned long long* cursor;    // [nparts] next free row of each region
  uint64_t* keys;                // key words, key_words per row
  void* vals[kMaxValCols];       // value bits per column (column width per row)
  uint8_t* bits;                 // validity byte per row (bit v = value column v), or null
  unsigned int* counters;        // [5] region overflow, [8] partition work counter
};

struct DenseRef {
  uint8_t* T;                    // dense slots
  int64_t cap;
  unsigned long long* count;     // slots written
  unsigned int* overflow;
};

__device__ __forceinline__ void prefetch_l2(const void* p)
{
  asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

// Pass 1.  Each CTA takes tiles of RPT*256 rows.  A tile's rows are counting-
// sorted by partition in shared memory (keys staged there, then each value
// column in turn), so every (tile, partition) run leaves as one contiguous
// write of ~tile/nparts rows instead of scattered 8-byte stores.  256 threads
// and a 4K-row tile keep the footprint at ~64 KB so three CTAs share an SM;
// each column's RPT loads per thread are issued back to back.
// Shared memory: stage[tile * 8*KW] | inv u16[tile] | psort u16[tile] |
//                hist u32[nparts] | scan u32[nparts] | gbase u64[nparts]
constexpr int kScatterThreads = 256;
template <int KW, int RPT>
__global__ void __launch_bounds__(256, 3) k_part_scatter(const __grid_constant__ Plan P,
                                                      const __grid_constant__ PartArgs A)
{
  constexpr int T = kScatterThreads;
  constexpr int TILE = RPT * T;
  extern __shared__ __align__(16) uint8_t sh[];
  uint8_t* stage = sh;
  uint16_t* inv = (uint16_t*)(sh + (size_t)TILE * 8 * KW);
  uint16_t* psort = inv + TILE;
  unsigned int* hist = (unsigned int*)(psort + TILE);
  unsigned int* scan = hist + A.nparts;
  unsigned long long* gbase = (unsigned long long*)(scan + A.nparts + (A.nparts & 1));
  using Scan = cub::BlockScan<unsigned, T>;
  __shared__ typename Scan::TempStorage scan_tmp;
  __shared__ unsigned int s_valid;
  const int64_t n = P.num_rows;
  const bool any_bits = A.bits != nullptr;
  const int per = (A.nparts + T - 1) / T;  // partitions per thread in the scan
  for (int64_t t0 = (int64_t)blockIdx.x * TILE; t0 < n; t0 += (int64_t)gridDim.x * TILE) {
    const int cnt = (int)(n - t0 < (int64_t)TILE ? n - t0 : (int64_t)TILE);
    for (int i = threadIdx.x; i < A.nparts; i += T) hist[i] = 0;
    __syncthreads();
    // A: keys -> stage, partition ids and ranks
    uint32_t pr[RPT];
    if (P.num_keys == 1 && !P.keys[0].mask && P.keys[0].width == 8 && P.keys[0].cat != CAT_F64) {
      // one plain 64-bit key: load all RPT keys first
      const unsigned long long* kd = (const unsigned long long*)P.keys[0].data + P.keys[0].offset;
      uint64_t kk[RPT];
#pragma unroll
      for (int k = 0; k < RPT; ++k) {
        int i = k * T + threadIdx.x;
        kk[k] = i < cnt ? __ldg(kd + t0 + i) : 0;
      }
#pragma unroll
      for (int k = 0; k < RPT; ++k) {
        int i = k * T + threadIdx.x;
        pr[k] = 0xFFFFFFFFu;
        if (i < cnt) {
          ((uint64_t*)stage)[i] = kk[k];
          unsigned p = (unsigned)(hash_key(kk[k], 0, 1) >> A.shift);
          pr[k] = (p << 16) | atomicAdd(&hist[p], 1u);
        }
      }
    } else {
#pragma unroll
      for (int k = 0; k < RPT; ++k) {
        int i = k * T + threadIdx.x;
        pr[k] = 0xFFFFFFFFu;
        uint64_t w0, w1;
        if (i < cnt && pack_key(P, t0 + i, w0, w1)) {
          if (KW == 1) ((uint64_t*)stage)[i] = w0;
          else ((ulonglong2*)stage)[i] = make_ulonglong2(w0, w1);
          unsigned p = (unsigned)(hash_key(w0, w1, KW) >> A.shift);
          pr[k] = (p << 16) | atomicAdd(&hist[p], 1u);
        }
      }
    }
    __syncthreads();
    // B: reserve each partition's run; exclusive scan of the histogram
    unsigned mine = 0;
    for (int q = threadIdx.x * per; q < min(A.nparts, (threadIdx.x + 1) * per); ++q) {
      unsigned h = hist[q];
      mine += h;
      if (h) {
        unsigned long long g = atomicAdd(&A.cursor[q], (unsigned long long)h);
        gbase[q] = g;
        if ((int64_t)(g + h) > A.end[q]) atomicOr(A.counters + 5, 1u);
      }
    }
    unsigned off, total;
    Scan(scan_tmp).ExclusiveSum(mine, off, total);
    for (int q = threadIdx.x * per; q < min(A.nparts, (threadIdx.x + 1) * per); ++q) {
      scan[q] = off;
      off += hist[q];
    }
    if (threadIdx.x == 0) s_valid = total;
    __syncthreads();
    // C: sorted order
#pragma unroll
    for (int k = 0; k < RPT; ++k) {
      if (pr[k] == 0xFFFFFFFFu) continue;
      unsigned p = pr[k] >> 16;
      unsigned s = scan[p] + (pr[k] & 0xFFFFu);
      inv[s] = (uint16_t)(k * T + threadIdx.x);
      psort[s] = (uint16_t)p;
    }
    __syncthreads();
    const int nvalid = (int)s_valid;
    // D: keys out
    for (int s = threadIdx.x; s < nvalid; s += T) {
      unsigned p = psort[s];
      int64_t g = (int64_t)gbase[p] + (s - (int)scan[p]);
      if (g >= A.end[p]) continue;
      if (KW == 1) A.keys[g] = ((const uint64_t*)stage)[inv[s]];
      else ((ulonglong2*)A.keys)[g] = ((const ulonglong2*)stage)[inv[s]];
    }
    // E: each value column through the stage
    uint32_t vb[RPT];
#pragma unroll
    for (int k = 0; k < RPT; ++k) vb[k] = 0;
#pragma unroll 1
    for (int v = 0; v < P.num_vals; ++v) {
      const ValCol& c = P.vals[v];
      uint64_t x[RPT];
#pragma unroll
      for (int k = 0; k < RPT; ++k) {
        int i = k * T + threadIdx.x;
        x[k] = pr[k] != 0xFFFFFFFFu ? load_bits(c.data, t0 + i + c.offset, c.width) : 0;
      }
      if (any_bits && c.mask) {
#pragma unroll
        for (int k = 0; k < RPT; ++k)
          if (pr[k] != 0xFFFFFFFFu && bit_valid(c.mask, t0 + k * T + threadIdx.x + c.offset)) vb[k] |= 1u << v;
      } else if (any_bits) {
#pragma unroll
        for (int k = 0; k < RPT; ++k) vb[k] |= 1u << v;
      }
      __syncthreads();
#pragma unroll
      for (int k = 0; k < RPT; ++k)
        if (pr[k] != 0xFFFFFFFFu) store_width(stage, k * T + threadIdx.x, c.width, x[k]);
      __syncthreads();
      for (int s = threadIdx.x; s < nvalid; s += T) {
        unsigned p = psort[s];
        int64_t g = (int64_t)gbase[p] + (s - (int)scan[p]);
        if (g >= A.end[p]) continue;
        int i = inv[s];
        switch (c.width) {
          case 1: ((uint8_t*)A.vals[v])[g] = stage[i]; break;
          case 2: ((uint16_t*)A.vals[v])[g] = ((const uint16_t*)stage)[i]; break;
          case 4: ((uint32_t*)A.vals[v])[g] = ((const uint32_t*)stage)[i]; break;
          default: ((uint64_t*)A.vals[v])[g] = ((const uint64_t*)stage)[i]; break;
        }
      }
    }
    if (any_bits) {
      __syncthreads();
#pragma unroll
      for (int k = 0; k < RPT; ++k)
        if (pr[k] != 0xFFFFFFFFu) stage[k * T + threadIdx.x] = (uint8_t)vb[k];
      __syncthreads();
      for (int s = threadIdx.x; s < nvalid; s += T) {
        unsigned p = psort[s];
        int64_t g = (int64_t)gbase[p] + (s - (int)scan[p]);
        if (g < A.end[p]) A.bits[g] = stage[inv[s]];
      }
    }
    __syncthreads();
  }
}

// shared-memory bytes k_part_scatter<KW, RPT> needs
inline size_t part_scatter_smem(int kw, int rpt, int nparts)
{
  size_t tile = (size_t)rpt * kScatterThreads;
  return tile * 8 * kw + tile * 4 + (size_t)nparts * 8 + 8 + (size_t)nparts * 8;
}

// Shared-memory find-or-insert (bounded probes); null when the key does not
// fit (table at its fill limit or too many probes) or is the all-ones key.
__device__ __forceinline__ uint8_t* smem_slot(uint8_t* smem, int stride, uint64_t smask, int sfill,
                                              unsigned int* s_used, int words, uint64_t w0,
                                              uint64_t w1, uint64_t h)
{
  uint64_t i = h & smask;
  if (words == 1) {
    if (w0 == kEmpty) return nullptr;
    for (int p = 0; p < 64; ++p) {
      unsigned long long* kp = (unsigned long long*)(smem + i * stride);
      uint64_t cur = *(volatile unsigned long long*)kp;
      if (cur == w0) return (uint8_t*)kp;
      if (cur == kEmpty) {
        if (*(volatile unsigned int*)s_used >= (unsigned)sfill) return nullptr;
        uint64_t old = atomicCAS(kp, kEmpty, w0);
        if (old == kEmpty) { atomicAdd(s_used, 1u); return (uint8_t*)kp; }
        if (old == w0) return (uint8_t*)kp;
      }
      i = (i + 1) & smask;
    }
    return nullptr;
  }
  unsigned __int128 want = ((unsigned __int128)w1 << 64) | w0;
  const unsigned __int128 empty = ~(unsigned __int128)0;
  for (int p = 0; p < 64; ++p) {
    unsigned __int128* kp = (unsigned __int128*)(smem + i * stride);
    ulonglong2 cur = vload2(kp);
    if (cur.x == w0 && cur.y == w1 && w0 != kEmpty) return (uint8_t*)kp;
    if ((cur.y >> 63) || cur.x == kEmpty) {
      if ((cur.y >> 63) && *(volatile unsigned int*)s_used >= (unsigned)sfill) return nullptr;
      unsigned __int128 old = atomicCAS(kp, empty, want);
      if (old == empty) { atomicAdd(s_used, 1u); return (uint8_t*)kp; }
      if (old == want) return (uint8_t*)kp;
    }
    i = (i + 1) & smask;
  }
  return nullptr;
}

// ---- explicit shared-memory operations (32-bit shared-window addresses) ----
__device__ __forceinline__ void sred_add_u32(uint32_t a, uint32_t v) { asm volatile("red.shared.add.u32 [%0], %1;" ::"r"(a), "r"(v)); }
__device__ __forceinline__ void sred_add_u64(uint32_t a, uint64_t v) { asm volatile("red.shared.add.u64 [%0], %1;" ::"r"(a), "l"(v)); }
__device__ __forceinline__ void sred_add_f32(uint32_t a, float v) { asm volatile("red.shared.add.f32 [%0], %1;" ::"r"(a), "f"(v)); }
__device__ __forceinline__ void sred_add_f64(uint32_t a, double v) { asm volatile("red.shared.add.f64 [%0], %1;" ::"r"(a), "d"(v)); }
__device__ __forceinline__ void sred_min_u32(uint32_t a, uint32_t v) { asm volatile("red.shared.min.u32 [%0], %1;" ::"r"(a), "r"(v)); }
__device__ __forceinline__ void sred_max_u32(uint32_t a, uint32_t v) { asm volatile("red.shared.max.u32 [%0], %1;" ::"r"(a), "r"(v)); }
__device__ __forceinline__ void sred_min_u64(uint32_t a, uint64_t v) { asm volatile("red.shared.min.u64 [%0], %1;" ::"r"(a), "l"(v)); }
__device__ __forceinline__ void sred_max_u64(uint32_t a, uint64_t v) { asm volatile("red.shared.max.u64 [%0], %1;" ::"r"(a), "l"(v)); }
__device__ __forceinline__ uint32_t sld_u32(uint32_t a)
{
  uint32_t v;
  asm volatile("ld.volatile.shared.u32 %0, [%1];" : "=r"(v) : "r"(a));
  return v;
}
__device__ __forceinline__ uint64_t sld_u64(uint32_t a)
{
  uint64_t v;
  asm volatile("ld.volatile.shared.u64 %0, [%1];" : "=l"(v) : "r"(a));
  return v;
}

// Ops the partitioned path supports (PRODUCT and ARGMIN/ARGMAX plans use the
// other modes).
__device__ __forceinline__ bool part_op_ok(uint8_t op)
{
  return op <= OP_MAX_U64 || op == OP_SQ_I64 || op == OP_SQ_F32 || op == OP_SQ_F64;
}

// Applies one valid value (raw bits) of column c to a shared slot at `sa`.
__device__ __noinline__ void sapply(const Plan& P, const ValCol& c, uint32_t sa, uint64_t bits)
{
  int64_t iv = 0;
  float f = 0.f;
  double d = 0.0;
  switch (c.cat) {
    case CAT_SIGNED: iv = sign_extend(bits, c.width); break;
    case CAT_BOOL: iv = bits != 0; break;
    case CAT_UNSIGNED: iv = (int64_t)bits; break;
    case CAT_F32: f = __uint_as_float((uint32_t)bits); d = f; break;
    default: d = __longlong_as_double((long long)bits); break;
  }
#pragma unroll 1
  for (int a = c.acc_begin; a < c.acc_end; ++a) {
    const Acc A = P.accs[a];
    uint32_t p = sa + A.off;
    switch (A.op) {
      case OP_SUM_I64: sred_add_u64(p, (uint64_t)iv); break;
      case OP_SUM_I32: sred_add_u32(p, (uint32_t)iv); break;
      case OP_SUM_F32: sred_add_f32(p, f); break;
      case OP_SUM_F64: sred_add_f64(p, d); break;
      case OP_MIN_U32: case OP_MAX_U32: {
        bool mn = A.op == OP_MIN_U32;
        uint32_t v = c.cat == CAT_F32 ? ord32_f(f, mn)
                     : (c.cat == CAT_UNSIGNED || c.cat == CAT_BOOL) ? (uint32_t)iv
                                                                    : ((uint32_t)(int32_t)iv ^ 0x80000000u);
        uint32_t cur = sld_u32(p);
        if (mn ? v < cur : v > cur) { if (mn) sred_min_u32(p, v); else sred_max_u32(p, v); }
        break;
      }
      case OP_MIN_U64: case OP_MAX_U64: {
        bool mn = A.op == OP_MIN_U64;
        uint64_t v = c.cat == CAT_F64 ? ord64_f(d, mn)
                     : c.cat == CAT_UNSIGNED ? bits : ((uint64_t)iv ^ 0x8000000000000000ull);
        uint64_t cur = sld_u64(p);
        if (mn ? v < cur : v > cur) { if (mn) sred_min_u64(p, v); else sred_max_u64(p, v); }
        break;
      }
      case OP_SQ_I64: sred_add_u64(p, (uint64_t)iv * (uint64_t)iv); break;
      case OP_SQ_F32: sred_add_f32(p, f * f); break;
      case OP_SQ_F64: sred_add_f64(p, d * d); break;
      default: break;
    }
  }
}

// Same as sapply for a column whose accumulators are only SUM/MIN/MAX/sum of
// squares: the value is converted once and each accumulator is a fixed
// offset, without the per-accumulator dispatch.
__device__ __forceinline__ void sapply_basic(const ValCol& c, uint32_t sa, uint64_t bits)
{
  const uint8_t cat = c.cat;
  int64_t iv = 0;
  float f = 0.f;
  double d = 0.0;
  if (cat == CAT_F32) { f = __uint_as_float((uint32_t)bits); d = f; }
  else if (cat == CAT_F64) d = __longlong_as_double((long long)bits);
  else if (cat == CAT_SIGNED) iv = sign_extend(bits, c.width);
  else if (cat == CAT_BOOL) iv = bits != 0;
  else iv = (int64_t)bits;
  switch (c.sum_op) {
    case OP_SUM_I64: sred_add_u64(sa + c.sum_off, (uint64_t)iv); break;
    case OP_SUM_I32: sred_add_u32(sa + c.sum_off, (uint32_t)iv); break;
    case OP_SUM_F32: sred_add_f32(sa + c.sum_off, f); break;
    case OP_SUM_F64: sred_add_f64(sa + c.sum_off, d); break;
    default: break;
  }
  if (c.min_off >= 0 || c.max_off >= 0) {
    if (c.width == 8) {
      uint64_t lo, hi;
      if (cat == CAT_F64) { lo = ord64_f(d, true); hi = ord64_f(d, false); }
      else if (cat == CAT_UNSIGNED) lo = hi = bits;
      else lo = hi = (uint64_t)iv ^ 0x8000000000000000ull;
      if (c.min_off >= 0) sred_min_u64(sa + c.min_off, lo);
      if (c.max_off >= 0) sred_max_u64(sa + c.max_off, hi);
    } else {
      uint32_t lo, hi;
      if (cat == CAT_F32) { lo = ord32_f(f, true); hi = ord32_f(f, false); }
      else if (cat == CAT_UNSIGNED || cat == CAT_BOOL) lo = hi = (uint32_t)iv;
      else lo = hi = (uint32_t)(int32_t)iv ^ 0x80000000u;
      if (c.min_off >= 0) sred_min_u32(sa + c.min_off, lo);
      if (c.max_off >= 0) sred_max_u32(sa + c.max_off, hi);
    }
  }
  if (c.sq_off >= 0) {
    if (cat == CAT_F32) sred_add_f32(sa + c.sq_off, f * f);
    else if (cat == CAT_F64) sred_add_f64(sa + c.sq_off, d * d);
    else sred_add_u64(sa + c.sq_off, (uint64_t)iv * (uint64_t)iv);
  }
}

// A row whose key did not fit the shared table: global table, generic update.
__device__ __noinline__ void spill_row(const Plan& P2, const TableRef& G, uint64_t w0, uint64_t w1,
                                       uint64_t h, int64_t r, unsigned int* s_new)
{
  int64_t gi = global_slot(P2, G, w0, w1, h, s_new);
  if (gi < 0) {
    atomicOr(G.counters + 1, 1u);
    return;
  }
  update_slot(P2, G.T + gi * (int64_t)G.stride, r);
}

// ---- pass 2 ----
// Per-partition prologue: claim a partition, reset the shared table.  Returns
// the partition id (>= nparts: no work left).
template <int NT>
__device__ __forceinline__ int p2_claim(const PartArgs& A, uint8_t* smem, int scap, int nw,
                                        const SlotTemplate& tmpl, int* s_part, unsigned int* s_used,
                                        unsigned int* s_spill)
{
  if (threadIdx.x == 0) {
    *s_part = (int)atomicAdd(A.counters + 8, 1u);
    *s_used = 0;
    *s_spill = 0;
  }
  for (int i = threadIdx.x; i < scap * nw; i += NT) {
    int s = i / nw;
    *(unsigned long long*)(smem + (size_t)s * nw * 8 + (i - s * nw) * 8) = tmpl.w[i - s * nw];
  }
  __syncthreads();
  return *s_part;
}

// Per-partition epilogue: the partition's groups leave as dense slots, or are
// merged into the global spill table when some of its rows went there.
template <int NT, typename ScanT>
__device__ __forceinline__ void p2_flush(const Plan& P2, const TableRef& G, const DenseRef& D,
                                         const uint8_t* smem, int scap, bool spilled,
                                         typename ScanT::TempStorage& scan_tmp,
                                         unsigned long long* s_base, unsigned int* s_new)
{
  const int stride = G.stride;
  const int nw = stride / 8;
  if (spilled) {
    for (int i = threadIdx.x; i < scap; i += NT) {
      const uint8_t* s = smem + i * stride;
      if (slot_occupied(P2, s, false)) merge_slot(P2, G, s, s_new);
    }
    return;
  }
  const int per = (scap + NT - 1) / NT;
  int first = threadIdx.x * per;
  unsigned mine = 0;
  for (int i = first; i < min(first + per, scap); ++i) mine += slot_occupied(P2, smem + i * stride, false);
  unsigned off, total;
  ScanT(scan_tmp).ExclusiveSum(mine, off, total);
  if (threadIdx.x == 0) *s_base = total ? atomicAdd(D.count, (unsigned long long)total) : 0ull;
  __syncthreads();
  unsigned long long o = *s_base + off;
  for (int i = first; i < min(first + per, scap); ++i) {
    const uint8_t* s = smem + i * stride;
    if (!slot_occupied(P2, s, false)) continue;
    if ((int64_t)o >= D.cap) {
      atomicOr(D.overflow, 1u);
      break;
    }
    unsigned long long* dst = (unsigned long long*)(D.T + o * stride);
    for (int w = 0; w < nw; ++w) dst[w] = ((const unsigned long long*)s)[w];
    ++o;
  }
}

// Pass 2.  P2 is the plan with value columns redirected to the partitioned
// arrays (offset 0, `bits` validity) and packed_keys set.  One CTA owns a
// partition at a time and aggregates it in a shared-memory table.  The row
// loop is software-pipelined: while step t's rows are placed in the table,
// step t's values (every column) and step t+1's keys are already in flight,
// and step t+2 is prefetched into L2.  MAXV bounds the value columns.
template <int R, int NT, int MAXV>
__global__ void __launch_bounds__(NT, 1) k_part_aggregate(const __grid_constant__ Plan P2,
                                                          const __grid_constant__ PartArgs A,
                                                          TableRef G, DenseRef D, int scap, int sfill,
                                                          const __grid_constant__ SlotTemplate tmpl)
{
  extern __shared__ __align__(16) uint8_t smem[];
  using ScanT = cub::BlockScan<unsigned, NT>;
  __shared__ typename ScanT::TempStorage scan_tmp;
  __shared__ int s_part;
  __shared__ unsigned int s_used, s_spill, s_new;
  __shared__ unsigned long long s_base;
  if (threadIdx.x == 0) s_new = 0;
  const int stride = G.stride;
  const int nw = stride / 8;
  const uint64_t smask = (uint64_t)scap - 1;
  const bool have_bits = A.bits != nullptr;
  const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(smem);
  const int kw = P2.key_words;
  const int nv = P2.num_vals;
  for (;;) {
    const int p = p2_claim<NT>(A, smem, scap, nw, tmpl, &s_part, &s_used, &s_spill);
    if (p >= A.nparts) break;
    const int64_t b = A.base[p];
    const int64_t e = min((int64_t)A.cursor[p], A.end[p]);
    constexpr int64_t STEP = (int64_t)R * NT;
    auto load_keys = [&](int64_t r0, uint64_t (&k0)[R], uint64_t (&k1)[R], uint32_t (&vb)[R]) {
#pragma unroll
      for (int j = 0; j < R; ++j) {
        int64_t r = r0 + (int64_t)j * NT + threadIdx.x;
        k0[j] = kEmpty;
        k1[j] = 0;
        vb[j] = 0xFFFFFFFFu;
        if (r < e) {
          if (kw == 1) k0[j] = __ldg(P2.packed_keys + r);
          else {
            ulonglong2 kk = __ldg((const ulonglong2*)(P2.packed_keys + 2 * r));
            k0[j] = kk.x;
            k1[j] = kk.y;
          }
          if (have_bits) vb[j] = __ldg(A.bits + r);
        }
      }
    };
    uint64_t k0[R], k1[R];
    uint32_t vb[R];
    load_keys(b, k0, k1, vb);
    for (int64_t r0 = b; r0 < e; r0 += STEP) {
      // step t+2 into L2
      {
        const int64_t n0 = r0 + 2 * STEP;
        const int64_t n1 = min(e, n0 + STEP);
        if (n0 < n1) {
          const int64_t t = threadIdx.x;
          if (t * 128 < (n1 - n0) * 8 * kw) prefetch_l2((const uint8_t*)(P2.packed_keys + n0 * kw) + t * 128);
#pragma unroll
          for (int v = 0; v < MAXV; ++v) {
            if (v >= nv) break;
            if (t * 128 < (n1 - n0) * P2.vals[v].width)
              prefetch_l2((const uint8_t*)P2.vals[v].data + n0 * P2.vals[v].width + t * 128);
          }
          if (have_bits && t * 128 < n1 - n0) prefetch_l2(A.bits + n0 + t * 128);
        }
      }
      // place this step's rows
      uint32_t sa[R];
#pragma unroll
      for (int j = 0; j < R; ++j) {
        int64_t r = r0 + (int64_t)j * NT + threadIdx.x;
        sa[j] = 0;
        if (r >= e) continue;
        uint64_t h = hash_key(k0[j], k1[j], kw);
        uint8_t* slot = smem_slot(smem, stride, smask, sfill, &s_used, kw, k0[j], k1[j], h);
        if (slot == nullptr) {
          s_spill = 1;
          spill_row(P2, G, k0[j], k1[j], h, r, &s_new);
          continue;
        }
        sa[j] = sbase + (uint32_t)(slot - smem);
      }
      // this step's values and the next step's keys in flight together
      uint64_t x[R][MAXV];
#pragma unroll
      for (int j = 0; j < R; ++j) {
        int64_t r = r0 + (int64_t)j * NT + threadIdx.x;
#pragma unroll
        for (int v = 0; v < MAXV; ++v) {
          x[j][v] = 0;
          if (v < nv && sa[j] && ((vb[j] >> v) & 1)) x[j][v] = load_bits(P2.vals[v].data, r, P2.vals[v].width);
        }
      }
      uint64_t nk0[R], nk1[R];
      uint32_t nvb[R];
      load_keys(r0 + STEP, nk0, nk1, nvb);
#pragma unroll
      for (int j = 0; j < R; ++j) {
        if (!sa[j]) continue;
        sred_add_u32(sa[j] + P2.rows_off, 1u);
#pragma unroll
        for (int v = 0; v < MAXV; ++v) {
          if (v >= nv) break;
          const ValCol& c = P2.vals[v];
          if (!((vb[j] >> v) & 1)) {
            if (c.nulls_off >= 0) sred_add_u32(sa[j] + c.nulls_off, 1u);
            continue;
          }
          if (c.basic) sapply_basic(c, sa[j], x[j][v]);
          else sapply(P2, c, sa[j], x[j][v]);
        }
      }
#pragma unroll
      for (int j = 0; j < R; ++j) {
        k0[j] = nk0[j];
        k1[j] = nk1[j];
        vb[j] = nvb[j];
      }
    }
    __syncthreads();
    p2_flush<NT, ScanT>(P2, G, D, smem, scap, s_spill != 0, scan_tmp, &s_base, &s_new);
    __syncthreads();
  }
  if (threadIdx.x == 0 && s_new) atomicAdd(G.counters, s_new);
}

}  // namespace gb
