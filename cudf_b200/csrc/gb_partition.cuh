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
//   k_part_aggregate  pass 2: one CTA at a time owns a work item -- a
//                     partition, or a row range of a heavy partition -- and
//                     aggregates it in a shared-memory table; its groups are
//                     then copied out as dense slots (or merged into a global
//                     spill table for split partitions and partitions that did
//                     not fit).  Items of split partitions combine the rows of
//                     one slot per warp before the shared update.  The same
//                     kernel over row ranges of the caller's own columns is
//                     the shared-stage mode for groups that fit one CTA.
//   k_part_spill      applies the rows listed as not fitting their table to
//                     the global spill table.
#pragma once
#include <cub/block/block_scan.cuh>

#include "gb_kernels.cuh"

namespace gb {

// One unit of pass-2 work: rows [begin, end) of partition `part`'s region.
// `merge` = 1 when the partition is split over several items, whose tables
// then all go to the global table.
struct PartItem {
  int32_t part;
  int32_t merge;
  int64_t begin, end;
};

struct PartArgs {
  int32_t nparts;
  int32_t shift;                 // partition = hash >> shift
  const int64_t* base;           // [nparts] first row of each region
  const int64_t* end;            // [nparts] one past the last row of each region
  unsigned long long* cursor;    // [nparts] next free row of each region
  uint64_t* keys;                // key words, key_words per row
  void* vals[kMaxValCols];       // value bits per column (column width per row)
  uint8_t* bits;                 // validity byte per row (bit v = value column v), or null
  unsigned int* counters;        // [5] region overflow, [8] partition work counter,
                                 // [12] spill list length, [13] spill list overflow
  int64_t* spill_rows;           // pass 2: rows that did not fit their shared table
  unsigned int spill_cap;
  const PartItem* items;         // pass 2 work list
  int32_t nitems;
  unsigned int* work;            // pass 2 claim counter of this item list
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

// Pass 1.  Each CTA takes tiles of RPT*NT rows.  A tile's rows are counting-
// sorted by partition in shared memory, so every (tile, partition) run leaves
// as one contiguous write of ~tile/nparts rows instead of scattered stores:
//   A  keys loaded (all RPT per thread at once), partition id = top hash bits,
//      rank within the tile's partition from a shared histogram;
//   B  one global reservation per (tile, partition) on the region cursor,
//      exclusive scan of the histogram; per partition, `delta` maps a sorted
//      position to its global row and `send` bounds the rows that fit;
//   C  keys, then each value column, then the validity bytes are stored into
//      the stage at their sorted position and written out in sorted order
//      (consecutive threads, consecutive rows of a run).  The next column's
//      loads are issued before the current column's write-out.
// Shared memory: stage[tile * 8] | psort u16[tile] | hist u32[nparts] |
//                send u32[nparts] | delta i64[nparts]
template <int KW, int RPT, int NT, int MINB, bool PF = true>
__global__ void __launch_bounds__(NT, MINB) k_part_scatter(const __grid_constant__ Plan P,
                                                         const __grid_constant__ PartArgs A)
{
  constexpr int TILE = RPT * NT;
  static_assert(TILE <= 65536, "sorted positions are 16-bit");
  extern __shared__ __align__(16) uint8_t sh[];
  uint8_t* stage = sh;
  uint16_t* psort = (uint16_t*)(sh + (size_t)TILE * 8);
  unsigned int* hist = (unsigned int*)(psort + TILE);
  unsigned int* send = hist + A.nparts;
  long long* delta = (long long*)(send + A.nparts + (A.nparts & 1));
  using Scan = cub::BlockScan<unsigned, NT>;
  __shared__ typename Scan::TempStorage scan_tmp;
  __shared__ unsigned int s_valid;
  const int64_t n = P.num_rows;
  const bool any_bits = A.bits != nullptr;
  const int nv = P.num_vals;
  const int per = (A.nparts + NT - 1) / NT;  // partitions per thread in the scan
  for (int64_t t0 = (int64_t)blockIdx.x * TILE; t0 < n; t0 += (int64_t)gridDim.x * TILE) {
    const int cnt = (int)(n - t0 < (int64_t)TILE ? n - t0 : (int64_t)TILE);
    for (int i = threadIdx.x; i < A.nparts; i += NT) hist[i] = 0;
    __syncthreads();
    // A
    uint32_t pr[RPT];  // partition << 16 | rank, later partition << 16 | sorted position
    const bool plain_key =
      P.num_keys == 1 && !P.keys[0].mask && P.keys[0].width == 8 && P.keys[0].cat != CAT_F64;
    const unsigned long long* kd = (const unsigned long long*)P.keys[0].data + P.keys[0].offset;
    if (plain_key) {
      // one plain 64-bit key: its bits are the key word
      uint64_t k0[RPT];
#pragma unroll
      for (int k = 0; k < RPT; ++k) {
        const int i = k * NT + threadIdx.x;
        k0[k] = i < cnt ? __ldg(kd + t0 + i) : 0;
      }
#pragma unroll
      for (int k = 0; k < RPT; ++k) {
        const int i = k * NT + threadIdx.x;
        pr[k] = 0xFFFFFFFFu;
        if (i < cnt) {
          const unsigned p = (unsigned)(hash_key(k0[k], 0, 1) >> A.shift);
          pr[k] = (p << 16) | atomicAdd(&hist[p], 1u);
        }
      }
    } else {
#pragma unroll
      for (int k = 0; k < RPT; ++k) {
        const int i = k * NT + threadIdx.x;
        pr[k] = 0xFFFFFFFFu;
        uint64_t w0 = 0, w1 = 0;
        if (i < cnt && pack_key(P, t0 + i, w0, w1)) {
          const unsigned p = (unsigned)(hash_key(w0, w1, KW) >> A.shift);
          pr[k] = (p << 16) | atomicAdd(&hist[p], 1u);
        }
      }
    }
    __syncthreads();
    // B: reservations (independent atomics, issued before their results are
    // used), then the scan
    unsigned mine = 0;
    for (int q0 = threadIdx.x * per; q0 < min(A.nparts, (threadIdx.x + 1) * per); q0 += 4) {
      unsigned h[4];
      unsigned long long g[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int q = q0 + j;
        h[j] = (j < per && q < min(A.nparts, (threadIdx.x + 1) * per)) ? hist[q] : 0u;
        g[j] = h[j] ? atomicAdd(&A.cursor[q], (unsigned long long)h[j]) : 0ull;
        mine += h[j];
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int q = q0 + j;
        if (!h[j]) continue;
        const long long room = (long long)A.end[q] - (long long)g[j];
        if ((long long)h[j] > room) atomicOr(A.counters + 5, 1u);
        delta[q] = (long long)g[j];                      // minus the scan offset below
        send[q] = room <= 0 ? 0u : (unsigned)min((long long)h[j], room);  // plus the offset below
      }
    }
    unsigned off, total;
    Scan(scan_tmp).ExclusiveSum(mine, off, total);
    for (int q = threadIdx.x * per; q < min(A.nparts, (threadIdx.x + 1) * per); ++q) {
      const unsigned h = hist[q];
      if (h) {
        delta[q] -= (long long)off;
        send[q] += off;
      }
      hist[q] = off;  // partition start in the sorted tile
      off += h;
    }
    if (threadIdx.x == 0) s_valid = total;
    __syncthreads();
    const int nvalid = (int)s_valid;
    // C: sorted positions; keys (read again: the tile was just loaded, so
    // they come from cache) through the stage
#pragma unroll
    for (int k = 0; k < RPT; ++k) {
      if (pr[k] == 0xFFFFFFFFu) continue;
      const unsigned p = pr[k] >> 16;
      const unsigned s = hist[p] + (pr[k] & 0xFFFFu);
      pr[k] = (p << 16) | s;
      psort[s] = (uint16_t)p;
    }
    // two-word keys go through the 8-byte stage one word at a time (word 1
    // waits in registers), which halves the stage and lets two CTAs share an SM
    uint64_t kw1[KW == 2 ? RPT : 1];
    if (plain_key) {
      uint64_t k0[RPT];
#pragma unroll
      for (int k = 0; k < RPT; ++k) k0[k] = pr[k] != 0xFFFFFFFFu ? __ldg(kd + t0 + k * NT + threadIdx.x) : 0;
#pragma unroll
      for (int k = 0; k < RPT; ++k)
        if (pr[k] != 0xFFFFFFFFu) ((uint64_t*)stage)[pr[k] & 0xFFFFu] = k0[k];
    } else {
#pragma unroll
      for (int k = 0; k < RPT; ++k) {
        if (pr[k] == 0xFFFFFFFFu) continue;
        uint64_t w0 = 0, w1 = 0;
        pack_key(P, t0 + k * NT + threadIdx.x, w0, w1);
        ((uint64_t*)stage)[pr[k] & 0xFFFFu] = w0;
        if (KW == 2) kw1[k] = w1;
      }
    }
    // first value column's loads in flight with the key write-out
    uint64_t x[RPT];
    auto load_col = [&](int v) {
      const ValCol& c = P.vals[v];
#pragma unroll
      for (int k = 0; k < RPT; ++k) {
        const int i = k * NT + threadIdx.x;
        x[k] = pr[k] != 0xFFFFFFFFu ? load_bits(c.data, t0 + i + c.offset, c.width) : 0;
      }
    };
    // a column of at most 4 bytes shares its round with the validity bytes
    // (value at +0 and validity at +4 of an 8-byte stage slot), saving the
    // validity bytes' own round; it goes last, once every column's validity
    // bit is known
    int vn = -1;
    if (any_bits)
      for (int v = 0; v < nv; ++v)
        if (P.vals[v].width <= 4) vn = v;
    auto col_at = [&](int vi) { return vn < 0 || vi < vn ? vi : (vi == nv - 1 ? vn : vi + 1); };
    if (PF && nv > 0) load_col(col_at(0));
    __syncthreads();
    for (int s = threadIdx.x; s < nvalid; s += NT) {
      const unsigned p = psort[s];
      if ((unsigned)s >= send[p]) continue;
      const int64_t g = delta[p] + s;
      A.keys[KW * g] = ((const uint64_t*)stage)[s];
    }
    if (KW == 2) {
      __syncthreads();
#pragma unroll
      for (int k = 0; k < RPT; ++k)
        if (pr[k] != 0xFFFFFFFFu) ((uint64_t*)stage)[pr[k] & 0xFFFFu] = kw1[k];
      __syncthreads();
      for (int s = threadIdx.x; s < nvalid; s += NT) {
        const unsigned p = psort[s];
        if ((unsigned)s >= send[p]) continue;
        A.keys[2 * (delta[p] + s) + 1] = ((const uint64_t*)stage)[s];
      }
    }
    // validity bytes of this thread's rows, four to a register
    uint32_t vb[(RPT + 3) / 4];
#pragma unroll
    for (int k = 0; k < (RPT + 3) / 4; ++k) vb[k] = 0;
#pragma unroll 1
    for (int vi = 0; vi < nv; ++vi) {
      const int v = col_at(vi);
      const ValCol& c = P.vals[v];
      if (any_bits) {
#pragma unroll
        for (int k = 0; k < RPT; ++k)
          if (pr[k] != 0xFFFFFFFFu && (!c.mask || bit_valid(c.mask, t0 + k * NT + threadIdx.x + c.offset)))
            vb[k >> 2] |= 1u << (v + 8 * (k & 3));
      }
      if (!PF) load_col(v);
      __syncthreads();  // the previous write-out has read the stage
      void* dst = A.vals[v];
      if (v == vn) {
#pragma unroll
        for (int k = 0; k < RPT; ++k)
          if (pr[k] != 0xFFFFFFFFu) {
            const unsigned s = pr[k] & 0xFFFFu;
            ((uint32_t*)stage)[2 * s] = (uint32_t)x[k];
            stage[8 * s + 4] = (uint8_t)(vb[k >> 2] >> (8 * (k & 3)));
          }
        __syncthreads();
        for (int s = threadIdx.x; s < nvalid; s += NT) {
          const unsigned p = psort[s];
          if ((unsigned)s >= send[p]) continue;
          const int64_t g = delta[p] + s;
          const uint32_t w = ((const uint32_t*)stage)[2 * s];
          if (c.width == 4) ((uint32_t*)dst)[g] = w;
          else if (c.width == 2) ((uint16_t*)dst)[g] = (uint16_t)w;
          else ((uint8_t*)dst)[g] = (uint8_t)w;
          A.bits[g] = stage[8 * s + 4];
        }
        continue;
      }
#pragma unroll
      for (int k = 0; k < RPT; ++k)
        if (pr[k] != 0xFFFFFFFFu) store_width(stage, pr[k] & 0xFFFFu, c.width, x[k]);
      __syncthreads();
      if (PF && vi + 1 < nv) load_col(col_at(vi + 1));
      switch (c.width) {
        case 8:
          for (int s = threadIdx.x; s < nvalid; s += NT) {
            const unsigned p = psort[s];
            if ((unsigned)s < send[p]) ((uint64_t*)dst)[delta[p] + s] = ((const uint64_t*)stage)[s];
          }
          break;
        case 4:
          for (int s = threadIdx.x; s < nvalid; s += NT) {
            const unsigned p = psort[s];
            if ((unsigned)s < send[p]) ((uint32_t*)dst)[delta[p] + s] = ((const uint32_t*)stage)[s];
          }
          break;
        case 2:
          for (int s = threadIdx.x; s < nvalid; s += NT) {
            const unsigned p = psort[s];
            if ((unsigned)s < send[p]) ((uint16_t*)dst)[delta[p] + s] = ((const uint16_t*)stage)[s];
          }
          break;
        default:
          for (int s = threadIdx.x; s < nvalid; s += NT) {
            const unsigned p = psort[s];
            if ((unsigned)s < send[p]) ((uint8_t*)dst)[delta[p] + s] = stage[s];
          }
          break;
      }
    }
    if (any_bits && vn < 0) {
      __syncthreads();
#pragma unroll
      for (int k = 0; k < RPT; ++k)
        if (pr[k] != 0xFFFFFFFFu) stage[pr[k] & 0xFFFFu] = (uint8_t)(vb[k >> 2] >> (8 * (k & 3)));
      __syncthreads();
      for (int s = threadIdx.x; s < nvalid; s += NT) {
        const unsigned p = psort[s];
        if ((unsigned)s < send[p]) A.bits[delta[p] + s] = stage[s];
      }
    }
    __syncthreads();
  }
}

// shared-memory bytes of k_part_scatter for a tile of `tile` rows
inline size_t part_scatter_smem(int kw, int tile, int nparts)
{
  (void)kw;
  return (size_t)tile * 8 + (size_t)tile * 2 + (size_t)nparts * 8 + 8 + (size_t)nparts * 8;
}

// Shared-memory find-or-insert; null when the key does not fit (table at its
// fill limit) or is the all-ones key.  Probes take two slots per step for the
// first 64 slots, then continue one slot at a time up to the table size: at
// ~70% fill linear probing's longest runs in a table of a few thousand slots
// pass 64, and a key cut off there would send all its rows of the item to the
// spill list.
// The table has `scap` slots, any count: the start slot is the low 32 hash
// bits scaled to [0, scap) (multiply-shift), so the table can fill all the
// shared memory a CTA has instead of the largest power of two below it.
__device__ __forceinline__ uint8_t* smem_slot(uint8_t* smem, int stride, uint32_t scap, int sfill,
                                              unsigned int* s_used, int words, uint64_t w0,
                                              uint64_t w1, uint64_t h)
{
  uint32_t i = (uint32_t)(((uint64_t)(uint32_t)h * scap) >> 32);
  if (words == 1) {
    if (w0 == kEmpty) return nullptr;
    // two consecutive slots per step, both keys loaded together: a warp
    // runs as many steps as its longest probe, so halving the steps halves
    // the divergent tail.  A key sits at or before the first empty slot of
    // its sequence (no deletions), so an empty first slot is claimed before
    // the second is looked at.
    auto claim = [&](unsigned long long* kp) -> int {  // 1 mine, 0 taken by another key, -1 full
      if (*(volatile unsigned int*)s_used >= (unsigned)sfill) return -1;
      const uint64_t old = atomicCAS(kp, kEmpty, w0);
      if (old == kEmpty) { atomicAdd(s_used, 1u); return 1; }
      return old == w0 ? 1 : 0;
    };
    for (int p = 0; p < 64; p += 2) {
      const uint32_t i1 = i + 1 == scap ? 0 : i + 1;
      unsigned long long* k0p = (unsigned long long*)(smem + (size_t)i * stride);
      unsigned long long* k1p = (unsigned long long*)(smem + (size_t)i1 * stride);
      const uint64_t c0 = *(volatile unsigned long long*)k0p;
      const uint64_t c1 = *(volatile unsigned long long*)k1p;
      if (c0 == w0) return (uint8_t*)k0p;
      if (c0 == kEmpty) {
        const int r = claim(k0p);
        if (r > 0) return (uint8_t*)k0p;
        if (r < 0) return nullptr;
        i = i1;  // taken meanwhile: the sequence continues at the second slot
        continue;
      }
      if (c1 == w0) return (uint8_t*)k1p;
      if (c1 == kEmpty) {
        const int r = claim(k1p);
        if (r > 0) return (uint8_t*)k1p;
        if (r < 0) return nullptr;
      }
      i = i1 + 1 == scap ? 0 : i1 + 1;
    }
    // a run longer than 64 slots (a table near its fill limit): keep walking
    // one slot at a time; below the fill limit an empty slot is always ahead
    for (uint32_t p = 64; p < scap; ++p) {
      unsigned long long* kp = (unsigned long long*)(smem + (size_t)i * stride);
      const uint64_t c = *(volatile unsigned long long*)kp;
      if (c == w0) return (uint8_t*)kp;
      if (c == kEmpty) {
        const int r = claim(kp);
        if (r > 0) return (uint8_t*)kp;
        if (r < 0) return nullptr;
      }
      i = i + 1 == scap ? 0 : i + 1;
    }
    return nullptr;
  }
  // two-word keys: an empty slot has the top bit of its second word set
  // (never set in a packed key); a first word of all ones is a valid key
  // and is matched through the compare-and-swap.  Two slots per step, as for
  // one-word keys.
  unsigned __int128 want = ((unsigned __int128)w1 << 64) | w0;
  const unsigned __int128 empty = ~(unsigned __int128)0;
  // 1: the key's slot, 0: another key's, -1: table at its fill limit
  auto look = [&](unsigned __int128* kp, ulonglong2 cur) -> int {
    if (cur.x == w0 && cur.y == w1 && w0 != kEmpty) return 1;
    if ((cur.y >> 63) || cur.x == kEmpty) {
      if ((cur.y >> 63) && *(volatile unsigned int*)s_used >= (unsigned)sfill) return -1;
      unsigned __int128 old = atomicCAS(kp, empty, want);
      if (old == empty) { atomicAdd(s_used, 1u); return 1; }
      if (old == want) return 1;
    }
    return 0;
  };
  for (int p = 0; p < 64; p += 2) {
    const uint32_t i1 = i + 1 == scap ? 0 : i + 1;
    unsigned __int128* kp0 = (unsigned __int128*)(smem + (size_t)i * stride);
    unsigned __int128* kp1 = (unsigned __int128*)(smem + (size_t)i1 * stride);
    const ulonglong2 c0 = vload2(kp0);
    const ulonglong2 c1 = vload2(kp1);
    // the first slot is settled (ours, or another key's) before the second
    // is looked at; a second slot seen empty is claimed by compare-and-swap
    int r = look(kp0, c0);
    if (r > 0) return (uint8_t*)kp0;
    if (r < 0) return nullptr;
    r = look(kp1, c1);
    if (r > 0) return (uint8_t*)kp1;
    if (r < 0) return nullptr;
    i = i1 + 1 == scap ? 0 : i1 + 1;
  }
  // longer runs: one slot at a time, as for one-word keys
  for (uint32_t p = 64; p < scap; ++p) {
    unsigned __int128* kp = (unsigned __int128*)(smem + (size_t)i * stride);
    const int r = look(kp, vload2(kp));
    if (r > 0) return (uint8_t*)kp;
    if (r < 0) return nullptr;
    i = i + 1 == scap ? 0 : i + 1;
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

// MIN/MAX updates that skip the shared reduction when a plain read of the
// field shows the value cannot change it.  A MIN field only decreases and a
// MAX field only increases, so a stale read can let a useless update through
// but never drops a needed one; on this architecture the 64-bit reductions
// are compare-and-swap loops, and after a group's first rows most values no
// longer improve its MIN or MAX.
__device__ __forceinline__ void smin_u64(uint32_t a, uint64_t v) { if (v < sld_u64(a)) sred_min_u64(a, v); }
__device__ __forceinline__ void smax_u64(uint32_t a, uint64_t v) { if (v > sld_u64(a)) sred_max_u64(a, v); }
__device__ __forceinline__ void smin_u32(uint32_t a, uint32_t v) { if (v < sld_u32(a)) sred_min_u32(a, v); }
__device__ __forceinline__ void smax_u32(uint32_t a, uint32_t v) { if (v > sld_u32(a)) sred_max_u32(a, v); }

// Rows whose key did not fit their partition's shared table (a partition
// with more groups than the sample predicted) are listed by pass 2 and
// applied to the global spill table afterwards by k_part_spill, so the hot
// loop carries no call into the generic update code.  The list count lives in
// counters[12]; counters[13] is set when the list itself overflowed (the host
// then re-runs pass 2 with a longer list).
template <bool RAW = false>
__global__ void __launch_bounds__(256) k_part_spill(const __grid_constant__ Plan P2, TableRef G,
                                                    const __grid_constant__ PartArgs A)
{
  __shared__ unsigned int s_new;
  if (threadIdx.x == 0) s_new = 0;
  __syncthreads();
  const unsigned cnt = min(*(volatile unsigned int*)(A.counters + 12), A.spill_cap);
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += gridDim.x * blockDim.x) {
    const int64_t r = A.spill_rows[i];
    uint64_t w0, w1;
    if (RAW) {
      if (!pack_key(P2, r, w0, w1)) continue;  // not listed: null keys are skipped first
    } else {
      w0 = P2.packed_keys[r * P2.key_words];
      w1 = P2.key_words == 2 ? P2.packed_keys[r * 2 + 1] : 0;
    }
    const uint64_t h = hash_key(w0, w1, P2.key_words);
    const int64_t gi = global_slot(P2, G, w0, w1, h, &s_new);
    if (gi < 0) {
      atomicOr(G.counters + 1, 1u);
      continue;
    }
    update_slot(P2, G.T + gi * (int64_t)G.stride, r);
  }
  __syncthreads();
  if (threadIdx.x == 0 && s_new) atomicAdd(G.counters, s_new);
}

// ---- pass 2 ----
// Per-item prologue: claim a work item, reset the shared table (`scap`
// slots plus, for one-word keys, the slot of the all-ones key).  Returns the
// item index (>= nitems: no work left).
template <int NT>
__device__ __forceinline__ int p2_claim(const PartArgs& A, uint8_t* smem, int scap, int nw,
                                        const SlotTemplate& tmpl, int* s_part, unsigned int* s_used,
                                        unsigned int* s_spill)
{
  if (threadIdx.x == 0) {
    *s_part = (int)atomicAdd(A.work, 1u);
    *s_used = 0;
    *s_spill = 0;
  }
  // word by word: every thread reads the same template word (no divergent
  // parameter loads, no division by the slot width)
  for (int w = 0; w < nw; ++w) {
    const unsigned long long t = tmpl.w[w];
    for (int s = threadIdx.x; s < scap; s += NT) *(unsigned long long*)(smem + ((size_t)s * nw + w) * 8) = t;
  }
  __syncthreads();
  return *s_part;
}

// Per-partition epilogue: the partition's groups leave as dense slots, or are
// merged into the global spill table when some of its rows went there.  The
// all-ones key's slot (one-word keys; it cannot be told from an empty slot)
// is always merged into the global table's dedicated slot.
template <int NT, typename ScanT>
__device__ __forceinline__ void p2_flush(const Plan& P2, const TableRef& G, const DenseRef& D,
                                         const uint8_t* smem, int scap, bool spilled,
                                         typename ScanT::TempStorage& scan_tmp,
                                         unsigned long long* s_base, unsigned int* s_new)
{
  const int stride = G.stride;
  const int nw = stride / 8;
  if (P2.key_words == 1 && threadIdx.x == 0) {
    const uint8_t* sp = smem + (size_t)scap * stride;
    if (*(const uint32_t*)(sp + P2.rows_off) > 0) merge_slot(P2, G, sp, s_new);
  }
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

// Combines `v` over the lanes of `grp` (lanes sharing one slot); the result
// is meaningful at the group's lowest lane.  A whole-warp group (one hot key)
// folds in five butterfly steps, other groups through one shuffle per member.
template <typename T, typename F>
__device__ __forceinline__ T grp_reduce(unsigned grp, T v, F op)
{
  if (grp == 0xFFFFFFFFu) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = op(v, __shfl_xor_sync(0xFFFFFFFFu, v, o));
    return v;
  }
  unsigned rest = grp & (grp - 1);
  T acc = v;
  while (rest) {
    const int src = __ffs(rest) - 1;
    rest &= rest - 1;
    acc = op(acc, __shfl_sync(grp, v, src));
  }
  return acc;
}

// One value column of a chunk of R rows per thread (values already loaded),
// with the column's type fixed at compile time: each accumulator present
// (sum, min, max, sum of squares) is one shared-memory reduction per row.
// `ok` = 0 marks rows that are absent, null in this column, or were listed
// as spills.
// With WAGG, lanes whose rows hit the same slot (`peers`, from one match per
// row) first combine their values in registers and the group's lowest lane
// makes the single shared update: rows of one hot key no longer queue on one
// shared address (64-bit and floating-point shared reductions are
// compare-and-swap loops on this architecture, which such contention makes
// retry up to 32 times).
template <int CAT, int W, int R, int MAXV, bool WAGG>
__device__ __forceinline__ void p2_column(const ValCol& c, const uint32_t (&sa)[R], const uint32_t (&ok)[R],
                                          const uint64_t (&xv)[R][MAXV], int v, const unsigned (&peers)[R])
{
  // the caller rotates its preloaded values: this column's are element 0
  (void)v;
  uint64_t x[R];
#pragma unroll
  for (int j = 0; j < R; ++j) x[j] = xv[j][0];
  const int so = c.sum_off, mo = c.min_off, xo = c.max_off, qo = c.sq_off;
  const bool sum32 = c.sum_op == OP_SUM_I32;
  bool grouped[R];
#pragma unroll
  for (int j = 0; j < R; ++j) grouped[j] = false;
  if (WAGG) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int j = 0; j < R; ++j) {
      const unsigned grp = peers[j] & __ballot_sync(0xFFFFFFFFu, ok[j] != 0);
      if (!ok[j] || __popc(grp) == 1) continue;  // singles take the plain path below
      grouped[j] = true;
      const bool lead = lane == __ffs(grp) - 1;
      const uint32_t a = sa[j];
      auto add64 = [](uint64_t p, uint64_t q) { return p + q; };
      auto min64 = [](uint64_t p, uint64_t q) { return p < q ? p : q; };
      auto max64 = [](uint64_t p, uint64_t q) { return p > q ? p : q; };
      auto min32 = [](uint32_t p, uint32_t q) { return p < q ? p : q; };
      auto max32 = [](uint32_t p, uint32_t q) { return p > q ? p : q; };
      if (CAT == CAT_F64) {
        const double d = __longlong_as_double((long long)x[j]);
        if (so >= 0) { const double t = grp_reduce(grp, d, [](double p, double q) { return p + q; }); if (lead) sred_add_f64(a + so, t); }
        if (mo >= 0) { const uint64_t t = grp_reduce(grp, ord64_f(d, true), min64); if (lead) smin_u64(a + mo, t); }
        if (xo >= 0) { const uint64_t t = grp_reduce(grp, ord64_f(d, false), max64); if (lead) smax_u64(a + xo, t); }
        if (qo >= 0) { const double t = grp_reduce(grp, d * d, [](double p, double q) { return p + q; }); if (lead) sred_add_f64(a + qo, t); }
      } else if (CAT == CAT_F32) {
        const float f = __uint_as_float((uint32_t)x[j]);
        if (so >= 0) { const float t = grp_reduce(grp, f, [](float p, float q) { return p + q; }); if (lead) sred_add_f32(a + so, t); }
        if (mo >= 0) { const uint32_t t = grp_reduce(grp, ord32_f(f, true), min32); if (lead) smin_u32(a + mo, t); }
        if (xo >= 0) { const uint32_t t = grp_reduce(grp, ord32_f(f, false), max32); if (lead) smax_u32(a + xo, t); }
        if (qo >= 0) { const float t = grp_reduce(grp, f * f, [](float p, float q) { return p + q; }); if (lead) sred_add_f32(a + qo, t); }
      } else {
        int64_t iv;
        if (CAT == CAT_SIGNED) iv = W == 8 ? (int64_t)x[j] : W == 4 ? (int64_t)(int32_t)x[j]
                                          : W == 2 ? (int64_t)(int16_t)x[j] : (int64_t)(int8_t)x[j];
        else if (CAT == CAT_BOOL) iv = x[j] != 0;
        else iv = (int64_t)x[j];
        if (so >= 0) {
          const uint64_t t = grp_reduce(grp, (uint64_t)iv, add64);  // wrapping, as the atomics
          if (lead) {
            if (sum32) sred_add_u32(a + so, (uint32_t)t);
            else sred_add_u64(a + so, t);
          }
        }
        if (W == 8) {
          const uint64_t o = CAT == CAT_SIGNED ? ((uint64_t)iv ^ 0x8000000000000000ull) : (uint64_t)iv;
          if (mo >= 0) { const uint64_t t = grp_reduce(grp, o, min64); if (lead) smin_u64(a + mo, t); }
          if (xo >= 0) { const uint64_t t = grp_reduce(grp, o, max64); if (lead) smax_u64(a + xo, t); }
        } else {
          const uint32_t o = CAT == CAT_SIGNED ? ((uint32_t)(int32_t)iv ^ 0x80000000u) : (uint32_t)iv;
          if (mo >= 0) { const uint32_t t = grp_reduce(grp, o, min32); if (lead) smin_u32(a + mo, t); }
          if (xo >= 0) { const uint32_t t = grp_reduce(grp, o, max32); if (lead) smax_u32(a + xo, t); }
        }
        if (qo >= 0) {
          const uint64_t t = grp_reduce(grp, (uint64_t)iv * (uint64_t)iv, add64);
          if (lead) sred_add_u64(a + qo, t);
        }
      }
    }
  }
#pragma unroll
  for (int j = 0; j < R; ++j) {
    if (!ok[j] || grouped[j]) continue;
    const uint32_t a = sa[j];
    if (CAT == CAT_F64) {
      const double d = __longlong_as_double((long long)x[j]);
      if (so >= 0) sred_add_f64(a + so, d);
      if (mo >= 0) smin_u64(a + mo, ord64_f(d, true));
      if (xo >= 0) smax_u64(a + xo, ord64_f(d, false));
      if (qo >= 0) sred_add_f64(a + qo, d * d);
    } else if (CAT == CAT_F32) {
      const float f = __uint_as_float((uint32_t)x[j]);
      if (so >= 0) sred_add_f32(a + so, f);
      if (mo >= 0) smin_u32(a + mo, ord32_f(f, true));
      if (xo >= 0) smax_u32(a + xo, ord32_f(f, false));
      if (qo >= 0) sred_add_f32(a + qo, f * f);
    } else {
      // integers: sign- or zero-extended to 64 bits; min/max in the
      // order-preserving unsigned encoding of the slot's width
      int64_t iv;
      if (CAT == CAT_SIGNED) iv = W == 8 ? (int64_t)x[j] : W == 4 ? (int64_t)(int32_t)x[j]
                                        : W == 2 ? (int64_t)(int16_t)x[j] : (int64_t)(int8_t)x[j];
      else if (CAT == CAT_BOOL) iv = x[j] != 0;
      else iv = (int64_t)x[j];
      if (so >= 0) {
        if (sum32) sred_add_u32(a + so, (uint32_t)iv);
        else sred_add_u64(a + so, (uint64_t)iv);
      }
      if (W == 8) {
        const uint64_t o = CAT == CAT_SIGNED ? ((uint64_t)iv ^ 0x8000000000000000ull) : (uint64_t)iv;
        if (mo >= 0) smin_u64(a + mo, o);
        if (xo >= 0) smax_u64(a + xo, o);
      } else {
        const uint32_t o = CAT == CAT_SIGNED ? ((uint32_t)(int32_t)iv ^ 0x80000000u) : (uint32_t)iv;
        if (mo >= 0) smin_u32(a + mo, o);
        if (xo >= 0) smax_u32(a + xo, o);
      }
      if (qo >= 0) sred_add_u64(a + qo, (uint64_t)iv * (uint64_t)iv);
    }
  }
}

// Pass 2.  P2 is the plan with value columns redirected to the partitioned
// arrays (offset 0, `bits` validity) and packed_keys set.  One CTA owns a
// partition at a time and aggregates it in a shared-memory table.  Rows are
// taken in chunks of R per thread: the chunk's keys are placed in the table
// (the next chunk's keys and validity bytes are loaded meanwhile, and the
// chunk after that is prefetched into L2, each thread owning one fixed
// 128-byte line of the key, value and validity arrays), then the columns are
// applied one at a time, each through code specialised for its type, so the
// per-type dispatch happens once per column and chunk instead of per row.
//
// With RAW the rows are the caller's own columns (P2 is the plan itself):
// keys are packed per row, values read at their column offsets and validity
// taken from the null masks; each item is a row range whose table is merged
// into the global table.  This is the shared-stage mode for groups that fit
// one CTA's table.
template <int KW, int R, int NT, int MAXV, bool WAGG, bool RAW = false>
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
  const bool have_bits = A.bits != nullptr;
  const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(smem);
  const int nv = P2.num_vals;
  constexpr int64_t STEP = (int64_t)R * NT;
  // this thread's prefetch line: array base, bytes per row, byte offset in a step
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
    if (!RAW) {
      take(P2.packed_keys, 8 * KW);
      for (int v = 0; v < nv; ++v) take(P2.vals[v].data, P2.vals[v].width);
      if (have_bits) take(A.bits, 1);
    }
  }
  for (;;) {
    const int it = p2_claim<NT>(A, smem, scap + (KW == 1), nw, tmpl, &s_part, &s_used, &s_spill);
    if (it >= A.nitems) break;
    const PartItem item = A.items[it];
    const int64_t b = item.begin;
    const int64_t e = RAW ? item.end : min(item.end, min((int64_t)A.cursor[item.part], A.end[item.part]));
    auto load_keys = [&](int64_t r0, uint64_t (&k0)[R], uint64_t (&k1)[R], uint32_t (&vb)[R]) {
#pragma unroll
      for (int j = 0; j < R; ++j) {
        const int64_t r = r0 + (int64_t)j * NT + threadIdx.x;
        k0[j] = kEmpty;
        k1[j] = 0;
        vb[j] = 0xFFFFFFFFu;
        if (r < e) {
          if (RAW) {
            // the caller's columns: a row whose key is null under EXCLUDE
            // takes no part (vb = 0 marks it); validity bits from the masks
            uint64_t w0, w1;
            if (!pack_key(P2, r, w0, w1)) {
              vb[j] = 0;
              k0[j] = kEmpty;
              continue;
            }
            k0[j] = w0;
            k1[j] = w1;
            uint32_t bits = 0;
#pragma unroll
            for (int v = 0; v < MAXV; ++v)
              if (v < nv && bit_valid(P2.vals[v].mask, r + P2.vals[v].offset)) bits |= 1u << v;
            vb[j] = bits | 0x80000000u;
          } else {
            if (KW == 1) k0[j] = __ldg(P2.packed_keys + r);
            else {
              const ulonglong2 kk = __ldg((const ulonglong2*)(P2.packed_keys + 2 * r));
              k0[j] = kk.x;
              k1[j] = kk.y;
            }
            if (have_bits) vb[j] = __ldg(A.bits + r);
          }
        }
      }
    };
    uint64_t k0[R], k1[R];
    uint32_t vb[R];
    load_keys(b, k0, k1, vb);
    const int64_t pf_end = e * pf_w;
    for (int64_t r0 = b; r0 < e; r0 += STEP) {
      if (pf_base) {
        const int64_t at = (r0 + 2 * STEP) * pf_w + pf_off;
        if (at < pf_end) prefetch_l2(pf_base + at);
      }
      // place this chunk's rows
      uint32_t sa[R];
      int64_t row[R];
#pragma unroll
      for (int j = 0; j < R; ++j) {
        row[j] = r0 + (int64_t)j * NT + threadIdx.x;
        sa[j] = 0;
        if (row[j] >= e) continue;
        if (RAW && vb[j] == 0) continue;  // null key, EXCLUDE
        const uint64_t h = hash_key(k0[j], k1[j], KW);
        uint8_t* slot = (KW == 1 && k0[j] == kEmpty)
                          ? smem + (size_t)scap * stride
                          : smem_slot(smem, stride, (uint32_t)scap, sfill, &s_used, KW, k0[j], k1[j], h);
        if (slot == nullptr) {
          // listed for the global table; one list reservation per warp
          s_spill = 1;
          const unsigned mates = __activemask();
          const int leader = __ffs(mates) - 1;
          const int lane = threadIdx.x & 31;
          unsigned at = 0;
          if (lane == leader) at = atomicAdd(A.counters + 12, (unsigned)__popc(mates));
          at = __shfl_sync(mates, at, leader) + __popc(mates & ((1u << lane) - 1));
          if (at < A.spill_cap) A.spill_rows[at] = row[j];
          else atomicOr(A.counters + 13, 1u);
          continue;
        }
        sa[j] = sbase + (uint32_t)(slot - smem);
      }
      // lanes sharing a slot (WAGG): one match per row; rows counted by the
      // group's lowest lane
      unsigned peers[R];
#pragma unroll
      for (int j = 0; j < R; ++j) {
        peers[j] = 1u << (threadIdx.x & 31);
        if (WAGG) peers[j] = __match_any_sync(0xFFFFFFFFu, sa[j] ? sa[j] : (0x80000000u | (threadIdx.x & 31)));
        if (!sa[j]) continue;
        if (!WAGG) sred_add_u32(sa[j] + P2.rows_off, 1u);
        else if ((threadIdx.x & 31) == __ffs(peers[j]) - 1) sred_add_u32(sa[j] + P2.rows_off, __popc(peers[j]));
      }
      uint32_t cur_vb[R];
#pragma unroll
      for (int j = 0; j < R; ++j) cur_vb[j] = vb[j];
      // every column's values of this chunk, and the next chunk's keys, in
      // flight together
      uint64_t xv[R][MAXV];
#pragma unroll
      for (int j = 0; j < R; ++j) {
#pragma unroll
        for (int v = 0; v < MAXV; ++v) {
          xv[j][v] = 0;
          if (v < nv && sa[j] && ((cur_vb[j] >> v) & 1))
            xv[j][v] = load_bits(P2.vals[v].data, row[j] + (RAW ? P2.vals[v].offset : 0), P2.vals[v].width);
        }
      }
      load_keys(r0 + STEP, k0, k1, vb);
      // one copy of the per-type column code, looped over the columns (each
      // column's preloaded values are rotated into element 0 of the register
      // array after the previous column), keeps the kernel small enough for
      // the instruction cache
#pragma unroll 1
      for (int v = 0; v < MAXV; ++v) {
        if (v >= nv) break;
        const ValCol& c = P2.vals[v];
        uint32_t ok[R];
#pragma unroll
        for (int j = 0; j < R; ++j) {
          const bool valid = (cur_vb[j] >> v) & 1;
          ok[j] = sa[j] != 0 && valid;
          if (WAGG) {
            const unsigned ng = peers[j] & __ballot_sync(0xFFFFFFFFu, sa[j] != 0 && !valid);
            if (sa[j] != 0 && !valid && c.nulls_off >= 0 && (threadIdx.x & 31) == __ffs(ng) - 1)
              sred_add_u32(sa[j] + c.nulls_off, __popc(ng));
          } else if (sa[j] != 0 && !valid && c.nulls_off >= 0) {
            sred_add_u32(sa[j] + c.nulls_off, 1u);
          }
        }
        switch ((c.cat << 4) | c.width) {
          case (CAT_F64 << 4) | 8: p2_column<CAT_F64, 8, R, MAXV, WAGG>(c, sa, ok, xv, v, peers); break;
          case (CAT_F32 << 4) | 4: p2_column<CAT_F32, 4, R, MAXV, WAGG>(c, sa, ok, xv, v, peers); break;
          case (CAT_SIGNED << 4) | 8: p2_column<CAT_SIGNED, 8, R, MAXV, WAGG>(c, sa, ok, xv, v, peers); break;
          case (CAT_SIGNED << 4) | 4: p2_column<CAT_SIGNED, 4, R, MAXV, WAGG>(c, sa, ok, xv, v, peers); break;
          case (CAT_SIGNED << 4) | 2: p2_column<CAT_SIGNED, 2, R, MAXV, WAGG>(c, sa, ok, xv, v, peers); break;
          case (CAT_SIGNED << 4) | 1: p2_column<CAT_SIGNED, 1, R, MAXV, WAGG>(c, sa, ok, xv, v, peers); break;
          case (CAT_UNSIGNED << 4) | 8: p2_column<CAT_UNSIGNED, 8, R, MAXV, WAGG>(c, sa, ok, xv, v, peers); break;
          case (CAT_UNSIGNED << 4) | 4: p2_column<CAT_UNSIGNED, 4, R, MAXV, WAGG>(c, sa, ok, xv, v, peers); break;
          case (CAT_UNSIGNED << 4) | 2: p2_column<CAT_UNSIGNED, 2, R, MAXV, WAGG>(c, sa, ok, xv, v, peers); break;
          case (CAT_UNSIGNED << 4) | 1: p2_column<CAT_UNSIGNED, 1, R, MAXV, WAGG>(c, sa, ok, xv, v, peers); break;
          default: p2_column<CAT_BOOL, 1, R, MAXV, WAGG>(c, sa, ok, xv, v, peers); break;
        }
        // next column's values to element 0 (register moves, no indexed selection)
#pragma unroll
        for (int j = 0; j < R; ++j) {
#pragma unroll
          for (int u = 0; u + 1 < MAXV; ++u) xv[j][u] = xv[j][u + 1];
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
