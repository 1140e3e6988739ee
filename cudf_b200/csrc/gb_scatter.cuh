// gb_scatter.cuh -- pass 1 of the partitioned path with bulk-copy staging.
//
// Each CTA takes tiles of T rows.  One thread stages a whole tile into shared
// memory with cp.async.bulk (global -> shared, completion counted in bytes on
// an mbarrier): every key column, every value column and every validity mask
// the plan reads, each as one contiguous copy (the tile's rows of a column are
// contiguous in HBM).  From the staged tile the threads then
//   A  pack each row's key, take the top hash bits as partition and the rank
//      within the tile's partition from a shared histogram;
//   B  reserve each (tile, partition) run in its region (one global atomic per
//      partition present) and scan the histogram;
//   C  write the packed keys at their sorted position, and the inverse
//      permutation (sorted position -> row) with each position's partition;
//   D  write every output array of the tile in sorted order: consecutive
//      threads write consecutive rows of a run, the values gathered from the
//      staged columns, so no column needs a barrier of its own.
// The staged arrays form two groups, each completing on its own mbarrier: the
// key group (key columns and their masks, read only by A) and the value group
// (value columns and their masks, read only by D).  The next tile's key group
// is copied in as soon as A is done with this tile's, so it lands during B-D;
// the next tile's value group as soon as D is done, so it lands during the
// next tile's A-C.  Tiles are 16-byte aligned only when every staged column
// starts on a suitable row (see part_scatter_bulk_ok); the last, partial tile
// is staged with plain loads.
//
// Waits on the mbarrier are bounded: a copy that has not landed after the
// limit sets counters[14] (the host reports a CUDA error) and the CTA stops
// after waiting, again bounded, for its copies in flight.
#pragma once
#include <cub/block/block_scan.cuh>

#include <cstring>

#include "gb_partition.cuh"

namespace gb {

constexpr int kMaxStaged = 2 * (kMaxKeyCols + 8);

// Arrays a tile stages: data columns (bytes per row = width) and validity
// masks (one bit per row).  src points at the column's row 0 (offset applied;
// masks: the word holding row 0, whose bit 0 is row 0).
struct StageSpec {
  int32_t narr;
  int32_t key_data[kMaxKeyCols];  // staged array of key column k
  int32_t key_mask[kMaxKeyCols];  // its mask array, or -1
  int32_t val_data[8];
  int32_t val_mask[8];
  const uint8_t* src[kMaxStaged];
  int32_t width[kMaxStaged];      // bytes per row; 0 for a mask
  int32_t soff[kMaxStaged];       // byte offset in shared memory
  int32_t group[kMaxStaged];      // 0: read by the key phase (keys, key masks), 1: by the write-out
  int32_t stage_bytes;            // all arrays of one tile, with their alignment
  int32_t tx_bytes[2];            // bytes a full tile's copies of each group deliver
  int32_t tile_rows;              // rows per tile the layout was made for
  int32_t key8;                   // one 8-byte integer key column without a mask:
                                  // its staged value is the packed key
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes)
{
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// Waits for phase `parity` of the barrier to complete; false after `limit` tries.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity, int limit)
{
  for (int i = 0; i < limit; ++i) {
    unsigned done;
    asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(done)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
    if (done) return true;
  }
  return false;
}
// Global -> shared bulk copy of `bytes` (multiple of 16; both addresses
// 16-byte aligned), counted on `bar`.  The source is this GPU's memory.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar)
{
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                 smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void fence_async_shared() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Staged element / validity of a row of the tile.
__device__ __forceinline__ uint64_t staged_bits(const uint8_t* a, int w, int row)
{
  switch (w) {
    case 1: return a[row];
    case 2: return ((const uint16_t*)a)[row];
    case 4: return ((const uint32_t*)a)[row];
    default: return ((const uint64_t*)a)[row];
  }
}
__device__ __forceinline__ bool staged_valid(const uint8_t* m, int row)
{
  return (((const uint32_t*)m)[row >> 5] >> (row & 31)) & 1u;
}

// Copies the staged elements rows[k] of one column to their destinations
// dst[g[k]] (g < 0: nothing to write).
template <typename W, int RPT>
__device__ __forceinline__ void scatter_col(void* dst, const uint8_t* src, const int64_t (&g)[RPT],
                                            const int (&rows)[RPT])
{
#pragma unroll
  for (int k = 0; k < RPT; ++k)
    if (g[k] >= 0) ((W*)dst)[g[k]] = ((const W*)src)[rows[k]];
}

// Packs the key of staged row `row` (as pack_key does from HBM).
__device__ __forceinline__ bool pack_key_staged(const Plan& P, const StageSpec& S, const uint8_t* sm, int row,
                                                uint64_t& w0, uint64_t& w1)
{
  w0 = 0;
  w1 = 0;
#pragma unroll 1
  for (int k = 0; k < P.num_keys; ++k) {
    const KeyCol& c = P.keys[k];
    if (S.key_mask[k] >= 0 && !staged_valid(sm + S.soff[S.key_mask[k]], row)) {
      if (!P.include_nulls) return false;
      const uint64_t nb = 1ull << c.null_shift;
      if (c.null_word == 0) w0 |= nb;
      else w1 |= nb;
      continue;
    }
    uint64_t b = staged_bits(sm + S.soff[S.key_data[k]], c.width, row);
    if (c.cat == CAT_F32) {
      const float f = __uint_as_float((uint32_t)b);
      b = f != f ? 0x7FC00000u : (f == 0.0f ? 0 : b);
    } else if (c.cat == CAT_F64) {
      const double d = __longlong_as_double((long long)b);
      b = d != d ? 0x7FF8000000000000ull : (d == 0.0 ? 0 : b);
    } else if (c.cat == CAT_BOOL) {
      b = b != 0;
    }
    if (c.word == 0) w0 |= b << c.shift;
    else w1 |= b << c.shift;
  }
  return true;
}

// Shared memory of k_part_scatter_bulk: staged tile | sorted keys (8*KW per
// row) | order u16[T] | psort u16[T] | hist u32[nparts] | send u32[nparts] |
// delta i64[nparts]
inline size_t part_scatter_bulk_smem(const StageSpec& S, int kw, int T, int nparts)
{
  auto a16 = [](size_t x) { return (x + 15) & ~(size_t)15; };
  size_t b = a16((size_t)S.stage_bytes);
  b += a16((size_t)T * 8 * kw);
  b += a16((size_t)T * 2) * 2;
  b += a16((size_t)nparts * 4) * 2;
  b += (size_t)nparts * 8;
  return b;
}

template <int KW, int NT, int T, int MINB>
__global__ void __launch_bounds__(NT, MINB) k_part_scatter_bulk(const __grid_constant__ Plan P,
                                                             const __grid_constant__ PartArgs A,
                                                             const __grid_constant__ StageSpec S)
{
  static_assert(T % 128 == 0 && T % NT == 0 && T <= 65536, "tile rows");
  constexpr int RPT = T / NT;
  extern __shared__ __align__(128) uint8_t sm[];
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ unsigned int s_valid, s_stop;
  using Scan = cub::BlockScan<unsigned, NT>;
  __shared__ typename Scan::TempStorage scan_tmp;
  auto a16 = [](size_t x) { return (x + 15) & ~(size_t)15; };
  size_t off = a16((size_t)S.stage_bytes);
  uint64_t* kst = (uint64_t*)(sm + off);
  off += a16((size_t)T * 8 * KW);
  uint16_t* order = (uint16_t*)(sm + off);
  off += a16((size_t)T * 2);
  uint16_t* psort = (uint16_t*)(sm + off);
  off += a16((size_t)T * 2);
  unsigned int* hist = (unsigned int*)(sm + off);
  off += a16((size_t)A.nparts * 4);
  unsigned int* send = (unsigned int*)(sm + off);
  off += a16((size_t)A.nparts * 4);
  long long* delta = (long long*)(sm + off);
  const int64_t n = P.num_rows;
  const int64_t ntiles = (n + T - 1) / T;
  const int nv = P.num_vals;
  const bool any_bits = A.bits != nullptr;
  const int per = (A.nparts + NT - 1) / NT;
  constexpr int kWaitLimit = 1 << 22;
  if (threadIdx.x == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    s_stop = 0;
  }
  __syncthreads();
  // one thread issues the copies of a full tile's group g
  auto issue = [&](int g, int64_t t0) {
    mbar_expect_tx(&bar[g], (unsigned)S.tx_bytes[g]);
#pragma unroll 1
    for (int a = 0; a < S.narr; ++a) {
      if (S.group[a] != g) continue;
      const int w = S.width[a];
      const uint8_t* src = w ? S.src[a] + t0 * w : S.src[a] + (t0 >> 3);
      bulk_g2s(sm + S.soff[a], src, w ? (unsigned)(T * w) : (unsigned)(T / 8), &bar[g]);
    }
  };
  // plain loads of group g of a partial tile into the same layout
  auto plain = [&](int g, int64_t t0, int cnt) {
#pragma unroll 1
    for (int a = 0; a < S.narr; ++a) {
      if (S.group[a] != g) continue;
      const int w = S.width[a];
      uint8_t* d = sm + S.soff[a];
      if (w) {
        for (int i = threadIdx.x; i < cnt; i += NT) {
          const uint8_t* s = S.src[a] + (t0 + i) * w;
          switch (w) {
            case 1: d[i] = __ldg(s); break;
            case 2: ((uint16_t*)d)[i] = __ldg((const uint16_t*)s); break;
            case 4: ((uint32_t*)d)[i] = __ldg((const uint32_t*)s); break;
            default: ((uint64_t*)d)[i] = __ldg((const unsigned long long*)s); break;
          }
        }
      } else {
        const uint32_t* s = (const uint32_t*)(S.src[a] + (t0 >> 3));
        for (int i = threadIdx.x; i < (cnt + 31) / 32; i += NT) ((uint32_t*)d)[i] = __ldg(s + i);
      }
    }
  };
  unsigned phase[2] = {0, 0};
  bool pending[2] = {false, false};  // thread 0's view: copies issued, not yet waited for
  auto wait_group = [&](int g) {
    if (mbar_wait(&bar[g], phase[g], kWaitLimit)) {
      phase[g] ^= 1;
      pending[g] = false;
    } else {  // still in flight: reported, and waited for again before exit
      atomicOr(A.counters + 14, 1u);
      s_stop = 1;
    }
  };
  int64_t tile = blockIdx.x;
  if (threadIdx.x == 0 && tile < ntiles && (tile + 1) * T <= n) {
    issue(0, tile * T);
    issue(1, tile * T);
  }
  pending[0] = pending[1] = tile < ntiles && (tile + 1) * T <= n;
  for (; tile < ntiles; tile += gridDim.x) {
    const int64_t t0 = tile * T;
    const int cnt = (int)min((int64_t)T, n - t0);
    const int64_t nt = tile + gridDim.x;
    const bool next_full = nt < ntiles && (nt + 1) * T <= n;
    for (int i = threadIdx.x; i < A.nparts; i += NT) hist[i] = 0;
    if (cnt == T) {
      wait_group(0);  // issued one tile earlier, after A
    } else {
      plain(0, t0, cnt);
      plain(1, t0, cnt);
    }
    __syncthreads();
    if (s_stop) break;
    // A: partition and rank of every row (packed keys kept in registers)
    uint32_t pr[RPT];
    uint64_t kw0[RPT], kw1[KW == 2 ? RPT : 1];
    const uint64_t* k8 = (KW == 1 && S.key8) ? (const uint64_t*)(sm + S.soff[S.key_data[0]]) : nullptr;
#pragma unroll
    for (int k = 0; k < RPT; ++k) {
      const int i = k * NT + threadIdx.x;
      pr[k] = 0xFFFFFFFFu;
      uint64_t w0 = 0, w1 = 0;
      if (i < cnt && (k8 ? (w0 = k8[i], true) : pack_key_staged(P, S, sm, i, w0, w1))) {
        const unsigned p = (unsigned)(hash_key(w0, w1, KW) >> A.shift);
        pr[k] = (p << 16) | atomicAdd(&hist[p], 1u);
      }
      kw0[k] = w0;
      if (KW == 2) kw1[k] = w1;
    }
    __syncthreads();
    // the key group is free: the next full tile's keys land during B-D
    if (next_full) {
      if (threadIdx.x == 0) {
        fence_async_shared();
        issue(0, nt * T);
      }
      pending[0] = true;
    }
    // B: the tile's positions (exclusive scan of the histogram) and one
    // reservation per partition present on its region cursor.  With at most
    // four partitions per thread the reservations are issued before the scan
    // and their results are first used after C, so their round trip to L2
    // overlaps the scan and the placement of the keys; with more, each is
    // used as it returns.
    const int q0 = threadIdx.x * per;
    const int qe = min(A.nparts, q0 + per);
    const bool early = per <= 4;
    unsigned long long g4[4];
    unsigned mine = 0;
    if (early) {
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int q = q0 + j;
        const unsigned h = q < qe ? hist[q] : 0u;
        g4[j] = h ? atomicAdd(&A.cursor[q], (unsigned long long)h) : 0ull;
        mine += h;
      }
    } else {
      for (int qa = q0; qa < qe; qa += 4) {
        unsigned h[4];
        unsigned long long g[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int q = qa + j;
          h[j] = q < qe ? hist[q] : 0u;
          g[j] = h[j] ? atomicAdd(&A.cursor[q], (unsigned long long)h[j]) : 0ull;
          mine += h[j];
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int q = qa + j;
          if (!h[j]) continue;
          const long long room = (long long)A.end[q] - (long long)g[j];
          if ((long long)h[j] > room) atomicOr(A.counters + 5, 1u);
          delta[q] = (long long)g[j];
          send[q] = room <= 0 ? 0u : (unsigned)min((long long)h[j], room);
        }
      }
    }
    unsigned pre, total;
    Scan(scan_tmp).ExclusiveSum(mine, pre, total);
    if (early) {
      for (int q = q0; q < qe; ++q) {
        const unsigned h = hist[q];
        hist[q] = pre;
        pre += h;
      }
    } else {
      for (int q = q0; q < qe; ++q) {
        const unsigned h = hist[q];
        if (h) {
          delta[q] -= (long long)pre;
          send[q] += pre;
        }
        hist[q] = pre;
        pre += h;
      }
    }
    if (threadIdx.x == 0) s_valid = total;
    __syncthreads();
    // C: sorted positions; packed keys at their position
#pragma unroll
    for (int k = 0; k < RPT; ++k) {
      if (pr[k] == 0xFFFFFFFFu) continue;
      const int i = k * NT + threadIdx.x;
      const unsigned p = pr[k] >> 16;
      const unsigned s = hist[p] + (pr[k] & 0xFFFFu);
      order[s] = (uint16_t)i;
      psort[s] = (uint16_t)p;
      kst[KW * s] = kw0[k];
      if (KW == 2) kst[2 * s + 1] = kw1[k];
    }
    // the early reservations have returned by now: destinations and bounds
    // per partition (read by D after the next barrier); a partition's tile
    // position and row count come back from the scanned histogram
    if (early) {
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int q = q0 + j;
        if (q >= qe) break;
        const unsigned pq = hist[q];
        const unsigned h = (q + 1 < A.nparts ? hist[q + 1] : s_valid) - pq;
        if (!h) continue;
        const long long room = (long long)A.end[q] - (long long)g4[j];
        if ((long long)h > room) atomicOr(A.counters + 5, 1u);
        delta[q] = (long long)g4[j] - (long long)pq;
        send[q] = pq + (room <= 0 ? 0u : (unsigned)min((long long)h, room));
      }
    }
    if (cnt == T) wait_group(1);  // issued after the previous tile's write-out
    __syncthreads();
    if (s_stop) break;
    // D: every output array in sorted order.  Each thread keeps the
    // destination and the staged row of its sorted positions in registers and
    // writes the columns one at a time, so the width dispatch is taken once
    // per column instead of once per row.
    const int nvalid = (int)s_valid;
    int64_t gdst[RPT];
    int srow[RPT];
    uint32_t vb[RPT];
#pragma unroll
    for (int k = 0; k < RPT; ++k) {
      const int s = k * NT + threadIdx.x;
      gdst[k] = -1;
      srow[k] = 0;
      vb[k] = 0;
      if (s >= nvalid) continue;
      const unsigned p = psort[s];
      if ((unsigned)s >= send[p]) continue;
      gdst[k] = delta[p] + s;
      srow[k] = order[s];
      if (KW == 1) A.keys[gdst[k]] = kst[s];
      else *(ulonglong2*)(A.keys + 2 * gdst[k]) = make_ulonglong2(kst[2 * s], kst[2 * s + 1]);
    }
#pragma unroll 1
    for (int v = 0; v < nv; ++v) {
      const uint8_t* src = sm + S.soff[S.val_data[v]];
      switch (P.vals[v].width) {
        case 1: scatter_col<uint8_t, RPT>(A.vals[v], src, gdst, srow); break;
        case 2: scatter_col<uint16_t, RPT>(A.vals[v], src, gdst, srow); break;
        case 4: scatter_col<uint32_t, RPT>(A.vals[v], src, gdst, srow); break;
        default: scatter_col<uint64_t, RPT>(A.vals[v], src, gdst, srow); break;
      }
      if (!any_bits) continue;
      if (S.val_mask[v] < 0) {
#pragma unroll
        for (int k = 0; k < RPT; ++k) vb[k] |= 1u << v;
      } else {
        const uint8_t* m = sm + S.soff[S.val_mask[v]];
#pragma unroll
        for (int k = 0; k < RPT; ++k) vb[k] |= (uint32_t)staged_valid(m, srow[k]) << v;
      }
    }
    if (any_bits) {
#pragma unroll
      for (int k = 0; k < RPT; ++k)
        if (gdst[k] >= 0) A.bits[gdst[k]] = (uint8_t)vb[k];
    }
    __syncthreads();
    // the value group is free: the next full tile's values land during its A-C
    if (next_full) {
      if (threadIdx.x == 0) {
        fence_async_shared();
        issue(1, nt * T);
      }
      pending[1] = true;
    }
  }
  // leave no copy in flight: a CTA that stopped early waits (bounded) for
  // the groups it had issued
  if (s_stop && threadIdx.x == 0)
    for (int g = 0; g < 2; ++g)
      if (pending[g]) mbar_wait(&bar[g], phase[g], kWaitLimit);
}

// Whether every array the plan reads can be bulk-copied tile by tile: data
// 16-byte aligned at row 0 with tile rows a multiple of 16 bytes, masks with
// row 0 at bit 0 of a 16-byte aligned word; fixed-width types of 1-8 bytes; at
// most 8 value columns.  Fills S (soff/stage_bytes for tiles of T rows).
inline bool part_scatter_bulk_ok(const Plan& P, int T, StageSpec& S)
{
  std::memset(&S, 0, sizeof(S));
  if (P.num_vals > 8 || P.num_keys > kMaxKeyCols) return false;
  int a = 0;
  size_t off = 0, tx[2] = {0, 0};
  int grp = 0;
  auto add = [&](const void* data, int64_t offset, int width) -> int {
    if (a >= kMaxStaged) return -2;
    const uint8_t* src;
    if (width) {
      src = (const uint8_t*)data + offset * width;
      if (((uintptr_t)src & 15) != 0) return -2;
    } else {
      if (offset & 127) return -2;  // row 0 at bit 0 of a 16-byte aligned word
      src = (const uint8_t*)data + (offset >> 3);
      if (((uintptr_t)src & 15) != 0) return -2;
    }
    S.src[a] = src;
    S.width[a] = width;
    S.soff[a] = (int32_t)off;
    S.group[a] = grp;
    const size_t bytes = width ? (size_t)T * width : (size_t)T / 8;
    off = (off + bytes + 15) & ~(size_t)15;
    tx[grp] += bytes;
    return a++;
  };
  for (int k = 0; k < P.num_keys; ++k) {
    const KeyCol& c = P.keys[k];
    if (c.width != 1 && c.width != 2 && c.width != 4 && c.width != 8) return false;
    S.key_data[k] = add(c.data, c.offset, c.width);
    S.key_mask[k] = c.mask ? add(c.mask, c.offset, 0) : -1;
    if (S.key_data[k] == -2 || S.key_mask[k] == -2) return false;
  }
  grp = 1;
  for (int v = 0; v < P.num_vals; ++v) {
    const ValCol& c = P.vals[v];
    if (c.width != 1 && c.width != 2 && c.width != 4 && c.width != 8) return false;
    S.val_data[v] = add(c.data, c.offset, c.width);
    S.val_mask[v] = c.mask ? add(c.mask, c.offset, 0) : -1;
    if (S.val_data[v] == -2 || S.val_mask[v] == -2) return false;
  }
  S.narr = a;
  S.key8 = P.num_keys == 1 && P.keys[0].width == 8 && P.keys[0].mask == nullptr && P.keys[0].word == 0 &&
           P.keys[0].shift == 0 && (P.keys[0].cat == CAT_SIGNED || P.keys[0].cat == CAT_UNSIGNED);
  S.stage_bytes = (int32_t)off;
  S.tx_bytes[0] = (int32_t)tx[0];
  S.tx_bytes[1] = (int32_t)tx[1];
  S.tile_rows = T;
  return true;
}

}  // namespace gb
