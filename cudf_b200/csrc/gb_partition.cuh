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

template <int R, int KW>
__global__ void __launch_bounds__(512, 1) k_part_scatter(const __grid_constant__ Plan P,
                                                         const __grid_constant__ PartArgs A)
{
  extern __shared__ __align__(16) uint8_t sh_raw[];
  unsigned long long* pbase = (unsigned long long*)sh_raw;
  unsigned int* hist = (unsigned int*)(pbase + A.nparts);
  const int64_t n = P.num_rows;
  const int64_t tile = (int64_t)blockDim.x * R;
  const bool any_bits = A.bits != nullptr;
  for (int64_t t0 = (int64_t)blockIdx.x * tile; t0 < n; t0 += (int64_t)gridDim.x * tile) {
    for (int i = threadIdx.x; i < A.nparts; i += blockDim.x) hist[i] = 0;
    __syncthreads();
    uint64_t k0[R], k1[R];
    int part[R];
    unsigned rank[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      int64_t row = t0 + (int64_t)r * blockDim.x + threadIdx.x;
      part[r] = -1;
      rank[r] = 0;
      k0[r] = 0;
      k1[r] = 0;
      if (row < n) {
        uint64_t w0, w1;
        if (pack_key(P, row, w0, w1)) {
          k0[r] = w0;
          k1[r] = w1;
          part[r] = (int)(hash_key(w0, w1, KW) >> A.shift);
        }
      }
    }
#pragma unroll
    for (int r = 0; r < R; ++r)
      if (part[r] >= 0) rank[r] = atomicAdd(&hist[part[r]], 1u);
    __syncthreads();
    for (int i = threadIdx.x; i < A.nparts; i += blockDim.x) {
      unsigned c = hist[i];
      pbase[i] = c ? atomicAdd(&A.cursor[i], (unsigned long long)c) : 0ull;
    }
    __syncthreads();
    int64_t pos[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      pos[r] = -1;
      if (part[r] < 0) continue;
      int64_t p = (int64_t)(pbase[part[r]] + rank[r]);
      if (p >= A.end[part[r]]) {
        atomicOr(A.counters + 5, 1u);
        continue;
      }
      pos[r] = p;
      if (KW == 1) A.keys[p] = k0[r];
      else *(ulonglong2*)(A.keys + 2 * p) = make_ulonglong2(k0[r], k1[r]);
    }
    uint32_t vb[R];
#pragma unroll
    for (int r = 0; r < R; ++r) vb[r] = 0;
#pragma unroll 1
    for (int v = 0; v < P.num_vals; ++v) {
      const ValCol& c = P.vals[v];
      uint64_t x[R];
#pragma unroll
      for (int r = 0; r < R; ++r) {
        int64_t row = t0 + (int64_t)r * blockDim.x + threadIdx.x + c.offset;
        x[r] = pos[r] >= 0 ? load_bits(c.data, row, c.width) : 0;
        if (any_bits && pos[r] >= 0 && bit_valid(c.mask, row)) vb[r] |= 1u << v;
      }
#pragma unroll
      for (int r = 0; r < R; ++r)
        if (pos[r] >= 0) store_width(A.vals[v], pos[r], c.width, x[r]);
    }
    if (any_bits) {
#pragma unroll
      for (int r = 0; r < R; ++r)
        if (pos[r] >= 0) A.bits[pos[r]] = (uint8_t)vb[r];
    }
    __syncthreads();
  }
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

// P2 is the plan with value columns redirected to the partitioned arrays
// (offset 0, `bits` validity) and packed_keys set.
__global__ void __launch_bounds__(512, 1) k_part_aggregate(const __grid_constant__ Plan P2,
                                                           const __grid_constant__ PartArgs A,
                                                           TableRef G, DenseRef D, int scap, int sfill,
                                                           const __grid_constant__ SlotTemplate tmpl)
{
  extern __shared__ __align__(16) uint8_t smem[];
  using Scan = cub::BlockScan<unsigned, 512>;
  __shared__ typename Scan::TempStorage scan_tmp;
  __shared__ int s_part;
  __shared__ unsigned int s_used, s_spill, s_new;
  __shared__ unsigned long long s_base;
  if (threadIdx.x == 0) s_new = 0;
  const int stride = G.stride;
  const int nw = stride / 16;
  const uint64_t smask = (uint64_t)scap - 1;
  const int per = (scap + blockDim.x - 1) / blockDim.x;
  for (;;) {
    if (threadIdx.x == 0) {
      s_part = (int)atomicAdd(A.counters + 8, 1u);
      s_used = 0;
      s_spill = 0;
    }
    for (int i = threadIdx.x; i < scap * nw; i += blockDim.x) {
      int s = i / nw;
      *(uint4*)(smem + s * stride + (i - s * nw) * 16) = tmpl.w[i - s * nw];
    }
    __syncthreads();
    const int p = s_part;
    if (p >= A.nparts) break;
    const int64_t b = A.base[p];
    const int64_t e = min((int64_t)A.cursor[p], A.end[p]);
    for (int64_t r = b + threadIdx.x; r < e; r += blockDim.x) {
      uint64_t w0, w1 = 0;
      if (P2.key_words == 1) w0 = P2.packed_keys[r];
      else {
        ulonglong2 kk = *(const ulonglong2*)(P2.packed_keys + 2 * r);
        w0 = kk.x;
        w1 = kk.y;
      }
      uint64_t h = hash_key(w0, w1, P2.key_words);
      uint8_t* slot = smem_slot(smem, stride, smask, sfill, &s_used, P2.key_words, w0, w1, h);
      if (slot == nullptr) {
        s_spill = 1;
        int64_t gi = global_slot(P2, G, w0, w1, h, &s_new);
        if (gi < 0) {
          atomicOr(G.counters + 1, 1u);
          continue;
        }
        slot = G.T + gi * (int64_t)stride;
      }
      update_slot(P2, slot, r);
    }
    __syncthreads();
    if (s_spill) {
      for (int i = threadIdx.x; i < scap; i += blockDim.x) {
        const uint8_t* s = smem + i * stride;
        if (slot_occupied(P2, s, false)) merge_slot(P2, G, s, &s_new);
      }
    } else {
      // copy this partition's groups out as dense slots, in slot order
      int first = threadIdx.x * per;
      unsigned mine = 0;
      for (int i = first; i < min(first + per, scap); ++i) mine += slot_occupied(P2, smem + i * stride, false);
      unsigned off, total;
      Scan(scan_tmp).ExclusiveSum(mine, off, total);
      if (threadIdx.x == 0) s_base = total ? atomicAdd(D.count, (unsigned long long)total) : 0ull;
      __syncthreads();
      unsigned long long o = s_base + off;
      for (int i = first; i < min(first + per, scap); ++i) {
        const uint8_t* s = smem + i * stride;
        if (!slot_occupied(P2, s, false)) continue;
        if ((int64_t)o >= D.cap) {
          atomicOr(D.overflow, 1u);
          break;
        }
        uint4* dst = (uint4*)(D.T + o * stride);
        for (int w = 0; w < nw; ++w) dst[w] = ((const uint4*)s)[w];
        ++o;
      }
    }
    __syncthreads();
  }
  if (threadIdx.x == 0 && s_new) atomicAdd(G.counters, s_new);
}

}  // namespace gb
