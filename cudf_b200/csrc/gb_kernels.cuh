// gb_kernels.cuh -- kernels of the hash groupby engine.
//
//   k_init_slots     fill table slots with the identity template
//   k_aggregate<S>   one pass over the rows: optional per-CTA shared-memory
//                    table (S = true) that spills to the global table; fused
//                    SUM/COUNT/MIN/MAX/... updates with null handling
//   k_var_pass       second pass of VARIANCE/STD
//   k_finish_count   adds the all-ones-key slot to the group count
//   k_compact        gathers occupied slots into dense key and result columns
//   k_sketch         full-pass HyperLogLog + per-bucket row counts (group
//                    estimate, partition region sizes)
#pragma once
#include <cub/block/block_scan.cuh>

#include "gb_device.cuh"

namespace gb {

constexpr int kMaxSlotBytes = 1024;
// Longest probe run of a global table.  At load <= 0.5 linear probing needs a
// few probes; a run this long means the table is (nearly) full, which is
// reported as overflow (the host regrows the table) instead of scanning it.
constexpr uint64_t kMaxProbes = 4096;

// Identity contents of an empty slot, as 8-byte words (slot strides are
// multiples of 8; an odd multiple spreads a field of consecutive slots over
// all shared-memory banks).
struct SlotTemplate {
  unsigned long long w[kMaxSlotBytes / 8];
};

struct TableRef {
  uint8_t* T;          // capacity + 1 slots (the last one is the all-ones-key slot)
  uint64_t cap_mask;   // capacity - 1 (capacity is a power of two)
  int32_t stride;
  int32_t words;
  unsigned int* counters;  // [0] groups, [1] overflow flag
};

static __global__ void k_init_slots(uint8_t* T, int64_t nslots, int stride, const __grid_constant__ SlotTemplate tmpl)
{
  int nw = stride / 8;
  int64_t total = nslots * nw;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    int64_t s = i / nw;
    int w = (int)(i - s * nw);
    *(unsigned long long*)(T + s * stride + w * 8) = tmpl.w[w];
  }
}

__device__ __forceinline__ bool slot_occupied(const Plan& P, const uint8_t* slot, bool special)
{
  if (special) return *(const uint32_t*)(slot + P.rows_off) > 0;
  if (P.key_words == 1) return *(const uint64_t*)slot != kEmpty;
  return (((const uint64_t*)slot)[1] >> 63) == 0;
}

// Updates the slot of one row: rows counter, per-column null counters and the
// column's accumulators.
__device__ __forceinline__ void update_slot(const Plan& P, uint8_t* slot, int64_t row)
{
  atomicAdd((unsigned int*)(slot + P.rows_off), 1u);
#pragma unroll 1
  for (int v = 0; v < P.num_vals; ++v) {
    const ValCol& c = P.vals[v];
    int64_t r = row + c.offset;
    bool valid = c.bits ? ((c.bits[r] >> c.bit) & 1) : bit_valid(c.mask, r);
    if (!valid) {
      if (c.nulls_off >= 0) atomicAdd((unsigned int*)(slot + c.nulls_off), 1u);
      continue;
    }
    if (c.acc_begin == c.acc_end) continue;
    Elem e = load_elem(c, r);
    apply_elem(P, c, c.acc_begin, c.acc_end, slot, e, (uint32_t)row);
  }
}

__device__ __forceinline__ int64_t global_slot(const Plan& P, const TableRef& G, uint64_t w0,
                                               uint64_t w1, uint64_t h, unsigned int* s_new)
{
  bool ins;
  int64_t i = P.key_words == 1
                ? find_or_insert1(G.T, G.stride, G.cap_mask, w0, h, (int)min(kMaxProbes, G.cap_mask + 1), ins)
                : find_or_insert2(G.T, G.stride, G.cap_mask, w0, w1, h, (int)min(kMaxProbes, G.cap_mask + 1), ins);
  if (ins) atomicAdd(s_new, 1u);
  return i;
}

// Merges a shared-memory slot into the global table.
__device__ __forceinline__ void merge_slot(const Plan& P, const TableRef& G, const uint8_t* s,
                                           unsigned int* s_new)
{
  uint64_t w0 = ((const uint64_t*)s)[0];
  uint64_t w1 = P.key_words == 2 ? ((const uint64_t*)s)[1] : 0;
  uint64_t h = hash_key(w0, w1, P.key_words);
  int64_t gi = global_slot(P, G, w0, w1, h, s_new);
  if (gi < 0) {
    atomicOr(G.counters + 1, 1u);
    return;
  }
  uint8_t* d = G.T + gi * (int64_t)G.stride;
  atomicAdd((unsigned int*)(d + P.rows_off), *(const uint32_t*)(s + P.rows_off));
#pragma unroll 1
  for (int v = 0; v < P.num_vals; ++v) {
    int off = P.vals[v].nulls_off;
    if (off < 0) continue;
    uint32_t nn = *(const uint32_t*)(s + off);
    if (nn) atomicAdd((unsigned int*)(d + off), nn);
  }
#pragma unroll 1
  for (int a = 0; a < P.num_accs; ++a) merge_acc(P, P.accs[a], d, s);
}

// One pass over rows [0, num_rows).  With USE_SMEM each CTA first aggregates
// into its own shared-memory table of `scap` slots (at most `sfill` of them
// claimed); keys that do not fit go to the global table directly.  At the end
// the CTA merges its table into the global one.
template <bool USE_SMEM>
__global__ void __launch_bounds__(512) k_aggregate(const __grid_constant__ Plan P, TableRef G,
                                                   int scap, int sfill,
                                                   const __grid_constant__ SlotTemplate tmpl)
{
  extern __shared__ __align__(16) uint8_t smem[];
  __shared__ unsigned int s_new, s_used;
  if (threadIdx.x == 0) { s_new = 0; s_used = 0; }
  if (USE_SMEM) {
    int nw = G.stride / 8;
    for (int i = threadIdx.x; i < scap * nw; i += blockDim.x) {
      int s = i / nw;
      int w = i - s * nw;
      *(unsigned long long*)(smem + s * G.stride + w * 8) = tmpl.w[w];
    }
  }
  __syncthreads();
  const uint64_t smask = (uint64_t)scap - 1;
  const int64_t n = P.num_rows;
  int since_check = 0;
  for (int64_t row = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; row < n;
       row += (int64_t)gridDim.x * blockDim.x) {
    // once the table overflowed the host re-runs with a larger one: stop early
    if (++since_check == 64) {
      since_check = 0;
      if (*(volatile unsigned int*)(G.counters + 1)) break;
    }
    uint64_t w0, w1;
    if (!pack_key(P, row, w0, w1)) continue;
    uint64_t h = hash_key(w0, w1, P.key_words);
    uint8_t* slot = nullptr;
    if (USE_SMEM) {
      uint64_t i = (h >> 20) & smask;
      if (P.key_words == 1) {
        if (w0 != kEmpty) {
          for (int p = 0; p < 32; ++p) {
            unsigned long long* kp = (unsigned long long*)(smem + i * G.stride);
            uint64_t cur = *(volatile unsigned long long*)kp;
            if (cur == w0) { slot = (uint8_t*)kp; break; }
            if (cur == kEmpty) {
              if (*(volatile unsigned int*)&s_used >= (unsigned)sfill) break;
              uint64_t old = atomicCAS(kp, kEmpty, w0);
              if (old == kEmpty) { atomicAdd(&s_used, 1u); slot = (uint8_t*)kp; break; }
              if (old == w0) { slot = (uint8_t*)kp; break; }
            }
            i = (i + 1) & smask;
          }
        }
      } else {
        unsigned __int128 want = ((unsigned __int128)w1 << 64) | w0;
        const unsigned __int128 empty = ~(unsigned __int128)0;
        for (int p = 0; p < 32; ++p) {
          unsigned __int128* kp = (unsigned __int128*)(smem + i * G.stride);
          ulonglong2 cur = vload2(kp);
          if (cur.x == w0 && cur.y == w1 && w0 != kEmpty) { slot = (uint8_t*)kp; break; }
          if ((cur.y >> 63) || cur.x == kEmpty) {
            // a slot read as empty is only claimed while the table has room;
            // a torn read (cur.x == kEmpty only) goes through the CAS compare
            if ((cur.y >> 63) && *(volatile unsigned int*)&s_used >= (unsigned)sfill) break;
            unsigned __int128 old = atomicCAS(kp, empty, want);
            if (old == empty) { atomicAdd(&s_used, 1u); slot = (uint8_t*)kp; break; }
            if (old == want) { slot = (uint8_t*)kp; break; }
          }
          i = (i + 1) & smask;
        }
      }
    }
    if (slot == nullptr) {
      int64_t gi = global_slot(P, G, w0, w1, h, &s_new);
      if (gi < 0) {
        atomicOr(G.counters + 1, 1u);
        continue;
      }
      slot = G.T + gi * (int64_t)G.stride;
    }
    update_slot(P, slot, row);
  }
  __syncthreads();
  if (USE_SMEM) {
    for (int i = threadIdx.x; i < scap; i += blockDim.x) {
      const uint8_t* s = smem + i * G.stride;
      if (!slot_occupied(P, s, false)) continue;
      merge_slot(P, G, s, &s_new);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0 && s_new) atomicAdd(G.counters, s_new);
}

// VARIANCE/STD second pass (cpp/src/groupby/hash/multi_pass_kernels.cuh:79-94):
// per valid value, (x - mean)^2 / (n - ddof) added to the group's M2.
static __global__ void __launch_bounds__(256) k_var_pass(const __grid_constant__ Plan P, TableRef G)
{
  const int64_t n = P.num_rows;
  for (int64_t row = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; row < n;
       row += (int64_t)gridDim.x * blockDim.x) {
    uint64_t w0, w1;
    if (!pack_key(P, row, w0, w1)) continue;
    uint64_t h = hash_key(w0, w1, P.key_words);
    int64_t gi = P.key_words == 1 ? find1(G.T, G.stride, G.cap_mask, w0, h)
                                  : find2(G.T, G.stride, G.cap_mask, w0, w1, h);
    if (gi < 0) continue;
    uint8_t* slot = G.T + gi * (int64_t)G.stride;
    uint32_t rows = *(const uint32_t*)(slot + P.rows_off);
    for (int v = 0; v < P.num_vals; ++v) {
      const ValCol& c = P.vals[v];
      if (c.m2_off < 0) continue;
      int64_t r = row + c.offset;
      if (!bit_valid(c.mask, r)) continue;
      int64_t cnt = (int64_t)rows - (c.nulls_off >= 0 ? *(const uint32_t*)(slot + c.nulls_off) : 0u);
      if (cnt == 0 || cnt - c.ddof <= 0) continue;
      Elem e = load_elem(c, r);
      double x = (c.cat == CAT_F32 || c.cat == CAT_F64) ? e.d : (c.cat == CAT_UNSIGNED ? (double)e.bits : (double)e.i);
      double sum;
      switch (c.cat) {
        case CAT_F32: sum = *(const float*)(slot + c.sum_off); break;
        case CAT_F64: sum = *(const double*)(slot + c.sum_off); break;
        default: sum = (double)*(const int64_t*)(slot + c.sum_off); break;
      }
      double mean = sum / (double)cnt;
      double t = (x - mean) * (x - mean) / (double)(cnt - c.ddof);
      atomicAdd((double*)(slot + c.m2_off), t);
    }
  }
}

static __global__ void k_finish_count(const __grid_constant__ Plan P, TableRef G)
{
  const uint8_t* special = G.T + (int64_t)(G.cap_mask + 1) * G.stride;
  if (*(const uint32_t*)(special + P.rows_off) > 0) atomicAdd(G.counters, 1u);
}

struct OutPtrs {
  void* key_data[kMaxKeyCols];
  uint32_t* key_mask[kMaxKeyCols];
  void* out_data[kMaxOutputs];
  uint32_t* out_mask[kMaxOutputs];
  unsigned int* counters;  // [2] output position, [4 + j] null count of output column j
};

__device__ __forceinline__ void store_width(void* base, int64_t i, int width, uint64_t bits)
{
  switch (width) {
    case 1: ((uint8_t*)base)[i] = (uint8_t)bits; break;
    case 2: ((uint16_t*)base)[i] = (uint16_t)bits; break;
    case 4: ((uint32_t*)base)[i] = (uint32_t)bits; break;
    default: ((uint64_t*)base)[i] = bits; break;
  }
}

__device__ __forceinline__ void count_nulls(bool is_null, unsigned int* counter)
{
  unsigned m = __ballot_sync(__activemask(), is_null);
  if (m && (threadIdx.x & 31) == (__ffs(m) - 1)) atomicAdd(counter, __popc(m));
}

// Sets the validity bits of a warp's output rows.  The occupied lanes of a
// warp write consecutive positions (pos of the lowest occupied lane, + 1 per
// occupied lane), so their bits form one run: assembled with one warp OR
// reduction and stored with at most two atomic ORs instead of one per row.
// Every lane of the warp calls it.
__device__ __forceinline__ void warp_mask_or(uint32_t* mask, bool occ, bool bit, int64_t pos)
{
  const unsigned full = 0xFFFFFFFFu;
  const unsigned occm = __ballot_sync(full, occ);
  if (!occm) return;
  const int lane = threadIdx.x & 31;
  const unsigned rank = __popc(occm & ((1u << lane) - 1));
  const unsigned word = __reduce_or_sync(full, (occ && bit) ? (1u << rank) : 0u);
  if (lane == __ffs(occm) - 1 && word) {
    const int sh = (int)(pos & 31);
    atomicOr(mask + (pos >> 5), word << sh);
    if (sh && (word >> (32 - sh))) atomicOr(mask + (pos >> 5) + 1, word >> (32 - sh));
  }
}

// Value bits of output j for a slot, and whether it is valid.
__device__ __forceinline__ uint64_t finalize(const Plan& P, const OutSpec& o, const uint8_t* slot,
                                             bool& valid)
{
  const ValCol& c = P.vals[o.col];
  uint32_t rows = *(const uint32_t*)(slot + P.rows_off);
  uint32_t nulls = c.nulls_off >= 0 ? *(const uint32_t*)(slot + c.nulls_off) : 0u;
  int64_t cnt = (int64_t)rows - nulls;
  valid = cnt > 0;
  const uint8_t* a = slot + (o.acc_off >= 0 ? o.acc_off : 0);
  switch (o.kind) {
    case K_COUNT_VALID: valid = true; return (uint64_t)cnt;
    case K_COUNT_ALL: valid = true; return rows;
    case K_SUM: case K_SUM_OF_SQUARES: case K_PRODUCT:
      return o.out_width == 8 ? *(const uint64_t*)a : *(const uint32_t*)a;
    case K_MIN: case K_MAX: {
      bool is_min = o.kind == K_MIN;
      if (c.width == 8) {
        uint64_t e = *(const uint64_t*)a;
        if (c.cat == CAT_F64) return (uint64_t)__double_as_longlong(dec64_f(e));
        if (c.cat == CAT_UNSIGNED) return e;
        return e ^ 0x8000000000000000ull;
      }
      (void)is_min;
      uint32_t e = *(const uint32_t*)a;
      if (c.cat == CAT_F32) return __float_as_uint(dec32_f(e));
      if (c.cat == CAT_UNSIGNED || c.cat == CAT_BOOL) return e;
      return (uint64_t)(int64_t)(int32_t)(e ^ 0x80000000u);
    }
    case K_MEAN: {
      if (cnt == 0) return 0;
      if (o.out_type >= T_DUR_D) {  // durations: integer mean in the duration's type
        int64_t s = c.width == 8 ? *(const int64_t*)a : (int64_t) * (const int32_t*)a;
        return (uint64_t)(s / cnt);
      }
      double s;
      if (c.cat == CAT_F32) s = *(const float*)a;
      else if (c.cat == CAT_F64) s = *(const double*)a;
      else s = (double)*(const int64_t*)a;
      return (uint64_t)__double_as_longlong(s / (double)cnt);
    }
    case K_VARIANCE: case K_STD: {
      valid = cnt - o.ddof > 0;
      double m2 = valid ? *(const double*)a : 0.0;
      if (o.kind == K_STD) m2 = sqrt(m2);
      return (uint64_t)__double_as_longlong(m2);
    }
    case K_ARGMIN: case K_ARGMAX: {
      uint64_t v = *(const uint64_t*)a;
      if (v == kEmpty || (o.kind == K_ARGMAX && v == 0 && c.width != 8)) return kNoRow32;
      if (c.width == 8) return (uint32_t)v;
      return o.kind == K_ARGMIN ? (uint32_t)v : (uint32_t)~(uint32_t)v;
    }
    default: return 0;
  }
}

// Writes the occupied slots among [base, base + blockDim.x) of one table into
// dense output columns (positions reserved per block on O.counters[2]).
// Every thread of the block calls it (it synchronises the block).
__device__ __forceinline__ void compact_block(const Plan& P, const uint8_t* T, int64_t nslots, int stride,
                                              int64_t limit, int dense, const OutPtrs& O, int64_t base,
                                              void* scan_storage, unsigned int* s_base)
{
  using Scan = cub::BlockScan<int, 256>;
  typename Scan::TempStorage& tmp = *(typename Scan::TempStorage*)scan_storage;
  int64_t i = base + threadIdx.x;
  const uint8_t* slot = T + i * (int64_t)stride;
  bool occ = i < nslots && (dense || slot_occupied(P, slot, i == nslots - 1));
  int local, total;
  Scan(tmp).ExclusiveSum(occ ? 1 : 0, local, total);
  if (threadIdx.x == 0) *s_base = total ? atomicAdd(O.counters + 2, (unsigned)total) : 0;
  __syncthreads();
  if (occ && (int64_t)*s_base + local >= limit) {
    atomicOr(O.counters + 1, 1u);  // more occupied slots than counted groups
    occ = false;
  }
  // every lane of the block runs what follows (warp-wide mask assembly)
  const int64_t pos = (int64_t)*s_base + local;
  uint64_t w[2] = {0, 0};
  if (occ) {
    w[0] = ((const uint64_t*)slot)[0];
    w[1] = P.key_words == 2 ? ((const uint64_t*)slot)[1] : 0;
  }
  for (int k = 0; k < P.num_keys; ++k) {
    const KeyCol& c = P.keys[k];
    const bool is_null = occ && c.has_null_bit && ((w[c.null_word] >> c.null_shift) & 1);
    if (occ) {
      const uint64_t bits = c.width == 8 ? w[c.word] : (w[c.word] >> c.shift) & ((1ull << (8 * c.width)) - 1);
      store_width(O.key_data[k], pos, c.width, is_null ? 0 : bits);
    }
    if (O.key_mask[k]) warp_mask_or(O.key_mask[k], occ, !is_null, pos);
    count_nulls(is_null, O.counters + 4 + k);
  }
  for (int j = 0; j < P.num_outs; ++j) {
    const OutSpec& o = P.outs[j];
    bool valid = true;
    uint64_t bits = 0;
    if (occ) {
      bits = finalize(P, o, slot, valid);
      store_width(O.out_data[j], pos, o.out_width, valid ? bits : 0);
    }
    if (O.out_mask[j]) warp_mask_or(O.out_mask[j], occ, valid, pos);
    count_nulls(occ && !valid, O.counters + 4 + P.num_keys + j);
  }
  __syncthreads();
}

// nslots_dev (optional): a device count that bounds nslots (dense slots
// written by the partitioned pass, read here instead of on the host).
static __global__ void __launch_bounds__(256) k_compact(const __grid_constant__ Plan P, const uint8_t* T,
                                                        int64_t nslots, int stride, int64_t limit, int dense,
                                                        const __grid_constant__ OutPtrs O,
                                                        const unsigned long long* nslots_dev = nullptr)
{
  using Scan = cub::BlockScan<int, 256>;
  __shared__ typename Scan::TempStorage tmp;
  __shared__ unsigned int s_base;
  if (nslots_dev) nslots = min(nslots, (int64_t)*(volatile const unsigned long long*)nslots_dev);
  const int64_t step = (int64_t)gridDim.x * blockDim.x;
  for (int64_t base = (int64_t)blockIdx.x * blockDim.x; base < nslots; base += step)
    compact_block(P, T, nslots, stride, limit, dense, O, base, &tmp, &s_base);
}

// ---- group-count estimate ----
// Hash buckets (top kBucketBits bits of a key's hash) of the sketch's row
// histogram; the partitioned path sizes its regions from them.
constexpr int kBucketBits = 14;

// Full-pass key sketch: per hash bucket (top kBucketBits bits) the exact
// number of rows with a valid key, and a HyperLogLog register array
// (Flajolet, Fusy, Gandouet, Meunier 2007) of 2^kHllBits registers over the
// same hashes: register index from hash bits 40-51, rank = position of the
// first set bit among bits 39..0.  Each CTA builds both in shared memory and
// merges them into `hll` (atomic max) and `buckets` (atomic add) at the end.
constexpr int kHllBits = 12;
inline size_t sketch_smem() { return ((size_t(1) << kHllBits) + (size_t(1) << kBucketBits)) * 4; }

static __global__ void __launch_bounds__(512) k_sketch(const __grid_constant__ Plan P, unsigned int* hll,
                                                       unsigned int* buckets)
{
  extern __shared__ unsigned int sk[];
  unsigned int* reg = sk;
  unsigned int* bk = sk + (1 << kHllBits);
  for (int i = threadIdx.x; i < (1 << kHllBits) + (1 << kBucketBits); i += blockDim.x) sk[i] = 0;
  __syncthreads();
  const int64_t n = P.num_rows;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  auto add = [&](uint64_t h, unsigned rows) {
    atomicAdd(&bk[h >> (64 - kBucketBits)], rows);
    const uint64_t low = h << 24;
    const unsigned rank = low ? (unsigned)__clzll((long long)low) + 1u : 41u;
    atomicMax(&reg[(h >> 40) & ((1u << kHllBits) - 1)], rank);
  };
  if (P.num_keys == 1 && !P.keys[0].mask && P.keys[0].width == 8 && P.keys[0].cat != CAT_F64) {
    // one plain 64-bit key: four rows per thread in flight
    const unsigned long long* kd = (const unsigned long long*)P.keys[0].data + P.keys[0].offset;
    int64_t row = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    for (; row + 3 * stride < n; row += 4 * stride) {
      uint64_t k[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) k[j] = __ldg(kd + row + j * stride);
#pragma unroll
      for (int j = 0; j < 4; ++j) add(fmix64(k[j]), 1u);
    }
    for (; row < n; row += stride) add(fmix64(__ldg(kd + row)), 1u);
  } else {
    // several key columns, nullable or floating-point keys: four rows per
    // thread, packed column by column so that the four rows' data and mask
    // loads of a column are in flight together (as pack_key, per row)
    constexpr int SR = 4;
    for (int64_t row0 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; row0 < n; row0 += SR * stride) {
      uint64_t w0[SR], w1[SR];
      bool ok[SR];
#pragma unroll
      for (int j = 0; j < SR; ++j) {
        w0[j] = 0;
        w1[j] = 0;
        ok[j] = row0 + j * stride < n;
      }
#pragma unroll 1
      for (int k = 0; k < P.num_keys; ++k) {
        const KeyCol& c = P.keys[k];
        uint64_t b[SR];
        uint32_t mw[SR];
#pragma unroll
        for (int j = 0; j < SR; ++j) {
          const int64_t r = row0 + j * stride + c.offset;
          b[j] = ok[j] ? load_bits(c.data, r, c.width) : 0;
          mw[j] = (ok[j] && c.mask) ? __ldg(c.mask + (r >> 5)) : 0xFFFFFFFFu;
        }
#pragma unroll
        for (int j = 0; j < SR; ++j) {
          if (!ok[j]) continue;
          const int64_t r = row0 + j * stride + c.offset;
          if (!((mw[j] >> (r & 31)) & 1u)) {
            if (!P.include_nulls) {
              ok[j] = false;
              continue;
            }
            const uint64_t nb = 1ull << c.null_shift;
            if (c.null_word == 0) w0[j] |= nb;
            else w1[j] |= nb;
            continue;
          }
          const uint64_t v = norm_key_bits(c, b[j]) << c.shift;
          if (c.word == 0) w0[j] |= v;
          else w1[j] |= v;
        }
      }
#pragma unroll
      for (int j = 0; j < SR; ++j)
        if (ok[j]) add(hash_key(w0[j], w1[j], P.key_words), 1u);
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < (1 << kHllBits); i += blockDim.x)
    if (reg[i]) atomicMax(hll + i, reg[i]);
  for (int i = threadIdx.x; i < (1 << kBucketBits); i += blockDim.x)
    if (bk[i]) atomicAdd(buckets + i, bk[i]);
}


}  // namespace gb
