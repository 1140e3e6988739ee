// gb_batch.cu -- many independent groupbys of one schema in one persistent launch.
//
// A batch is a list of instances (each its own key and value columns, all with
// the same key types, value types and aggregations).  Rows of every instance
// are cut into tiles; a persistent kernel pulls tiles from a device work
// counter, so instances of very different sizes share the GPU without one
// launch (and one host synchronisation) per instance.  Each instance has its
// own region of one global table buffer, sized from a per-instance key sample;
// low-cardinality instances first aggregate each tile in a shared-memory table.
// The sequence (table init, aggregate, count, compact, read-back) can be
// captured once in a CUDA graph and replayed for batches of the same shape.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/cudf_b200.h"
#include "gb_batch.h"
#include "gb_kernels.cuh"

namespace gb {

constexpr int kSampleRows = 2048;
constexpr int kSampleSlots = 4096;

struct BatchInst {
  const void* key_data[kMaxKeyCols];
  const uint32_t* key_mask[kMaxKeyCols];
  int64_t key_off[kMaxKeyCols];
  const void* val_data[kMaxValCols];
  const uint32_t* val_mask[kMaxValCols];
  int64_t val_off[kMaxValCols];
  int64_t n_rows;
  uint8_t* table;
  uint64_t cap_mask;
  unsigned int* counters;  // [0] groups [1] overflow [2] output position [4..] null counts
  int32_t scap;            // shared-memory slots per tile (0: global table only)
  int32_t sfill;
};

struct BatchTile {
  int32_t inst;
  int32_t pad;
  int64_t begin, end;
};

// Plan with instance `I`'s column pointers.
__device__ __forceinline__ void patch_plan(Plan& sp, const BatchInst& I)
{
  for (int k = 0; k < sp.num_keys; ++k) {
    sp.keys[k].data = I.key_data[k];
    sp.keys[k].mask = I.key_mask[k];
    sp.keys[k].offset = I.key_off[k];
  }
  for (int v = 0; v < sp.num_vals; ++v) {
    sp.vals[v].data = I.val_data[v];
    sp.vals[v].mask = I.val_mask[v];
    sp.vals[v].offset = I.val_off[v];
  }
  sp.num_rows = I.n_rows;
}

// One CTA per instance: up to kSampleRows strided rows into a shared table;
// distinct keys, keys seen once and twice, and rows that took part.
static __global__ void __launch_bounds__(256) k_batch_sample(const __grid_constant__ Plan P, const BatchInst* insts,
                                                             unsigned int* stats)
{
  extern __shared__ __align__(16) uint8_t sh[];
  __shared__ Plan sp;
  __shared__ unsigned int s_cnt[4];
  const BatchInst& I = insts[blockIdx.x];
  if (threadIdx.x == 0) {
    sp = P;
    patch_plan(sp, I);
    s_cnt[0] = s_cnt[1] = s_cnt[2] = s_cnt[3] = 0;
  }
  // slots: 16 B key | u32 count | pad  (32 B)
  for (int i = threadIdx.x; i < kSampleSlots * 4; i += blockDim.x) {
    int s = i >> 2, w = i & 3;
    ((unsigned long long*)sh)[s * 4 + w] = w < 2 ? kEmpty : 0ull;
  }
  __syncthreads();
  const int64_t n = I.n_rows;
  const int64_t m = n < kSampleRows ? n : kSampleRows;
  for (int64_t j = threadIdx.x; j < m; j += blockDim.x) {
    int64_t row = m >= n ? j : (j * n) / m;
    uint64_t w0, w1;
    if (!pack_key(sp, row, w0, w1)) continue;
    atomicAdd(&s_cnt[3], 1u);
    uint64_t h = hash_key(w0, w1, 2);  // both words always hashed here
    uint64_t i = h & (kSampleSlots - 1);
    const unsigned __int128 empty = ~(unsigned __int128)0;
    unsigned __int128 want = ((unsigned __int128)w1 << 64) | w0;
    for (int p = 0; p < kSampleSlots; ++p) {
      unsigned __int128* kp = (unsigned __int128*)(sh + i * 32);
      unsigned __int128 old = atomicCAS(kp, empty, want);
      if (old == empty || old == want) {
        atomicAdd((unsigned int*)(sh + i * 32 + 16), 1u);
        break;
      }
      i = (i + 1) & (kSampleSlots - 1);
    }
  }
  __syncthreads();
  for (int s = threadIdx.x; s < kSampleSlots; s += blockDim.x) {
    unsigned c = *(const unsigned int*)(sh + s * 32 + 16);
    if (c) atomicAdd(&s_cnt[0], 1u);
    if (c == 1) atomicAdd(&s_cnt[1], 1u);
    if (c == 2) atomicAdd(&s_cnt[2], 1u);
  }
  __syncthreads();
  if (threadIdx.x < 4) stats[blockIdx.x * 4 + threadIdx.x] = s_cnt[threadIdx.x];
}

static __global__ void k_batch_init(uint8_t* T, int64_t nslots, int stride, const __grid_constant__ SlotTemplate tmpl)
{
  int nw = stride / 8;
  int64_t total = nslots * nw;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    int64_t s = i / nw;
    *(unsigned long long*)(T + s * stride + (i - s * nw) * 8) = tmpl.w[i - s * nw];
  }
}

// Aggregation of the tile list: one CTA per tile (largest instances first), so
// that kernels of other streams (the serving loop's sketch) interleave at tile
// granularity.
template <int NT>
static __global__ void __launch_bounds__(NT) k_batch_aggregate(const __grid_constant__ Plan P,
                                                                          const BatchInst* insts,
                                                                          const BatchTile* tiles, int64_t ntiles,
                                                                          unsigned int* work,
                                                                          const __grid_constant__ SlotTemplate tmpl)
{
  extern __shared__ __align__(16) uint8_t smem[];
  __shared__ __align__(16) Plan sp;
  __shared__ unsigned int s_new, s_used;
  {
    const int4* src = (const int4*)&P;
    int4* dst = (int4*)&sp;
    for (int i = threadIdx.x; i < (int)(sizeof(Plan) / 16); i += blockDim.x) dst[i] = src[i];
    if (threadIdx.x == 0) {
      for (size_t b = (sizeof(Plan) / 16) * 16; b < sizeof(Plan); ++b) ((char*)&sp)[b] = ((const char*)&P)[b];
      s_new = 0;
      s_used = 0;
    }
  }
  (void)work;
  const int stride = P.slot_bytes;
  const int nw = stride / 8;
  for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    __syncthreads();
    if (threadIdx.x == 0) {
      s_new = 0;
      s_used = 0;
    }
    const BatchTile tl = tiles[t];
    const BatchInst& I = insts[tl.inst];
    const int scap = I.scap;
    if (threadIdx.x == 0) patch_plan(sp, I);
    for (int i = threadIdx.x; i < scap * nw; i += blockDim.x) {
      int s = i / nw;
      *(unsigned long long*)(smem + (size_t)s * stride + (i - s * nw) * 8) = tmpl.w[i - s * nw];
    }
    __syncthreads();
    TableRef G{I.table, I.cap_mask, stride, sp.key_words, I.counters};
    const uint64_t smask = (uint64_t)(scap > 0 ? scap : 1) - 1;
    // an instance whose table overflowed is re-run with a larger table: skip
    const int64_t row_end = *(volatile unsigned int*)(I.counters + 1) ? tl.begin : tl.end;
    int since_check = 0;
    for (int64_t row = tl.begin + threadIdx.x; row < row_end; row += blockDim.x) {
      if (++since_check == 64) {
        since_check = 0;
        if (*(volatile unsigned int*)(I.counters + 1)) break;
      }
      uint64_t w0, w1;
      if (!pack_key(sp, row, w0, w1)) continue;
      uint64_t h = hash_key(w0, w1, sp.key_words);
      uint8_t* slot = nullptr;
      if (scap > 0) {
        uint64_t i = (h >> 20) & smask;
        if (sp.key_words == 1) {
          if (w0 != kEmpty) {
            for (int p = 0; p < 32; ++p) {
              unsigned long long* kp = (unsigned long long*)(smem + i * stride);
              uint64_t cur = *(volatile unsigned long long*)kp;
              if (cur == w0) { slot = (uint8_t*)kp; break; }
              if (cur == kEmpty) {
                if (*(volatile unsigned int*)&s_used >= (unsigned)I.sfill) break;
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
            unsigned __int128* kp = (unsigned __int128*)(smem + i * stride);
            ulonglong2 cur = vload2(kp);
            if (cur.x == w0 && cur.y == w1 && w0 != kEmpty) { slot = (uint8_t*)kp; break; }
            if ((cur.y >> 63) || cur.x == kEmpty) {
              if ((cur.y >> 63) && *(volatile unsigned int*)&s_used >= (unsigned)I.sfill) break;
              unsigned __int128 old = atomicCAS(kp, empty, want);
              if (old == empty) { atomicAdd(&s_used, 1u); slot = (uint8_t*)kp; break; }
              if (old == want) { slot = (uint8_t*)kp; break; }
            }
            i = (i + 1) & smask;
          }
        }
      }
      if (slot == nullptr) {
        int64_t gi = global_slot(sp, G, w0, w1, h, &s_new);
        if (gi < 0) {
          atomicOr(I.counters + 1, 1u);
          continue;
        }
        slot = G.T + gi * (int64_t)stride;
      }
      update_slot(sp, slot, row);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < scap; i += blockDim.x) {
      const uint8_t* s = smem + (size_t)i * stride;
      if (slot_occupied(sp, s, false)) merge_slot(sp, G, s, &s_new);
    }
    __syncthreads();
    if (threadIdx.x == 0 && s_new) atomicAdd(I.counters, s_new);
    __syncthreads();
  }
}

static __global__ void k_batch_finish(const __grid_constant__ Plan P, const BatchInst* insts, int ninst)
{
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ninst) return;
  const BatchInst& I = insts[i];
  const uint8_t* special = I.table + (int64_t)(I.cap_mask + 1) * P.slot_bytes;
  if (*(const uint32_t*)(special + P.rows_off) > 0) atomicAdd(I.counters, 1u);
}

struct BatchChunk {
  int32_t inst;
  int32_t pad;
  int64_t base;
};

// Compaction of every instance's table into its outputs; chunks of 256 slots.
static __global__ void __launch_bounds__(256) k_batch_compact(const __grid_constant__ Plan P, const BatchInst* insts,
                                                              const OutPtrs* outs, const BatchChunk* chunks,
                                                              int64_t nchunks)
{
  using Scan = cub::BlockScan<int, 256>;
  __shared__ typename Scan::TempStorage tmp;
  __shared__ unsigned int s_base;
  for (int64_t c = blockIdx.x; c < nchunks; c += gridDim.x) {
    const BatchChunk ch = chunks[c];
    const BatchInst& I = insts[ch.inst];
    const int64_t nslots = (int64_t)I.cap_mask + 2;
    const int64_t limit = *(volatile const unsigned int*)I.counters;
    compact_block(P, I.table, nslots, P.slot_bytes, limit, 0, outs[ch.inst], ch.base, &tmp, &s_base);
  }
}

// ---------------------------------------------------------------------------
static void ck(cudaError_t e, const char* what)
{
  if (e == cudaSuccess) return;
  cudaGetLastError();
  throw Error(e == cudaErrorMemoryAllocation ? ERR_ALLOC : ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

static uint64_t pow2_at_least(uint64_t x)
{
  uint64_t p = 1;
  while (p < x) p <<= 1;
  return p;
}

static void slot_template(const Plan& P, SlotTemplate& t)
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

struct DevBuf {
  Allocator A;
  cudaStream_t s = nullptr;
  void* p = nullptr;
  size_t n = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  void get(const Allocator& a, size_t bytes, cudaStream_t st)
  {
    release();
    A = a;
    s = st;
    n = std::max<size_t>(bytes, 256);
    p = A.allocate(A.ctx, n, (void*)s);
    if (!p) throw Error(ERR_ALLOC, "device allocation of " + std::to_string(n) + " bytes failed");
  }
  void release()
  {
    if (p) A.deallocate(A.ctx, p, n, (void*)s);
    p = nullptr;
  }
  ~DevBuf() { release(); }
};

struct Batch::Impl {
  Plan P;
  std::vector<int> out_types;
  int ninst = 0;
  int nout = 0;
  std::vector<BatchInst> insts;
  std::vector<BatchTile> tiles;
  std::vector<BatchChunk> chunks;
  std::vector<OutPtrs> outs;
  std::vector<int64_t> caps;
  // device buffers
  DevBuf d_tables, d_counters, d_insts, d_tiles, d_chunks, d_outs, d_outputs, d_work, d_stats;
  unsigned int* h_counters = nullptr;  // pinned copy of the per-instance counters
  size_t counter_words = 128;
  SlotTemplate tmpl;
  int smem_bytes = 0;
  int grid_agg = 0, grid_compact = 0;
  int block = 512;
  int64_t total_slots = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaStream_t stream = nullptr;
  Allocator A;
  // output layout: per instance, per column: (data offset, mask offset) in d_outputs;
  // every mask lies in [mask_begin, mask_end) so one memset clears them all
  std::vector<std::vector<std::pair<size_t, size_t>>> out_off;
  size_t mask_begin = 0, mask_end = 0;
  int sms = 148;
  BatchStats stats;


  std::vector<int> key_types;
  std::vector<bool> key_nullable;

  // Tables, outputs, descriptors and compaction chunks for the current caps.
  void layout(cudaStream_t stream)
  {
    const int stride = P.slot_bytes;
    int64_t ts = 0;
    std::vector<int64_t> tbase(ninst);
    for (int i = 0; i < ninst; ++i) {
      tbase[i] = ts;
      ts += caps[i] + 1;
    }
    total_slots = ts;
    d_tables.get(A, (size_t)ts * stride, stream);
    for (int i = 0; i < ninst; ++i) {
      insts[i].table = (uint8_t*)d_tables.p + (size_t)tbase[i] * stride;
      insts[i].cap_mask = (uint64_t)caps[i] - 1;
      insts[i].counters = (unsigned int*)d_counters.p + (size_t)i * counter_words;
    }
    ck(cudaMemcpyAsync(d_insts.p, insts.data(), sizeof(BatchInst) * ninst, cudaMemcpyHostToDevice, stream), "h2d");
    // outputs, sized by table capacity (an upper bound on the group count):
    // all data arrays first, then all masks in one region
    size_t total = 0, mtotal = 0;
    auto take = [](size_t& t, size_t bytes) {
      size_t o = t;
      t += (bytes + 255) & ~(size_t)255;
      return o;
    };
    out_off.assign(ninst, {});
    for (int pass = 0; pass < 2; ++pass) {
      for (int i = 0; i < ninst; ++i) {
        int64_t rows = caps[i] + 1;
        size_t mw = (size_t)((rows + 31) / 32) * 4;
        int c = 0;
        for (int k = 0; k < P.num_keys + nout; ++k, ++c) {
          bool is_key = k < P.num_keys;
          int tid = is_key ? key_types[k] : out_types[k - P.num_keys];
          bool nullable = is_key ? (bool)key_nullable[k] : P.outs[k - P.num_keys].nullable != 0;
          if (pass == 0) out_off[i].push_back({take(total, (size_t)rows * type_width(tid)), (size_t)-1});
          else if (nullable) out_off[i][c].second = take(mtotal, mw);
        }
      }
    }
    mask_begin = total;
    mask_end = total + mtotal;
    for (int i = 0; i < ninst; ++i)
      for (auto& oo : out_off[i])
        if (oo.second != (size_t)-1) oo.second += total;
    total += mtotal;
    d_outputs.get(A, total, stream);
    outs.assign(ninst, OutPtrs{});
    for (int i = 0; i < ninst; ++i) {
      OutPtrs& O = outs[i];
      std::memset(&O, 0, sizeof(O));
      uint8_t* base = (uint8_t*)d_outputs.p;
      int c = 0;
      for (int k = 0; k < P.num_keys; ++k, ++c) {
        O.key_data[k] = base + out_off[i][c].first;
        O.key_mask[k] = out_off[i][c].second == (size_t)-1 ? nullptr : (uint32_t*)(base + out_off[i][c].second);
      }
      for (int j = 0; j < nout; ++j, ++c) {
        O.out_data[j] = base + out_off[i][c].first;
        O.out_mask[j] = out_off[i][c].second == (size_t)-1 ? nullptr : (uint32_t*)(base + out_off[i][c].second);
      }
      O.counters = insts[i].counters;
    }
    d_outs.get(A, sizeof(OutPtrs) * ninst, stream);
    ck(cudaMemcpyAsync(d_outs.p, outs.data(), sizeof(OutPtrs) * ninst, cudaMemcpyHostToDevice, stream), "h2d");
    chunks.clear();
    for (int i = 0; i < ninst; ++i)
      for (int64_t b = 0; b < caps[i] + 1; b += 256) chunks.push_back(BatchChunk{i, 0, b});
    d_chunks.get(A, sizeof(BatchChunk) * std::max<size_t>(1, chunks.size()), stream);
    if (!chunks.empty())
      ck(cudaMemcpyAsync(d_chunks.p, chunks.data(), sizeof(BatchChunk) * chunks.size(), cudaMemcpyHostToDevice, stream),
         "h2d");
    stats.table_bytes = (int64_t)ts * stride;
    stats.output_bytes = (int64_t)total;
    stats.kernels_per_run = 4 + (chunks.empty() ? 0 : 1);
  }

  ~Impl()
  {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (h_counters) cudaFreeHost(h_counters);
  }

  template <int NT>
  void launch_agg(cudaStream_t s)
  {
    k_batch_aggregate<NT><<<grid_agg, NT, smem_bytes, s>>>(P, (const BatchInst*)d_insts.p, (const BatchTile*)d_tiles.p,
                                                           (int64_t)tiles.size(), (unsigned int*)d_work.p, tmpl);
  }
  static const void* agg_kernel(int block)
  {
    switch (block) {
      case 256: return (const void*)k_batch_aggregate<256>;
      case 1024: return (const void*)k_batch_aggregate<1024>;
      default: return (const void*)k_batch_aggregate<512>;
    }
  }

  void enqueue(cudaStream_t s)
  {
    ck(cudaMemsetAsync(d_counters.p, 0, (size_t)ninst * counter_words * 4, s), "memset counters");
    ck(cudaMemsetAsync(d_work.p, 0, 16, s), "memset work");
    k_batch_init<<<sms * 8, 256, 0, s>>>((uint8_t*)d_tables.p, total_slots, P.slot_bytes, tmpl);
    switch (block) {
      case 256: launch_agg<256>(s); break;
      case 1024: launch_agg<1024>(s); break;
      default: launch_agg<512>(s); break;
    }
    k_batch_finish<<<(ninst + 255) / 256, 256, 0, s>>>(P, (const BatchInst*)d_insts.p, ninst);
    // output masks start at zero (compaction ORs bits in)
    if (mask_end > mask_begin)
      ck(cudaMemsetAsync((uint8_t*)d_outputs.p + mask_begin, 0, mask_end - mask_begin, s), "memset masks");
    if (!chunks.empty())
      k_batch_compact<<<grid_compact, 256, 0, s>>>(P, (const BatchInst*)d_insts.p, (const OutPtrs*)d_outs.p,
                                                   (const BatchChunk*)d_chunks.p, (int64_t)chunks.size());
    ck(cudaMemcpyAsync(h_counters, d_counters.p, (size_t)ninst * counter_words * 4, cudaMemcpyDeviceToHost, s),
       "counters d2h");
  }
};

std::vector<int64_t> batch_estimate_groups(const std::vector<std::vector<Column>>& keys, int null_policy,
                                           const std::vector<std::vector<Request>>&, cudaStream_t stream,
                                           const Allocator& A)
{
  const int ninst = (int)keys.size();
  std::vector<int64_t> out(ninst, 1);
  if (ninst == 0) return out;
  std::vector<Column> k0 = keys[0];
  static const uint32_t kAnyMask = 0;
  for (int i = 0; i < ninst; ++i) {
    if (keys[i].size() != k0.size()) throw Error(ERR_LOGIC, "key layouts differ");
    for (size_t k = 0; k < k0.size(); ++k) {
      if (keys[i][k].type_id != k0[k].type_id) throw Error(ERR_LOGIC, "key types differ");
      if (keys[i][k].mask) k0[k].mask = &kAnyMask;
    }
  }
  Plan P;
  std::vector<int> ot;
  build_plan(k0, null_policy, {}, P, ot);
  std::vector<BatchInst> insts(ninst);
  for (int i = 0; i < ninst; ++i) {
    std::memset(&insts[i], 0, sizeof(BatchInst));
    for (size_t k = 0; k < keys[i].size(); ++k) {
      insts[i].key_data[k] = keys[i][k].data;
      insts[i].key_mask[k] = keys[i][k].mask;
      insts[i].key_off[k] = keys[i][k].offset;
    }
    insts[i].n_rows = keys[i][0].size;
  }
  DevBuf d_insts, d_stats;
  d_insts.get(A, sizeof(BatchInst) * ninst, stream);
  d_stats.get(A, (size_t)ninst * 16, stream);
  ck(cudaMemcpyAsync(d_insts.p, insts.data(), sizeof(BatchInst) * ninst, cudaMemcpyHostToDevice, stream), "h2d");
  size_t sm = (size_t)kSampleSlots * 32;
  allow_max_smem((const void*)k_batch_sample);
  k_batch_sample<<<ninst, 256, sm, stream>>>(P, (const BatchInst*)d_insts.p, (unsigned int*)d_stats.p);
  ck(cudaGetLastError(), "sketch launch");
  std::vector<unsigned int> st((size_t)ninst * 4);
  ck(cudaMemcpyAsync(st.data(), d_stats.p, st.size() * 4, cudaMemcpyDeviceToHost, stream), "d2h");
  ck(cudaStreamSynchronize(stream), "sketch sync");
  for (int i = 0; i < ninst; ++i) {
    const int64_t n = insts[i].n_rows;
    double d = st[i * 4 + 0], f1 = st[i * 4 + 1], m = st[i * 4 + 3];
    double est = n <= kSampleRows ? std::max(1.0, d)
                                  : std::min<double>((double)n, std::max(d, std::sqrt((double)n / std::max(1.0, m)) * f1 + (d - f1)));
    out[i] = (int64_t)std::max(1.0, est);
  }
  return out;
}

Batch::Batch() : impl(new Impl) {}
Batch::~Batch() = default;

namespace {
std::mutex g_batch_mu;
std::vector<BatchRule> g_batch_rules;
BatchLaunch g_batch_launch;
}  // namespace

void set_batch_tuning(const std::vector<BatchRule>& rules, const BatchLaunch& launch)
{
  std::lock_guard<std::mutex> lk(g_batch_mu);
  g_batch_rules = rules;
  g_batch_launch = launch;
}

void Batch::prepare(const std::vector<std::vector<Column>>& keys, int null_policy,
                    const std::vector<std::vector<Request>>& reqs, cudaStream_t stream, const Allocator& A,
                    const BatchOptions& bo)
{
  Impl& B = *impl;
  std::vector<BatchRule> rules;
  BatchLaunch launch;
  {
    std::lock_guard<std::mutex> lk(g_batch_mu);
    rules = g_batch_rules;
    launch = g_batch_launch;
  }
  const int ninst = (int)keys.size();
  if (ninst < 1) throw Error(ERR_LOGIC, "a batch needs at least one instance");
  if (reqs.size() != keys.size()) throw Error(ERR_LOGIC, "one request list per instance is required");
  // schema: instance 0's columns, with a column nullable when any instance's is
  std::vector<Column> k0 = keys[0];
  std::vector<Request> r0 = reqs[0];
  static const uint32_t kAnyMask = 0;
  for (int i = 0; i < ninst; ++i) {
    if (keys[i].size() != k0.size() || reqs[i].size() != r0.size())
      throw Error(ERR_LOGIC, "every instance of a batch must have the same key and request layout");
    for (size_t k = 0; k < k0.size(); ++k) {
      if (keys[i][k].type_id != k0[k].type_id) throw Error(ERR_LOGIC, "key types differ between instances");
      if (keys[i][k].size != keys[i][0].size) throw Error(ERR_LOGIC, "Size mismatch between key columns.");
      if (keys[i][k].mask) k0[k].mask = &kAnyMask;
    }
    for (size_t r = 0; r < r0.size(); ++r) {
      if (reqs[i][r].values.type_id != r0[r].values.type_id || reqs[i][r].aggs.size() != r0[r].aggs.size())
        throw Error(ERR_LOGIC, "value types or aggregations differ between instances");
      for (size_t j = 0; j < r0[r].aggs.size(); ++j)
        if (reqs[i][r].aggs[j].kind != r0[r].aggs[j].kind || reqs[i][r].aggs[j].ddof != r0[r].aggs[j].ddof)
          throw Error(ERR_LOGIC, "aggregations differ between instances");
      if (reqs[i][r].values.size != keys[i][0].size)
        throw Error(ERR_LOGIC, "Size mismatch between request values and groupby keys.");
      if (reqs[i][r].values.mask) r0[r].values.mask = &kAnyMask;
    }
  }
  // distinct data pointers per request so build_plan keeps one value column per request
  for (size_t r = 0; r < r0.size(); ++r) r0[r].values.data = (const void*)(uintptr_t)(0x1000 + 64 * r);
  build_plan(k0, null_policy, r0, B.P, B.out_types);
  if (B.P.need_second_pass) throw Error(ERR_UNSUPPORTED, "VARIANCE/STD are not supported in batched mode");
  B.ninst = ninst;
  B.nout = B.P.num_outs;
  B.A = A;
  B.stream = stream;
  slot_template(B.P, B.tmpl);

  // instance descriptors (column pointers; tables filled in below)
  B.insts.assign(ninst, BatchInst{});
  // which schema value column each request maps to (build_plan dedups identical views)
  std::vector<int> vcol(r0.size(), 0);
  for (size_t r = 0; r < r0.size(); ++r)
    for (int v = 0; v < B.P.num_vals; ++v)
      if (B.P.vals[v].data == r0[r].values.data) vcol[r] = v;
  for (int i = 0; i < ninst; ++i) {
    BatchInst& I = B.insts[i];
    for (size_t k = 0; k < keys[i].size(); ++k) {
      I.key_data[k] = keys[i][k].data;
      I.key_mask[k] = keys[i][k].mask;
      I.key_off[k] = keys[i][k].offset;
    }
    for (size_t r = 0; r < reqs[i].size(); ++r) {
      int v = vcol[r];
      I.val_data[v] = reqs[i][r].values.data;
      I.val_mask[v] = reqs[i][r].values.mask;
      I.val_off[v] = reqs[i][r].values.offset;
    }
    I.n_rows = keys[i][0].size;
  }
  int dev = 0;
  ck(cudaGetDevice(&dev), "cudaGetDevice");
  int sms = 148, optin = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  B.sms = sms;

  auto tnow = [] { return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count(); };
  double t_begin = tnow();
  // ---- per-instance group-count estimates from one sample launch ----
  B.d_insts.get(A, sizeof(BatchInst) * ninst, stream);
  ck(cudaMemcpyAsync(B.d_insts.p, B.insts.data(), sizeof(BatchInst) * ninst, cudaMemcpyHostToDevice, stream), "h2d");
  std::vector<unsigned int> st((size_t)ninst * 4);
  if (bo.est_groups.empty()) {
    B.d_stats.get(A, (size_t)ninst * 16, stream);
    size_t sm = (size_t)kSampleSlots * 32;
    allow_max_smem((const void*)k_batch_sample);
    k_batch_sample<<<ninst, 256, sm, stream>>>(B.P, (const BatchInst*)B.d_insts.p, (unsigned int*)B.d_stats.p);
    ck(cudaGetLastError(), "batch sample");
    ck(cudaMemcpyAsync(st.data(), B.d_stats.p, st.size() * 4, cudaMemcpyDeviceToHost, stream), "d2h");
    ck(cudaStreamSynchronize(stream), "sample sync");
  }
  if (!bo.est_groups.empty() && (int)bo.est_groups.size() != ninst)
    throw Error(ERR_LOGIC, "one group estimate per instance is required");
  B.stats.sample_s = tnow() - t_begin;
  // ---- sizing ----
  const int stride = B.P.slot_bytes;
  int scap_max = 1;
  {
    int budget = std::min(bo.smem_bytes >= 0 ? bo.smem_bytes : launch.smem_bytes, optin - 8192 - (int)sizeof(Plan));
    while ((int64_t)scap_max * 2 * stride <= budget) scap_max *= 2;
    if (scap_max * stride > budget) scap_max = 0;
  }
  B.caps.resize(ninst);
  for (int i = 0; i < ninst; ++i) {
    const int64_t n = B.insts[i].n_rows;
    double d = st[i * 4 + 0], f1 = st[i * 4 + 1], m = st[i * 4 + 3];
    double est;
    if (!bo.est_groups.empty()) est = (double)std::max<int64_t>(1, bo.est_groups[i]);
    else if (n <= kSampleRows) est = std::max(1.0, d);
    else {
      // Guaranteed-Error Estimator (Charikar et al. 2000): sqrt(n/m)*f1 + the keys
      // seen more than once; within a factor sqrt(n/m) of the truth.  The
      // trial run below grows any table that still overflows.
      est = std::sqrt((double)n / std::max(1.0, m)) * f1 + (d - f1);
      est = std::min<double>((double)n, std::max(d, est));
    }
    est *= bo.growth;
    uint64_t cap = pow2_at_least((uint64_t)std::max(64.0, std::ceil(est / 0.5)));
    cap = std::min<uint64_t>(cap, pow2_at_least((uint64_t)(2 * n + 2)));
    cap = std::max<uint64_t>(cap, 64);
    B.caps[i] = (int64_t)cap;
    // shared-memory stage only when the instance's groups fit a tile's table
    // (a tuning rule of the instance's size bucket may cap the table or turn
    // the stage off)
    int slots_cap = scap_max;
    double headroom = 2.0;
    for (const BatchRule& r : rules) {
      if (n > r.max_rows || (int64_t)est > r.max_groups) continue;
      if (r.smem_slots >= 0) slots_cap = std::min(slots_cap, r.smem_slots);
      if (r.headroom > 0) headroom = r.headroom;
      ++B.stats.ruled_instances;
      break;
    }
    int sc = 0;
    if (slots_cap >= 64 && est * headroom <= slots_cap && n > 4096) {
      sc = 64;
      while (sc < slots_cap && sc < est * 2 * headroom) sc *= 2;
    }
    B.insts[i].scap = sc;
    B.insts[i].sfill = std::max(1, sc / 2);
    B.stats.est_groups_total += (int64_t)est;
    if (sc) ++B.stats.smem_instances;
  }
  B.d_counters.get(A, (size_t)ninst * B.counter_words * 4, stream);
  B.d_work.get(A, 16, stream);
  // tiles: instances cut into tile_rows-row pieces, largest first
  std::vector<int> order(ninst);
  for (int i = 0; i < ninst; ++i) order[i] = i;
  std::sort(order.begin(), order.end(), [&](int a, int b) { return B.insts[a].n_rows > B.insts[b].n_rows; });
  B.tiles.clear();
  for (int i : order)
    for (int64_t b = 0; b < B.insts[i].n_rows; b += launch.tile_rows)
      B.tiles.push_back(BatchTile{i, 0, b, std::min(B.insts[i].n_rows, b + launch.tile_rows)});
  B.d_tiles.get(A, sizeof(BatchTile) * std::max<size_t>(1, B.tiles.size()), stream);
  if (!B.tiles.empty())
    ck(cudaMemcpyAsync(B.d_tiles.p, B.tiles.data(), sizeof(BatchTile) * B.tiles.size(), cudaMemcpyHostToDevice, stream),
       "h2d");
  if (!B.h_counters) ck(cudaMallocHost((void**)&B.h_counters, (size_t)ninst * B.counter_words * 4), "cudaMallocHost");
  // launch shapes
  B.smem_bytes = scap_max * stride;
  B.block = launch.block;
  B.stats.block = launch.block;
  B.stats.tile_rows = launch.tile_rows;
  allow_max_smem(Impl::agg_kernel(B.block));
  int bps = 0;
  ck(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, Impl::agg_kernel(B.block), B.block, B.smem_bytes), "occ");
  B.grid_agg = (int)std::min<int64_t>(std::max<int64_t>(1, (int64_t)B.tiles.size()), 1 << 30);
  B.grid_compact = sms * 8;
  B.stats.instances = ninst;
  B.stats.tiles = (int64_t)B.tiles.size();
  B.key_types.clear();
  for (auto& k : keys[0]) B.key_types.push_back(k.type_id);
  B.key_nullable.clear();
  for (auto& k : k0) B.key_nullable.push_back(k.mask != nullptr);
  double t_lay = tnow();
  B.layout(stream);
  B.stats.layout_s = tnow() - t_lay;
  // trial runs: grow the tables (and outputs) of instances that overflowed
  double t_trial = tnow();
  for (int round = 0; bo.trial; ++round) {
    B.stats.trial_rounds = round + 1;
    B.enqueue(stream);
    ck(cudaStreamSynchronize(stream), "trial sync");
    std::vector<int> over;
    for (int i = 0; i < ninst; ++i) {
      const unsigned int* c = B.h_counters + (size_t)i * B.counter_words;
      // overflowed, or fuller than 0.7 (long probe runs; a later run could overflow)
      if (c[1] || (int64_t)c[0] * 10 > B.caps[i] * 7) over.push_back(i);
    }
    if (over.empty()) break;
    if (round >= 6) throw Error(ERR_CUDA, "batch tables keep overflowing");
    B.stats.regrown += (int64_t)over.size();
    for (int i : over) B.caps[i] *= 4;
    B.layout(stream);
  }
  B.stats.trial_s = tnow() - t_trial;
  if (std::getenv("GB_TRACE")) {
    int64_t rows = 0;
    for (auto& I : B.insts) rows += I.n_rows;
    std::fprintf(stderr, "[gb batch] %d inst %lld rows: sample %.3fs layout %.3fs trial %.3fs x%d tables %.2fGB out %.2fGB\n",
                 ninst, (long long)rows, B.stats.sample_s, B.stats.layout_s, B.stats.trial_s, B.stats.trial_rounds,
                 B.stats.table_bytes / 1e9, B.stats.output_bytes / 1e9);
  }
  if (bo.use_graph) {
    cudaStream_t cs;
    ck(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking), "stream");
    ck(cudaStreamSynchronize(stream), "sync");
    ck(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal), "begin capture");
    try {
      B.enqueue(cs);
    } catch (...) {
      cudaGraph_t g;
      cudaStreamEndCapture(cs, &g);
      if (g) cudaGraphDestroy(g);
      cudaStreamDestroy(cs);
      throw;
    }
    ck(cudaStreamEndCapture(cs, &B.graph), "end capture");
    cudaStreamDestroy(cs);
    ck(cudaGraphInstantiate(&B.exec, B.graph, 0), "graph instantiate");
  }
}

void Batch::run(cudaStream_t stream)
{
  Impl& B = *impl;
  auto t0 = std::chrono::steady_clock::now();
  if (B.exec) ck(cudaGraphLaunch(B.exec, stream), "graph launch");
  else B.enqueue(stream);
  ck(cudaStreamSynchronize(stream), "batch sync");
  B.stats.run_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  int over = 0;
  for (int i = 0; i < B.ninst; ++i) {
    const unsigned int* c = B.h_counters + (size_t)i * B.counter_words;
    if (c[1]) ++over;
  }
  B.stats.overflowed = over;
  if (!over) return;
  if (B.exec) throw Error(ERR_CUDA, std::to_string(over) + " batch instance table(s) overflowed; prepare the batch again");
  // grow the overflowed tables and run again (the run is idempotent)
  for (int round = 0; over && round < 6; ++round) {
    for (int i = 0; i < B.ninst; ++i)
      if (B.h_counters[(size_t)i * B.counter_words + 1]) {
        B.caps[i] *= 4;
        ++B.stats.regrown;
      }
    B.layout(stream);
    B.enqueue(stream);
    ck(cudaStreamSynchronize(stream), "batch sync");
    over = 0;
    for (int i = 0; i < B.ninst; ++i) over += B.h_counters[(size_t)i * B.counter_words + 1] ? 1 : 0;
  }
  if (over) throw Error(ERR_CUDA, std::to_string(over) + " batch instance table(s) overflowed");
}

int Batch::num_instances() const { return impl->ninst; }

void Batch::result(int i, Result& R) const
{
  const Impl& B = *impl;
  if (i < 0 || i >= B.ninst) throw Error(ERR_LOGIC, "instance index out of range");
  const unsigned int* c = B.h_counters + (size_t)i * B.counter_words;
  R.num_groups = c[0];
  R.keys.clear();
  R.results.clear();
  R.alloc = Allocator{nullptr, nullptr, nullptr};  // buffers belong to the batch
  uint8_t* base = (uint8_t*)B.d_outputs.p;
  int col = 0;
  for (int k = 0; k < B.P.num_keys; ++k, ++col) {
    OutColumn o;
    o.type_id = B.P.keys[k].type_id;
    o.size = c[0];
    o.data = base + B.out_off[i][col].first;
    o.mask = B.out_off[i][col].second == (size_t)-1 ? nullptr : (uint32_t*)(base + B.out_off[i][col].second);
    o.null_count = c[4 + k];
    R.keys.push_back(o);
  }
  std::vector<OutColumn> flat;
  for (int j = 0; j < B.nout; ++j, ++col) {
    OutColumn o;
    o.type_id = B.out_types[j];
    o.size = c[0];
    o.data = base + B.out_off[i][col].first;
    o.mask = B.out_off[i][col].second == (size_t)-1 ? nullptr : (uint32_t*)(base + B.out_off[i][col].second);
    o.null_count = c[4 + B.P.num_keys + j];
    flat.push_back(o);
  }
  R.results.push_back(flat);
}

const BatchStats& Batch::stats() const { return impl->stats; }

}  // namespace gb

// ---------------------------------------------------------------------------
// C ABI
struct gb_batch {
  gb::Batch b;
  std::vector<gb_out_column> cols;  // scratch for gb_batch_result
};

namespace {
gb::Column to_col(const gb_column& c) { return gb::Column{c.type_id, c.size, c.data, c.null_mask, c.offset}; }

template <typename F>
int guarded(F&& f)
{
  try {
    gb::set_last_error("");
    f();
    return GB_OK;
  } catch (const gb::Error& e) {
    gb::set_last_error(e.what());
    return e.code;
  } catch (const std::bad_alloc& e) {
    gb::set_last_error(e.what());
    return GB_ERR_ALLOC;
  } catch (const std::exception& e) {
    gb::set_last_error(e.what());
    return GB_ERR_LOGIC;
  }
}
}  // namespace

extern "C" {

int gb_batch_prepare(int32_t num_instances, const gb_column* keys, int32_t num_keys, int32_t null_policy,
                     const gb_request* requests, int32_t num_requests, int32_t use_graph, void* stream,
                     const gb_allocator* mr, gb_batch** out)
{
  return guarded([&] {
    if (!out) throw gb::Error(gb::ERR_LOGIC, "null output pointer");
    *out = nullptr;
    if (num_instances < 1 || num_keys < 1 || !keys) throw gb::Error(gb::ERR_LOGIC, "empty batch");
    if (num_requests < 0 || (num_requests > 0 && !requests)) throw gb::Error(gb::ERR_LOGIC, "invalid request list");
    std::vector<std::vector<gb::Column>> kc(num_instances);
    std::vector<std::vector<gb::Request>> rq(num_instances);
    for (int i = 0; i < num_instances; ++i) {
      for (int k = 0; k < num_keys; ++k) kc[i].push_back(to_col(keys[(size_t)i * num_keys + k]));
      for (int r = 0; r < num_requests; ++r) {
        const gb_request& q = requests[(size_t)i * num_requests + r];
        gb::Request R;
        R.values = to_col(q.values);
        if (q.num_aggs < 0 || (q.num_aggs > 0 && !q.aggs)) throw gb::Error(gb::ERR_LOGIC, "invalid aggregation list");
        for (int j = 0; j < q.num_aggs; ++j) R.aggs.push_back(gb::AggSpec{q.aggs[j].kind, q.aggs[j].param});
        rq[i].push_back(R);
      }
    }
    gb::Allocator A = mr ? gb::Allocator{mr->allocate, mr->deallocate, mr->ctx} : gb::default_allocator();
    std::unique_ptr<gb_batch> b(new gb_batch);
    gb::BatchOptions bo;
    bo.use_graph = use_graph != 0;
    b->b.prepare(kc, null_policy, rq, (cudaStream_t)stream, A, bo);
    *out = b.release();
  });
}

int gb_batch_run(gb_batch* b, void* stream)
{
  return guarded([&] {
    if (!b) throw gb::Error(gb::ERR_LOGIC, "null batch");
    b->b.run((cudaStream_t)stream);
  });
}

int gb_batch_result(gb_batch* b, int32_t instance, int64_t* num_groups, gb_out_column* keys, gb_out_column* results)
{
  return guarded([&] {
    if (!b || !num_groups) throw gb::Error(gb::ERR_LOGIC, "null argument");
    gb::Result R;
    b->b.result(instance, R);
    *num_groups = R.num_groups;
    auto put = [](gb_out_column& o, const gb::OutColumn& c) {
      o.type_id = c.type_id;
      o.size = c.size;
      o.data = c.data;
      o.null_mask = c.mask;
      o.null_count = c.null_count;
    };
    if (keys)
      for (size_t k = 0; k < R.keys.size(); ++k) put(keys[k], R.keys[k]);
    if (results)
      for (size_t j = 0; j < R.results[0].size(); ++j) put(results[j], R.results[0][j]);
  });
}

int gb_batch_get_stats(const gb_batch* b, gb_batch_stats* out)
{
  return guarded([&] {
    if (!b || !out) throw gb::Error(gb::ERR_LOGIC, "null argument");
    const gb::BatchStats& s = b->b.stats();
    out->instances = s.instances;
    out->tiles = s.tiles;
    out->smem_instances = s.smem_instances;
    out->table_bytes = s.table_bytes;
    out->output_bytes = s.output_bytes;
    out->kernels_per_run = s.kernels_per_run;
    out->regrown = s.regrown;
    out->block = s.block;
    out->tile_rows = s.tile_rows;
    out->ruled_instances = s.ruled_instances;
  });
}

int gb_batch_set_tuning(const gb_batch_rule* rules, int32_t num_rules, const gb_batch_launch* launch)
{
  return guarded([&] {
    if (num_rules < 0 || (num_rules > 0 && !rules)) throw gb::Error(gb::ERR_LOGIC, "bad batch tuning rules");
    gb::BatchLaunch L;
    if (launch) {
      if (launch->block != 256 && launch->block != 512 && launch->block != 1024)
        throw gb::Error(gb::ERR_LOGIC, "batch block must be 256, 512 or 1024");
      if (launch->tile_rows < 1024) throw gb::Error(gb::ERR_LOGIC, "batch tile_rows must be >= 1024");
      if (launch->smem_bytes < 0) throw gb::Error(gb::ERR_LOGIC, "batch smem_bytes must be >= 0");
      L.block = launch->block;
      L.tile_rows = launch->tile_rows;
      L.smem_bytes = launch->smem_bytes;
    }
    std::vector<gb::BatchRule> v;
    for (int i = 0; i < num_rules; ++i)
      v.push_back(gb::BatchRule{rules[i].max_rows, rules[i].max_groups, rules[i].smem_slots,
                                rules[i].headroom_pct > 0 ? rules[i].headroom_pct / 100.0 : -1.0});
    gb::set_batch_tuning(v, L);
  });
}

void gb_batch_destroy(gb_batch* b) { delete b; }

}  // extern "C"
