// gb_sorted.h -- host side of the sorted-chunk pass 2 (gb_sorted.cuh):
// shared-memory sizing and the launcher, compiled in gb_sorted.cu.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>

#include "gb_plan.h"

namespace gb {

struct PartArgs;
struct TableRef;
struct DenseRef;
struct SlotTemplate;

// Staged width of a value column: 8-byte columns keep 8 bytes, narrower ones
// are staged as 4 (zero-extended bits).
__host__ __device__ inline int sorted_stage_width(int w) { return w == 8 ? 8 : 4; }

// Shared-memory bytes of k_part_sorted: the table (scap slots, plus the
// all-ones key's slot for one-word keys), two per-slot count arrays, and the
// sorted stage of a chunk of C rows.
inline size_t part_sorted_smem(const Plan& P, int scap, int C, bool have_bits)
{
  auto a16 = [](size_t x) { return (x + 15) & ~(size_t)15; };
  const int nslots = scap + (P.key_words == 1);
  size_t b = a16((size_t)nslots * P.slot_bytes);
  b += 2 * a16((size_t)(nslots + 1) * 4);
  b += a16((size_t)C * 2);
  if (have_bits) b += a16((size_t)C);
  for (int v = 0; v < P.num_vals; ++v) b += (size_t)C * sorted_stage_width(P.vals[v].width);
  return b;
}

// Rows per chunk (threads x rows per thread) of the sorted kernel the variant
// and column count select: 0 512x4 (default), 3 256x8; more than four value
// columns take 512x2.
int part_sorted_rows(int variant, int num_vals);

// Launches k_part_sorted over A's work items (A.items, A.nitems, A.work).
// wagg: rank rows per warp with one atomic (items of heavy partitions).
void launch_part_sorted(int variant, const Plan& P2, const PartArgs& A, const TableRef& G, const DenseRef& D,
                        int scap, int sfill, const SlotTemplate& tmpl, size_t smem, bool wagg, cudaStream_t stream);

}  // namespace gb
