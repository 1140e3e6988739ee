// gb_scatter.cu -- launcher of the bulk-copy pass 1 (gb_scatter.cuh), in its
// own compilation unit.
#include "gb_engine.h"
#include "gb_scatter.cuh"
#include "gb_scatter.h"

namespace gb {

namespace {
constexpr int kBulkThreads = 512;
constexpr int kBulkRows = 2048;

template <int KW>
const void* bulk_kernel()
{
  return (const void*)k_part_scatter_bulk<KW, kBulkThreads, kBulkRows>;
}
}  // namespace

size_t part_scatter_bulk_plan(const Plan& P, int nparts, int smem_optin, void* spec_out)
{
  StageSpec& S = *(StageSpec*)spec_out;
  if (!part_scatter_bulk_ok(P, kBulkRows, S)) return 0;
  const size_t sm = part_scatter_bulk_smem(S, P.key_words, kBulkRows, nparts);
  // static shared memory of the kernel (barrier, scan temporaries) plus slack
  if (sm + 4096 > (size_t)smem_optin) return 0;
  return sm;
}

size_t part_scatter_spec_bytes() { return sizeof(StageSpec); }

void launch_part_scatter_bulk(const Plan& P, const PartArgs& A, const void* spec, size_t smem, cudaStream_t stream)
{
  const StageSpec& S = *(const StageSpec*)spec;
  const void* k = P.key_words == 1 ? bulk_kernel<1>() : bulk_kernel<2>();
  allow_max_smem(k);
  const int64_t ntiles = (P.num_rows + kBulkRows - 1) / kBulkRows;
  const int grid = (int)std::min<int64_t>(grid_for(k, kBulkThreads, smem, 2), ntiles);
  if (P.key_words == 1)
    k_part_scatter_bulk<1, kBulkThreads, kBulkRows><<<grid, kBulkThreads, smem, stream>>>(P, A, S);
  else
    k_part_scatter_bulk<2, kBulkThreads, kBulkRows><<<grid, kBulkThreads, smem, stream>>>(P, A, S);
}

}  // namespace gb
