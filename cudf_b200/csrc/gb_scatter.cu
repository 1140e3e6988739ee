// gb_scatter.cu -- launcher of the bulk-copy pass 1 (gb_scatter.cuh), in its
// own compilation unit.
#include "gb_engine.h"
#include "gb_scatter.cuh"
#include "gb_scatter.h"

namespace gb {

namespace {
// Launch shapes: 4096-row tiles with one 1024-thread CTA per SM where the
// tile's layout fits shared memory, else 2048-row tiles with two 512-thread
// CTAs per SM.
constexpr int kBigRows = 4096, kBigThreads = 1024;
constexpr int kMidRows = 3072;  // 1024 threads, 3 rows each
constexpr int kRows = 2048, kThreads = 512;
}  // namespace

size_t part_scatter_bulk_plan(const Plan& P, int nparts, int smem_optin, void* spec_out, bool small_only)
{
  StageSpec& S = *(StageSpec*)spec_out;
  // static shared memory of the kernel (barriers, scan temporaries) plus slack
  const size_t limit = (size_t)smem_optin - 8192;
  // one 1024-thread CTA per SM on 4096-row tiles where they fit, else on
  // 3072-row tiles (wide keys with many partitions), else two CTAs of 512 on
  // 2048-row tiles: the per-tile partition work is paid per tile, so the
  // largest tile that fits wins
  for (int T : {kBigRows, kMidRows}) {
    if (small_only || !part_scatter_bulk_ok(P, T, S)) continue;
    const size_t sm = part_scatter_bulk_smem(S, P.key_words, T, nparts);
    if (sm <= limit) return sm;
  }
  if (!part_scatter_bulk_ok(P, kRows, S)) return 0;
  const size_t sm = part_scatter_bulk_smem(S, P.key_words, kRows, nparts);
  return 2 * sm <= limit ? sm : 0;
}

size_t part_scatter_spec_bytes() { return sizeof(StageSpec); }

namespace {
template <int KW, int NT, int T, int MINB>
void launch_bulk(const Plan& P, const PartArgs& A, const StageSpec& S, size_t smem, cudaStream_t stream)
{
  const void* k = (const void*)k_part_scatter_bulk<KW, NT, T, MINB>;
  allow_max_smem(k);
  const int64_t ntiles = (P.num_rows + T - 1) / T;
  const int grid = (int)std::min<int64_t>(grid_for(k, NT, smem, MINB), ntiles);
  k_part_scatter_bulk<KW, NT, T, MINB><<<grid, NT, smem, stream>>>(P, A, S);
}
}  // namespace

void launch_part_scatter_bulk(const Plan& P, const PartArgs& A, const void* spec, size_t smem, cudaStream_t stream)
{
  const StageSpec& S = *(const StageSpec*)spec;
  const bool is_big = S.tile_rows == kBigRows;
  if (S.tile_rows == kMidRows) {
    if (P.key_words == 1) launch_bulk<1, kBigThreads, kMidRows, 1>(P, A, S, smem, stream);
    else launch_bulk<2, kBigThreads, kMidRows, 1>(P, A, S, smem, stream);
    return;
  }
  if (P.key_words == 1) {
    if (is_big) launch_bulk<1, kBigThreads, kBigRows, 1>(P, A, S, smem, stream);
    else launch_bulk<1, kThreads, kRows, 2>(P, A, S, smem, stream);
  } else {
    if (is_big) launch_bulk<2, kBigThreads, kBigRows, 1>(P, A, S, smem, stream);
    else launch_bulk<2, kThreads, kRows, 2>(P, A, S, smem, stream);
  }
}

}  // namespace gb
