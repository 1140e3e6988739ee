// gb_sorted.cu -- instantiations and launcher of the sorted-chunk pass 2
// (gb_sorted.cuh), kept in their own compilation unit.
#include "gb_engine.h"
#include "gb_sorted.cuh"

namespace gb {

int grid_for(const void* kernel, int block, size_t smem, int bps_cap);

int part_sorted_rows(int variant, int num_vals)
{
  if (num_vals > 4) return 2 * 512;
  return variant == 3 ? 8 * 256 : 4 * 512;
}

namespace {
template <int KW, int R, int NT, int MAXV>
void launch_one(const Plan& P2, const PartArgs& A, const TableRef& G, const DenseRef& D, int scap, int sfill,
                const SlotTemplate& tmpl, size_t smem, bool wagg, cudaStream_t stream)
{
  const void* k = wagg ? (const void*)k_part_sorted<KW, R, NT, MAXV, true>
                       : (const void*)k_part_sorted<KW, R, NT, MAXV, false>;
  allow_max_smem(k);
  int grid = std::min(grid_for(k, NT, smem, 0), A.nitems);
  // runs longer than two threads' shares are cut into pieces at the thread ranges
  const int L = 2 * R;
  if (wagg)
    k_part_sorted<KW, R, NT, MAXV, true><<<grid, NT, smem, stream>>>(P2, A, G, D, scap, sfill, L, tmpl);
  else
    k_part_sorted<KW, R, NT, MAXV, false><<<grid, NT, smem, stream>>>(P2, A, G, D, scap, sfill, L, tmpl);
}
}  // namespace

void launch_part_sorted(int variant, const Plan& P2, const PartArgs& A, const TableRef& G, const DenseRef& D,
                        int scap, int sfill, const SlotTemplate& tmpl, size_t smem, bool wagg, cudaStream_t stream)
{
  if (A.nitems <= 0) return;
  const bool kw1 = P2.key_words == 1;
  if (P2.num_vals > 4) {
    if (kw1) launch_one<1, 2, 512, 8>(P2, A, G, D, scap, sfill, tmpl, smem, wagg, stream);
    else launch_one<2, 2, 512, 8>(P2, A, G, D, scap, sfill, tmpl, smem, wagg, stream);
  } else if (variant == 3) {
    if (kw1) launch_one<1, 8, 256, 4>(P2, A, G, D, scap, sfill, tmpl, smem, wagg, stream);
    else launch_one<2, 8, 256, 4>(P2, A, G, D, scap, sfill, tmpl, smem, wagg, stream);
  } else {
    if (kw1) launch_one<1, 4, 512, 4>(P2, A, G, D, scap, sfill, tmpl, smem, wagg, stream);
    else launch_one<2, 4, 512, 4>(P2, A, G, D, scap, sfill, tmpl, smem, wagg, stream);
  }
}

}  // namespace gb
