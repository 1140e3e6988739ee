// gb_scatter.h -- host side of the bulk-copy pass 1 (gb_scatter.cuh).
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>

#include "gb_plan.h"

namespace gb {

struct PartArgs;

// Bytes of a StageSpec (the tile layout the kernel reads).
size_t part_scatter_spec_bytes();

// Shared-memory bytes of the bulk-copy pass 1 for this plan and partition
// count, with its tile layout written to spec_out (part_scatter_spec_bytes()
// bytes); 0 when a column cannot be bulk-copied tile by tile or the layout
// does not fit.  Tiles of 4096 rows with one CTA of 1024 threads per SM where
// they fit (unless small_only), else 2048 rows with two CTAs of 512 per SM.
size_t part_scatter_bulk_plan(const Plan& P, int nparts, int smem_optin, void* spec_out, bool small_only = false);

// Launches the bulk-copy pass 1 over all rows of P in the tile shape the plan chose.
void launch_part_scatter_bulk(const Plan& P, const PartArgs& A, const void* spec, size_t smem, cudaStream_t stream);

}  // namespace gb
