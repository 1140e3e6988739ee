// gb_batch.h -- batched groupby (many instances of one schema per launch).
#pragma once
#include <memory>
#include <vector>

#include "gb_engine.h"

namespace gb {

// Batch tuning (an autotuner picks these; see cudf_b200.autotune):
//  launch-wide: threads per CTA of the aggregation kernel (256, 512 or 1024),
//  rows per tile, and the shared-memory budget of a tile's table;
//  per instance, by the first rule with rows <= max_rows and estimated
//  groups <= max_groups: at most smem_slots shared slots (0: the global table
//  only) and the shared stage only when groups * headroom <= slots.
struct BatchRule {
  int64_t max_rows;
  int64_t max_groups;
  int smem_slots;    // -1: unset
  double headroom;   // <= 0: unset
};
struct BatchLaunch {
  int block = 512;
  int64_t tile_rows = 65536;
  int smem_bytes = 160 * 1024;
};
void set_batch_tuning(const std::vector<BatchRule>& rules, const BatchLaunch& launch);

struct BatchOptions {
  bool use_graph = false;  // capture the run sequence once, replay it
  int smem_bytes = -1;     // shared-memory budget of a tile's table (-1: the tuned launch's)
  double growth = 1.0;     // multiplies every instance's group estimate (tables size from it)
  bool trial = true;       // run once at prepare time and regrow overflowing / overfull tables
  std::vector<int64_t> est_groups;  // per-instance estimates from the caller (skips sampling)
};

struct BatchStats {
  int64_t instances = 0;
  int64_t tiles = 0;
  int64_t smem_instances = 0;
  int64_t est_groups_total = 0;
  int64_t table_bytes = 0;
  int64_t output_bytes = 0;
  int64_t overflowed = 0;
  int64_t regrown = 0;  // instance tables grown after a trial run overflowed
  int trial_rounds = 0;
  double sample_s = 0, layout_s = 0, trial_s = 0, run_s = 0;
  int kernels_per_run = 0;
  int block = 0;             // launch used
  int64_t tile_rows = 0;
  int64_t ruled_instances = 0;  // instances a tuning rule sized
};

// Device-side key sketch: estimated group count of each instance (one
// sampling launch; every instance must share the key layout).
std::vector<int64_t> batch_estimate_groups(const std::vector<std::vector<Column>>& keys, int null_policy,
                                           const std::vector<std::vector<Request>>& reqs, cudaStream_t stream,
                                           const Allocator& A);

class Batch {
 public:
  Batch();
  ~Batch();
  // Samples every instance, sizes the per-instance tables and outputs, and
  // (with use_graph) captures the run sequence.  Column views must stay valid
  // and keep their shapes for every later run().
  void prepare(const std::vector<std::vector<Column>>& keys, int null_policy,
               const std::vector<std::vector<Request>>& reqs, cudaStream_t stream, const Allocator& A,
               const BatchOptions& opt);
  // Aggregates every instance (graph replay when captured); synchronises.
  void run(cudaStream_t stream);
  int num_instances() const;
  // Views of instance i's results (buffers owned by the batch, valid until the
  // next run or destruction).
  void result(int i, Result& R) const;
  const BatchStats& stats() const;

  struct Impl;

 private:
  std::unique_ptr<Impl> impl;
};

}  // namespace gb
