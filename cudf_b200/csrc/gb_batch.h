// gb_batch.h -- batched groupby (many instances of one schema per launch).
#pragma once
#include <memory>
#include <vector>

#include "gb_engine.h"

namespace gb {

struct BatchOptions {
  bool use_graph = false;  // capture the run sequence once, replay it
  int smem_bytes = 160 * 1024;
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
