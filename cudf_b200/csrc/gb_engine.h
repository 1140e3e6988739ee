// gb_engine.h -- host side of the groupby engine (C++; no torch types).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <stdexcept>
#include <string>
#include <vector>

#include "gb_plan.h"

namespace gb {

// Error classes mirroring libcudf's (cpp/include/cudf/utilities/error.hpp:177-228):
// LOGIC = cudf::logic_error, CUDA = cudf::cuda_error, ALLOC = std::bad_alloc.
enum ErrCode : int { OK = 0, ERR_LOGIC = 1, ERR_CUDA = 2, ERR_ALLOC = 3, ERR_UNSUPPORTED = 4 };

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

struct Column {
  int32_t type_id;
  int64_t size;
  const void* data;
  const uint32_t* mask;
  int64_t offset;
};

struct AggSpec {
  int32_t kind;
  int32_t ddof;
};

struct Request {
  Column values;
  std::vector<AggSpec> aggs;
};

// Stream-ordered device memory resource (the role of rmm's
// device_memory_resource in cudf::groupby::aggregate).
struct Allocator {
  void* (*allocate)(void* ctx, size_t bytes, void* stream);
  void (*deallocate)(void* ctx, void* p, size_t bytes, void* stream);
  void* ctx;
};
Allocator default_allocator();

struct OutColumn {
  int32_t type_id = 0;
  int64_t size = 0;
  void* data = nullptr;
  uint32_t* mask = nullptr;
  int64_t null_count = 0;
  size_t data_bytes = 0;
  size_t mask_bytes = 0;
};

struct Result {
  int64_t num_groups = 0;
  std::vector<OutColumn> keys;
  std::vector<std::vector<OutColumn>> results;
  Allocator alloc{};
  cudaStream_t stream = nullptr;
  void release();  // frees every buffer through alloc
};

// Engine tunables (an autotuner picks these per size bucket).
struct Options {
  int block = 512;             // threads per CTA of the global-table and shared-stage kernels
  int blocks_per_sm = 0;       // 0 = occupancy limited
  int smem_bytes = 96 * 1024;  // shared-memory table bytes per CTA (0 disables the smem stage)
  double smem_fill = 0.5;      // fraction of smem slots a CTA may claim
  int64_t smem_max_groups = -1;  // use the smem stage when est. groups <= this (-1: derived)
  double load_factor = 0.5;    // global table target load
  int64_t groups_hint = -1;    // caller's group-count estimate (-1: sample)
  int force_mode = -1;         // -1 auto, 0 global only, 1 smem stage
  int profile = 0;             // time kernels with CUDA events
  int scatter = 7;             // partitioned pass 1: 7 bulk-copy tiles where the columns allow (else 0), 0-6 launch shapes of the per-thread scatter
  double part_fill = 0.7;      // partitioned mode: expected groups per partition / shared-table slots (sets the partition count)
  int pass2 = 1;               // partitioned pass 2: 1 per-row shared reductions, 0/2 sorted chunks 512x4, 3 sorted 256x8
  int wagg_pct = 125;          // partitioned pass 2: warp-combined updates for partitions above this % of the average rows
  uint32_t set_mask = 0;       // OPT_* bits of the fields a caller set explicitly
  // internal: 0 reads every outcome (group counts, overflow flags, null
  // counts) back once, after the compaction, sizing the outputs by an upper
  // bound; a call whose flags show an overflow is redone with 1, which checks
  // after each stage and regrows tables as it goes
  int sync_checks = 0;
};

// Option fields, as bits of Options::set_mask and TuningRule::mask.
enum OptBits : uint32_t {
  OPT_BLOCK = 1, OPT_BPS = 2, OPT_SMEM = 4, OPT_FILL = 8, OPT_SMEM_MAX = 16, OPT_LOAD = 32,
  OPT_MODE = 64, OPT_SCATTER = 128, OPT_PASS2 = 256, OPT_PART_FILL = 512, OPT_WAGG = 1024
};

// A process-wide tuning rule: for calls with at most max_rows rows and at most
// max_groups estimated groups, the fields in `mask` take `opt`'s values unless
// the handle set them itself.  The first matching rule applies.
struct TuningRule {
  int64_t max_rows;
  int64_t max_groups;
  int key_words;  // 0 any, else the packed key width the rule was tuned for
  Options opt;
  uint32_t mask;
};
void set_tuning_rules(const std::vector<TuningRule>& rules);
// Applies the first rule matching (rows, groups) to `o`; returns its index or -1.
int apply_tuning_rules(Options& o, int64_t rows, int64_t groups, int key_words, uint32_t* applied = nullptr);

struct Stats {
  int64_t est_groups = 0;
  int64_t capacity = 0;
  int mode = 0;     // 0 global, 1 smem stage
  int retries = 0;
  int kernels = 0;  // kernels launched by this call
  double agg_kernel_ms = 0;  // aggregation kernels (partitioned mode: both passes)
  double compact_ms = 0;
  double scatter_ms = 0;     // partitioned mode: pass 1 alone
  int rule = -1;             // tuning rule applied (-1: none)
};

// Builds the plan (validates like cudf::groupby::aggregate,
// cpp/src/groupby/groupby.cu:202-219, and cpp/src/groupby/groupby.cu:174-190).
void build_plan(const std::vector<Column>& keys, int null_policy, const std::vector<Request>& reqs,
                Plan& P, std::vector<int>& out_types);

// The groupby: keys table + requests -> unique keys and one column per
// requested aggregation, in request order.
Result aggregate(const std::vector<Column>& keys, int null_policy, const std::vector<Request>& reqs,
                 cudaStream_t stream, const Allocator& alloc, const Options& opt, Stats* stats);

// Global-table aggregation with its table in caller-provided device scratch
// and its results in caller-provided columns; makes no device allocation.
int64_t aggregate_into_scratch(const std::vector<Column>& keys, int null_policy,
                               const std::vector<Request>& reqs, cudaStream_t stream, void* scratch,
                               size_t scratch_bytes, int64_t max_groups,
                               std::vector<OutColumn>& out_keys, std::vector<OutColumn>& out_results);

// Sets the message gb_last_error() returns on this thread.
void set_last_error(const std::string& msg);

// type helpers
int type_width(int type_id);
bool valid_agg(int type_id, int kind);
int target_type(int type_id, int kind);

// Lets `kernel` take up to the device's opt-in shared memory per block.  Set
// once per (device, kernel) at that maximum, not per launch at the size the
// launch needs: engine calls on several host threads launch the same kernels
// with different shared-memory sizes, and a per-launch attribute set by one
// thread could be lowered by another between its set and its launch.
void allow_max_smem(const void* kernel);
// CTAs that fill the device for a kernel at this block size and shared memory
int grid_for(const void* kernel, int block, size_t smem, int bps_cap);

}  // namespace gb
