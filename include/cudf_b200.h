/*
 * cudf_b200.h -- C ABI of the B200 hash groupby-aggregate engine.
 *
 * A drop-in for libcudf's hash groupby path:
 *   cudf::groupby::groupby(keys, null_policy).aggregate(requests, stream, mr)
 *   (cpp/include/cudf/groupby.hpp:126-197, cpp/src/groupby/groupby.cu:51-62,202-219)
 * as bound from Python by pylibcudf.groupby.GroupBy.aggregate
 *   (python/cudf/cudf/_lib/pylibcudf/groupby.pyx:94-155)
 * and from Java by TableJni.cpp:3124-3155.
 *
 * Conventions (the same as libcudf's column_view, cpp/include/cudf/types.hpp):
 *  - type ids are cudf::type_id values, aggregation kinds cudf::aggregation::Kind
 *  - null masks are LSB-first 32-bit words (bit i of word i/32 set = row i valid),
 *    NULL when the column has no nulls; `offset` shifts both data and mask
 *  - every pointer in a gb_column / gb_out_column is device memory
 *  - functions return 0 on success or a GB_ERR_* code; gb_last_error() gives the
 *    message of the calling thread's last failure.  Nothing throws across the ABI.
 *  - work is stream-ordered on the given cudaStream_t (passed as void*); the call
 *    returns when the results are complete.
 */
#ifndef CUDF_B200_H
#define CUDF_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define GB_API __attribute__((visibility("default")))
#else
#define GB_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define GB_OK 0
#define GB_ERR_LOGIC 1       /* cudf::logic_error: bad arguments, size mismatch, invalid type/agg */
#define GB_ERR_CUDA 2        /* cudf::cuda_error */
#define GB_ERR_ALLOC 3       /* std::bad_alloc / rmm::bad_alloc */
#define GB_ERR_UNSUPPORTED 4 /* outside this engine's scope (e.g. key rows wider than 127 bits) */

#define GB_NULL_EXCLUDE 0    /* cudf::null_policy::EXCLUDE */
#define GB_NULL_INCLUDE 1    /* cudf::null_policy::INCLUDE */

/* A non-owning column view (cudf::column_view, cpp/include/cudf/column/column_view.hpp). */
typedef struct gb_column {
  int32_t type_id;
  int64_t size;
  const void* data;
  const uint32_t* null_mask;
  int64_t offset;
} gb_column;

/* One aggregation: cudf::aggregation::Kind plus its parameter (ddof for VARIANCE/STD,
 * ignored otherwise).  COUNT with null_policy::INCLUDE is kind COUNT_ALL (5). */
typedef struct gb_agg {
  int32_t kind;
  int32_t param;
} gb_agg;

/* cudf::groupby::aggregation_request (cpp/include/cudf/groupby.hpp:59-62). */
typedef struct gb_request {
  gb_column values;
  int32_t num_aggs;
  const gb_agg* aggs;
} gb_request;

/* An owning output column (cudf::column). */
typedef struct gb_out_column {
  int32_t type_id;
  int64_t size;
  void* data;
  uint32_t* null_mask;  /* NULL when the column is not nullable */
  int64_t null_count;
} gb_out_column;

/* pair<unique_ptr<table>, vector<aggregation_result>> (cpp/include/cudf/groupby.hpp:189-192):
 * keys[num_keys] are the unique key rows; results[r][j] is aggregation j of request r. */
typedef struct gb_result {
  int64_t num_groups;
  int32_t num_keys;
  gb_out_column* keys;
  int32_t num_requests;
  const int32_t* num_results;
  gb_out_column** results;
  void* impl;
} gb_result;

/* Stream-ordered device memory resource (the `mr` of cudf::groupby::aggregate).
 * allocate returns NULL on failure, else a block aligned to at least 16 bytes
 * (RMM's resources give 256). */
typedef struct gb_allocator {
  void* (*allocate)(void* ctx, size_t bytes, void* stream);
  void (*deallocate)(void* ctx, void* ptr, size_t bytes, void* stream);
  void* ctx;
} gb_allocator;

typedef struct gb_handle gb_handle;

/* cudf::groupby::groupby::groupby (cpp/src/groupby/groupby.cu:51-62).  The handle does
 * not own the key columns (cpp/include/cudf/groupby.hpp:111-113).  keys_are_sorted is
 * accepted for API parity and does not change the results of the hash path. */
GB_API int gb_create(const gb_column* keys, int32_t num_keys, int32_t null_policy,
              int32_t keys_are_sorted, gb_handle** out);

/* cudf::groupby::groupby::aggregate (cpp/src/groupby/groupby.cu:202-219).
 * mr may be NULL (stream-ordered cudaMallocAsync pool). */
GB_API int gb_aggregate(gb_handle* handle, const gb_request* requests, int32_t num_requests,
                 void* stream, const gb_allocator* mr, gb_result** out);

/* Frees a result and every column it owns (through the allocator that made it). */
GB_API void gb_result_free(gb_result* result);

/* Destroys a handle (cudf::groupby::groupby::~groupby). */
GB_API void gb_destroy(gb_handle* handle);

/* Message of the calling thread's last error ("" if none). */
GB_API const char* gb_last_error(void);

/* Result type id of an aggregation (cudf::detail::target_type,
 * cpp/include/cudf/detail/aggregation/aggregation.hpp:1168-1290); 0 if invalid. */
GB_API int32_t gb_target_type(int32_t type_id, int32_t kind);

/* 1 when the (type, aggregation) pair is supported by the hash path
 * (cpp/src/groupby/hash/groupby.cu:633-649), else 0. */
GB_API int32_t gb_is_valid_aggregation(int32_t type_id, int32_t kind);

/* Engine tuning of a handle (no counterpart in libcudf, whose hash path has no
 * tunables: cpp/src/groupby/hash/groupby.cu:64-67,570-572).  Fields < 0 keep
 * the default.  force_mode: -1 auto, 0 global table only, 1 shared-memory stage,
 * 2 hash-partitioned shared-memory aggregation. */
typedef struct gb_tuning {
  int32_t block;            /* threads per CTA of the aggregation kernel */
  int32_t blocks_per_sm;    /* CTAs per SM (0 = occupancy limit) */
  int32_t smem_bytes;       /* shared-memory table bytes per CTA */
  int32_t smem_fill_pct;    /* percent of shared slots a CTA may claim */
  int64_t smem_max_groups;  /* use the shared-memory stage up to this many groups */
  int32_t load_factor_pct;  /* global table load factor in percent */
  int32_t force_mode;
  int64_t groups_hint;      /* caller's estimate of the number of groups (skips sampling) */
  int32_t profile;          /* 1: time the aggregation and compaction kernels with CUDA events */
  int32_t scatter;          /* partitioned pass 1: 7 (default) tiles of 4096 (or 2048) rows staged in
                               shared memory by bulk copies when every column allows it (16-byte
                               aligned rows), else 0; 0-6 the per-thread launch shapes, threads x
                               rows per thread: 0 512x8, 1 256x16, 2 512x16, 3 1024x8, 4 512x8 with
                               the next column's loads issued early, 5 1024x4, 6 256x8; 8 as 7 with
                               2048-row tiles, two CTAs per SM */
  int32_t pass2;            /* partitioned pass 2: 1 per-row shared reductions (default); 0 (or 2)
                               chunks counting-sorted by slot, 512 threads x 4 rows; 3 sorted,
                               256 threads x 8 rows; 4 per-row, 512 threads x 2 rows (plans of
                               up to four value columns, else as 1) */
  int32_t part_fill_pct;    /* partitioned mode: expected groups per partition as a percentage of
                               the pass-2 shared table's slots (default 70; sets the partition
                               count, a power of two) */
  int32_t wagg_pct;         /* partitioned pass 2: a partition holding more rows than this percentage
                               of the average partition (a heavy key) has the rows of one slot
                               combined per warp before each shared update (default 125; 0: every
                               partition; when unset and the sketch finds many heavy hitters -- at
                               least 32 of its row-count buckets above four times the mean of the
                               non-empty ones -- every partition); negative: unset */
} gb_tuning;

/* What the last gb_aggregate on a handle did. */
typedef struct gb_stats {
  int64_t est_groups;
  int64_t capacity;
  int32_t mode;             /* 0 global table, 1 shared-memory stage, 2 partitioned */
  int32_t retries;          /* table-overflow retries */
  int32_t kernels;          /* kernels launched */
  double agg_kernel_ms;     /* device time of the aggregation kernel(s) (profile = 1) */
  double compact_ms;        /* device time of the compaction kernel (profile = 1) */
  double scatter_ms;        /* partitioned mode: device time of the partition pass (profile = 1) */
  int32_t rule;             /* index of the tuning rule applied, -1 if none */
} gb_stats;

GB_API int gb_set_tuning(gb_handle* handle, const gb_tuning* tuning);

/* Process-wide tuning by size bucket (no counterpart in libcudf).  Each call
 * of gb_aggregate, once it has estimated its number of groups, takes the first
 * rule with rows <= max_rows, groups <= max_groups and a matching key width,
 * and applies the rule's
 * set fields (block, blocks_per_sm, smem_bytes, smem_fill_pct, smem_max_groups,
 * load_factor_pct, force_mode, scatter, pass2, part_fill_pct, wagg_pct) except those its
 * handle set with
 * gb_set_tuning.  Replaces all rules; NULL/0 clears them.  The rules come
 * from cudf_b200.autotune, which times the candidates per bucket. */
typedef struct gb_tuning_rule {
  int64_t max_rows;
  int64_t max_groups;
  int32_t key_words;        /* 1 or 2: only calls whose keys pack into that many 64-bit
                               words (single 64-bit key: 1); 0: any */
  gb_tuning tuning;         /* fields < 0 (block, smem_fill_pct, load_factor_pct: <= 0) unset */
} gb_tuning_rule;
GB_API int gb_set_tuning_rules(const gb_tuning_rule* rules, int32_t num_rules);
GB_API int gb_get_stats(const gb_handle* handle, gb_stats* out);

/* Allocation-free groupby.  No counterpart in libcudf: its groupby always
 * allocates its hash table and results through `mr`.  This entry point is for
 * callers that cannot allocate device memory where they run -- code whose GPU
 * memory belongs to another allocator that forbids outside allocations (a
 * JVM or framework pool sized to the whole device), or loops where
 * cudaMalloc/cudaFree are off limits because they synchronise the device.
 * It runs the global-hash-table aggregation with its table in a fixed,
 * file-scope device array of GB_NOALLOC_SCRATCH_BYTES (held by every GPU that
 * loads the library until the process exits) and writes into caller-allocated
 * outputs: it calls no cudaMalloc, cudaFree or other allocating routine.
 *  - out_keys[num_keys] and out_results[sum of num_aggs] (request order): the
 *    caller sets `data` (room for max_groups rows of the result type, see
 *    gb_target_type) and, for nullable outputs, `null_mask` (room for
 *    ceil(max_groups/32) words); the call fills type_id, size and null_count.
 *  - the table needs (next_pow2(2*max_groups)+1) slots of the plan's slot size
 *    plus 4 KiB of counters; larger requests are rejected with GB_ERR_LOGIC,
 *    and so is a groupby that finds more than max_groups groups.
 *  - the first call on a device looks up the array's device address
 *    (cudaGetSymbolAddress; again if the device's context was recreated);
 *    make that call before any stream capture.
 *  - the call is synchronous: it waits for its stream and returns with the
 *    results complete.
 *  - all calls share the array: calls that overlap on the GPU race and must be
 *    serialised by the caller. */
#define GB_NOALLOC_SCRATCH_BYTES (16u * 1024u * 1024u)
GB_API int gb_aggregate_noalloc(const gb_column* keys, int32_t num_keys, int32_t null_policy,
                                const gb_request* requests, int32_t num_requests, int64_t max_groups,
                                gb_out_column* out_keys, gb_out_column* out_results,
                                int64_t* num_groups, void* stream);

/* Batched groupby: many independent groupbys with one schema (same key types,
 * value types and aggregations) aggregated by one persistent launch over a work
 * queue of row tiles, optionally captured once as a CUDA graph and replayed.
 * No counterpart in libcudf, where each groupby is its own call.
 *  keys:     [num_instances * num_keys] column views, instance-major
 *  requests: [num_instances * num_requests], instance-major
 * gb_batch_prepare samples every instance and sizes its table and outputs;
 * the views must stay valid (same shapes) for every gb_batch_run.  Results of
 * instance i (views into batch-owned buffers, valid until the next run or
 * gb_batch_destroy) come from gb_batch_result: keys[num_keys] and results in
 * request order.  VARIANCE/STD are not supported in a batch. */
typedef struct gb_batch gb_batch;
typedef struct gb_batch_stats {
  int64_t instances;
  int64_t tiles;
  int64_t smem_instances;   /* instances that use the shared-memory stage */
  int64_t table_bytes;
  int64_t output_bytes;
  int32_t kernels_per_run;
  int64_t regrown;          /* instance tables grown after a trial run overflowed */
  int32_t block;            /* threads per CTA of the aggregation launch */
  int64_t tile_rows;        /* rows per tile of the work queue */
  int64_t ruled_instances;  /* instances a gb_batch_rule sized */
} gb_batch_stats;
GB_API int gb_batch_prepare(int32_t num_instances, const gb_column* keys, int32_t num_keys,
                            int32_t null_policy, const gb_request* requests, int32_t num_requests,
                            int32_t use_graph, void* stream, const gb_allocator* mr, gb_batch** out);
GB_API int gb_batch_run(gb_batch* batch, void* stream);
GB_API int gb_batch_result(gb_batch* batch, int32_t instance, int64_t* num_groups,
                           gb_out_column* keys, gb_out_column* results);
GB_API int gb_batch_get_stats(const gb_batch* batch, gb_batch_stats* out);
GB_API void gb_batch_destroy(gb_batch* batch);

/* Process-wide tuning of batched launches (no counterpart in libcudf).
 * launch (NULL: defaults 512 threads, 64 Ki-row tiles, 160 KiB tables): the
 * aggregation kernel's threads per CTA (256, 512 or 1024), rows per tile of
 * the work queue, shared-memory bytes of a tile's table.  rules: for each
 * instance, the first rule with rows <= max_rows and estimated groups <=
 * max_groups caps its shared table at smem_slots slots (0: global table
 * only; -1: no cap) and takes the shared stage only when groups *
 * headroom_pct / 100 <= slots (<= 0: 200).  Applies to batches prepared
 * afterwards; replaces earlier settings.  cudf_b200.autotune times the
 * candidates per size bucket. */
typedef struct gb_batch_rule {
  int64_t max_rows;
  int64_t max_groups;
  int32_t smem_slots;
  int32_t headroom_pct;
} gb_batch_rule;
typedef struct gb_batch_launch {
  int32_t block;
  int32_t tile_rows;
  int32_t smem_bytes;
} gb_batch_launch;
GB_API int gb_batch_set_tuning(const gb_batch_rule* rules, int32_t num_rules, const gb_batch_launch* launch);

/* Serving loop: continuous batching of groupby queries (no counterpart in
 * libcudf).  gb_server_submit enqueues a query whose columns are resident on
 * the device (they must stay valid until the query is released).  A
 * dispatcher thread admits queries in arrival order while the estimated device
 * memory (hash table + results, from the row count and a device-side key
 * sketch) of all admitted, unreleased queries stays under memory_cap_bytes, and
 * packs each round of admitted queries into one batched launch run by the next
 * idle worker (each worker has its own stream, so batches overlap on the GPU).
 * gb_server_wait blocks until a query completes; gb_server_result gives views
 * of its results (valid until gb_server_release). */
typedef struct gb_server gb_server;
typedef struct gb_server_options {
  int64_t memory_cap_bytes;   /* admission cap (default 150 GiB) */
  int32_t max_batch_queries;  /* queries per batched launch (default 256) */
  int64_t max_batch_rows;     /* rows per batched launch (default 400 Mi) */
  int32_t workers;            /* worker threads / streams (default 4) */
  int64_t direct_rows;        /* queries with at least this many rows run alone through the
                                 single-query engine (default 64 Ki) ... */
  int64_t direct_groups;      /* ... as do queries with more estimated groups (default 64 Ki) */
  int64_t reserve_bytes;      /* device memory admission leaves free (cudaMemGetInfo), beside the
                                 cap (default 2 GiB) */
} gb_server_options;
typedef struct gb_query_info {
  int32_t status;             /* 2 done, 3 failed */
  double latency_s;           /* arrival to completion */
  double queue_s;             /* arrival to admission */
  int64_t num_groups;
} gb_query_info;
typedef struct gb_server_stats {
  int64_t completed;
  int64_t failed;
  int64_t batches;
  double p50_s;
  double p99_s;
  double queries_per_s;       /* completed / (last completion - first arrival) */
  int64_t peak_admitted_bytes;
  double sketch_s;            /* dispatcher time in the key sketch */
  double prepare_s;           /* workers' batch sizing time (sample, layout, trial runs) */
  double run_s;               /* workers' batch run time */
  int64_t trial_rounds;
  int64_t direct_runs;        /* large, many-group queries run alone instead of batched */
  int64_t held_for_memory;    /* admission rounds that stopped at free device memory */
  int64_t min_free_bytes;     /* lowest free device memory seen at admission */
} gb_server_stats;
GB_API int gb_server_create(const gb_server_options* opt, gb_server** out);
GB_API int gb_server_submit(gb_server* server, const gb_column* keys, int32_t num_keys, int32_t null_policy,
                            const gb_request* requests, int32_t num_requests, int64_t* query_id);
GB_API int gb_server_wait(gb_server* server, int64_t query_id, double timeout_s, gb_query_info* info);
GB_API int gb_server_result(gb_server* server, int64_t query_id, int64_t* num_groups,
                            gb_out_column* keys, gb_out_column* results);
GB_API int gb_server_release(gb_server* server, int64_t query_id);
GB_API int gb_server_get_stats(gb_server* server, gb_server_stats* out);
GB_API void gb_server_destroy(gb_server* server);

/* Library version string. */
GB_API const char* gb_version(void);

#ifdef __cplusplus
}
#endif
#endif /* CUDF_B200_H */
