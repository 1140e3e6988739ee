// gb_noalloc.cu -- gb_aggregate_noalloc: a groupby that allocates no memory.
//
// Some callers of this library cannot allocate device memory at the point
// where they run a groupby: code whose device memory is owned by another
// allocator that forbids allocations from outside (a JVM-side or framework
// memory pool sized to the whole GPU), and latency-bound loops in which
// cudaMalloc/cudaFree are off limits because they synchronise the device.
// For them this entry point runs the global-hash-table aggregation with its
// table in a file-scope device array of fixed size, and writes the results into
// output buffers the caller has already allocated.
//
// The array is static __device__ memory of this module, so every GPU that loads
// the library holds GB_NOALLOC_SCRATCH_BYTES of it until the process exits.  In
// host code the array's name is only a host-side stand-in, not a device
// address: its device address is looked up once per device (and again if the
// device's context was recreated, e.g. after cudaDeviceReset) with
// cudaGetSymbolAddress, with that device current.  That lookup happens on the
// first call on each device, so the first call on a device should come before
// any stream capture.  The call is synchronous: it waits for its stream and
// returns with the results complete.  Every call shares the one array and leaves its contents
// behind; each call clears the counters (and the caller's null masks) it relies
// on before use.  Calls that overlap on the GPU -- on different streams, or
// from different threads -- race on the array and must be serialised by the
// caller.
#include <cuda_runtime.h>

#include <mutex>
#include <string>
#include <vector>

#include "../../include/cudf_b200.h"
#include "gb_engine.h"

namespace {

static __device__ __align__(256) unsigned char g_noalloc_scratch[GB_NOALLOC_SCRATCH_BYTES];

// The current CUDA context (driver entry point fetched through the runtime,
// so the library needs no link-time dependency on libcuda).
void* current_context()
{
  using get_ctx_fn = int (*)(void**);
  static get_ctx_fn fn = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      f = nullptr;
    return reinterpret_cast<get_ctx_fn>(f);
  }();
  void* ctx = nullptr;
  if (!fn || fn(&ctx) != 0) return nullptr;
  return ctx;
}

// Device address of g_noalloc_scratch on the current device.  It is looked up
// once per device and context: a context made after cudaDeviceReset has the
// array at a new address, so a change of context repeats the lookup.
void* scratch_address()
{
  static std::mutex mu;
  static void* addr[64] = {};
  static void* ctx_of[64] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) throw gb::Error(gb::ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= 64) throw gb::Error(gb::ERR_UNSUPPORTED, "device ordinal out of range");
  std::lock_guard<std::mutex> g(mu);
  void* ctx = current_context();
  if (!addr[dev] || ctx_of[dev] != ctx || !ctx) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      throw gb::Error(gb::ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    }
    addr[dev] = p;
    ctx_of[dev] = current_context();
  }
  return addr[dev];
}

gb::Column to_col(const gb_column& c) { return gb::Column{c.type_id, c.size, c.data, c.null_mask, c.offset}; }

}  // namespace

extern "C" int gb_aggregate_noalloc(const gb_column* keys, int32_t num_keys, int32_t null_policy,
                                    const gb_request* requests, int32_t num_requests, int64_t max_groups,
                                    gb_out_column* out_keys, gb_out_column* out_results,
                                    int64_t* num_groups, void* stream)
{
  try {
    gb::set_last_error("");
    if (!keys || num_keys < 1) throw gb::Error(gb::ERR_LOGIC, "groupby needs at least one key column");
    if (null_policy != GB_NULL_EXCLUDE && null_policy != GB_NULL_INCLUDE)
      throw gb::Error(gb::ERR_LOGIC, "invalid null_policy");
    if (num_requests < 0 || (num_requests > 0 && !requests)) throw gb::Error(gb::ERR_LOGIC, "invalid request list");
    if (!out_keys || !num_groups) throw gb::Error(gb::ERR_LOGIC, "null output pointer");
    std::vector<gb::Column> kc;
    for (int i = 0; i < num_keys; ++i) kc.push_back(to_col(keys[i]));
    std::vector<gb::Request> reqs(num_requests);
    int total_aggs = 0;
    for (int r = 0; r < num_requests; ++r) {
      reqs[r].values = to_col(requests[r].values);
      if (requests[r].num_aggs < 0 || (requests[r].num_aggs > 0 && !requests[r].aggs))
        throw gb::Error(gb::ERR_LOGIC, "invalid aggregation list");
      for (int j = 0; j < requests[r].num_aggs; ++j)
        reqs[r].aggs.push_back(gb::AggSpec{requests[r].aggs[j].kind, requests[r].aggs[j].param});
      total_aggs += requests[r].num_aggs;
    }
    if (total_aggs > 0 && !out_results) throw gb::Error(gb::ERR_LOGIC, "null output result columns");
    std::vector<gb::OutColumn> ok(num_keys), orr(total_aggs);
    for (int i = 0; i < num_keys; ++i) {
      ok[i].data = out_keys[i].data;
      ok[i].mask = out_keys[i].null_mask;
    }
    for (int j = 0; j < total_aggs; ++j) {
      orr[j].data = out_results[j].data;
      orr[j].mask = out_results[j].null_mask;
    }
    void* scratch = scratch_address();
    int64_t g = gb::aggregate_into_scratch(kc, null_policy, reqs, (cudaStream_t)stream, scratch,
                                           (size_t)GB_NOALLOC_SCRATCH_BYTES, max_groups, ok, orr);
    for (int i = 0; i < num_keys; ++i) {
      out_keys[i].type_id = ok[i].type_id;
      out_keys[i].size = ok[i].size;
      out_keys[i].null_mask = ok[i].mask;
      out_keys[i].null_count = ok[i].null_count;
    }
    for (int j = 0; j < total_aggs; ++j) {
      out_results[j].type_id = orr[j].type_id;
      out_results[j].size = orr[j].size;
      out_results[j].null_mask = orr[j].mask;
      out_results[j].null_count = orr[j].null_count;
    }
    *num_groups = g;
    return GB_OK;
  } catch (const gb::Error& e) {
    gb::set_last_error(e.what());
    return e.code;
  } catch (const std::exception& e) {
    gb::set_last_error(e.what());
    return GB_ERR_LOGIC;
  } catch (...) {
    gb::set_last_error("unknown error");
    return GB_ERR_LOGIC;
  }
}
