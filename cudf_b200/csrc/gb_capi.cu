// gb_capi.cu -- the extern "C" boundary (include/cudf_b200.h) over the engine.
#include <algorithm>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/cudf_b200.h"
#include "gb_engine.h"

namespace {
thread_local std::string t_err;

int fail(int code, const std::string& msg)
{
  t_err = msg;
  return code;
}

template <typename F>
int guarded(F&& f)
{
  try {
    t_err.clear();
    f();
    return GB_OK;
  } catch (const gb::Error& e) {
    return fail(e.code, e.what());
  } catch (const std::bad_alloc& e) {
    return fail(GB_ERR_ALLOC, e.what());
  } catch (const std::exception& e) {
    return fail(GB_ERR_LOGIC, e.what());
  } catch (...) {
    return fail(GB_ERR_LOGIC, "unknown error");
  }
}

gb::Column to_col(const gb_column& c)
{
  return gb::Column{c.type_id, c.size, c.data, c.null_mask, c.offset};
}

struct ResultImpl {
  gb::Result r;
  std::vector<gb_out_column> keys;
  std::vector<std::vector<gb_out_column>> cols;
  std::vector<gb_out_column*> col_ptrs;
  std::vector<int32_t> counts;
};

gb_out_column to_out(const gb::OutColumn& c)
{
  gb_out_column o;
  o.type_id = c.type_id;
  o.size = c.size;
  o.data = c.data;
  o.null_mask = c.mask;
  o.null_count = c.null_count;
  return o;
}
}  // namespace

namespace gb {
void set_last_error(const std::string& msg) { t_err = msg; }
}  // namespace gb

struct gb_handle {
  std::vector<gb::Column> keys;
  int null_policy;
  int sorted;
  gb::Options opt;
  gb::Stats stats;
};

extern "C" {

int gb_create(const gb_column* keys, int32_t num_keys, int32_t null_policy, int32_t keys_are_sorted,
              gb_handle** out)
{
  return guarded([&] {
    if (!out) throw gb::Error(gb::ERR_LOGIC, "null output handle pointer");
    *out = nullptr;
    if (num_keys < 1 || !keys) throw gb::Error(gb::ERR_LOGIC, "groupby needs at least one key column");
    if (null_policy != GB_NULL_EXCLUDE && null_policy != GB_NULL_INCLUDE)
      throw gb::Error(gb::ERR_LOGIC, "invalid null_policy");
    auto* h = new gb_handle;
    for (int i = 0; i < num_keys; ++i) h->keys.push_back(to_col(keys[i]));
    h->null_policy = null_policy;
    h->sorted = keys_are_sorted;
    *out = h;
  });
}

void gb_destroy(gb_handle* h) { delete h; }

int gb_aggregate(gb_handle* h, const gb_request* requests, int32_t num_requests, void* stream,
                 const gb_allocator* mr, gb_result** out)
{
  return guarded([&] {
    if (!h || !out) throw gb::Error(gb::ERR_LOGIC, "null handle or output pointer");
    *out = nullptr;
    if (num_requests < 0 || (num_requests > 0 && !requests))
      throw gb::Error(gb::ERR_LOGIC, "invalid request list");
    std::vector<gb::Request> reqs(num_requests);
    for (int r = 0; r < num_requests; ++r) {
      reqs[r].values = to_col(requests[r].values);
      if (requests[r].num_aggs < 0 || (requests[r].num_aggs > 0 && !requests[r].aggs))
        throw gb::Error(gb::ERR_LOGIC, "invalid aggregation list");
      for (int j = 0; j < requests[r].num_aggs; ++j)
        reqs[r].aggs.push_back(gb::AggSpec{requests[r].aggs[j].kind, requests[r].aggs[j].param});
    }
    gb::Allocator A = mr ? gb::Allocator{mr->allocate, mr->deallocate, mr->ctx} : gb::default_allocator();
    auto* impl = new ResultImpl;
    try {
      impl->r = gb::aggregate(h->keys, h->null_policy, reqs, (cudaStream_t)stream, A, h->opt, &h->stats);
    } catch (...) {
      delete impl;
      throw;
    }
    for (auto& k : impl->r.keys) impl->keys.push_back(to_out(k));
    for (auto& rc : impl->r.results) {
      std::vector<gb_out_column> v;
      for (auto& c : rc) v.push_back(to_out(c));
      impl->cols.push_back(v);
    }
    for (auto& v : impl->cols) {
      impl->col_ptrs.push_back(v.data());
      impl->counts.push_back((int32_t)v.size());
    }
    auto* res = new gb_result;
    res->num_groups = impl->r.num_groups;
    res->num_keys = (int32_t)impl->keys.size();
    res->keys = impl->keys.data();
    res->num_requests = (int32_t)impl->cols.size();
    res->num_results = impl->counts.data();
    res->results = impl->col_ptrs.data();
    res->impl = impl;
    *out = res;
  });
}

void gb_result_free(gb_result* res)
{
  if (!res) return;
  auto* impl = (ResultImpl*)res->impl;
  if (impl) {
    impl->r.release();
    delete impl;
  }
  delete res;
}

const char* gb_last_error(void) { return t_err.c_str(); }

// Copies the fields of `t` that are set into `o`; returns their OPT_* bits.
static uint32_t apply_tuning(const gb_tuning* t, gb::Options& o)
{
  uint32_t m = 0;
  if (t->block > 0) {
    if (t->block % 32 || t->block > 1024) throw gb::Error(gb::ERR_LOGIC, "block must be a multiple of 32, <= 1024");
    o.block = t->block;
    m |= gb::OPT_BLOCK;
  }
  if (t->blocks_per_sm >= 0) o.blocks_per_sm = t->blocks_per_sm, m |= gb::OPT_BPS;
  if (t->smem_bytes >= 0) o.smem_bytes = t->smem_bytes, m |= gb::OPT_SMEM;
  if (t->smem_fill_pct > 0) o.smem_fill = std::min(95, t->smem_fill_pct) / 100.0, m |= gb::OPT_FILL;
  if (t->smem_max_groups >= 0) o.smem_max_groups = t->smem_max_groups, m |= gb::OPT_SMEM_MAX;
  if (t->load_factor_pct > 0) o.load_factor = std::min(90, t->load_factor_pct) / 100.0, m |= gb::OPT_LOAD;
  if (t->force_mode >= -1) {
    if (t->force_mode > 2) throw gb::Error(gb::ERR_LOGIC, "force_mode must be in [-1, 2]");
    o.force_mode = t->force_mode;
    m |= gb::OPT_MODE;
  }
  if (t->groups_hint >= 0) o.groups_hint = t->groups_hint;
  if (t->profile >= 0) o.profile = t->profile;
  if (t->scatter >= 0) {
    if (t->scatter > 8) throw gb::Error(gb::ERR_LOGIC, "scatter must be in [0, 8]");
    o.scatter = t->scatter;
    m |= gb::OPT_SCATTER;
  }
  if (t->part_fill_pct > 0) {
    if (t->part_fill_pct > 95) throw gb::Error(gb::ERR_LOGIC, "part_fill_pct must be in [1, 95]");
    o.part_fill = t->part_fill_pct / 100.0;
    m |= gb::OPT_PART_FILL;
  }
  if (t->wagg_pct >= 0) o.wagg_pct = t->wagg_pct, m |= gb::OPT_WAGG;
  if (t->pass2 >= 0) {
    if (t->pass2 > 4) throw gb::Error(gb::ERR_LOGIC, "pass2 must be in [0, 4]");
    o.pass2 = t->pass2;
    m |= gb::OPT_PASS2;
  }
  return m;
}

int gb_set_tuning(gb_handle* h, const gb_tuning* t)
{
  return guarded([&] {
    if (!h || !t) throw gb::Error(gb::ERR_LOGIC, "null handle or tuning");
    h->opt.set_mask |= apply_tuning(t, h->opt);
  });
}

int gb_set_tuning_rules(const gb_tuning_rule* rules, int32_t num_rules)
{
  return guarded([&] {
    if (num_rules < 0 || (num_rules > 0 && !rules)) throw gb::Error(gb::ERR_LOGIC, "bad tuning rules");
    std::vector<gb::TuningRule> v;
    for (int i = 0; i < num_rules; ++i) {
      gb::TuningRule r;
      r.max_rows = rules[i].max_rows;
      r.max_groups = rules[i].max_groups;
      if (rules[i].key_words < 0 || rules[i].key_words > 2) throw gb::Error(gb::ERR_LOGIC, "key_words must be 0, 1 or 2");
      r.key_words = rules[i].key_words;
      r.mask = apply_tuning(&rules[i].tuning, r.opt);
      v.push_back(r);
    }
    gb::set_tuning_rules(v);
  });
}

int gb_get_stats(const gb_handle* h, gb_stats* out)
{
  return guarded([&] {
    if (!h || !out) throw gb::Error(gb::ERR_LOGIC, "null handle or stats");
    out->est_groups = h->stats.est_groups;
    out->capacity = h->stats.capacity;
    out->mode = h->stats.mode;
    out->retries = h->stats.retries;
    out->kernels = h->stats.kernels;
    out->agg_kernel_ms = h->stats.agg_kernel_ms;
    out->compact_ms = h->stats.compact_ms;
    out->scatter_ms = h->stats.scatter_ms;
    out->rule = h->stats.rule;
  });
}

int32_t gb_target_type(int32_t type_id, int32_t kind)
{
  return gb::valid_agg(type_id, kind) ? gb::target_type(type_id, kind) : 0;
}

int32_t gb_is_valid_aggregation(int32_t type_id, int32_t kind) { return gb::valid_agg(type_id, kind) ? 1 : 0; }

const char* gb_version(void) { return "cudf_b200 0.1.0 (sm_100a)"; }

}  // extern "C"
