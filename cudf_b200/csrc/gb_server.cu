// gb_server.cu -- serving loop: continuous batching of groupby queries.
//
// Queries arrive on any thread (gb_server_submit) with their columns already
// resident on the device.  A dispatcher thread admits them in arrival order
// while the estimated device memory of everything admitted stays under the
// cap: the estimate comes from the row count and a device-side key sketch
// (the batch sampler run once over the newly arrived queries), sized as the
// hash table plus the result columns.  Admitted queries are packed into one
// batched launch (gb_batch) handed to the next idle worker; each worker runs
// on its own stream, so batches that were admitted while others run overlap
// on the GPU.  Results stay on the device until the caller releases them.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <climits>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/cudf_b200.h"
#include "gb_batch.h"

namespace gb {
namespace {

using Clock = std::chrono::steady_clock;

double now_s()
{
  return std::chrono::duration<double>(Clock::now().time_since_epoch()).count();
}

struct Query {
  int64_t id;
  std::vector<Column> keys;
  std::vector<Request> reqs;
  int null_policy;
  double arrive, admit = 0, launch = 0, done = 0;
  int64_t est_bytes = 0;
  int64_t est_groups = 1;
  int status = 0;  // 0 pending, 1 admitted, 2 done, 3 failed
  std::string error;
  std::shared_ptr<Batch> batch;  // keeps the result buffers alive
  int index_in_batch = 0;
  bool run_direct = false;          // routed to the single-query engine
  std::shared_ptr<Result> direct;   // its result
  ~Query()
  {
    if (direct) direct->release();
  }
};

struct WorkItem {
  std::vector<std::shared_ptr<Query>> queries;
};

}  // namespace

struct Server {
  gb_server_options opt;
  int device = 0;
  std::mutex mu;
  std::condition_variable cv_submit, cv_done, cv_worker;
  std::deque<std::shared_ptr<Query>> pending;
  std::map<int64_t, std::shared_ptr<Query>> queries;
  std::deque<WorkItem> work;
  int64_t next_id = 1;
  int64_t in_use = 0;  // estimated bytes of admitted, unreleased queries
  int64_t peak_in_use = 0;
  bool stop = false;
  int idle_workers = 0;
  std::vector<std::thread> threads;
  std::vector<double> latencies;
  int64_t completed = 0, failed = 0, batches = 0;
  double first_arrive = -1, last_done = 0;
  double sketch_s = 0, prepare_s = 0, run_s = 0, trial_s = 0;
  int64_t trial_rounds = 0, direct_runs = 0;
  int64_t held_for_memory = 0, min_free = -1;
  cudaStream_t sketch_stream = nullptr;

  // device-side sketch of a set of queries: estimated groups per query, one
  // sampling launch per key layout among the arrivals
  std::vector<double> sketch(const std::vector<std::shared_ptr<Query>>& qs)
  {
    std::vector<double> est(qs.size(), 1.0);
    std::map<std::string, std::vector<size_t>> by_layout;
    for (size_t i = 0; i < qs.size(); ++i) {
      std::string sig = std::to_string(qs[i]->null_policy) + ":";
      for (auto& k : qs[i]->keys) sig += std::to_string(k.type_id) + ",";
      by_layout[sig].push_back(i);
    }
    for (auto& kv : by_layout) {
      std::vector<std::vector<Column>> ks;
      std::vector<std::vector<Request>> rs;
      for (size_t i : kv.second) {
        ks.push_back(qs[i]->keys);
        rs.push_back(qs[i]->reqs);
      }
      std::vector<int64_t> e =
        batch_estimate_groups(ks, qs[kv.second[0]]->null_policy, rs, sketch_stream, default_allocator());
      for (size_t j = 0; j < kv.second.size(); ++j) est[kv.second[j]] = (double)e[j];
    }
    return est;
  }

  int64_t bytes_for(const Query& q, double groups)
  {
    // table at load 0.5 plus result columns: ~slot_guess bytes per group each
    int64_t per = 16 + 24 * (int64_t)q.reqs.size() * 2;
    int64_t g = (int64_t)std::max(64.0, groups);
    return 2 * g * per + g * per;
  }

  void dispatcher()
  {
    cudaSetDevice(device);
    // the sketch must not wait behind whole batches: highest stream priority
    int lo = 0, hi = 0;
    cudaDeviceGetStreamPriorityRange(&lo, &hi);
    cudaStreamCreateWithPriority(&sketch_stream, cudaStreamNonBlocking, hi);
    std::deque<std::shared_ptr<Query>> waiting;  // sketched, not admitted yet
    for (;;) {
      std::vector<std::shared_ptr<Query>> arrivals;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv_submit.wait_for(lk, std::chrono::microseconds(200), [&] { return stop || !pending.empty(); });
        if (stop && pending.empty() && waiting.empty()) break;
        while (!pending.empty()) {
          arrivals.push_back(pending.front());
          pending.pop_front();
        }
      }
      if (!arrivals.empty()) {
        // group arrivals by schema-compatible runs (same layout as the first)
        std::vector<double> est;
        try {
          double t0 = now_s();
          est = sketch(arrivals);
          sketch_s += now_s() - t0;
        } catch (const std::exception& ex) {
          est.assign(arrivals.size(), 0.0);
          for (auto& q : arrivals) q->est_bytes = -1, q->error = ex.what();
        }
        for (size_t i = 0; i < arrivals.size(); ++i) {
          if (arrivals[i]->est_bytes == 0) {
            arrivals[i]->est_bytes = bytes_for(*arrivals[i], est[i]);
            arrivals[i]->est_groups = (int64_t)est[i];
          }
          waiting.push_back(arrivals[i]);
        }
      }
      // admission in arrival order under the memory cap and the device's free
      // memory (less a reserve); pack into batches.  Free memory already
      // counts what running queries allocated; this round's admissions are
      // charged against it as they are admitted.
      std::vector<std::shared_ptr<Query>> admitted;
      int64_t free_budget = INT64_MAX;
      if (!waiting.empty()) {
        size_t fr = 0, tot = 0;
        if (cudaMemGetInfo(&fr, &tot) == cudaSuccess) {
          free_budget = (int64_t)fr - opt.reserve_bytes;
          std::lock_guard<std::mutex> lk(mu);
          min_free = min_free < 0 ? (int64_t)fr : std::min(min_free, (int64_t)fr);
        } else {
          cudaGetLastError();
        }
      }
      {
        std::unique_lock<std::mutex> lk(mu);
        int64_t rows = 0;
        while (!waiting.empty()) {
          auto& q = waiting.front();
          if (q->est_bytes < 0) {  // sketch failed: report the error
            q->status = 3;
            q->done = now_s();
            ++failed;
            waiting.pop_front();
            cv_done.notify_all();
            continue;
          }
          if (in_use + q->est_bytes > opt.memory_cap_bytes && in_use > 0) break;
          if (q->est_bytes > free_budget && in_use > 0) {
            ++held_for_memory;
            break;
          }
          free_budget -= q->est_bytes;
          if ((int)admitted.size() >= opt.max_batch_queries) break;
          in_use += q->est_bytes;
          peak_in_use = std::max(peak_in_use, in_use);
          q->status = 1;
          q->admit = now_s();
          rows += q->keys[0].size;
          admitted.push_back(q);
          waiting.pop_front();
          if (rows >= opt.max_batch_rows) break;
        }
        if (!admitted.empty()) {
          // large or many-group queries run alone through the single-query
          // engine (hash-partitioned for many groups), one work item each so
          // idle workers take them in parallel; the rest share one batched
          // launch.  Never queue more than one item per idle worker ahead.
          std::vector<WorkItem> items;
          WorkItem batched;
          for (auto& q : admitted) {
            q->run_direct = q->keys[0].size >= opt.direct_rows || q->est_groups > opt.direct_groups;
            if (q->run_direct) {
              WorkItem w;
              w.queries.push_back(q);
              items.push_back(std::move(w));
            } else {
              batched.queries.push_back(q);
            }
          }
          if (!batched.queries.empty()) items.push_back(std::move(batched));
          for (auto& w : items) {
            cv_worker.wait(lk, [&] { return stop || (int64_t)work.size() < std::max(1, idle_workers); });
            work.push_back(std::move(w));
            cv_worker.notify_all();
          }
        }
      }
    }
    cudaStreamDestroy(sketch_stream);
  }

  void worker()
  {
    cudaSetDevice(device);
    cudaStream_t s;
    cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    for (;;) {
      WorkItem w;
      {
        std::unique_lock<std::mutex> lk(mu);
        ++idle_workers;
        cv_worker.notify_all();
        cv_worker.wait(lk, [&] { return stop || !work.empty(); });
        --idle_workers;
        if (work.empty()) break;
        w = std::move(work.front());
        work.pop_front();
        cv_worker.notify_all();
      }
      double t_launch = now_s();
      // queries of one batch must share a schema: split by null policy / layout
      std::map<std::string, std::vector<std::shared_ptr<Query>>> groups;
      for (auto& q : w.queries) {
        std::string sig = std::to_string(q->null_policy) + ":";
        for (auto& k : q->keys) sig += std::to_string(k.type_id) + ",";
        sig += "|";
        for (auto& r : q->reqs) {
          sig += std::to_string(r.values.type_id) + "(";
          for (auto& a : r.aggs) sig += std::to_string(a.kind) + "." + std::to_string(a.ddof) + ",";
          sig += ")";
        }
        groups[sig].push_back(q);
      }
      // large queries with many groups run alone through the single-query
      // engine (its hash-partitioned path); the rest share one batched launch
      for (auto& kv : groups) {
        std::vector<std::shared_ptr<Query>> rest;
        for (auto& q : kv.second) {
          if (q->run_direct) {
            std::string err;
            auto R = std::make_shared<Result>();
            try {
              // the engine's own full-pass sketch sizes the tables (the
              // dispatcher's sample only routes the query)
              Options o;
              *R = aggregate(q->keys, q->null_policy, q->reqs, s, default_allocator(), o, nullptr);
            } catch (const std::exception& ex) {
              err = ex.what();
            }
            double t_done = now_s();
            std::lock_guard<std::mutex> lk(mu);
            q->launch = t_launch;
            q->done = t_done;
            if (err.empty()) {
              q->status = 2;
              q->direct = R;
              ++completed;
              ++direct_runs;
              latencies.push_back(q->done - q->arrive);
            } else {
              q->status = 3;
              q->error = err;
              ++failed;
              in_use -= q->est_bytes;
            }
            last_done = std::max(last_done, t_done);
            cv_done.notify_all();
          } else {
            rest.push_back(q);
          }
        }
        kv.second.swap(rest);
      }
      for (auto& kv : groups) {
        auto& qs = kv.second;
        if (qs.empty()) continue;
        auto b = std::make_shared<Batch>();
        std::string err;
        try {
          std::vector<std::vector<Column>> ks;
          std::vector<std::vector<Request>> rs;
          for (auto& q : qs) {
            ks.push_back(q->keys);
            rs.push_back(q->reqs);
          }
          BatchOptions bo;
          bo.trial = false;  // size from the dispatcher's sketch; run() regrows on overflow
          for (auto& q : qs) bo.est_groups.push_back(q->est_groups);
          bo.growth = 2.0;
          b->prepare(ks, qs[0]->null_policy, rs, s, default_allocator(), bo);
          b->run(s);
        } catch (const std::exception& ex) {
          err = ex.what();
        }
        double t_done = now_s();
        std::lock_guard<std::mutex> lk(mu);
        ++batches;
        {
          const BatchStats& bs = b->stats();
          prepare_s += bs.sample_s + bs.layout_s + bs.trial_s;
          trial_s += bs.trial_s;
          run_s += bs.run_s;
          trial_rounds += bs.trial_rounds;
        }
        for (size_t i = 0; i < qs.size(); ++i) {
          auto& q = qs[i];
          q->launch = t_launch;
          q->done = t_done;
          if (err.empty()) {
            q->status = 2;
            q->batch = b;
            q->index_in_batch = (int)i;
            ++completed;
            latencies.push_back(q->done - q->arrive);
          } else {
            q->status = 3;
            q->error = err;
            ++failed;
            in_use -= q->est_bytes;
          }
          last_done = std::max(last_done, t_done);
        }
        cv_done.notify_all();
      }
    }
    cudaStreamDestroy(s);
  }
};

}  // namespace gb

struct gb_server {
  gb::Server s;
};

namespace {
gb::Column to_col(const gb_column& c) { return gb::Column{c.type_id, c.size, c.data, c.null_mask, c.offset}; }

template <typename F>
int guarded(F&& f)
{
  try {
    gb::set_last_error("");
    f();
    return GB_OK;
  } catch (const gb::Error& e) {
    gb::set_last_error(e.what());
    return e.code;
  } catch (const std::exception& e) {
    gb::set_last_error(e.what());
    return GB_ERR_LOGIC;
  }
}

double pct(std::vector<double> v, double p)
{
  if (v.empty()) return 0;
  std::sort(v.begin(), v.end());
  size_t i = (size_t)std::min<double>((double)v.size() - 1, std::ceil(p / 100.0 * v.size()) - 1);
  return v[i];
}
}  // namespace

extern "C" {

int gb_server_create(const gb_server_options* opt, gb_server** out)
{
  return guarded([&] {
    if (!out) throw gb::Error(gb::ERR_LOGIC, "null output pointer");
    std::unique_ptr<gb_server> sv(new gb_server);
    gb::Server& S = sv->s;
    S.opt.memory_cap_bytes = 150ll << 30;
    S.opt.max_batch_queries = 256;
    S.opt.max_batch_rows = 400ll << 20;
    S.opt.workers = 4;
    S.opt.direct_rows = 64 << 10;
    S.opt.direct_groups = 64 << 10;
    S.opt.reserve_bytes = 2ll << 30;
    if (opt) {
      if (opt->memory_cap_bytes > 0) S.opt.memory_cap_bytes = opt->memory_cap_bytes;
      if (opt->max_batch_queries > 0) S.opt.max_batch_queries = opt->max_batch_queries;
      if (opt->max_batch_rows > 0) S.opt.max_batch_rows = opt->max_batch_rows;
      if (opt->workers > 0) S.opt.workers = std::min(8, opt->workers);
      if (opt->direct_rows > 0) S.opt.direct_rows = opt->direct_rows;
      if (opt->direct_groups > 0) S.opt.direct_groups = opt->direct_groups;
      if (opt->reserve_bytes > 0) S.opt.reserve_bytes = opt->reserve_bytes;
    }
    if (cudaGetDevice(&S.device) != cudaSuccess) throw gb::Error(gb::ERR_CUDA, "cudaGetDevice failed");
    S.threads.emplace_back([&S] { S.dispatcher(); });
    for (int i = 0; i < S.opt.workers; ++i) S.threads.emplace_back([&S] { S.worker(); });
    *out = sv.release();
  });
}

int gb_server_submit(gb_server* sv, const gb_column* keys, int32_t num_keys, int32_t null_policy,
                     const gb_request* requests, int32_t num_requests, int64_t* query_id)
{
  return guarded([&] {
    if (!sv || !keys || num_keys < 1 || !query_id) throw gb::Error(gb::ERR_LOGIC, "invalid arguments");
    auto q = std::make_shared<gb::Query>();
    for (int k = 0; k < num_keys; ++k) q->keys.push_back(to_col(keys[k]));
    for (int r = 0; r < num_requests; ++r) {
      gb::Request R;
      R.values = to_col(requests[r].values);
      for (int j = 0; j < requests[r].num_aggs; ++j)
        R.aggs.push_back(gb::AggSpec{requests[r].aggs[j].kind, requests[r].aggs[j].param});
      q->reqs.push_back(R);
    }
    // the checks aggregate() does, so that a bad query fails at submit
    gb::Plan P;
    std::vector<int> ot;
    gb::build_plan(q->keys, null_policy, q->reqs, P, ot);
    q->null_policy = null_policy;
    q->arrive = gb::now_s();
    gb::Server& S = sv->s;
    std::lock_guard<std::mutex> lk(S.mu);
    q->id = S.next_id++;
    if (S.first_arrive < 0) S.first_arrive = q->arrive;
    S.queries[q->id] = q;
    S.pending.push_back(q);
    *query_id = q->id;
    S.cv_submit.notify_all();
  });
}

int gb_server_wait(gb_server* sv, int64_t id, double timeout_s, gb_query_info* info)
{
  return guarded([&] {
    if (!sv) throw gb::Error(gb::ERR_LOGIC, "null server");
    gb::Server& S = sv->s;
    std::unique_lock<std::mutex> lk(S.mu);
    auto it = S.queries.find(id);
    if (it == S.queries.end()) throw gb::Error(gb::ERR_LOGIC, "unknown query id");
    auto q = it->second;
    bool ok = S.cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s > 0 ? timeout_s : 1e9),
                                 [&] { return q->status >= 2; });
    if (!ok) throw gb::Error(gb::ERR_LOGIC, "timed out waiting for the query");
    if (info) {
      info->status = q->status;
      info->latency_s = q->done - q->arrive;
      info->queue_s = q->admit - q->arrive;
      info->num_groups = 0;
      if (q->status == 2) {
        if (q->direct) info->num_groups = q->direct->num_groups;
        else {
          gb::Result R;
          q->batch->result(q->index_in_batch, R);
          info->num_groups = R.num_groups;
        }
      }
    }
    if (q->status == 3) throw gb::Error(gb::ERR_CUDA, q->error);
  });
}

int gb_server_result(gb_server* sv, int64_t id, int64_t* num_groups, gb_out_column* keys, gb_out_column* results)
{
  return guarded([&] {
    if (!sv || !num_groups) throw gb::Error(gb::ERR_LOGIC, "null argument");
    gb::Server& S = sv->s;
    std::shared_ptr<gb::Query> q;
    {
      std::lock_guard<std::mutex> lk(S.mu);
      auto it = S.queries.find(id);
      if (it == S.queries.end()) throw gb::Error(gb::ERR_LOGIC, "unknown query id");
      q = it->second;
    }
    if (q->status != 2) throw gb::Error(gb::ERR_LOGIC, "query not complete");
    gb::Result R;
    if (q->direct) {
      R.num_groups = q->direct->num_groups;
      R.keys = q->direct->keys;
      R.results.push_back({});
      for (auto& rc : q->direct->results)
        for (auto& c : rc) R.results[0].push_back(c);
    } else {
      q->batch->result(q->index_in_batch, R);
    }
    *num_groups = R.num_groups;
    auto put = [](gb_out_column& o, const gb::OutColumn& c) {
      o.type_id = c.type_id;
      o.size = c.size;
      o.data = c.data;
      o.null_mask = c.mask;
      o.null_count = c.null_count;
    };
    if (keys)
      for (size_t k = 0; k < R.keys.size(); ++k) put(keys[k], R.keys[k]);
    if (results)
      for (size_t j = 0; j < R.results[0].size(); ++j) put(results[j], R.results[0][j]);
  });
}

int gb_server_release(gb_server* sv, int64_t id)
{
  return guarded([&] {
    if (!sv) throw gb::Error(gb::ERR_LOGIC, "null server");
    gb::Server& S = sv->s;
    std::lock_guard<std::mutex> lk(S.mu);
    auto it = S.queries.find(id);
    if (it == S.queries.end()) throw gb::Error(gb::ERR_LOGIC, "unknown query id");
    if (it->second->status == 2) S.in_use -= it->second->est_bytes;
    S.queries.erase(it);  // the batch's buffers go with its last query
  });
}

int gb_server_get_stats(gb_server* sv, gb_server_stats* out)
{
  return guarded([&] {
    if (!sv || !out) throw gb::Error(gb::ERR_LOGIC, "null argument");
    gb::Server& S = sv->s;
    std::lock_guard<std::mutex> lk(S.mu);
    out->completed = S.completed;
    out->failed = S.failed;
    out->batches = S.batches;
    out->p50_s = pct(S.latencies, 50);
    out->p99_s = pct(S.latencies, 99);
    double span = S.last_done - S.first_arrive;
    out->queries_per_s = span > 0 ? S.completed / span : 0;
    out->peak_admitted_bytes = S.peak_in_use;
    out->sketch_s = S.sketch_s;
    out->prepare_s = S.prepare_s;
    out->run_s = S.run_s;
    out->trial_rounds = S.trial_rounds;
    out->direct_runs = S.direct_runs;
    out->held_for_memory = S.held_for_memory;
    out->min_free_bytes = S.min_free;
  });
}

void gb_server_destroy(gb_server* sv)
{
  if (!sv) return;
  gb::Server& S = sv->s;
  {
    std::lock_guard<std::mutex> lk(S.mu);
    S.stop = true;
  }
  S.cv_submit.notify_all();
  S.cv_worker.notify_all();
  S.cv_done.notify_all();
  for (auto& t : S.threads) t.join();
  delete sv;
}

}  // extern "C"
