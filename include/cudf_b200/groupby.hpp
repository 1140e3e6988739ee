/*
 * cudf_b200/groupby.hpp -- libcudf's groupby C++ API over the B200 engine.
 *
 * Minimal, header-only definitions of the libcudf types a groupby caller
 * touches, so that code written against
 *     cudf::groupby::groupby(keys, null_policy).aggregate(requests, stream, mr)
 * compiles and runs unchanged against this engine (it links libcudf_b200.so
 * instead of libcudf.so).  Each type keeps the reference's name, namespace,
 * argument order and ownership rules:
 *   cudf::groupby::aggregation_request / aggregation_result / groupby
 *       cpp/include/cudf/groupby.hpp:59-62,86-89,94-197
 *   make_{sum,product,min,max,count,sum_of_squares,mean,variance,std,argmax,
 *   argmin}_aggregation   cpp/include/cudf/aggregation.hpp:257-306 (and the
 *       factories after it); aggregation::Kind numbering  :86-102
 *   cudf::column_view / table_view   cpp/include/cudf/column/column_view.hpp,
 *       cpp/include/cudf/table/table_view.hpp (non-owning views)
 *   cudf::type_id, data_type, size_type, bitmask_type, null_policy, sorted,
 *       order, null_order   cpp/include/cudf/types.hpp:93-94,124,149,201-233
 *   cudf::logic_error / cuda_error   cpp/include/cudf/utilities/error.hpp
 *   host_span   cpp/include/cudf/utilities/span.hpp
 *   rmm::cuda_stream_view, rmm::mr::device_memory_resource (only the members
 *       a groupby caller uses; define CUDF_B200_HAVE_RMM to use the real RMM
 *       headers instead)
 * Everything forwards to the C ABI in cudf_b200.h (gb_create, gb_aggregate,
 * gb_result_free, gb_destroy, gb_last_error).  Result columns own their device
 * memory: they share the engine's result buffers, which are freed (through
 * the `mr` that allocated them) when the last column of a call is destroyed.
 */
#ifndef CUDF_B200_GROUPBY_HPP
#define CUDF_B200_GROUPBY_HPP

#include <cuda_runtime_api.h>

#include <cstddef>
#include <cstdint>
#include <memory>
#include <new>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../cudf_b200.h"

#ifdef CUDF_B200_HAVE_RMM
#include <rmm/cuda_stream_view.hpp>
#include <rmm/mr/device/device_memory_resource.hpp>
#include <rmm/mr/device/per_device_resource.hpp>
#else
namespace rmm {
/* The stream wrapper libcudf's API takes (rmm/cuda_stream_view.hpp). */
class cuda_stream_view {
 public:
  constexpr cuda_stream_view() = default;
  constexpr cuda_stream_view(cudaStream_t s) noexcept : s_(s) {}
  constexpr cudaStream_t value() const noexcept { return s_; }
  constexpr operator cudaStream_t() const noexcept { return s_; }
  void synchronize() const
  {
    if (cudaStreamSynchronize(s_) != cudaSuccess) throw std::runtime_error("cudaStreamSynchronize failed");
  }

 private:
  cudaStream_t s_{nullptr};
};
namespace mr {
/* Stream-ordered device allocator (rmm/mr/device/device_memory_resource.hpp):
 * subclasses implement do_allocate / do_deallocate. */
class device_memory_resource {
 public:
  virtual ~device_memory_resource() = default;
  void* allocate(std::size_t bytes, cuda_stream_view stream) { return do_allocate(bytes, stream); }
  void deallocate(void* p, std::size_t bytes, cuda_stream_view stream) { do_deallocate(p, bytes, stream); }

 private:
  virtual void* do_allocate(std::size_t bytes, cuda_stream_view stream) = 0;
  virtual void do_deallocate(void* p, std::size_t bytes, cuda_stream_view stream) = 0;
};
/* cudaMallocAsync / cudaFreeAsync on the call's stream. */
class cuda_async_memory_resource final : public device_memory_resource {
  void* do_allocate(std::size_t bytes, cuda_stream_view stream) override
  {
    void* p = nullptr;
    if (cudaMallocAsync(&p, bytes, stream.value()) != cudaSuccess) throw std::bad_alloc();
    return p;
  }
  void do_deallocate(void* p, std::size_t, cuda_stream_view stream) override { cudaFreeAsync(p, stream.value()); }
};
inline cuda_async_memory_resource& default_async_resource()
{
  static cuda_async_memory_resource r;
  return r;
}
inline device_memory_resource* get_current_device_resource() { return &default_async_resource(); }
}  // namespace mr
}  // namespace rmm
#endif

namespace cudf {

using size_type = int32_t;
using bitmask_type = uint32_t;

/* cudf::type_id (cpp/include/cudf/types.hpp:201-233): the engine's C ABI takes
 * the same numbers. */
enum class type_id : int32_t {
  EMPTY = 0, INT8, INT16, INT32, INT64, UINT8, UINT16, UINT32, UINT64, FLOAT32, FLOAT64, BOOL8,
  TIMESTAMP_DAYS, TIMESTAMP_SECONDS, TIMESTAMP_MILLISECONDS, TIMESTAMP_MICROSECONDS,
  TIMESTAMP_NANOSECONDS, DURATION_DAYS, DURATION_SECONDS, DURATION_MILLISECONDS,
  DURATION_MICROSECONDS, DURATION_NANOSECONDS, DICTIONARY32, STRING, LIST, DECIMAL32, DECIMAL64,
  DECIMAL128, STRUCT, NUM_TYPE_IDS
};

class data_type {
 public:
  data_type() = default;
  explicit constexpr data_type(type_id id) : id_(id) {}
  constexpr type_id id() const noexcept { return id_; }
  constexpr int32_t scale() const noexcept { return 0; }
  constexpr bool operator==(data_type o) const noexcept { return id_ == o.id_; }
  constexpr bool operator!=(data_type o) const noexcept { return id_ != o.id_; }

 private:
  type_id id_{type_id::EMPTY};
};

enum class null_policy : bool { EXCLUDE, INCLUDE };
enum class sorted : bool { NO, YES };
enum class order : bool { ASCENDING, DESCENDING };
enum class null_order : bool { AFTER, BEFORE };

/* Sentinel null count: "compute it when asked" (cpp/include/cudf/types.hpp). */
constexpr size_type UNKNOWN_NULL_COUNT = -1;

/* Bytes per element of a fixed-width type (0 otherwise). */
inline std::size_t size_of(data_type t)
{
  switch (t.id()) {
    case type_id::INT8: case type_id::UINT8: case type_id::BOOL8: return 1;
    case type_id::INT16: case type_id::UINT16: return 2;
    case type_id::INT32: case type_id::UINT32: case type_id::FLOAT32: case type_id::TIMESTAMP_DAYS:
    case type_id::DURATION_DAYS: return 4;
    case type_id::INT64: case type_id::UINT64: case type_id::FLOAT64: case type_id::TIMESTAMP_SECONDS:
    case type_id::TIMESTAMP_MILLISECONDS: case type_id::TIMESTAMP_MICROSECONDS:
    case type_id::TIMESTAMP_NANOSECONDS: case type_id::DURATION_SECONDS:
    case type_id::DURATION_MILLISECONDS: case type_id::DURATION_MICROSECONDS:
    case type_id::DURATION_NANOSECONDS: return 8;
    default: return 0;
  }
}

/* cudf::logic_error (CUDF_EXPECTS / CUDF_FAIL) and cudf::cuda_error. */
struct logic_error : public std::logic_error {
  using std::logic_error::logic_error;
};
struct cuda_error : public std::runtime_error {
  cuda_error(std::string const& what, cudaError_t e = cudaErrorUnknown) : std::runtime_error(what), code(e) {}
  cudaError_t error_code() const noexcept { return code; }
  cudaError_t code;
};

/* A non-owning view of a contiguous sequence (cudf::host_span). */
template <typename T>
class host_span {
 public:
  constexpr host_span() noexcept = default;
  constexpr host_span(T* data, std::size_t size) noexcept : p_(data), n_(size) {}
  template <typename C, typename = decltype(std::declval<C&>().data())>
  constexpr host_span(C& c) noexcept : p_(c.data()), n_(c.size()) {}
  template <typename C, typename = decltype(std::declval<C const&>().data())>
  constexpr host_span(C const& c) noexcept : p_(c.data()), n_(c.size()) {}
  template <std::size_t N>
  constexpr host_span(T (&a)[N]) noexcept : p_(a), n_(N) {}
  constexpr T* begin() const noexcept { return p_; }
  constexpr T* end() const noexcept { return p_ + n_; }
  constexpr T* data() const noexcept { return p_; }
  constexpr std::size_t size() const noexcept { return n_; }
  constexpr bool empty() const noexcept { return n_ == 0; }
  constexpr T& operator[](std::size_t i) const { return p_[i]; }

 private:
  T* p_{nullptr};
  std::size_t n_{0};
};

/* cudf::column_view: a non-owning fixed-width column -- element data, optional
 * LSB-first validity words, and a row offset applied to both. */
class column_view {
 public:
  column_view() = default;
  column_view(data_type type, size_type size, void const* data, bitmask_type const* null_mask = nullptr,
              size_type null_count = UNKNOWN_NULL_COUNT, size_type offset = 0)
    : type_(type), size_(size), data_(data), mask_(null_mask), null_count_(null_count), offset_(offset)
  {
    if (size < 0) throw logic_error("Column size cannot be negative.");
    if (size > 0 && data == nullptr && type.id() != type_id::EMPTY)
      throw logic_error("Null data pointer.");
  }
  data_type type() const noexcept { return type_; }
  size_type size() const noexcept { return size_; }
  bool is_empty() const noexcept { return size_ == 0; }
  size_type offset() const noexcept { return offset_; }
  bool nullable() const noexcept { return mask_ != nullptr; }
  bitmask_type const* null_mask() const noexcept { return mask_; }
  /* The count given at construction (UNKNOWN_NULL_COUNT if none was). */
  size_type null_count() const noexcept { return mask_ ? null_count_ : 0; }
  bool has_nulls() const noexcept { return mask_ != nullptr && null_count_ != 0; }
  template <typename T = void>
  T const* head() const noexcept { return static_cast<T const*>(data_); }
  /* First element of the view (offset applied). */
  template <typename T>
  T const* data() const noexcept { return head<T>() + offset_; }

 private:
  data_type type_{};
  size_type size_{0};
  void const* data_{nullptr};
  bitmask_type const* mask_{nullptr};
  size_type null_count_{0};
  size_type offset_{0};
};

/* cudf::table_view: equal-length column views. */
class table_view {
 public:
  table_view() = default;
  table_view(std::vector<column_view> const& cols) : cols_(cols)
  {
    for (auto const& c : cols_)
      if (c.size() != cols_.front().size()) throw logic_error("Column size mismatch.");
  }
  table_view(std::initializer_list<column_view> cols) : table_view(std::vector<column_view>(cols)) {}
  size_type num_columns() const noexcept { return static_cast<size_type>(cols_.size()); }
  size_type num_rows() const noexcept { return cols_.empty() ? 0 : cols_.front().size(); }
  column_view const& column(size_type i) const { return cols_.at(static_cast<std::size_t>(i)); }
  auto begin() const noexcept { return cols_.begin(); }
  auto end() const noexcept { return cols_.end(); }

 private:
  std::vector<column_view> cols_;
};

namespace detail {
/* Maps a C-ABI status to the exception libcudf throws for it. */
inline void throw_on_error(int rc)
{
  if (rc == GB_OK) return;
  std::string msg = gb_last_error();
  switch (rc) {
    case GB_ERR_ALLOC: throw std::bad_alloc();
    case GB_ERR_CUDA: throw cuda_error(msg);
    default: throw logic_error(msg);
  }
}
using result_owner = std::shared_ptr<gb_result>;
}  // namespace detail

/* cudf::column: an owning column.  Columns produced by one aggregate() call
 * share that call's device buffers, released with the last of them. */
class column {
 public:
  column(column const&) = delete;
  column& operator=(column const&) = delete;
  column(detail::result_owner owner, gb_out_column const& c)
    : owner_(std::move(owner)),
      view_(data_type{static_cast<type_id>(c.type_id)}, static_cast<size_type>(c.size), c.data, c.null_mask,
            static_cast<size_type>(c.null_count))
  {
  }
  data_type type() const noexcept { return view_.type(); }
  size_type size() const noexcept { return view_.size(); }
  size_type null_count() const noexcept { return view_.null_count(); }
  bool nullable() const noexcept { return view_.nullable(); }
  bool has_nulls() const noexcept { return null_count() > 0; }
  column_view view() const noexcept { return view_; }
  operator column_view() const noexcept { return view_; }

 private:
  detail::result_owner owner_;
  column_view view_;
};

/* cudf::table: owning columns of equal length. */
class table {
 public:
  explicit table(std::vector<std::unique_ptr<column>>&& cols) : cols_(std::move(cols)) {}
  size_type num_columns() const noexcept { return static_cast<size_type>(cols_.size()); }
  size_type num_rows() const noexcept { return cols_.empty() ? 0 : cols_.front()->size(); }
  column& get_column(size_type i) { return *cols_.at(static_cast<std::size_t>(i)); }
  column const& get_column(size_type i) const { return *cols_.at(static_cast<std::size_t>(i)); }
  table_view view() const
  {
    std::vector<column_view> v;
    for (auto const& c : cols_) v.push_back(c->view());
    return table_view(v);
  }
  std::vector<std::unique_ptr<column>> release() { return std::move(cols_); }

 private:
  std::vector<std::unique_ptr<column>> cols_;
};

/* Default stream of libcudf calls (the legacy default stream). */
inline rmm::cuda_stream_view get_default_stream() { return rmm::cuda_stream_view{}; }

/* cudf::aggregation and its kinds (cpp/include/cudf/aggregation.hpp:86-102). */
class aggregation {
 public:
  enum Kind {
    SUM, PRODUCT, MIN, MAX, COUNT_VALID, COUNT_ALL, ANY, ALL, SUM_OF_SQUARES, MEAN, M2, VARIANCE, STD,
    MEDIAN, QUANTILE, ARGMAX, ARGMIN, NUNIQUE, NTH_ELEMENT, ROW_NUMBER, EWMA, RANK, COLLECT_LIST,
    COLLECT_SET, LEAD, LAG, PTX, CUDA, MERGE_LISTS, MERGE_SETS, MERGE_M2, COVARIANCE, CORRELATION,
    TDIGEST, MERGE_TDIGEST, HISTOGRAM, MERGE_HISTOGRAM
  };
  explicit aggregation(Kind k) : kind(k) {}
  virtual ~aggregation() = default;
  virtual std::unique_ptr<aggregation> clone() const { return std::make_unique<aggregation>(*this); }
  Kind kind;
  /* ddof of VARIANCE / STD (unused by the other kinds) */
  size_type ddof{1};
};
/* Aggregations usable in a groupby (the engine's hash path). */
class groupby_aggregation : public virtual aggregation {
 public:
  explicit groupby_aggregation(Kind k) : aggregation(k) {}
};

namespace detail {
template <typename Base>
std::unique_ptr<Base> make_agg(aggregation::Kind k, size_type ddof = 1)
{
  auto a = std::make_unique<groupby_aggregation>(k);
  a->ddof = ddof;
  return std::unique_ptr<Base>(a.release());
}
}  // namespace detail

template <typename Base = aggregation>
std::unique_ptr<Base> make_sum_aggregation() { return detail::make_agg<Base>(aggregation::SUM); }
template <typename Base = aggregation>
std::unique_ptr<Base> make_product_aggregation() { return detail::make_agg<Base>(aggregation::PRODUCT); }
template <typename Base = aggregation>
std::unique_ptr<Base> make_min_aggregation() { return detail::make_agg<Base>(aggregation::MIN); }
template <typename Base = aggregation>
std::unique_ptr<Base> make_max_aggregation() { return detail::make_agg<Base>(aggregation::MAX); }
/* COUNT_VALID when nulls are excluded, COUNT_ALL when included. */
template <typename Base = aggregation>
std::unique_ptr<Base> make_count_aggregation(null_policy nulls = null_policy::EXCLUDE)
{
  return detail::make_agg<Base>(nulls == null_policy::INCLUDE ? aggregation::COUNT_ALL : aggregation::COUNT_VALID);
}
template <typename Base = aggregation>
std::unique_ptr<Base> make_sum_of_squares_aggregation() { return detail::make_agg<Base>(aggregation::SUM_OF_SQUARES); }
template <typename Base = aggregation>
std::unique_ptr<Base> make_mean_aggregation() { return detail::make_agg<Base>(aggregation::MEAN); }
template <typename Base = aggregation>
std::unique_ptr<Base> make_variance_aggregation(size_type ddof = 1) { return detail::make_agg<Base>(aggregation::VARIANCE, ddof); }
template <typename Base = aggregation>
std::unique_ptr<Base> make_std_aggregation(size_type ddof = 1) { return detail::make_agg<Base>(aggregation::STD, ddof); }
template <typename Base = aggregation>
std::unique_ptr<Base> make_argmax_aggregation() { return detail::make_agg<Base>(aggregation::ARGMAX); }
template <typename Base = aggregation>
std::unique_ptr<Base> make_argmin_aggregation() { return detail::make_agg<Base>(aggregation::ARGMIN); }

namespace groupby {

/* cpp/include/cudf/groupby.hpp:59-62 */
struct aggregation_request {
  column_view values;
  std::vector<std::unique_ptr<groupby_aggregation>> aggregations;
};

/* cpp/include/cudf/groupby.hpp:86-89 */
struct aggregation_result {
  std::vector<std::unique_ptr<column>> results{};
};

namespace detail {
/* Bridges an rmm device_memory_resource to the engine's allocator hooks. */
struct mr_bridge {
  static void* allocate(void* ctx, std::size_t bytes, void* stream)
  {
    try {
      return static_cast<rmm::mr::device_memory_resource*>(ctx)->allocate(
        bytes, rmm::cuda_stream_view{static_cast<cudaStream_t>(stream)});
    } catch (...) {
      return nullptr;
    }
  }
  static void deallocate(void* ctx, void* p, std::size_t bytes, void* stream)
  {
    static_cast<rmm::mr::device_memory_resource*>(ctx)->deallocate(
      p, bytes, rmm::cuda_stream_view{static_cast<cudaStream_t>(stream)});
  }
};
inline gb_column to_abi(column_view const& c)
{
  return gb_column{static_cast<int32_t>(c.type().id()), c.size(), c.head(), c.null_mask(), c.offset()};
}
}  // namespace detail

/* cudf::groupby::groupby (cpp/include/cudf/groupby.hpp:94-197): groups the
 * rows of `keys` (not owned: the caller keeps them alive) and aggregates
 * values by group on the engine.  keys_are_sorted, column_order and
 * null_precedence are accepted for API parity; the hash path's results do not
 * depend on them.  Unique-key order of the output is arbitrary. */
class groupby {
 public:
  groupby() = delete;
  ~groupby()
  {
    if (h_) gb_destroy(h_);
  }
  groupby(groupby const&) = delete;
  groupby(groupby&&) = delete;
  groupby& operator=(groupby const&) = delete;
  groupby& operator=(groupby&&) = delete;

  explicit groupby(table_view const& keys, null_policy include_null_keys = null_policy::EXCLUDE,
                   sorted keys_are_sorted = sorted::NO, std::vector<order> const& column_order = {},
                   std::vector<null_order> const& null_precedence = {})
    : keys_(keys)
  {
    (void)column_order;
    (void)null_precedence;
    std::vector<gb_column> k;
    for (auto const& c : keys) k.push_back(detail::to_abi(c));
    cudf::detail::throw_on_error(gb_create(k.data(), static_cast<int32_t>(k.size()),
                                           include_null_keys == null_policy::INCLUDE ? GB_NULL_INCLUDE
                                                                                     : GB_NULL_EXCLUDE,
                                           keys_are_sorted == sorted::YES ? 1 : 0, &h_));
  }

  /* Aggregates every request on `stream`; results are allocated from `mr`.
   * Throws cudf::logic_error when a request's row count differs from the
   * keys' or a (type, aggregation) pair is not supported by the hash path,
   * cudf::cuda_error on a CUDA failure, std::bad_alloc when `mr` fails. */
  std::pair<std::unique_ptr<table>, std::vector<aggregation_result>> aggregate(
    host_span<aggregation_request const> requests,
    rmm::cuda_stream_view stream = cudf::get_default_stream(),
    rmm::mr::device_memory_resource* mr = rmm::mr::get_current_device_resource())
  {
    std::vector<std::vector<gb_agg>> aggs(requests.size());
    std::vector<gb_request> reqs;
    for (std::size_t r = 0; r < requests.size(); ++r) {
      for (auto const& a : requests[r].aggregations) {
        if (!a) throw logic_error("Null aggregation.");
        aggs[r].push_back(gb_agg{static_cast<int32_t>(a->kind), a->ddof});
      }
      reqs.push_back(gb_request{detail::to_abi(requests[r].values), static_cast<int32_t>(aggs[r].size()),
                                aggs[r].data()});
    }
    gb_allocator bridge{&detail::mr_bridge::allocate, &detail::mr_bridge::deallocate, mr};
    bool default_mr = mr == nullptr;
#ifndef CUDF_B200_HAVE_RMM
    default_mr = default_mr || mr == &rmm::mr::default_async_resource();
#endif
    gb_result* raw = nullptr;
    cudf::detail::throw_on_error(gb_aggregate(h_, reqs.data(), static_cast<int32_t>(reqs.size()),
                                              static_cast<void*>(stream.value()), default_mr ? nullptr : &bridge,
                                              &raw));
    cudf::detail::result_owner owner(raw, [](gb_result* p) { gb_result_free(p); });
    std::vector<std::unique_ptr<column>> kc;
    for (int32_t k = 0; k < raw->num_keys; ++k) kc.push_back(std::make_unique<column>(owner, raw->keys[k]));
    std::vector<aggregation_result> out(static_cast<std::size_t>(raw->num_requests));
    for (int32_t r = 0; r < raw->num_requests; ++r)
      for (int32_t j = 0; j < raw->num_results[r]; ++j)
        out[static_cast<std::size_t>(r)].results.push_back(std::make_unique<column>(owner, raw->results[r][j]));
    return {std::make_unique<table>(std::move(kc)), std::move(out)};
  }

 private:
  table_view keys_;
  gb_handle* h_{nullptr};
};

}  // namespace groupby
}  // namespace cudf

#endif  // CUDF_B200_GROUPBY_HPP
