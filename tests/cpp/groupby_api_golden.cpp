// groupby_api_golden.cpp -- drives the engine through the libcudf-shaped C++
// API (include/cudf_b200/groupby.hpp) the way a libcudf caller would:
// column_views over device buffers, aggregation_requests built with the
// make_*_aggregation factories, cudf::groupby::groupby(...).aggregate(...) on
// a non-default stream, owning result columns.
//
// Test harness, not product: tests/test_gpu_cpp_api.py writes libcudf's own
// known-answer cases (tests/golden/golden_vectors.json) to stdin in a line
// format and checks what this program prints.
//
// stdin, per case:
//   case <name>
//   policy <0 exclude | 1 include>
//   key <type_id> <n> <hex element bits>...      keyvalid - | <0/1>...
//   val <type_id> <n> <hex element bits>...      valvalid - | <0/1>...
//   aggs <kind>...
//   run
// stdout, per case:
//   case <name>
//   error <logic|cuda|alloc> <message>        (on an exception), or
//   groups <G> / key <type> <G> <hex>... / keyvalid ... /
//   result <j> <type> <G> <hex>... / resultvalid ...
//   end
// A final "mr <allocations> <live bytes after release>" line reports a run of
// the last case through a counting device_memory_resource.
#include <cudf_b200/groupby.hpp>

#include <cstdio>
#include <cstring>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

namespace {

void check(cudaError_t e, const char* what)
{
  if (e != cudaSuccess) {
    std::fprintf(stderr, "%s: %s\n", what, cudaGetErrorString(e));
    std::exit(2);
  }
}

struct DevCol {
  cudf::data_type type{};
  int n = 0;
  void* data = nullptr;
  cudf::bitmask_type* mask = nullptr;
  int nulls = 0;
  cudf::column_view view() const
  {
    return cudf::column_view(type, n, data, mask, mask ? nulls : 0);
  }
  void free_all()
  {
    if (data) cudaFree(data);
    if (mask) cudaFree(mask);
    data = nullptr;
    mask = nullptr;
  }
};

DevCol upload(int type_id, const std::vector<unsigned long long>& bits, const std::vector<int>* valid)
{
  DevCol c;
  c.type = cudf::data_type{static_cast<cudf::type_id>(type_id)};
  c.n = static_cast<int>(bits.size());
  const size_t w = cudf::size_of(c.type);
  std::vector<unsigned char> host(bits.size() * w + 8);
  for (size_t i = 0; i < bits.size(); ++i) std::memcpy(host.data() + i * w, &bits[i], w);
  check(cudaMalloc(&c.data, host.size()), "cudaMalloc data");
  check(cudaMemcpy(c.data, host.data(), host.size(), cudaMemcpyHostToDevice), "copy data");
  if (valid) {
    std::vector<cudf::bitmask_type> words((bits.size() + 31) / 32 + 1, 0u);
    for (size_t i = 0; i < valid->size(); ++i) {
      if ((*valid)[i]) words[i / 32] |= 1u << (i % 32);
      else ++c.nulls;
    }
    check(cudaMalloc(reinterpret_cast<void**>(&c.mask), words.size() * 4), "cudaMalloc mask");
    check(cudaMemcpy(c.mask, words.data(), words.size() * 4, cudaMemcpyHostToDevice), "copy mask");
  }
  return c;
}

std::unique_ptr<cudf::groupby_aggregation> make(int kind)
{
  using cudf::groupby_aggregation;
  switch (kind) {
    case cudf::aggregation::SUM: return cudf::make_sum_aggregation<groupby_aggregation>();
    case cudf::aggregation::PRODUCT: return cudf::make_product_aggregation<groupby_aggregation>();
    case cudf::aggregation::MIN: return cudf::make_min_aggregation<groupby_aggregation>();
    case cudf::aggregation::MAX: return cudf::make_max_aggregation<groupby_aggregation>();
    case cudf::aggregation::COUNT_VALID: return cudf::make_count_aggregation<groupby_aggregation>();
    case cudf::aggregation::COUNT_ALL:
      return cudf::make_count_aggregation<groupby_aggregation>(cudf::null_policy::INCLUDE);
    case cudf::aggregation::SUM_OF_SQUARES: return cudf::make_sum_of_squares_aggregation<groupby_aggregation>();
    case cudf::aggregation::MEAN: return cudf::make_mean_aggregation<groupby_aggregation>();
    case cudf::aggregation::VARIANCE: return cudf::make_variance_aggregation<groupby_aggregation>();
    case cudf::aggregation::STD: return cudf::make_std_aggregation<groupby_aggregation>();
    case cudf::aggregation::ARGMAX: return cudf::make_argmax_aggregation<groupby_aggregation>();
    case cudf::aggregation::ARGMIN: return cudf::make_argmin_aggregation<groupby_aggregation>();
    default: return std::make_unique<groupby_aggregation>(static_cast<cudf::aggregation::Kind>(kind));
  }
}

void print_column(const char* tag, int j, cudf::column_view v)
{
  const size_t w = cudf::size_of(v.type());
  std::vector<unsigned char> host(static_cast<size_t>(v.size()) * w);
  if (!host.empty())
    check(cudaMemcpy(host.data(), v.data<unsigned char>(), host.size(), cudaMemcpyDeviceToHost), "copy out");
  std::printf("%s", tag);
  if (j >= 0) std::printf(" %d", j);
  std::printf(" %d %d", static_cast<int>(v.type().id()), v.size());
  for (int i = 0; i < v.size(); ++i) {
    unsigned long long b = 0;
    std::memcpy(&b, host.data() + static_cast<size_t>(i) * w, w);
    std::printf(" %llx", b);
  }
  std::printf("\n%svalid", tag);
  if (!v.nullable()) {
    std::printf(" -\n");
    return;
  }
  std::vector<cudf::bitmask_type> words((v.size() + 31) / 32);
  if (!words.empty())
    check(cudaMemcpy(words.data(), v.null_mask(), words.size() * 4, cudaMemcpyDeviceToHost), "copy mask");
  for (int i = 0; i < v.size(); ++i) std::printf(" %u", (words[i / 32] >> (i % 32)) & 1u);
  std::printf("\n");
}

// A device_memory_resource that counts what passes through it.
class counting_resource final : public rmm::mr::device_memory_resource {
 public:
  long allocations = 0;
  long long live = 0;

 private:
  void* do_allocate(std::size_t bytes, rmm::cuda_stream_view stream) override
  {
    void* p = nullptr;
    if (cudaMallocAsync(&p, bytes, stream.value()) != cudaSuccess) throw std::bad_alloc();
    ++allocations;
    live += static_cast<long long>(bytes);
    return p;
  }
  void do_deallocate(void* p, std::size_t bytes, rmm::cuda_stream_view stream) override
  {
    cudaFreeAsync(p, stream.value());
    live -= static_cast<long long>(bytes);
  }
};

struct Case {
  std::string name;
  int policy = 0;
  int ktype = 0, vtype = 0;
  std::vector<unsigned long long> keys, vals;
  bool kvalid_set = false, vvalid_set = false;
  std::vector<int> kvalid, vvalid;
  std::vector<int> aggs;
};

std::vector<unsigned long long> read_hex(std::istringstream& is, int n)
{
  std::vector<unsigned long long> v(static_cast<size_t>(n));
  for (int i = 0; i < n; ++i) is >> std::hex >> v[static_cast<size_t>(i)] >> std::dec;
  return v;
}

std::vector<int> read_valid(std::istringstream& is, bool& set)
{
  std::vector<int> v;
  std::string t;
  set = false;
  while (is >> t) {
    if (t == "-") return v;
    set = true;
    v.push_back(std::stoi(t));
  }
  return v;
}

// Runs one case and prints its results (quiet: runs it without printing).
void run_case(const Case& c, cudaStream_t stream, rmm::mr::device_memory_resource* mr, bool quiet)
{
  DevCol k = upload(c.ktype, c.keys, c.kvalid_set ? &c.kvalid : nullptr);
  DevCol v = upload(c.vtype, c.vals, c.vvalid_set ? &c.vvalid : nullptr);
  if (!quiet) std::printf("case %s\n", c.name.c_str());
  try {
    cudf::groupby::groupby gb(cudf::table_view({k.view()}),
                              c.policy ? cudf::null_policy::INCLUDE : cudf::null_policy::EXCLUDE);
    std::vector<cudf::groupby::aggregation_request> requests(1);
    requests[0].values = v.view();
    for (int a : c.aggs) requests[0].aggregations.push_back(make(a));
    auto result = gb.aggregate(requests, rmm::cuda_stream_view{stream},
                               mr ? mr : rmm::mr::get_current_device_resource());
    check(cudaStreamSynchronize(stream), "sync");
    if (!quiet) {
      std::printf("groups %d\n", result.first->num_rows());
      print_column("key", -1, result.first->get_column(0).view());
      for (size_t j = 0; j < result.second[0].results.size(); ++j)
        print_column("result", static_cast<int>(j), result.second[0].results[j]->view());
    }
  } catch (cudf::logic_error const& e) {
    if (!quiet) std::printf("error logic %s\n", e.what());
  } catch (cudf::cuda_error const& e) {
    if (!quiet) std::printf("error cuda %s\n", e.what());
  } catch (std::bad_alloc const&) {
    if (!quiet) std::printf("error alloc\n");
  }
  if (!quiet) std::printf("end\n");
  k.free_all();
  v.free_all();
}

}  // namespace

int main()
{
  cudaStream_t stream;
  check(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "stream");
  std::string line;
  Case c;
  Case last;
  bool have_last = false;
  while (std::getline(std::cin, line)) {
    std::istringstream is(line);
    std::string tag;
    is >> tag;
    if (tag == "case") {
      c = Case{};
      is >> c.name;
    } else if (tag == "policy") {
      is >> c.policy;
    } else if (tag == "key") {
      int n;
      is >> c.ktype >> n;
      c.keys = read_hex(is, n);
    } else if (tag == "keyvalid") {
      c.kvalid = read_valid(is, c.kvalid_set);
    } else if (tag == "val") {
      int n;
      is >> c.vtype >> n;
      c.vals = read_hex(is, n);
    } else if (tag == "valvalid") {
      c.vvalid = read_valid(is, c.vvalid_set);
    } else if (tag == "aggs") {
      int a;
      while (is >> a) c.aggs.push_back(a);
    } else if (tag == "run") {
      run_case(c, stream, nullptr, false);
      last = c;
      have_last = true;
    }
  }
  if (have_last) {
    counting_resource mr;
    run_case(last, stream, &mr, true);
    check(cudaStreamSynchronize(stream), "sync");
    std::printf("mr %ld %lld\n", mr.allocations, mr.live);
  }
  std::fflush(stdout);
  cudaStreamDestroy(stream);
  return 0;
}
