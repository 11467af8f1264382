// The GPU task bodies of legate-dataframe's join, groupby_aggregation, sort,
// the local step of repartition_by_hash and CSV read, rewritten over the C ABI
// of libldf_b200.so.  INTEGRATION.md shows this code; the test suite type-checks
// it against include/ldf_b200.h and the stand-in declarations of the
// reference's task-side API (reference_api.hpp).
#include "reference_api.hpp"

#include <ldf_b200.h>

#include <fstream>
#include <iterator>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

namespace ldf_integration {

using legate::dataframe::JoinType;
using legate::dataframe::TaskContext;
using legate::dataframe::TaskMemoryResource;
using legate::dataframe::task::PhysicalColumn;
using legate::dataframe::task::PhysicalTable;
namespace argument = legate::dataframe::argument;

// ---- status -> the reference's exception types --------------------------------
inline void ldf_check(int st)
{
  if (st == LDF_OK) return;
  std::string msg = ldf_b200_last_error();
  if (st == LDF_ERR_INVALID_ARGUMENT || st == LDF_ERR_UNSUPPORTED) throw std::invalid_argument(msg);
  throw std::runtime_error(msg);
}

// ---- column types (the Arrow ids of utils.cpp:30-139) ---------------------------
int32_t ldf_type_of(const PhysicalColumn& col)
{
  switch (col.arrow_type()->id()) {
    case arrow::Type::BOOL: return LDF_BOOL8;
    case arrow::Type::INT8: return LDF_INT8;
    case arrow::Type::INT16: return LDF_INT16;
    case arrow::Type::INT32: return LDF_INT32;
    case arrow::Type::INT64: return LDF_INT64;
    case arrow::Type::UINT8: return LDF_UINT8;
    case arrow::Type::UINT16: return LDF_UINT16;
    case arrow::Type::UINT32: return LDF_UINT32;
    case arrow::Type::UINT64: return LDF_UINT64;
    case arrow::Type::FLOAT: return LDF_FLOAT32;
    case arrow::Type::DOUBLE: return LDF_FLOAT64;
    case arrow::Type::STRING:
    case arrow::Type::LARGE_STRING: return LDF_STRING;
    case arrow::Type::TIMESTAMP: return LDF_TIMESTAMP_US;
    default: throw std::invalid_argument("column type not supported by the B200 task bodies");
  }
}

// ---- a bound input column as an ldf_column (replaces column_view(),
// column.cu:319-363: no null-mask or offsets conversion) -------------------------
ldf_column to_ldf(const PhysicalColumn& col)
{
  ldf_column c{};
  const legate::PhysicalArray& arr = col.physical_array();
  c.type     = ldf_type_of(col);
  c.size     = static_cast<int64_t>(col.num_rows());
  c.nullable = arr.nullable() ? 1 : 0;
  if (c.type == LDF_STRING) {
    legate::StringPhysicalArray s = arr.as_string_array();
    legate::PhysicalStore ranges  = s.ranges().data();
    legate::PhysicalStore chars   = s.chars().data();
    legate::Rect<1> cshape        = chars.shape<1>();
    c.data       = const_cast<legate::Rect<1>*>(
      ranges.read_accessor<legate::Rect<1>, 1>().ptr(ranges.shape<1>().lo));  // inclusive global ranges
    c.chars      = const_cast<char*>(reinterpret_cast<const char*>(chars.read_accessor<int8_t, 1>().ptr(cshape.lo)));
    c.chars_base = cshape.lo[0];
    c.num_chars  = static_cast<int64_t>(cshape.volume());
  } else {
    legate::PhysicalStore d = arr.data();
    c.data = const_cast<int8_t*>(d.read_accessor<int8_t, 1, false>().ptr(d.shape<1>().lo));  // untyped bytes
  }
  if (c.nullable) {
    legate::PhysicalStore m = arr.null_mask();  // one bool per row
    c.valid = const_cast<uint8_t*>(reinterpret_cast<const uint8_t*>(m.read_accessor<bool, 1>().ptr(m.shape<1>().lo)));
  }
  return c;
}

// ---- outputs: the library allocates through the task's memory resource
// (legate buffers, allocator.cu:27-52); the task binds them zero-copy -----------
struct TaskAlloc {
  static void* allocate(void* ctx, size_t n, void* stream)
  {
    return static_cast<TaskMemoryResource*>(ctx)->allocate(n, static_cast<cudaStream_t>(stream));
  }
  static void deallocate(void* ctx, void* p, size_t n, void* stream)
  {
    static_cast<TaskMemoryResource*>(ctx)->deallocate(p, n, static_cast<cudaStream_t>(stream));
  }
};

inline ldf_allocator task_allocator(TaskContext& ctx)
{
  return ldf_allocator{ctx.mr(), TaskAlloc::allocate, TaskAlloc::deallocate};
}

// Bind one library-allocated buffer to an unbound store and take it out of the
// resource's ownership (as release_buffer does for cudf columns, column.cu:63-68).
void bind_buffer(const legate::PhysicalStore& store, TaskMemoryResource& mr, const void* ptr, size_t extent)
{
  legate::dataframe::MemAlloc* found = mr.find_buffer(ptr);
  if (found == nullptr || !found->valid()) throw std::runtime_error("output buffer not owned by the task");
  legate::dataframe::MemAlloc owned = std::move(*found);  // a later deallocate() leaves it alone
  store.bind_untyped_data(owned.buffer(), legate::Point<1>(static_cast<int64_t>(extent)));
}

void bind_output(PhysicalColumn& out, const ldf_column& c, TaskMemoryResource& mr, cudaStream_t stream)
{
  legate::PhysicalArray& arr = out.physical_array();
  if (c.size == 0) {
    out.bind_empty_data();
    return;
  }
  if (c.type == LDF_STRING) {
    legate::StringPhysicalArray s = arr.as_string_array();
    bind_buffer(s.ranges().data(), mr, c.data, static_cast<size_t>(c.size));  // local ranges, chars_base 0
    if (c.num_chars > 0) bind_buffer(s.chars().data(), mr, c.chars, static_cast<size_t>(c.num_chars));
    else s.chars().data().bind_empty_data();
  } else {
    bind_buffer(arr.data(), mr, c.data, static_cast<size_t>(c.size));
  }
  if (arr.nullable()) {
    if (c.valid != nullptr) {
      bind_buffer(arr.null_mask(), mr, c.valid, static_cast<size_t>(c.size));
    } else {  // no nulls in the result: a mask of ones, as move_into writes (column.cu:58-60)
      legate::PhysicalStore m = arr.null_mask();
      bool* ones = m.create_output_buffer<bool, 1>(legate::Point<1>(c.size), true).ptr(legate::Point<1>(0));
      cudaMemsetAsync(ones, 1, static_cast<size_t>(c.size), stream);
    }
  }
}

std::vector<ldf_column> inputs_of(std::vector<PhysicalColumn>& cols)
{
  std::vector<ldf_column> v;
  v.reserve(cols.size());
  for (auto& c : cols) v.push_back(to_ldf(c));
  return v;
}

void bind_outputs(std::vector<PhysicalColumn>& cols, const std::vector<ldf_column>& res, TaskContext& ctx)
{
  for (size_t i = 0; i < cols.size(); ++i) bind_output(cols[i], res[i], *ctx.mr(), ctx.stream());
}

// ---- JoinTask::gpu_variant (join.cu:187-244), one rank or no repartition ------
void join_gpu_body(TaskContext& ctx)
{
  auto lhs               = argument::get_next_input<PhysicalTable>(ctx);
  auto rhs               = argument::get_next_input<PhysicalTable>(ctx);
  const auto lhs_keys    = argument::get_next_scalar_vector<int32_t>(ctx);
  const auto rhs_keys    = argument::get_next_scalar_vector<int32_t>(ctx);
  const auto join_type   = argument::get_next_scalar<JoinType>(ctx);
  const bool nulls_equal = argument::get_next_scalar<bool>(ctx);
  const auto lhs_out     = argument::get_next_scalar_vector<int32_t>(ctx);
  const auto rhs_out     = argument::get_next_scalar_vector<int32_t>(ctx);
  auto output            = argument::get_next_output<PhysicalTable>(ctx);

  auto lcols = lhs.release();
  auto rcols = rhs.release();
  auto L     = inputs_of(lcols);
  auto R     = inputs_of(rcols);
  std::vector<ldf_column> res(lhs_out.size() + rhs_out.size());
  ldf_allocator alloc = task_allocator(ctx);
  ldf_check(ldf_b200_join(L.data(), static_cast<int32_t>(L.size()), R.data(), static_cast<int32_t>(R.size()),
                          lhs_keys.data(), rhs_keys.data(), static_cast<int32_t>(lhs_keys.size()),
                          static_cast<int32_t>(join_type), nulls_equal ? 1 : 0, lhs_out.data(),
                          static_cast<int32_t>(lhs_out.size()), rhs_out.data(), static_cast<int32_t>(rhs_out.size()),
                          res.data(), &alloc, ctx.stream()));
  auto ocols = output.release();
  bind_outputs(ocols, res, ctx);
}

// ---- GroupByAggregationTask::gpu_variant (groupby_aggregation.cu:90-167) -----
int32_t agg_kind(const std::string& name)  // the names of groupby_aggregation.cu:46-87
{
  static const std::map<std::string, int32_t> kinds{
    {"sum", LDF_AGG_SUM},     {"min", LDF_AGG_MIN},           {"max", LDF_AGG_MAX},
    {"count", LDF_AGG_COUNT}, {"count_all", LDF_AGG_COUNT_ALL}, {"mean", LDF_AGG_MEAN},
    {"count_distinct", LDF_AGG_COUNT_DISTINCT}, {"product", LDF_AGG_PRODUCT},
    {"variance", LDF_AGG_VARIANCE}, {"stddev", LDF_AGG_STDDEV}};
  auto it = kinds.find(name);
  if (it == kinds.end()) throw std::invalid_argument("Unsupported groupby aggregation");
  return it->second;
}

void groupby_gpu_body(TaskContext& ctx)
{
  auto table         = argument::get_next_input<PhysicalTable>(ctx);
  auto output        = argument::get_next_output<PhysicalTable>(ctx);
  const auto keys_sz = argument::get_next_scalar_vector<size_t>(ctx);
  std::vector<int32_t> keys(keys_sz.begin(), keys_sz.end());
  const auto naggs = argument::get_next_scalar<size_t>(ctx);
  auto ocols       = output.release();
  std::vector<ldf_aggregation> aggs;
  std::vector<size_t> out_idx;
  for (size_t i = 0; i < naggs; ++i) {
    const auto in_col  = argument::get_next_scalar<size_t>(ctx);
    const auto kind    = argument::get_next_scalar<std::string>(ctx);
    const auto options = argument::get_next_scalar<std::optional<std::shared_ptr<arrow::compute::FunctionOptions>>>(ctx);
    const auto out_col = argument::get_next_scalar<size_t>(ctx);
    ldf_aggregation a{};
    a.in_col     = static_cast<int32_t>(in_col);
    a.kind       = agg_kind(kind);
    a.count_mode = LDF_COUNT_ONLY_VALID;
    if (options.has_value()) {
      if (auto* co = dynamic_cast<const arrow::compute::CountOptions*>(options->get())) {
        a.count_mode = co->mode == arrow::compute::CountOptions::ONLY_NULL ? LDF_COUNT_ONLY_NULL
                       : co->mode == arrow::compute::CountOptions::ALL     ? LDF_COUNT_ALL
                                                                           : LDF_COUNT_ONLY_VALID;
      }
    }
    a.out_type = ldf_type_of(ocols.at(out_col));  // computed by make_output_column (groupby_aggregation.cpp:100-132)
    aggs.push_back(a);
    out_idx.push_back(out_col);
  }
  auto cols = table.release();
  auto in   = inputs_of(cols);
  std::vector<ldf_column> res(keys.size() + aggs.size());
  ldf_allocator alloc = task_allocator(ctx);
  ldf_check(ldf_b200_groupby_aggregation(in.data(), static_cast<int32_t>(in.size()), keys.data(),
                                         static_cast<int32_t>(keys.size()), aggs.data(),
                                         static_cast<int32_t>(aggs.size()), res.data(), &alloc, ctx.stream()));
  // the library returns the keys, then the aggregations in request order
  for (size_t k = 0; k < keys.size(); ++k) bind_output(ocols.at(k), res[k], *ctx.mr(), ctx.stream());
  for (size_t i = 0; i < aggs.size(); ++i)
    bind_output(ocols.at(out_idx[i]), res[keys.size() + i], *ctx.mr(), ctx.stream());
}

// ---- SortTask::gpu_variant (sort.cu:295-379), the local sort -----------------
void sort_gpu_body(TaskContext& ctx)
{
  auto tbl             = argument::get_next_input<PhysicalTable>(ctx);
  const auto keys_sz   = argument::get_next_scalar_vector<std::size_t>(ctx);
  const auto ascending = argument::get_next_scalar_vector<bool>(ctx);
  const bool nulls_at_end = argument::get_next_scalar<bool>(ctx);
  const bool stable       = argument::get_next_scalar<bool>(ctx);
  const int64_t limit     = argument::get_next_scalar<int64_t>(ctx);
  auto output             = argument::get_next_output<PhysicalTable>(ctx);

  std::vector<int32_t> keys(keys_sz.begin(), keys_sz.end());
  std::vector<uint8_t> asc(ascending.begin(), ascending.end());
  auto cols = tbl.release();
  auto in   = inputs_of(cols);
  std::vector<ldf_column> res(in.size());
  ldf_allocator alloc = task_allocator(ctx);
  ldf_check(ldf_b200_sort(in.data(), static_cast<int32_t>(in.size()), keys.data(), asc.data(),
                          static_cast<int32_t>(keys.size()), nulls_at_end ? 1 : 0, stable ? 1 : 0, limit, res.data(),
                          &alloc, ctx.stream()));
  auto ocols = output.release();
  bind_outputs(ocols, res, ctx);
}

// ---- repartition_by_hash local step (core/repartition_by_hash.cu:296-310) ----
// The partitioned columns and the nparts + 1 bucket offsets, which the
// existing exchange then sends (bucket b to rank b).
std::vector<ldf_column> hash_partition_local(TaskContext& ctx, std::vector<PhysicalColumn>& cols,
                                             const std::vector<int32_t>& keys, std::vector<int64_t>& offsets)
{
  auto in = inputs_of(cols);
  std::vector<ldf_column> res(in.size());
  offsets.assign(static_cast<size_t>(ctx.nranks) + 1, 0);
  ldf_allocator alloc = task_allocator(ctx);
  ldf_check(ldf_b200_hash_partition(in.data(), static_cast<int32_t>(in.size()), keys.data(),
                                    static_cast<int32_t>(keys.size()), ctx.nranks, res.data(), offsets.data(),
                                    &alloc, ctx.stream()));
  return res;
}

// ---- CSVRead::gpu_variant (csv.cu:53-139) --------------------------------------
// Each rank parses whole files (as the CPU variant splits the files,
// csv.cpp:87-88): the bytes go to a device buffer from the task's resource
// and ldf_b200_csv_read parses them there.  This sketch binds one file per
// rank; several files per rank would concatenate the columns.
void csv_read_gpu_body(TaskContext& ctx)
{
  const auto file_paths   = argument::get_next_scalar_vector<std::string>(ctx);
  const auto column_names = argument::get_next_scalar_vector<std::string>(ctx);
  const auto use_cols     = argument::get_next_scalar_vector<int>(ctx);
  const bool na_filter    = argument::get_next_scalar<bool>(ctx);
  const auto delimiter    = static_cast<char>(argument::get_next_scalar<int32_t>(ctx));
  const auto nbytes       = argument::get_next_scalar_vector<size_t>(ctx);
  const auto nbytes_total = argument::get_next_scalar<size_t>(ctx);
  const bool read_header  = argument::get_next_scalar<bool>(ctx);
  auto output             = argument::get_next_output<PhysicalTable>(ctx);
  argument::get_parallel_launch_task(ctx);
  (void)nbytes;
  (void)nbytes_total;
  (void)column_names;

  auto ocols = output.release();
  auto [first_file, nfiles] =
    legate::dataframe::evenly_partition_work(file_paths.size(), static_cast<size_t>(ctx.rank),
                                             static_cast<size_t>(ctx.nranks));
  if (nfiles == 0) {
    for (auto& c : ocols) c.bind_empty_data();
    return;
  }
  std::ifstream in(file_paths[first_file], std::ios::binary);
  const std::vector<char> bytes((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
  TaskMemoryResource& mr = *ctx.mr();
  void* text             = mr.allocate(bytes.size() + 16, ctx.stream());  // 16-byte aligned legate buffer
  cudaMemcpyAsync(text, bytes.data(), bytes.size(), cudaMemcpyHostToDevice, ctx.stream());
  // Arrow's default null spellings (ConvertOptions::null_values), NUL-separated
  static const char kNulls[] =
    "\0#N/A\0#N/A N/A\0#NA\0-1.#IND\0-1.#QNAN\0-NaN\0-nan\0001.#IND\0001.#QNAN\0N/A\0NA\0NULL\0NaN\0n/a\0nan\0null";
  std::vector<int32_t> types;
  for (auto& c : ocols) types.push_back(ldf_type_of(c));
  std::vector<ldf_column> res(ocols.size());
  int64_t nrows       = 0;
  ldf_allocator alloc = task_allocator(ctx);
  ldf_check(ldf_b200_csv_read(static_cast<const uint8_t*>(text), static_cast<int64_t>(bytes.size()), delimiter,
                              read_header ? 1 : 0, use_cols.data(), types.data(), static_cast<int32_t>(types.size()),
                              kNulls, na_filter ? static_cast<int32_t>(sizeof(kNulls)) : 0, na_filter ? 17 : 0,
                              res.data(), &nrows, &alloc, ctx.stream()));
  mr.deallocate(text, bytes.size() + 16, ctx.stream());
  bind_outputs(ocols, res, ctx);
}

// ---- ParquetRead::gpu_variant (parquet.cu:48-101) ----------------------------------
// The rank's row groups (find_files_and_row_groups, parquet.cpp:60-93) are
// decoded on the device: Arrow's metadata reader gives the column chunks'
// extents, ldf_b200_parquet_pages walks their page headers on the host and
// ldf_b200_parquet_decode decodes the pages from a device copy of the file.
// This sketch binds one file per rank; several files per rank would
// concatenate the columns, and a chunk in another codec would take the CPU
// reader's path.
void parquet_read_gpu_body(TaskContext& ctx)
{
  const auto file_paths        = argument::get_next_scalar_vector<std::string>(ctx);
  const auto columns           = argument::get_next_scalar_vector<std::string>(ctx);
  const auto column_indices    = argument::get_next_scalar_vector<int>(ctx);
  const auto ngroups_per_file  = argument::get_next_scalar_vector<size_t>(ctx);
  const auto nrow_groups_total = argument::get_next_scalar<size_t>(ctx);
  auto output                  = argument::get_next_output<PhysicalTable>(ctx);
  argument::get_parallel_launch_task(ctx);
  (void)columns;

  auto ocols = output.release();
  auto [first_group, ngroups] = legate::dataframe::evenly_partition_work(
    nrow_groups_total, static_cast<size_t>(ctx.rank), static_cast<size_t>(ctx.nranks));
  if (ngroups == 0) {
    for (auto& c : ocols) c.bind_empty_data();
    return;
  }
  auto [files, row_groups] =
    legate::dataframe::task::find_files_and_row_groups(file_paths, ngroups_per_file, first_group, ngroups);
  auto metadata = parquet::ParquetFileReader::Open(arrow::io::ReadableFile::Open(files.at(0)))->metadata();
  std::vector<int64_t> start, bytes, row0;
  std::vector<int32_t> column, codec, physical;
  int64_t nrows = 0;
  for (int g : row_groups.at(0)) {
    auto rg = metadata->RowGroup(g);
    for (size_t j = 0; j < column_indices.size(); ++j) {
      auto cc = rg->ColumnChunk(column_indices[j]);
      if (cc->compression() != parquet::Compression::SNAPPY && cc->compression() != parquet::Compression::UNCOMPRESSED)
        throw std::invalid_argument("codec not decoded on the device");
      start.push_back(cc->has_dictionary_page() ? cc->dictionary_page_offset() : cc->data_page_offset());
      bytes.push_back(cc->total_compressed_size());
      row0.push_back(nrows);
      column.push_back(static_cast<int32_t>(j));
      codec.push_back(cc->compression() == parquet::Compression::SNAPPY ? LDF_PQ_SNAPPY : LDF_PQ_UNCOMPRESSED);
      if (g == row_groups.at(0).front()) physical.push_back(static_cast<int32_t>(cc->type()));
    }
    nrows += rg->num_rows();
  }
  std::ifstream in(files.at(0), std::ios::binary);
  const std::vector<uint8_t> file((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
  const auto nchunks = static_cast<int32_t>(start.size());
  int32_t npages     = 0;
  std::vector<int32_t> chunk_physical;
  for (int32_t k = 0; k < nchunks; ++k) chunk_physical.push_back(physical.at(column[k]));
  ldf_check(ldf_b200_parquet_pages(file.data(), static_cast<int64_t>(file.size()), start.data(), bytes.data(),
                                   row0.data(), column.data(), codec.data(), chunk_physical.data(), nchunks,
                                   nullptr, 0, &npages));
  std::vector<ldf_parquet_page> pages(static_cast<size_t>(npages));
  ldf_check(ldf_b200_parquet_pages(file.data(), static_cast<int64_t>(file.size()), start.data(), bytes.data(),
                                   row0.data(), column.data(), codec.data(), chunk_physical.data(), nchunks,
                                   pages.data(), npages, &npages));
  TaskMemoryResource& mr = *ctx.mr();
  void* dfile            = mr.allocate(file.size() + 16, ctx.stream());
  cudaMemcpyAsync(dfile, file.data(), file.size(), cudaMemcpyHostToDevice, ctx.stream());
  std::vector<int32_t> types, nullable;
  for (auto& c : ocols) {
    types.push_back(ldf_type_of(c));
    nullable.push_back(c.nullable() ? 1 : 0);
  }
  std::vector<ldf_column> res(ocols.size());
  ldf_allocator alloc = task_allocator(ctx);
  ldf_check(ldf_b200_parquet_decode(static_cast<const uint8_t*>(dfile), static_cast<int64_t>(file.size()),
                                    pages.data(), npages, physical.data(), types.data(), nullable.data(),
                                    static_cast<int32_t>(ocols.size()), nrows, res.data(), &alloc, ctx.stream()));
  mr.deallocate(dfile, file.size() + 16, ctx.stream());
  bind_outputs(ocols, res, ctx);
}

}  // namespace ldf_integration
