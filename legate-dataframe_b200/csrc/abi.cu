// extern "C" entry points (include/ldf_b200.h): argument checks, exception ->
// status translation, one OpContext per call.
#include "radix.cuh"

namespace ldf {
void join(const ldf_column* lhs, int lhs_ncols, const ldf_column* rhs, int rhs_ncols,
          const int32_t* lhs_keys, const int32_t* rhs_keys, int nkeys, int join_type,
          bool nulls_equal, const int32_t* lhs_out, int n_lhs_out, const int32_t* rhs_out,
          int n_rhs_out, ldf_column* out, const OpContext& ctx);
void groupby_aggregation(const ldf_column* table, int ncols, const int32_t* keys, int nkeys,
                         const ldf_aggregation* aggs, int naggs, ldf_column* out, const OpContext& ctx);
void sort_table(const ldf_column* table, int ncols, const int32_t* keys, const uint8_t* ascending, int nkeys,
                bool nulls_at_end, int64_t limit, ldf_column* out, const OpContext& ctx);
void hash_partition(const ldf_column* table, int ncols, const int32_t* keys, int nkeys, int nparts,
                    ldf_column* out, int64_t* offsets, const OpContext& ctx);
void distinct(const ldf_column* table, int ncols, const int32_t* keys, int nkeys, ldf_column* out,
              const OpContext& ctx);
void arrow_bits_to_bytes(const uint8_t* bits, int64_t bit_offset, int64_t n, uint8_t* out, cudaStream_t s);
void arrow_offsets_to_ranges(const void* offsets, int offset_bytes, int64_t n, ldf_range* out, cudaStream_t s);
void csv_read(const uint8_t* text, int64_t n, char delimiter, int skip_first, const int32_t* fields,
              const int32_t* types, int ncols, const char* nulls, int nulls_bytes, int n_nulls, ldf_column* out,
              int64_t* nrows, const OpContext& ctx);
void parquet_pages(const uint8_t* file, int64_t file_bytes, const int64_t* chunk_start, const int64_t* chunk_bytes,
                   const int64_t* chunk_row0, const int32_t* chunk_column, const int32_t* chunk_codec,
                   const int32_t* chunk_physical, int nchunks, ldf_parquet_page* pages, int max_pages, int* npages);
void parquet_decode(const uint8_t* file, int64_t file_bytes, const ldf_parquet_page* pages, int npages,
                    const int32_t* physical, const int32_t* types, const int32_t* nullable, int ncols, int64_t nrows,
                    ldf_column* out, const OpContext& ctx);
}  // namespace ldf

namespace {
thread_local std::string g_last_error;

template <typename F>
int guarded(F&& f)
{
  g_last_error.clear();
  try {
    f();
    return LDF_OK;
  } catch (const ldf::LdfError& e) {
    g_last_error = e.what();
    return e.code;
  } catch (const std::exception& e) {
    g_last_error = e.what();
    return LDF_ERR_INTERNAL;
  } catch (...) {
    g_last_error = "unknown error";
    return LDF_ERR_INTERNAL;
  }
}

void check_table(const ldf_column* t, int32_t ncols, const char* what)
{
  LDF_REQUIRE(ncols >= 0, std::string(what) + ": negative column count");
  LDF_REQUIRE(ncols == 0 || t != nullptr, std::string(what) + ": null column array");
  for (int i = 0; i < ncols; ++i) {
    ldf::type_width(t[i].type);
    LDF_REQUIRE(t[i].size == t[0].size, std::string(what) + ": columns differ in length");
    LDF_REQUIRE(t[i].size == 0 || t[i].data != nullptr, std::string(what) + ": column without data");
    if (t[i].type == LDF_STRING)
      LDF_REQUIRE(t[i].size == 0 || t[i].chars != nullptr || t[i].num_chars == 0,
                  std::string(what) + ": string column without chars");
  }
}
}  // namespace

namespace ldf {
void set_last_error(const std::string& msg) { g_last_error = msg; }
}  // namespace ldf

extern "C" {

const char* ldf_b200_last_error(void) { return g_last_error.c_str(); }
const char* ldf_b200_version(void) { return "ldf_b200 0.1.0 (sm_100a)"; }

int ldf_b200_join(const ldf_column* lhs, int32_t lhs_ncols, const ldf_column* rhs, int32_t rhs_ncols,
                  const int32_t* lhs_keys, const int32_t* rhs_keys, int32_t nkeys, int32_t join_type,
                  int32_t nulls_equal, const int32_t* lhs_out, int32_t n_lhs_out, const int32_t* rhs_out,
                  int32_t n_rhs_out, ldf_column* out, const ldf_allocator* alloc, void* stream)
{
  return guarded([&] {
    check_table(lhs, lhs_ncols, "lhs");
    check_table(rhs, rhs_ncols, "rhs");
    LDF_REQUIRE(out != nullptr || n_lhs_out + n_rhs_out == 0, "null output array");
    ldf::OpContext ctx(alloc, static_cast<cudaStream_t>(stream));
    ldf::join(lhs, lhs_ncols, rhs, rhs_ncols, lhs_keys, rhs_keys, nkeys, join_type, nulls_equal != 0,
              lhs_out, n_lhs_out, rhs_out, n_rhs_out, out, ctx);
  });
}

int ldf_b200_groupby_aggregation(const ldf_column* table, int32_t ncols, const int32_t* keys, int32_t nkeys,
                                 const ldf_aggregation* aggs, int32_t naggs, ldf_column* out,
                                 const ldf_allocator* alloc, void* stream)
{
  return guarded([&] {
    check_table(table, ncols, "table");
    LDF_REQUIRE(naggs >= 0 && (naggs == 0 || aggs != nullptr), "bad aggregation list");
    ldf::OpContext ctx(alloc, static_cast<cudaStream_t>(stream));
    ldf::groupby_aggregation(table, ncols, keys, nkeys, aggs, naggs, out, ctx);
  });
}

int ldf_b200_sort(const ldf_column* table, int32_t ncols, const int32_t* keys, const uint8_t* ascending,
                  int32_t nkeys, int32_t nulls_at_end, int32_t stable, int64_t limit, ldf_column* out,
                  const ldf_allocator* alloc, void* stream)
{
  (void)stable;  // the radix sort is always stable
  return guarded([&] {
    check_table(table, ncols, "table");
    ldf::OpContext ctx(alloc, static_cast<cudaStream_t>(stream));
    ldf::sort_table(table, ncols, keys, ascending, nkeys, nulls_at_end != 0, limit, out, ctx);
  });
}

int ldf_b200_hash_partition(const ldf_column* table, int32_t ncols, const int32_t* keys, int32_t nkeys,
                            int32_t nparts, ldf_column* out, int64_t* offsets, const ldf_allocator* alloc,
                            void* stream)
{
  return guarded([&] {
    check_table(table, ncols, "table");
    LDF_REQUIRE(offsets != nullptr, "null offsets array");
    ldf::OpContext ctx(alloc, static_cast<cudaStream_t>(stream));
    ldf::hash_partition(table, ncols, keys, nkeys, nparts, out, offsets, ctx);
  });
}

int ldf_b200_distinct(const ldf_column* table, int32_t ncols, const int32_t* keys, int32_t nkeys, ldf_column* out,
                      const ldf_allocator* alloc, void* stream)
{
  return guarded([&] {
    check_table(table, ncols, "table");
    LDF_REQUIRE(out != nullptr || ncols == 0, "null output array");
    ldf::OpContext ctx(alloc, static_cast<cudaStream_t>(stream));
    ldf::distinct(table, ncols, keys, nkeys, out, ctx);
  });
}

int ldf_b200_arrow_bits_to_bytes(const uint8_t* bits, int64_t bit_offset, int64_t n, uint8_t* out, void* stream)
{
  return guarded([&] { ldf::arrow_bits_to_bytes(bits, bit_offset, n, out, static_cast<cudaStream_t>(stream)); });
}

int ldf_b200_arrow_offsets_to_ranges(const void* offsets, int32_t offset_bytes, int64_t n, ldf_range* ranges,
                                     void* stream)
{
  return guarded([&] {
    ldf::arrow_offsets_to_ranges(offsets, offset_bytes, n, ranges, static_cast<cudaStream_t>(stream));
  });
}

int ldf_b200_csv_read(const uint8_t* text, int64_t nbytes, char delimiter, int32_t skip_first, const int32_t* fields,
                      const int32_t* types, int32_t ncols, const char* nulls, int32_t nulls_bytes, int32_t n_nulls,
                      ldf_column* out, int64_t* nrows, const ldf_allocator* alloc, void* stream)
{
  return guarded([&] {
    ldf::OpContext ctx(alloc, static_cast<cudaStream_t>(stream));
    ldf::csv_read(text, nbytes, delimiter, skip_first != 0, fields, types, ncols, nulls, nulls_bytes, n_nulls, out,
                  nrows, ctx);
  });
}

int ldf_b200_parquet_pages(const uint8_t* file_host, int64_t file_bytes, const int64_t* chunk_start,
                           const int64_t* chunk_bytes, const int64_t* chunk_row0, const int32_t* chunk_column,
                           const int32_t* chunk_codec, const int32_t* chunk_physical, int32_t nchunks,
                           ldf_parquet_page* pages, int32_t max_pages, int32_t* npages)
{
  return guarded([&] {
    int n = 0;
    ldf::parquet_pages(file_host, file_bytes, chunk_start, chunk_bytes, chunk_row0, chunk_column, chunk_codec,
                       chunk_physical, nchunks, pages, max_pages, &n);
    *npages = n;
  });
}

int ldf_b200_parquet_decode(const uint8_t* file, int64_t file_bytes, const ldf_parquet_page* pages, int32_t npages,
                            const int32_t* physical, const int32_t* types, const int32_t* nullable, int32_t ncols,
                            int64_t nrows, ldf_column* out, const ldf_allocator* alloc, void* stream)
{
  return guarded([&] {
    LDF_REQUIRE(physical != nullptr && types != nullptr && nullable != nullptr && out != nullptr,
                "parquet_decode: null argument");
    ldf::OpContext ctx(alloc, static_cast<cudaStream_t>(stream));
    ldf::parquet_decode(file, file_bytes, pages, npages, physical, types, nullable, ncols, nrows, out, ctx);
  });
}

int ldf_b200_free_column(ldf_column* col, const ldf_allocator* alloc, void* stream)
{
  return guarded([&] {
    if (col == nullptr) return;
    ldf::Allocator a(alloc, static_cast<cudaStream_t>(stream));
    ldf::free_out_column(a, *col);
  });
}

}  // extern "C"
