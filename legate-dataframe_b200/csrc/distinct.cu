// distinct: one row per distinct combination of the key columns.
//
// Reference: legate::dataframe::distinct (cpp/src/stream_compaction.cpp:121-150)
// and DistinctTask (cpp/src/stream_compaction.cu:45-76, .cpp:45-96): every
// column of the input is returned; for columns that are not keys any value
// of the group is allowed (cudf distinct KEEP_ANY, Arrow hash_one).  Here
// whole rows are kept: the groupby key kernels give every group a
// representative row (MAX of the row index), then every column is gathered
// through the representative rows.  Keys follow the groupby's equality: null
// keys form one group, floats compare by bit pattern.
#include "table_ops.cuh"

namespace ldf {
void groupby_aggregation(const ldf_column* table, int ncols, const int32_t* keys, int nkeys,
                         const ldf_aggregation* aggs, int naggs, ldf_column* out, const OpContext& ctx);

namespace {
__global__ void iota_i32_kernel(int32_t* p, int64_t n)
{
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    p[i] = static_cast<int32_t>(i);
}
}  // namespace

void distinct(const ldf_column* table, int ncols, const int32_t* keys, int nkeys, ldf_column* out,
              const OpContext& ctx)
{
  LDF_REQUIRE(ncols >= 1, "distinct needs at least one column");
  if (nkeys < 1) fail(LDF_ERR_INVALID_ARGUMENT, "must pass at least one key column");
  for (int j = 0; j < nkeys; ++j) LDF_REQUIRE(keys[j] >= 0 && keys[j] < ncols, "key column out of range");
  const int64_t n = table[0].size;
  LDF_REQUIRE(n < (int64_t(1) << 31), "tables of 2^31 rows or more per task are not supported");
  const Allocator& al = ctx.alloc();
  cudaStream_t s      = ctx.stream();

  // row-index column appended to the table; its per-group MAX is the representative row
  Buffer<int32_t> rows(al, std::max<int64_t>(n, 1));
  if (n > 0) {
    const unsigned blocks = static_cast<unsigned>(std::min<int64_t>(ceil_div(n, 256), 8 * num_sms()));
    launch("iota", iota_i32_kernel, blocks, 256u, 0, s, rows.get(), n);
  }
  std::vector<ldf_column> t(table, table + ncols);
  ldf_column rc{};
  rc.type = LDF_INT32;
  rc.size = n;
  rc.data = rows.get();
  t.push_back(rc);
  ldf_aggregation ag{};
  ag.in_col   = ncols;
  ag.kind     = LDF_AGG_MAX;
  ag.out_type = LDF_INT32;
  std::vector<ldf_column> g(nkeys + 1);
  groupby_aggregation(t.data(), ncols + 1, keys, nkeys, &ag, 1, g.data(), ctx);
  const ldf_column& rep = g[nkeys];
  const int64_t groups  = rep.size;

  for (int j = 0; j < ncols; ++j) {
    const ldf_column& c = table[j];
    out[j]              = alloc_out_column(al, c.type, groups, c.valid != nullptr);
    if (c.type == LDF_STRING) gather_strings(ctx, make_dcol(c), static_cast<const int32_t*>(rep.data), groups, out[j]);
    else gather_fixed(ctx, make_dcol(c), static_cast<const int32_t*>(rep.data), groups, out[j]);
    out[j].size = groups;
  }
  for (auto& c : g) free_out_column(al, c);
}

}  // namespace ldf
