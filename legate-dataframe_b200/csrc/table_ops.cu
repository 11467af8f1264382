// Shared building blocks: key sets, output allocation, gathers.
#include "table_ops.cuh"

namespace ldf {

KeyCols make_keys(const ldf_column* cols, int ncols, const int32_t* idx, int nkeys)
{
  LDF_REQUIRE(nkeys >= 1 && nkeys <= kMaxKeys,
              "number of key columns must be in [1, " + std::to_string(kMaxKeys) + "]");
  KeyCols k{};
  k.n = nkeys;
  for (int j = 0; j < nkeys; ++j) {
    LDF_REQUIRE(idx[j] >= 0 && idx[j] < ncols, "key column index out of range");
    k.c[j] = make_dcol(cols[idx[j]]);
  }
  return k;
}

KeyMode key_mode(const KeyCols& k)
{
  if (k.n != 1 || k.c[0].type == LDF_STRING) return KeyMode::GEN;
  return k.c[0].width <= 4 ? KeyMode::K32 : KeyMode::K64;
}

ldf_column alloc_out_column(const Allocator& a, int type, int64_t rows, bool nullable)
{
  ldf_column c{};
  c.type     = type;
  c.nullable = nullable ? 1 : 0;
  c.size     = rows;
  int w      = type_width(type);
  c.data     = a.allocate(static_cast<size_t>(rows) * w);
  c.valid    = nullable ? static_cast<uint8_t*>(a.allocate(static_cast<size_t>(rows))) : nullptr;
  c.chars    = nullptr;
  c.chars_base = 0;
  c.num_chars  = 0;
  return c;
}

void free_out_column(const Allocator& a, ldf_column& c)
{
  if (c.data) a.deallocate(c.data, static_cast<size_t>(c.size) * type_width(c.type));
  if (c.valid) a.deallocate(c.valid, static_cast<size_t>(c.size));
  if (c.chars) a.deallocate(c.chars, static_cast<size_t>(c.num_chars));
  c.data  = nullptr;
  c.valid = nullptr;
  c.chars = nullptr;
}

namespace {

__global__ void string_lengths_kernel(DCol src, const int32_t* map, int64_t rows, int64_t* lens)
{
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < rows;
       i += (int64_t)gridDim.x * blockDim.x) {
    int64_t r = map ? map[i] : i;
    lens[i]   = (r >= 0 && dvalid(src, r)) ? dstr_len(src, r) : 0;
  }
}

// One warp per 32 rows; each lane copies its row's bytes.  Ranges are written
// as local offsets with chars_base = 0.
__global__ void string_copy_kernel(DCol src, const int32_t* map, int64_t rows,
                                   const int64_t* offs, ldf_range* dst_ranges, uint8_t* dst_valid,
                                   uint8_t* dst_chars)
{
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < rows;
       i += (int64_t)gridDim.x * blockDim.x) {
    int64_t r  = map ? map[i] : i;
    bool ok    = r >= 0 && dvalid(src, r);
    int64_t o  = offs[i];
    int64_t n  = ok ? dstr_len(src, r) : 0;
    dst_ranges[i] = ldf_range{o, o + n - 1};
    if (dst_valid) dst_valid[i] = ok ? 1 : 0;
    if (n > 0) {
      const uint8_t* p = dstr_ptr(src, r);
      for (int64_t b = 0; b < n; ++b) dst_chars[o + b] = p[b];
    }
  }
}

__global__ void gather_fixed_kernel(DCol src, const int32_t* map, int64_t rows, void* dst,
                                    uint8_t* dst_valid)
{
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < rows;
       i += (int64_t)gridDim.x * blockDim.x) {
    int64_t r = map[i];
    if (r >= 0) {
      copy_fixed(dst, i, src.data, r, src.width);
      if (dst_valid) dst_valid[i] = dvalid(src, r) ? 1 : 0;
    } else {
      zero_fixed(dst, i, src.width);
      if (dst_valid) dst_valid[i] = 0;
    }
  }
}

inline unsigned grid_for(int64_t n, int threads)
{
  int64_t b = ceil_div(n, threads);
  int64_t cap = static_cast<int64_t>(num_sms()) * 16;
  return static_cast<unsigned>(b < 1 ? 1 : (b > cap ? cap : b));
}

}  // namespace

void gather_strings(const OpContext& ctx, const DCol& src, const int32_t* map, int64_t rows,
                    ldf_column& dst)
{
  const Allocator& a = ctx.alloc();
  cudaStream_t s     = ctx.stream();
  if (rows == 0) {
    dst.chars     = static_cast<char*>(a.allocate(16));
    dst.num_chars = 0;
    return;
  }
  Buffer<int64_t> lens(a, rows);
  Buffer<int64_t> offs(a, rows);
  Buffer<int64_t> total(a, 1);
  launch("string_lengths", string_lengths_kernel, grid_for(rows, 256), 256, 0, s, src, map, rows, lens.get());
  LDF_CHECK_LAUNCH();
  exclusive_scan_i64(lens.get(), offs.get(), rows, total.get(), ctx);
  int64_t nchars = ctx.read_i64(total.get());
  dst.chars      = static_cast<char*>(a.allocate(static_cast<size_t>(nchars)));
  dst.num_chars  = nchars;
  dst.chars_base = 0;
  launch("string_copy", string_copy_kernel, grid_for(rows, 256), 256, 0, s, 
    src, map, rows, offs.get(), static_cast<ldf_range*>(dst.data), dst.valid,
    reinterpret_cast<uint8_t*>(dst.chars));
  LDF_CHECK_LAUNCH();
}

void gather_fixed(const OpContext& ctx, const DCol& src, const int32_t* map, int64_t rows,
                  ldf_column& dst)
{
  if (rows == 0) return;
  launch("gather_fixed", gather_fixed_kernel, grid_for(rows, 256), 256, 0, ctx.stream(), src, map, rows, dst.data,
                                                                      dst.valid);
  LDF_CHECK_LAUNCH();
}

}  // namespace ldf
