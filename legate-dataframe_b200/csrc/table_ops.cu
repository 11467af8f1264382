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

// Tiles of kStrTile x kStrRows rows.  Each thread handles kStrRows rows and
// issues their loads together: map entries, source ranges, then every
// string's bytes as at most kStrWords aligned 8-byte words (only words inside
// the chars buffer; longer strings and the buffer's edges go byte by byte).
// The tile's chars (a contiguous output range) are assembled in shared memory
// at the output's 16-byte phase and written with 16-byte stores (bytes at the
// range's two ends, shared with the neighbouring tiles, singly).  A tile whose
// chars exceed the staging buffer writes bytes directly.  Ranges are written
// as local offsets with chars_base = 0.
constexpr int kStrTile  = 256;
constexpr int kStrRows  = 2;
constexpr int kStrWords = 4;
constexpr int kStrStage = 16 * 1024;

__global__ void __launch_bounds__(kStrTile) string_copy_kernel(DCol src, const int32_t* map, int64_t rows,
                                                               const int64_t* offs, int64_t nchars,
                                                               ldf_range* dst_ranges, uint8_t* dst_valid,
                                                               uint8_t* dst_chars)
{
  __shared__ __align__(16) uint8_t stage[kStrStage + 16];
  const ldf_range* rg_src = static_cast<const ldf_range*>(src.data);
  const uintptr_t cbeg    = reinterpret_cast<uintptr_t>(src.chars);
  const uintptr_t cend    = cbeg + static_cast<uintptr_t>(src.num_chars);
  const int64_t per_tile  = static_cast<int64_t>(kStrTile) * kStrRows;
  for (int64_t tile = blockIdx.x; tile * per_tile < rows; tile += gridDim.x) {
    const int64_t i0 = tile * per_tile;
    int64_t r[kStrRows], o[kStrRows], n[kStrRows];
    const uint8_t* p[kStrRows];
#pragma unroll
    for (int j = 0; j < kStrRows; ++j) {
      const int64_t i = i0 + j * kStrTile + threadIdx.x;
      r[j]            = -2;
      if (i < rows) r[j] = map ? __ldg(map + i) : i;
    }
#pragma unroll
    for (int j = 0; j < kStrRows; ++j) {
      const int64_t i = i0 + j * kStrTile + threadIdx.x;
      n[j] = 0;
      o[j] = 0;
      p[j] = nullptr;
      if (r[j] == -2) continue;
      o[j]          = offs[i];
      const bool ok = r[j] >= 0 && dvalid(src, r[j]);
      if (ok) {
        const ldf_range rg = rg_src[r[j]];
        n[j]               = rg.hi - rg.lo + 1;
        p[j]               = reinterpret_cast<const uint8_t*>(src.chars) + (rg.lo - src.chars_base);
      }
      dst_ranges[i] = ldf_range{o[j], o[j] + n[j] - 1};
      if (dst_valid) dst_valid[i] = ok ? 1 : 0;
    }
    // the strings' words (all loads of the thread in flight together)
    unsigned long long w[kStrRows][kStrWords];
    int sh[kStrRows];
    bool fast[kStrRows];
#pragma unroll
    for (int j = 0; j < kStrRows; ++j) {
      const uintptr_t a  = reinterpret_cast<uintptr_t>(p[j]);
      const uintptr_t a0 = a & ~uintptr_t(7);
      sh[j]              = static_cast<int>(a - a0);
      fast[j]            = n[j] > 0 && sh[j] + n[j] <= 8 * kStrWords;
#pragma unroll
      for (int k = 0; k < kStrWords; ++k) {
        const uintptr_t wa = a0 + 8 * k;
        w[j][k]            = 0;
        if (fast[j] && 8 * k < sh[j] + n[j]) {
          if (wa >= cbeg && wa + 8 <= cend) w[j][k] = __ldg(reinterpret_cast<const unsigned long long*>(wa));
          else fast[j] = false;
        }
      }
    }
    const int64_t lo    = offs[i0];
    const int64_t hi    = i0 + per_tile < rows ? offs[i0 + per_tile] : nchars;
    // stage[k] <-> dst_chars[abase + k], with dst_chars + abase 16-byte aligned
    const int64_t abase = lo - static_cast<int64_t>(reinterpret_cast<uintptr_t>(dst_chars + lo) & 15);
    const bool staged   = hi - abase <= kStrStage;
#pragma unroll
    for (int j = 0; j < kStrRows; ++j) {
      uint8_t* q = staged ? stage + (o[j] - abase) : dst_chars + o[j];
      if (fast[j]) {
        // string word k = bytes [8k, 8k + 8) of the string (funnel shift by the
        // source misalignment); every index below is a compile-time constant
        const int s8 = 8 * sh[j];
#pragma unroll
        for (int k = 0; k < kStrWords; ++k) {
          const unsigned long long nxt = k + 1 < kStrWords ? w[j][k + 1] : 0ull;
          const unsigned long long wk  = s8 == 0 ? w[j][k] : ((w[j][k] >> s8) | (nxt << (64 - s8)));
#pragma unroll
          for (int bb = 0; bb < 8; ++bb)
            if (8 * k + bb < n[j]) q[8 * k + bb] = static_cast<uint8_t>(wk >> (8 * bb));
        }
      } else {
        for (int64_t b = 0; b < n[j]; ++b) q[b] = __ldg(p[j] + b);
      }
    }
    if (staged) {
      __syncthreads();
      // chunk c covers dst positions [abase + 16c, abase + 16c + 16)
      const int64_t nchunks = (hi - abase + 15) >> 4;
      for (int64_t c = threadIdx.x; c < nchunks; c += blockDim.x) {
        const int64_t a0 = abase + 16 * c;
        if (a0 >= lo && a0 + 16 <= hi) {
          *reinterpret_cast<uint4*>(dst_chars + a0) = *reinterpret_cast<const uint4*>(stage + 16 * c);
        } else {
          for (int k = 0; k < 16; ++k) {
            const int64_t a = a0 + k;
            if (a >= lo && a < hi) dst_chars[a] = stage[16 * c + k];
          }
        }
      }
      __syncthreads();
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
  launch("string_copy", string_copy_kernel, grid_for(ceil_div(rows, kStrRows), kStrTile), kStrTile, 0, s, src, map,
         rows,
         static_cast<const int64_t*>(offs.get()), nchars, static_cast<ldf_range*>(dst.data), dst.valid,
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
