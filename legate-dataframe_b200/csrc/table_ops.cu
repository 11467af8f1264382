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

// ---- host-resident inputs -----------------------------------------------------
namespace {
bool host_resident(const void* p)
{
  if (p == nullptr) return false;
  cudaPointerAttributes at{};
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    (void)cudaGetLastError();
    return true;  // unknown to CUDA: plain host memory
  }
  return at.type == cudaMemoryTypeHost || at.type == cudaMemoryTypeUnregistered;
}
}  // namespace

HostStaging::HostStaging(const OpContext& ctx, const ldf_column* table, int ncols, const std::vector<int>& order)
  : s_(ctx.stream()), table_(table, table + ncols), ready_(static_cast<size_t>(ncols), nullptr)
{
  try {
    stage_columns(ctx, order);
  } catch (...) {
    release();  // a copy already issued must finish before its buffer is freed
    throw;
  }
}

void HostStaging::stage_columns(const OpContext& ctx, const std::vector<int>& order)
{
  const int ncols     = static_cast<int>(table_.size());
  const Allocator& al = ctx.alloc();
  cudaStream_t& cs    = cs_;
  for (int c : order) {
    if (c < 0 || c >= ncols || ready_[c] != nullptr) continue;
    ldf_column& col  = table_[c];
    const bool str   = col.type == LDF_STRING;
    const bool h_dat = host_resident(col.data), h_val = host_resident(col.valid);
    const bool h_chr = str && host_resident(col.chars);
    if (!h_dat && !h_val && !h_chr) continue;
    if (cs == nullptr) {
      // the staging buffers may reuse memory that earlier work on the op's
      // stream still touches: the copies start after that work
      cs = staging_stream();
      cudaEvent_t e0;
      LDF_CUDA(cudaEventCreateWithFlags(&e0, cudaEventDisableTiming));
      LDF_CUDA(cudaEventRecord(e0, s_));
      LDF_CUDA(cudaStreamWaitEvent(cs, e0, 0));
      LDF_CUDA(cudaEventDestroy(e0));
    }
    auto stage = [&](void* src, size_t nbytes) -> void* {
      bufs_.emplace_back(al, std::max<size_t>(nbytes, 1));
      void* dst = bufs_.back().get();
      if (nbytes) LDF_CUDA(cudaMemcpyAsync(dst, src, nbytes, cudaMemcpyHostToDevice, cs));
      bytes_ += static_cast<int64_t>(nbytes);
      return dst;
    };
    const size_t rows = static_cast<size_t>(col.size);
    if (h_dat) col.data = stage(col.data, rows * (str ? sizeof(ldf_range) : static_cast<size_t>(type_width(col.type))));
    if (h_val) col.valid = static_cast<uint8_t*>(stage(col.valid, rows));
    if (h_chr) col.chars = static_cast<char*>(stage(col.chars, static_cast<size_t>(col.num_chars)));
    LDF_CUDA(cudaEventCreateWithFlags(&ready_[c], cudaEventDisableTiming));
    LDF_CUDA(cudaEventRecord(ready_[c], cs));
  }
}

HostStaging::~HostStaging() { release(); }

// The op's stream passes every copy before the staging buffers go back to the
// allocator (stream-ordered), also when the op failed part way.
void HostStaging::release() noexcept
{
  if (cs_ != nullptr) {  // every copy issued so far
    cudaEvent_t done;
    if (cudaEventCreateWithFlags(&done, cudaEventDisableTiming) == cudaSuccess) {
      cudaEventRecord(done, cs_);
      cudaStreamWaitEvent(s_, done, 0);
      cudaEventDestroy(done);
    }
    cs_ = nullptr;
  }
  for (cudaEvent_t& e : ready_)
    if (e != nullptr) {
      cudaEventDestroy(e);
      e = nullptr;
    }
}

void HostStaging::wait(int col) const
{
  if (col >= 0 && col < static_cast<int>(ready_.size()) && ready_[col] != nullptr)
    LDF_CUDA(cudaStreamWaitEvent(s_, ready_[col], 0));
}

namespace {

// Output length and source chars offset of each gathered string: srcoff[i] =
// offset of the row's first char in src.chars (0 for an empty string), -1
// for a null row.  The copy kernel then reads these sequentially instead of
// gathering the ranges a second time.  Four rows per thread, loads in flight
// together.
constexpr int kLenRows = 4;
__global__ void __launch_bounds__(256) string_lengths_kernel(DCol src, const int32_t* map, int64_t rows,
                                                             int64_t* lens, int64_t* srcoff)
{
  const ldf_range* rg    = static_cast<const ldf_range*>(src.data);
  const int64_t per_iter = static_cast<int64_t>(blockDim.x) * kLenRows;
  for (int64_t base = blockIdx.x * per_iter; base < rows; base += static_cast<int64_t>(gridDim.x) * per_iter) {
    int64_t r[kLenRows];
#pragma unroll
    for (int j = 0; j < kLenRows; ++j) {
      const int64_t i = base + j * blockDim.x + threadIdx.x;
      r[j]            = i < rows ? (map ? static_cast<int64_t>(__ldg(map + i)) : i) : -2;
    }
    ldf_range g[kLenRows];
    bool ok[kLenRows];
#pragma unroll
    for (int j = 0; j < kLenRows; ++j) {
      ok[j] = r[j] >= 0 && dvalid(src, r[j]);
      g[j]  = r[j] >= 0 ? rg[r[j]] : ldf_range{0, -1};
    }
#pragma unroll
    for (int j = 0; j < kLenRows; ++j) {
      if (r[j] == -2) continue;
      const int64_t i = base + j * blockDim.x + threadIdx.x;
      const int64_t n = ok[j] ? g[j].hi - g[j].lo + 1 : 0;
      lens[i]         = n;
      srcoff[i]       = ok[j] ? (n > 0 ? g[j].lo - src.chars_base : 0) : -1;
    }
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

__global__ void __launch_bounds__(kStrTile) string_copy_kernel(DCol src, const int64_t* srcoff, int64_t rows,
                                                               const int64_t* offs, int64_t nchars,
                                                               ldf_range* dst_ranges, uint8_t* dst_valid,
                                                               uint8_t* dst_chars)
{
  __shared__ __align__(16) uint8_t stage[kStrStage + 16];
  const uintptr_t cbeg    = reinterpret_cast<uintptr_t>(src.chars);
  const uintptr_t cend    = cbeg + static_cast<uintptr_t>(src.num_chars);
  const int64_t per_tile  = static_cast<int64_t>(kStrTile) * kStrRows;
  for (int64_t tile = blockIdx.x; tile * per_tile < rows; tile += gridDim.x) {
    const int64_t i0 = tile * per_tile;
    int64_t so[kStrRows], o[kStrRows], n[kStrRows];
    const uint8_t* p[kStrRows];
#pragma unroll
    for (int j = 0; j < kStrRows; ++j) {
      const int64_t i = i0 + j * kStrTile + threadIdx.x;
      so[j] = -2;
      n[j]  = 0;
      o[j]  = 0;
      if (i < rows) {
        so[j] = __ldg(srcoff + i);
        o[j]  = __ldg(offs + i);
        n[j]  = (i + 1 < rows ? __ldg(offs + i + 1) : nchars) - o[j];
      }
    }
#pragma unroll
    for (int j = 0; j < kStrRows; ++j) {
      const int64_t i = i0 + j * kStrTile + threadIdx.x;
      p[j]            = so[j] >= 0 ? reinterpret_cast<const uint8_t*>(src.chars) + so[j] : nullptr;
      if (so[j] == -2) continue;
      dst_ranges[i] = ldf_range{o[j], o[j] + n[j] - 1};
      if (dst_valid) dst_valid[i] = so[j] >= 0 ? 1 : 0;
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

// Gather of up to kGatherCols fixed-width columns through one index map
// (map[i] < 0 -> null).  Each thread owns kGatherRows rows (strided by the
// block, so map reads and output writes stay coalesced) and keeps all their
// source loads of one column in flight together.
constexpr int kGatherCols = 8;
constexpr int kGatherRows = 8;
struct GatherSet {
  int ncols;
  int width[kGatherCols];
  const void* src[kGatherCols];
  const uint8_t* valid[kGatherCols];
  void* dst[kGatherCols];
  uint8_t* dst_valid[kGatherCols];
};

template <typename T>
__device__ __forceinline__ void gather_one(const T* src, const uint8_t* valid, T* dst, uint8_t* dst_valid,
                                           const int64_t (&i)[kGatherRows], const int32_t (&r)[kGatherRows],
                                           int64_t rows)
{
  T v[kGatherRows];
  uint8_t ok[kGatherRows];
#pragma unroll
  for (int j = 0; j < kGatherRows; ++j) {
    v[j]  = r[j] >= 0 ? __ldg(src + r[j]) : T(0);
    ok[j] = r[j] >= 0 ? 1 : 0;
    if (valid != nullptr && r[j] >= 0) ok[j] = __ldg(valid + r[j]) != 0 ? 1 : 0;
  }
#pragma unroll
  for (int j = 0; j < kGatherRows; ++j) {
    if (i[j] >= rows) continue;
    dst[i[j]] = v[j];
    if (dst_valid) dst_valid[i[j]] = ok[j];
  }
}

__global__ void __launch_bounds__(256) gather_fixed_kernel(GatherSet g, const int32_t* map, int64_t rows)
{
  const int64_t per_iter = static_cast<int64_t>(blockDim.x) * kGatherRows;
  for (int64_t base = blockIdx.x * per_iter; base < rows; base += static_cast<int64_t>(gridDim.x) * per_iter) {
    int64_t i[kGatherRows];
    int32_t r[kGatherRows];
#pragma unroll
    for (int j = 0; j < kGatherRows; ++j) {
      i[j] = base + j * blockDim.x + threadIdx.x;
      r[j] = i[j] < rows ? __ldg(map + i[j]) : -1;
    }
    for (int c = 0; c < g.ncols; ++c) {
      switch (g.width[c]) {
        case 1:
          gather_one(static_cast<const uint8_t*>(g.src[c]), g.valid[c], static_cast<uint8_t*>(g.dst[c]),
                     g.dst_valid[c], i, r, rows);
          break;
        case 2:
          gather_one(static_cast<const uint16_t*>(g.src[c]), g.valid[c], static_cast<uint16_t*>(g.dst[c]),
                     g.dst_valid[c], i, r, rows);
          break;
        case 4:
          gather_one(static_cast<const uint32_t*>(g.src[c]), g.valid[c], static_cast<uint32_t*>(g.dst[c]),
                     g.dst_valid[c], i, r, rows);
          break;
        default:
          gather_one(static_cast<const unsigned long long*>(g.src[c]), g.valid[c],
                     static_cast<unsigned long long*>(g.dst[c]), g.dst_valid[c], i, r, rows);
          break;
      }
    }
  }
}

// dst[inv[r]] = src[r] for up to kGatherCols fixed-width columns: the source
// is read in order and every output row is written once.  Used where the
// output positions of consecutive rows fall into few runs (a partition by
// bucket: a tile's rows of one bucket land side by side), so the writes
// combine in L2 instead of the reads scattering.
template <typename T>
__device__ __forceinline__ void scatter_one(const T* src, const uint8_t* valid, T* dst, uint8_t* dst_valid,
                                            const int64_t (&i)[kGatherRows], const int32_t (&pos)[kGatherRows],
                                            int64_t rows)
{
  T v[kGatherRows];
  uint8_t ok[kGatherRows];
#pragma unroll
  for (int j = 0; j < kGatherRows; ++j) {
    v[j]  = i[j] < rows ? __ldg(src + i[j]) : T(0);
    ok[j] = (i[j] < rows && valid != nullptr) ? (__ldg(valid + i[j]) != 0 ? 1 : 0) : 1;
  }
#pragma unroll
  for (int j = 0; j < kGatherRows; ++j) {
    if (i[j] >= rows) continue;
    dst[pos[j]] = v[j];
    if (dst_valid) dst_valid[pos[j]] = ok[j];
  }
}

__global__ void __launch_bounds__(256) scatter_fixed_kernel(GatherSet g, const int32_t* inv, int64_t rows)
{
  const int64_t per_iter = static_cast<int64_t>(blockDim.x) * kGatherRows;
  for (int64_t base = blockIdx.x * per_iter; base < rows; base += static_cast<int64_t>(gridDim.x) * per_iter) {
    int64_t i[kGatherRows];
    int32_t pos[kGatherRows];
#pragma unroll
    for (int j = 0; j < kGatherRows; ++j) {
      i[j]   = base + j * blockDim.x + threadIdx.x;
      pos[j] = i[j] < rows ? __ldg(inv + i[j]) : 0;
    }
    for (int c = 0; c < g.ncols; ++c) {
      switch (g.width[c]) {
        case 1:
          scatter_one(static_cast<const uint8_t*>(g.src[c]), g.valid[c], static_cast<uint8_t*>(g.dst[c]),
                      g.dst_valid[c], i, pos, rows);
          break;
        case 2:
          scatter_one(static_cast<const uint16_t*>(g.src[c]), g.valid[c], static_cast<uint16_t*>(g.dst[c]),
                      g.dst_valid[c], i, pos, rows);
          break;
        case 4:
          scatter_one(static_cast<const uint32_t*>(g.src[c]), g.valid[c], static_cast<uint32_t*>(g.dst[c]),
                      g.dst_valid[c], i, pos, rows);
          break;
        default:
          scatter_one(static_cast<const unsigned long long*>(g.src[c]), g.valid[c],
                      static_cast<unsigned long long*>(g.dst[c]), g.dst_valid[c], i, pos, rows);
          break;
      }
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
  Buffer<int64_t> srcoff(a, rows);
  Buffer<int64_t> total(a, 1);
  launch("string_lengths", string_lengths_kernel, grid_for(ceil_div(rows, kLenRows), 256), 256, 0, s, src, map, rows,
         lens.get(), srcoff.get());
  LDF_CHECK_LAUNCH();
  exclusive_scan_i64(lens.get(), offs.get(), rows, total.get(), ctx);
  int64_t nchars = ctx.read_i64(total.get());
  dst.chars      = static_cast<char*>(a.allocate(static_cast<size_t>(nchars)));
  dst.num_chars  = nchars;
  dst.chars_base = 0;
  launch("string_copy", string_copy_kernel, grid_for(ceil_div(rows, kStrRows), kStrTile), kStrTile, 0, s, src,
         static_cast<const int64_t*>(srcoff.get()), rows,
         static_cast<const int64_t*>(offs.get()), nchars, static_cast<ldf_range*>(dst.data), dst.valid,
         reinterpret_cast<uint8_t*>(dst.chars));
  LDF_CHECK_LAUNCH();
}

void gather_fixed_columns(const OpContext& ctx, const DCol* src, const int32_t* map, int64_t rows,
                          ldf_column* const* dst, int ncols)
{
  if (rows == 0) return;
  for (int c0 = 0; c0 < ncols; c0 += kGatherCols) {
    GatherSet g{};
    g.ncols = ncols - c0 < kGatherCols ? ncols - c0 : kGatherCols;
    for (int k = 0; k < g.ncols; ++k) {
      const DCol& sc = src[c0 + k];
      LDF_REQUIRE(sc.width == 1 || sc.width == 2 || sc.width == 4 || sc.width == 8,
                  "gather: unsupported fixed width");
      g.width[k]     = sc.width;
      g.src[k]       = sc.data;
      g.valid[k]     = sc.valid;
      g.dst[k]       = dst[c0 + k]->data;
      g.dst_valid[k] = dst[c0 + k]->valid;
    }
    launch("gather_fixed", gather_fixed_kernel, grid_for(ceil_div(rows, kGatherRows), 256), 256, 0, ctx.stream(), g,
           map, rows);
  }
}

void scatter_fixed_columns(const OpContext& ctx, const DCol* src, const int32_t* inv, int64_t rows,
                           ldf_column* const* dst, int ncols)
{
  if (rows == 0) return;
  for (int c0 = 0; c0 < ncols; c0 += kGatherCols) {
    GatherSet g{};
    g.ncols = ncols - c0 < kGatherCols ? ncols - c0 : kGatherCols;
    for (int k = 0; k < g.ncols; ++k) {
      const DCol& sc = src[c0 + k];
      LDF_REQUIRE(sc.width == 1 || sc.width == 2 || sc.width == 4 || sc.width == 8,
                  "scatter: unsupported fixed width");
      g.width[k]     = sc.width;
      g.src[k]       = sc.data;
      g.valid[k]     = sc.valid;
      g.dst[k]       = dst[c0 + k]->data;
      g.dst_valid[k] = dst[c0 + k]->valid;
    }
    launch("scatter_fixed", scatter_fixed_kernel, grid_for(ceil_div(rows, kGatherRows), 256), 256, 0, ctx.stream(),
           g, inv, rows);
  }
}

void gather_fixed(const OpContext& ctx, const DCol& src, const int32_t* map, int64_t rows,
                  ldf_column& dst)
{
  ldf_column* d = &dst;
  gather_fixed_columns(ctx, &src, map, rows, &d, 1);
}

}  // namespace ldf
