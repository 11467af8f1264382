// Shared building blocks of the relational ops: key-column sets, output
// column specs, index compaction and the string gather.
#pragma once

#include "scan.cuh"

namespace ldf {

constexpr int kMaxKeys = 8;
constexpr int kMaxOut  = 16;

enum class KeyMode : int { K32 = 0, K64 = 1, GEN = 2 };

struct KeyCols {
  int n;
  DCol c[kMaxKeys];
};

// A set of output columns fed from one input table: dst[j][pos] = src[j][row].
// String columns are not copied here (their rows go through gather maps).
struct OutSpec {
  int n;
  int nullable_out[kMaxOut];
  DCol src[kMaxOut];
  OCol dst[kMaxOut];
};

KeyCols make_keys(const ldf_column* cols, int ncols, const int32_t* idx, int nkeys);

// Which fast key path a key set can use: one fixed-width column of <= 4 bytes
// -> K32, one 8-byte column -> K64, anything else (several columns, strings)
// -> GEN (64-bit row hash + column-wise equality).
KeyMode key_mode(const KeyCols& k);

// Seed of the row hash of a key set.
constexpr uint64_t kKeyHashSeed = 0x243f6a8885a308d3ull;

// Key bits / row hash for each mode.
template <KeyMode M>
__device__ __forceinline__ uint64_t key_bits(const KeyCols& k, int64_t r)
{
  if constexpr (M == KeyMode::GEN) {
    uint64_t h = kKeyHashSeed;
    for (int j = 0; j < k.n; ++j) h = hash_combine64(h, hash_value(k.c[j], r));
    return h;
  } else {
    return dbits(k.c[0], r);
  }
}

// True if any key column of row r is null.
__device__ __forceinline__ bool key_has_null(const KeyCols& k, int64_t r)
{
  for (int j = 0; j < k.n; ++j)
    if (!dvalid(k.c[j], r)) return true;
  return false;
}

__device__ __forceinline__ bool keys_equal(const KeyCols& a, int64_t ra, const KeyCols& b, int64_t rb)
{
  for (int j = 0; j < a.n; ++j)
    if (!values_equal(a.c[j], ra, b.c[j], rb)) return false;
  return true;
}

// Write one output row of an OutSpec from source row `src_row` (or nulls when
// src_row < 0).
__device__ __forceinline__ void write_out_row(const OutSpec& o, int64_t pos, int64_t src_row)
{
  for (int j = 0; j < o.n; ++j) {
    const OCol& d = o.dst[j];
    if (d.type == LDF_STRING) continue;
    if (src_row >= 0) {
      copy_fixed(d.data, pos, o.src[j].data, src_row, d.width);
      if (d.valid) d.valid[pos] = dvalid(o.src[j], src_row) ? 1 : 0;
    } else {
      zero_fixed(d.data, pos, d.width);
      if (d.valid) d.valid[pos] = 0;
    }
  }
}

// Input columns that live in host memory (pinned or pageable), copied to the
// device inside the op so that the copies overlap its kernels.  The columns
// named in `order` are copied in that order on the staging stream, one event
// after each; the op's stream waits on a column's event (`wait`) right before
// the first kernel that reads it.  `table` is the op's view of the input with
// device pointers.  Columns already on the device are used in place.  The
// host memory must stay valid until the op's stream has passed the end of
// the op.
class HostStaging {
 public:
  HostStaging(const OpContext& ctx, const ldf_column* table, int ncols, const std::vector<int>& order);
  ~HostStaging();
  HostStaging(const HostStaging&)            = delete;
  HostStaging& operator=(const HostStaging&) = delete;
  const ldf_column* table() const { return table_.data(); }
  void wait(int col) const;
  int64_t staged_bytes() const { return bytes_; }

 private:
  void stage_columns(const OpContext& ctx, const std::vector<int>& order);
  void release() noexcept;

  cudaStream_t s_;
  cudaStream_t cs_ = nullptr;  // staging stream, once a copy was issued
  std::vector<ldf_column> table_;
  std::vector<cudaEvent_t> ready_;
  std::vector<Buffer<uint8_t>> bufs_;
  int64_t bytes_ = 0;
};

// Allocate an output column of `rows` rows (fixed width or string ranges).
ldf_column alloc_out_column(const Allocator& a, int type, int64_t rows, bool nullable);
void free_out_column(const Allocator& a, ldf_column& c);

// Gather a string column: dst[i] = src[map[i]] (null when map[i] < 0 or the
// source row is null).  Allocates dst chars; dst ranges/valid must exist.
void gather_strings(const OpContext& ctx, const DCol& src, const int32_t* map, int64_t rows,
                    ldf_column& dst);

// Gather a fixed-width column by index map (map[i] < 0 -> null).
void gather_fixed(const OpContext& ctx, const DCol& src, const int32_t* map, int64_t rows,
                  ldf_column& dst);

// The same for several fixed-width columns through one map (one launch per
// eight columns).
void gather_fixed_columns(const OpContext& ctx, const DCol* src, const int32_t* map, int64_t rows,
                          ldf_column* const* dst, int ncols);

// dst[inv[r]] = src[r] for several fixed-width columns (inv: a permutation;
// one launch per eight columns).
void scatter_fixed_columns(const OpContext& ctx, const DCol* src, const int32_t* inv, int64_t rows,
                           ldf_column* const* dst, int ncols);

}  // namespace ldf
