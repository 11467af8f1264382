// Common device/host infrastructure of the B200 relational kernels:
// error handling, the allocator contract, device column views, key hashing.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstring>
#include <utility>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/ldf_b200.h"

namespace ldf {

// ---------------------------------------------------------------------------
// Errors.  Host code throws LdfError; the C-ABI layer turns it into a status
// code plus a thread-local message.
// ---------------------------------------------------------------------------
struct LdfError : std::runtime_error {
  int code;
  LdfError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

[[noreturn]] inline void fail(int code, const std::string& msg) { throw LdfError(code, msg); }

#define LDF_CUDA(call)                                                                    \
  do {                                                                                    \
    cudaError_t e__ = (call);                                                             \
    if (e__ != cudaSuccess) {                                                             \
      ::ldf::fail(LDF_ERR_CUDA, std::string("CUDA error ") + cudaGetErrorString(e__) +    \
                                  " at " + __FILE__ + ":" + std::to_string(__LINE__));    \
    }                                                                                     \
  } while (0)

#define LDF_CHECK_LAUNCH() LDF_CUDA(cudaGetLastError())

#define LDF_REQUIRE(cond, msg)                                                 \
  do {                                                                         \
    if (!(cond)) ::ldf::fail(LDF_ERR_INVALID_ARGUMENT, (msg));                 \
  } while (0)

// Number of SMs of the current device (148 on B200); grids are sized in
// multiples of it.
int num_sms();

// Non-blocking stream of the current device for host -> device staging copies
// (created on first use, one per device, kept until the process exits).
cudaStream_t staging_stream();

// ---------------------------------------------------------------------------
// Kernel launches.  Every kernel of the library goes through `launch`, which
// counts launches and, when profiling is on, brackets the launch with CUDA
// events on its own stream (per-kernel device time, read by the bench).
// ---------------------------------------------------------------------------
namespace prof {
void begin(const char* name, cudaStream_t s);
void end(const char* name, cudaStream_t s);
void count_launches(unsigned long long n);  // kernels launched by a graph replay
}  // namespace prof

template <typename... KArgs, typename... Args>
inline void launch(const char* name, void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem,
                   cudaStream_t s, Args&&... args)
{
  prof::begin(name, s);
  kernel<<<grid, block, smem, s>>>(std::forward<Args>(args)...);
  LDF_CHECK_LAUNCH();
  prof::end(name, s);
}

// ---------------------------------------------------------------------------
// Allocation.  All device memory (outputs and scratch) comes from the caller's
// allocator; with none, stream-ordered cudaMallocAsync.  Scratch buffers are
// RAII and released on the same stream, so no device-wide synchronisation.
// ---------------------------------------------------------------------------
// Device memory of one call.  allocate/deallocate go straight to the
// caller's allocator (outputs use them: the caller owns what they return).
// Scratch buffers (Buffer<T>) of at most kSmallScratch bytes are carved from
// kScratchChunk-byte chunks instead, which are handed back when the Allocator
// is destroyed at the end of the call: one allocator round trip per chunk
// rather than per buffer.
class Allocator {
 public:
  static constexpr size_t kSmallScratch = size_t(1) << 20;
  static constexpr size_t kScratchChunk = size_t(16) << 20;

  Allocator(const ldf_allocator* a, cudaStream_t s) : a_(a), s_(s) {}
  Allocator(const Allocator&)            = delete;
  Allocator& operator=(const Allocator&) = delete;
  ~Allocator();
  void* allocate(size_t nbytes) const;
  void deallocate(void* p, size_t nbytes) const;
  void* allocate_scratch(size_t nbytes) const;
  void deallocate_scratch(void* p, size_t nbytes) const;
  cudaStream_t stream() const { return s_; }

 private:
  const ldf_allocator* a_;
  cudaStream_t s_;
  mutable std::vector<void*> chunks_;
  mutable char* bump_  = nullptr;
  mutable size_t left_ = 0;
};

template <typename T>
class Buffer {
 public:
  Buffer() = default;
  Buffer(const Allocator& a, size_t n) : a_(&a), n_(n)
  {
    p_ = static_cast<T*>(a.allocate_scratch(bytes()));
  }
  Buffer(const Buffer&)            = delete;
  Buffer& operator=(const Buffer&) = delete;
  Buffer(Buffer&& o) noexcept { *this = std::move(o); }
  Buffer& operator=(Buffer&& o) noexcept
  {
    reset();
    a_ = o.a_;
    p_ = o.p_;
    n_ = o.n_;
    o.p_ = nullptr;
    o.n_ = 0;
    return *this;
  }
  ~Buffer() { reset(); }
  void reset()
  {
    if (p_ && a_) a_->deallocate_scratch(p_, bytes());
    p_ = nullptr;
    n_ = 0;
  }
  // Give up ownership (used for outputs that are handed back to the caller).
  T* release()
  {
    T* p = p_;
    p_   = nullptr;
    n_   = 0;
    return p;
  }
  T* get() const { return p_; }
  size_t size() const { return n_; }
  size_t bytes() const { return n_ == 0 ? 16 : n_ * sizeof(T); }

 private:
  const Allocator* a_ = nullptr;
  T* p_               = nullptr;
  size_t n_           = 0;
};

// ---------------------------------------------------------------------------
// Types.
// ---------------------------------------------------------------------------
inline int type_width(int t)
{
  switch (t) {
    case LDF_BOOL8:
    case LDF_INT8:
    case LDF_UINT8: return 1;
    case LDF_INT16:
    case LDF_UINT16: return 2;
    case LDF_INT32:
    case LDF_UINT32:
    case LDF_FLOAT32: return 4;
    case LDF_INT64:
    case LDF_UINT64:
    case LDF_FLOAT64:
    case LDF_TIMESTAMP_US: return 8;
    case LDF_STRING: return 16;  // one ldf_range per row
    default: fail(LDF_ERR_UNSUPPORTED, "unsupported column type id " + std::to_string(t));
  }
}
inline bool is_string(int t) { return t == LDF_STRING; }
inline bool is_float(int t) { return t == LDF_FLOAT32 || t == LDF_FLOAT64; }
inline bool is_signed_int(int t)
{
  return t == LDF_INT8 || t == LDF_INT16 || t == LDF_INT32 || t == LDF_INT64 ||
         t == LDF_TIMESTAMP_US;
}

// Device view of one input column (the legate layout, read directly: the
// bool-per-row null mask and the global Rect<1> string ranges are consumed
// as they are, no bitmask / offsets conversion pass).
struct DCol {
  const void* data;
  const uint8_t* valid;
  const char* chars;
  int64_t chars_base;
  int32_t type;
  int32_t width;
  int64_t num_chars;  // bytes of `chars` (strings)
};

inline DCol make_dcol(const ldf_column& c)
{
  DCol d;
  d.data       = c.data;
  d.valid      = c.valid;
  d.chars      = c.chars;
  d.chars_base = c.chars_base;
  d.type       = c.type;
  d.width      = type_width(c.type);
  d.num_chars  = c.type == LDF_STRING ? c.num_chars : 0;
  return d;
}

// Device view of one output column.
struct OCol {
  void* data;
  uint8_t* valid;
  int32_t type;
  int32_t width;
};

// ---------------------------------------------------------------------------
// Device helpers.
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool dvalid(const DCol& c, int64_t r)
{
  return c.valid == nullptr || __ldg(c.valid + r) != 0;
}

// Raw bits of a fixed-width value, zero-extended.  Hashing and equality of
// keys and distinct values use these bits, as Arrow's hash kernels do: 0.0 and
// -0.0 are different keys and a NaN equals only a NaN with the same bits.
__device__ __forceinline__ uint64_t dbits(const DCol& c, int64_t r)
{
  switch (c.width) {
    case 1: return __ldg(static_cast<const uint8_t*>(c.data) + r);
    case 2: return __ldg(static_cast<const uint16_t*>(c.data) + r);
    case 4: return __ldg(static_cast<const uint32_t*>(c.data) + r);
    default: return __ldg(reinterpret_cast<const unsigned long long*>(c.data) + r);
  }
}

// dvalid / dbits with an evict-first hint, for a column read once in row
// order: its lines leave L2 before the hash tables a pass probes.
__device__ __forceinline__ bool dvalid_stream(const DCol& c, int64_t r)
{
  return c.valid == nullptr || __ldcs(c.valid + r) != 0;
}
__device__ __forceinline__ uint64_t dbits_stream(const DCol& c, int64_t r)
{
  switch (c.width) {
    case 1: return __ldcs(static_cast<const uint8_t*>(c.data) + r);
    case 2: return __ldcs(static_cast<const uint16_t*>(c.data) + r);
    case 4: return __ldcs(static_cast<const uint32_t*>(c.data) + r);
    default: return __ldcs(reinterpret_cast<const unsigned long long*>(c.data) + r);
  }
}

__device__ __forceinline__ bool is_signed_int_dev(int t)
{
  return t == LDF_INT8 || t == LDF_INT16 || t == LDF_INT32 || t == LDF_INT64 ||
         t == LDF_TIMESTAMP_US;
}

// Sign-extended value of a signed integer column.
__device__ __forceinline__ int64_t signed_value(const DCol& c, int64_t r)
{
  switch (c.width) {
    case 1: return __ldg(static_cast<const signed char*>(c.data) + r);
    case 2: return __ldg(static_cast<const short*>(c.data) + r);
    case 4: return __ldg(static_cast<const int*>(c.data) + r);
    default: return __ldg(reinterpret_cast<const long long*>(c.data) + r);
  }
}

// MurmurHash3's 64-bit finaliser (public domain), used as the key mixer.
__device__ __host__ __forceinline__ uint64_t mix64(uint64_t x)
{
  x ^= x >> 33;
  x *= 0xff51afd7ed558ccdull;
  x ^= x >> 33;
  x *= 0xc4ceb9fe1a85ec53ull;
  x ^= x >> 33;
  return x;
}

__device__ __host__ __forceinline__ uint64_t hash_combine64(uint64_t seed, uint64_t h)
{
  return mix64(seed ^ (h + 0x9e3779b97f4a7c15ull + (seed << 6) + (seed >> 2)));
}

// Byte length of a string row (ranges are inclusive, so hi = lo - 1 is "").
__device__ __forceinline__ int64_t dstr_len(const DCol& c, int64_t r)
{
  const ldf_range* rg = static_cast<const ldf_range*>(c.data);
  return rg[r].hi - rg[r].lo + 1;
}
__device__ __forceinline__ const uint8_t* dstr_ptr(const DCol& c, int64_t r)
{
  const ldf_range* rg = static_cast<const ldf_range*>(c.data);
  return reinterpret_cast<const uint8_t*>(c.chars) + (rg[r].lo - c.chars_base);
}

// Hash of a byte string: 8-byte little-endian words folded through mix64.
// The same function is restated in the numpy oracle (hash partition parity).
__device__ __forceinline__ uint64_t hash_bytes(const uint8_t* p, int64_t n)
{
  uint64_t h = 0x27d4eb2f165667c5ull ^ (static_cast<uint64_t>(n) * 0x9e3779b97f4a7c15ull);
  int64_t i  = 0;
  for (; i + 8 <= n; i += 8) {
    uint64_t w = 0;
#pragma unroll
    for (int b = 0; b < 8; ++b) w |= static_cast<uint64_t>(p[i + b]) << (8 * b);
    h = mix64(h ^ w) + 0x165667b19e3779f9ull;
  }
  if (i < n) {
    uint64_t w = 0;
    for (int b = 0; i + b < n; ++b) w |= static_cast<uint64_t>(p[i + b]) << (8 * b);
    h = mix64(h ^ w) + 0x165667b19e3779f9ull;
  }
  return mix64(h);
}

__device__ __forceinline__ bool bytes_equal(const uint8_t* a, const uint8_t* b, int64_t n)
{
  for (int64_t i = 0; i < n; ++i)
    if (a[i] != b[i]) return false;
  return true;
}

// A string of at most 32 bytes as 4 little-endian words w[k] = bytes
// [8k, 8k + 8) (zero past the end), read with at most 5 aligned 8-byte loads
// that stay inside the column's chars buffer.  False (w untouched) when the
// string is longer or the loads would leave the buffer.
__device__ __forceinline__ bool str_words(const DCol& c, const uint8_t* p, int64_t n, uint64_t w[4])
{
  if (n > 32) return false;
  const uintptr_t a  = reinterpret_cast<uintptr_t>(p);
  const uintptr_t a0 = a & ~uintptr_t(7);
  const int sh       = static_cast<int>(a - a0);
  const int nw       = static_cast<int>((sh + n + 7) >> 3);
  const uintptr_t cb = reinterpret_cast<uintptr_t>(c.chars);
  if (n > 0 && (a0 < cb || a0 + 8 * static_cast<uintptr_t>(nw) > cb + static_cast<uintptr_t>(c.num_chars)))
    return false;
  uint64_t raw[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) raw[k] = k < nw ? __ldg(reinterpret_cast<const unsigned long long*>(a0) + k) : 0ull;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    uint64_t v      = sh ? ((raw[k] >> (8 * sh)) | (raw[k + 1] << (64 - 8 * sh))) : raw[k];
    const int64_t m = n - 8 * k;  // bytes of the string in word k
    if (m <= 0) v = 0;
    else if (m < 8) v &= (1ull << (8 * m)) - 1;
    w[k] = v;
  }
  return true;
}

// hash_bytes of a string given as str_words.
__device__ __forceinline__ uint64_t hash_words(const uint64_t w[4], int64_t n)
{
  uint64_t h = 0x27d4eb2f165667c5ull ^ (static_cast<uint64_t>(n) * 0x9e3779b97f4a7c15ull);
#pragma unroll
  for (int k = 0; k < 4; ++k)
    if (8 * k < n) h = mix64(h ^ w[k]) + 0x165667b19e3779f9ull;
  return mix64(h);
}

// Hash of a null value.
constexpr uint64_t kNullValueHash = 0x5bd1e9955bd1e995ull;

// Hash of one column value of a row, null-aware.  A null hashes to a fixed
// constant.
__device__ __forceinline__ uint64_t hash_value(const DCol& c, int64_t r)
{
  if (!dvalid(c, r)) return kNullValueHash;
  if (c.type == LDF_STRING) {
    const uint8_t* p = dstr_ptr(c, r);
    const int64_t n  = dstr_len(c, r);
    uint64_t w[4];
    if (str_words(c, p, n, w)) return hash_words(w, n);
    return hash_bytes(p, n);
  }
  return mix64(dbits(c, r) + 0x9e3779b97f4a7c15ull * static_cast<uint64_t>(c.width));
}

// Value equality between row ra of column a and row rb of column b (same
// type), nulls equal to nulls.
__device__ __forceinline__ bool values_equal(const DCol& a, int64_t ra, const DCol& b, int64_t rb)
{
  bool va = dvalid(a, ra), vb = dvalid(b, rb);
  if (va != vb) return false;
  if (!va) return true;
  if (a.type == LDF_STRING) {
    int64_t la = dstr_len(a, ra), lb = dstr_len(b, rb);
    if (la != lb) return false;
    const uint8_t* pa = dstr_ptr(a, ra);
    const uint8_t* pb = dstr_ptr(b, rb);
    uint64_t wa[4], wb[4];
    if (str_words(a, pa, la, wa) && str_words(b, pb, lb, wb))
      return wa[0] == wb[0] && wa[1] == wb[1] && wa[2] == wb[2] && wa[3] == wb[3];
    return bytes_equal(pa, pb, la);
  }
  return dbits(a, ra) == dbits(b, rb);
}

// Lemire's multiply-shift range reduction: hash -> [0, n).
__device__ __forceinline__ uint64_t fastrange(uint64_t h, uint64_t n)
{
  return __umul64hi(h, n);
}

// Copy one fixed-width value.
__device__ __forceinline__ void copy_fixed(void* dst, int64_t di, const void* src, int64_t si, int w)
{
  switch (w) {
    case 1: static_cast<uint8_t*>(dst)[di] = static_cast<const uint8_t*>(src)[si]; break;
    case 2: static_cast<uint16_t*>(dst)[di] = static_cast<const uint16_t*>(src)[si]; break;
    case 4: static_cast<uint32_t*>(dst)[di] = static_cast<const uint32_t*>(src)[si]; break;
    case 8: static_cast<uint64_t*>(dst)[di] = static_cast<const uint64_t*>(src)[si]; break;
    default: static_cast<ldf_range*>(dst)[di] = static_cast<const ldf_range*>(src)[si]; break;
  }
}
__device__ __forceinline__ void zero_fixed(void* dst, int64_t di, int w)
{
  switch (w) {
    case 1: static_cast<uint8_t*>(dst)[di] = 0; break;
    case 2: static_cast<uint16_t*>(dst)[di] = 0; break;
    case 4: static_cast<uint32_t*>(dst)[di] = 0; break;
    case 8: static_cast<uint64_t*>(dst)[di] = 0; break;
    default: static_cast<ldf_range*>(dst)[di] = ldf_range{0, -1}; break;
  }
}

// The 16-byte-aligned span inside bytes [lo, hi) of the buffer at address
// b0: its start in *addr, its size as the result (0: nothing to prefetch).
__host__ __device__ __forceinline__ uint32_t prefetch_span(uint64_t b0, int64_t lo, int64_t hi, uint64_t* addr)
{
  const uint64_t a = (b0 + static_cast<uint64_t>(lo) + 15) & ~15ull;
  const uint64_t e = (b0 + static_cast<uint64_t>(hi)) & ~15ull;
  *addr            = a;
  if (hi <= lo || e <= a || e - a > 0xfffffff0ull) return 0;
  return static_cast<uint32_t>(e - a);
}

// Prefetch bytes [lo, hi) of a buffer into L2 with one bulk-copy-engine
// instruction (cp.async.bulk.prefetch.L2, no registers held while it is in
// flight).  The range is shrunk inward to 16-byte bounds, as the instruction
// requires, so no byte outside [lo, hi) is touched; a range under 16 bytes is
// skipped.  A hint only: the data is still loaded by the caller.
__device__ __forceinline__ void l2_prefetch_bulk(const void* base, int64_t lo, int64_t hi)
{
  uint64_t a;
  const uint32_t bytes = prefetch_span(reinterpret_cast<uint64_t>(base), lo, hi, &a);
  if (bytes == 0) return;
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a), "r"(bytes) : "memory");
}

// Bounded spin budget for device-side waits (look-back).  A wait that runs
// out sets the call's error word and returns; it never traps or hangs.
constexpr uint32_t kSpinLimit = 1u << 22;

inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

}  // namespace ldf
