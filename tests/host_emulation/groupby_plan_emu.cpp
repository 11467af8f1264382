// Host emulation of the partitioned groupby plan (csrc/groupby.cu): the
// plan's device code compiled as host C++, one thread per block, blocks run
// one after another over host memory, so AddressSanitizer checks every access
// and the aggregates are compared with a direct per-key computation.  The
// test that builds it (tests/test_groupby_plan_emulated.py) extracts the
// plan's section from the CUDA source; this file supplies the CUDA built-ins
// and the library pieces the section uses.
#include <stdint.h>
#include <string.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string>
#include <vector>
#include <algorithm>
#include <stdexcept>
#include <map>
#include <cstring>
#include "ldf_b200.h"

#define __global__
#define __device__
#define __host__
#define __forceinline__ inline
#define __launch_bounds__(...)
#define __align__(x)
typedef void* cudaStream_t;
struct dim3 { unsigned x, y, z; dim3(unsigned a = 1, unsigned b = 1, unsigned c = 1) : x(a), y(b), z(c) {} };
static dim3 threadIdx(0), blockIdx(0), blockDim(1), gridDim(1);
static unsigned char* emu_smem = nullptr;
struct uint4 { unsigned x, y, z, w; };
static inline uint4 make_uint4(unsigned a, unsigned b, unsigned c, unsigned d) { return uint4{a, b, c, d}; }
struct ulonglong2 { unsigned long long x, y; };
static inline void __syncthreads() {}
static inline void __threadfence() {}
static inline void __threadfence_block() {}
static inline void __nanosleep(unsigned) {}
template <typename T> static inline T __ldg(const T* p) { return *p; }
static inline int __popc(unsigned x) { return __builtin_popcount(x); }
static inline int __popcll(unsigned long long x) { return __builtin_popcountll(x); }
static inline int __ffs(int x) { return __builtin_ffs(x); }
static inline int __clzll(long long x) { return x == 0 ? 64 : __builtin_clzll((unsigned long long)x); }
static inline unsigned __activemask() { return 1u; }
static inline unsigned __match_any_sync(unsigned, unsigned long long) { return 1u; }
template <typename T> static inline T __shfl_xor_sync(unsigned, T, int) { return T(0); }
static inline long long __double_as_longlong(double d) { long long x; memcpy(&x, &d, 8); return x; }
static inline double __longlong_as_double(long long x) { double d; memcpy(&d, &x, 8); return d; }
static inline float __uint_as_float(unsigned x) { float f; memcpy(&f, &x, 4); return f; }
static inline double __ull2double_rn(unsigned long long x) { return (double)x; }
static inline unsigned long long __umul64hi(unsigned long long a, unsigned long long b) { return (unsigned long long)(((unsigned __int128)a * b) >> 64); }
template <typename T> static inline T atomicAdd(T* p, T v) { T o = *p; *p = o + v; return o; }
static inline unsigned long long atomicAdd(unsigned long long* p, unsigned long long v) { auto o = *p; *p = o + v; return o; }
static inline unsigned atomicAdd(unsigned* p, unsigned v) { auto o = *p; *p = o + v; return o; }
template <typename T, typename U> static inline T atomicMax(T* p, U vv) { T v = (T)vv; T o = *p; if (v > o) *p = v; return o; }
template <typename T> static inline T atomicMin(T* p, T v) { T o = *p; if (v < o) *p = v; return o; }
template <typename T, typename U, typename V> static inline T atomicCAS(T* p, U c, V v) { T o = *p; if (o == (T)c) *p = (T)v; return o; }
template <typename T, typename U> static inline T atomicExch(T* p, U v) { T o = *p; *p = (T)v; return o; }
template <typename T> static inline T min(T a, T b) { return a < b ? a : b; }
template <typename T> static inline T max(T a, T b) { return a > b ? a : b; }

namespace ldf {
constexpr uint32_t kSpinLimit = 1u << 22;
struct LdfError : std::runtime_error { int code; LdfError(int c, const std::string& m) : std::runtime_error(m), code(c) {} };
[[noreturn]] inline void fail(int code, const std::string& msg) { throw LdfError(code, msg); }
#define LDF_CUDA(call) do { (void)(call); } while (0)
#define LDF_REQUIRE(c, m) do { if (!(c)) ::ldf::fail(LDF_ERR_INVALID_ARGUMENT, m); } while (0)
int num_sms() { return 4; }
inline int type_width(int t) {
  switch (t) { case LDF_BOOL8: case LDF_INT8: case LDF_UINT8: return 1; case LDF_INT16: case LDF_UINT16: return 2;
    case LDF_INT32: case LDF_UINT32: case LDF_FLOAT32: return 4; case LDF_STRING: return 16; default: return 8; }
}
inline bool is_float(int t) { return t == LDF_FLOAT32 || t == LDF_FLOAT64; }
inline bool is_signed_int(int t) { return t == LDF_INT8 || t == LDF_INT16 || t == LDF_INT32 || t == LDF_INT64 || t == LDF_TIMESTAMP_US; }
inline bool is_signed_int_dev(int t) { return is_signed_int(t); }
struct DCol { const void* data; const uint8_t* valid; const char* chars; int64_t chars_base; int32_t type; int32_t width; int64_t num_chars; };
inline DCol make_dcol(const ldf_column& c) { DCol d{c.data, c.valid, c.chars, c.chars_base, c.type, type_width(c.type), 0}; return d; }
struct OCol { void* data; uint8_t* valid; int32_t type; int32_t width; };
inline bool dvalid(const DCol& c, int64_t r) { return c.valid == nullptr || c.valid[r] != 0; }
inline uint64_t mix64(uint64_t x) { x ^= x >> 33; x *= 0xff51afd7ed558ccdull; x ^= x >> 33; x *= 0xc4ceb9fe1a85ec53ull; x ^= x >> 33; return x; }
inline uint64_t fastrange(uint64_t h, uint64_t n) { return __umul64hi(h, n); }
template <typename T> static inline T warp_reduce_sum(T v) { return v; }
inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }
constexpr int kMaxAggs = 32;
constexpr int kMaxProbe = 1024;
constexpr uint64_t kEmpty = ~0ull;
constexpr int kRows = 4;
enum : uint32_t { ST_SUM = 1, ST_MIN = 2, ST_MAX = 4, ST_NDIST = 8 };
static std::map<void*, size_t> g_live;
struct Allocator {
  void* allocate(size_t n) const { void* p = malloc(n ? n : 16); g_live[p] = n; return p; }
  void deallocate(void* p, size_t) const { g_live.erase(p); free(p); }
};
template <typename T> struct Buffer {
  const Allocator* a = nullptr; T* p = nullptr; size_t n = 0;
  Buffer() = default;
  Buffer(const Allocator& al, size_t cnt) : a(&al), n(cnt) { p = (T*)a->allocate(sizeof(T) * std::max<size_t>(cnt, 1)); }
  Buffer(const Buffer&) = delete;
  Buffer& operator=(Buffer&& o) { if (p) a->deallocate(p, 0); a = o.a; p = o.p; n = o.n; o.p = nullptr; return *this; }
  ~Buffer() { if (p) a->deallocate(p, 0); }
  T* get() const { return p; }
};
struct OpContext {
  Allocator al; int e = 0;
  const Allocator& alloc() const { return al; }
  cudaStream_t stream() const { return nullptr; }
  int* err() const { return const_cast<int*>(&e); }
  void finish() const { if (e) fail(LDF_ERR_TIMEOUT, "wait expired"); }
};
struct HostStaging { void wait(int) const {} };
ldf_column alloc_out_column(const Allocator& a, int type, int64_t rows, bool nullable) {
  ldf_column c{}; c.type = type; c.nullable = nullable; c.size = rows;
  c.data = a.allocate((size_t)rows * type_width(type)); c.valid = nullable ? (uint8_t*)a.allocate(rows) : nullptr; return c;
}
void free_out_column(const Allocator& a, ldf_column& c) { if (c.data) a.deallocate(c.data, 0); if (c.valid) a.deallocate(c.valid, 0); c.data = nullptr; c.valid = nullptr; }
struct ColPlan { DCol col; uint32_t states; int nullable; int fixed; };
struct GbPlan { int64_t n; int ncols; ColPlan c[8]; };
enum cudaMemcpyKind { cudaMemcpyHostToDevice, cudaMemcpyDeviceToHost, cudaMemcpyDeviceToDevice };
static int cudaMemsetAsync(void* p, int v, size_t n, cudaStream_t) { memset(p, v, n); return 0; }
static int cudaMemcpyAsync(void* d, const void* s, size_t n, cudaMemcpyKind, cudaStream_t) { memcpy(d, s, n); return 0; }
enum { cudaFuncAttributeMaxDynamicSharedMemorySize };
template <typename K> static int cudaFuncSetAttribute(K, int, int) { return 0; }
template <typename K> static int cudaOccupancyMaxActiveBlocksPerMultiprocessor(int* o, K, int, size_t) { *o = 1; return 0; }
static unsigned gs_blocks(int64_t n, int) { return (unsigned)std::max<int64_t>(1, std::min<int64_t>(n, 8)); }
template <typename... KArgs, typename... Args>
static void launch(const char*, void (*kernel)(KArgs...), dim3 grid, dim3, size_t smem, cudaStream_t, Args&&... args)
{
  std::vector<unsigned char> sm(smem + 64, 0xcd);
  gridDim = dim3(grid.x);
  blockDim = dim3(1);
  threadIdx = dim3(0);
  for (unsigned b = 0; b < grid.x; ++b) {
    blockIdx = dim3(b);
    std::vector<unsigned char> s(smem ? smem : 1, 0xcd);
    emu_smem = s.data();
    kernel(args...);
  }
}
template <int W>
void value_range_kernel(DCol col, int64_t n, uint32_t flip, unsigned int* out)
{
  if (blockIdx.x) return;
  for (int64_t r = 0; r < n; ++r) {
    if (!dvalid(col, r)) continue;
    uint32_t x = (W == 1 ? ((const uint8_t*)col.data)[r] : W == 2 ? ((const uint16_t*)col.data)[r] : ((const uint32_t*)col.data)[r]) ^ flip;
    out[0] = std::min(out[0], x); out[1] = std::max(out[1], x);
  }
}
inline void red_add(unsigned long long* p, uint64_t v) { *p += v; }
inline void red_max(unsigned long long* p, uint64_t v) { if (v > *p) *p = v; }
inline void red_or32(uint32_t* p, uint32_t v) { *p |= v; }
constexpr int kSumChunks = 6;
#include "section.inc"
}  // namespace ldf

using namespace ldf;

int main(int argc, char** argv)
{
  setenv("LDF_B200_GB_PART", "1", 1);
  setenv("LDF_B200_GB_PART_MIN_ROWS", "0", 1);
  const int64_t n = argc > 1 ? atoll(argv[1]) : 600000;
  const int64_t ng = argc > 2 ? atoll(argv[2]) : 50000;
  // Zipf(1.1)-like keys via inverse power
  std::vector<int64_t> k(n); std::vector<double> v(n); std::vector<int32_t> iv(n);
  std::vector<uint8_t> kv(n), vv(n), iv_ok(n);
  uint64_t s = 12345;
  auto rnd = [&]() { s = s * 6364136223846793005ull + 1442695040888963407ull; return (s >> 11) * (1.0 / 9007199254740992.0); };
  for (int64_t r = 0; r < n; ++r) {
    double u = rnd();
    int64_t rank = (int64_t)std::min<double>(ng - 1, floor(pow(1.0 - u, -1.0 / 0.1)) - 1);
    k[r] = (rank * 2654435761ll) % 1000003;
    kv[r] = rnd() >= 0.01; v[r] = rnd() * 2 - 1; vv[r] = rnd() >= 0.1; iv[r] = (int32_t)(rnd() * 1500) - 500; iv_ok[r] = rnd() >= 0.05;
  }
  ldf_column t[3]{};
  t[0].type = LDF_INT64; t[0].size = n; t[0].data = k.data(); t[0].valid = kv.data(); t[0].nullable = 1;
  t[1].type = LDF_FLOAT64; t[1].size = n; t[1].data = v.data(); t[1].valid = vv.data(); t[1].nullable = 1;
  t[2].type = LDF_INT32; t[2].size = n; t[2].data = iv.data(); t[2].valid = iv_ok.data(); t[2].nullable = 1;
  int32_t keys[1] = {0};
  // aggs: v sum, v mean, v count, count_all, v min, v max, i min, i max, i nunique, i sum, i mean, i nunique(all)
  std::vector<ldf_aggregation> aggs = {
    {1, LDF_AGG_SUM, 0, LDF_FLOAT64}, {1, LDF_AGG_MEAN, 0, LDF_FLOAT64}, {1, LDF_AGG_COUNT, 0, LDF_INT64},
    {-1, LDF_AGG_COUNT_ALL, 0, LDF_INT64}, {1, LDF_AGG_MIN, 0, LDF_FLOAT64}, {1, LDF_AGG_MAX, 0, LDF_FLOAT64},
    {2, LDF_AGG_MIN, 0, LDF_INT32}, {2, LDF_AGG_MAX, 0, LDF_INT32}, {2, LDF_AGG_COUNT_DISTINCT, 0, LDF_INT64},
    {2, LDF_AGG_SUM, 0, LDF_INT64}, {2, LDF_AGG_MEAN, 0, LDF_FLOAT64}, {2, LDF_AGG_COUNT_DISTINCT, 2, LDF_INT64}};
  GbPlan p{}; p.n = n;
  std::vector<int> agg_col(aggs.size(), -1), col_of_plan;
  for (size_t a = 0; a < aggs.size(); ++a) {
    if (aggs[a].kind == LDF_AGG_COUNT_ALL) continue;
    int ci = -1;
    for (size_t q = 0; q < col_of_plan.size(); ++q) if (col_of_plan[q] == aggs[a].in_col) ci = q;
    if (ci < 0) { ci = p.ncols++; col_of_plan.push_back(aggs[a].in_col); p.c[ci].col = make_dcol(t[aggs[a].in_col]);
      p.c[ci].nullable = 1; p.c[ci].fixed = is_float(t[aggs[a].in_col].type); }
    agg_col[a] = ci;
    switch (aggs[a].kind) { case LDF_AGG_SUM: case LDF_AGG_MEAN: p.c[ci].states |= ST_SUM; break;
      case LDF_AGG_MIN: p.c[ci].states |= ST_MIN; break; case LDF_AGG_MAX: p.c[ci].states |= ST_MAX; break;
      case LDF_AGG_COUNT_DISTINCT: p.c[ci].states |= ST_NDIST; break; default: break; }
  }
  OpContext ctx; HostStaging hs;
  std::vector<ldf_column> out(1 + aggs.size());
  bool ok = try_partitioned(ctx, p, t, keys, 1, aggs.data(), (int)aggs.size(), agg_col, out.data(), hs, col_of_plan);
  printf("partitioned=%d groups=%lld\n", ok, (long long)out[0].size);
  // reference counts per key
  std::map<int64_t, int64_t> cnt; int64_t nulls = 0;
  for (int64_t r = 0; r < n; ++r) { if (kv[r]) cnt[k[r]]++; else nulls++; }
  int64_t G = out[0].size, bad = 0;
  const int64_t* ok_keys = (const int64_t*)out[0].data; const int64_t* c_all = (const int64_t*)out[4].data;
  for (int64_t g = 0; g < G; ++g) {
    bool null = out[0].valid && !out[0].valid[g];
    int64_t want = null ? nulls : (cnt.count(ok_keys[g]) ? cnt[ok_keys[g]] : -1);
    if (want != c_all[g]) ++bad;
  }
  printf("expected groups %zu, count mismatches %lld\n", cnt.size() + (nulls > 0), (long long)bad);
  // full reference per key (null key = INT64_MIN sentinel)
  struct Ref { int64_t n = 0, cv = 0, ci = 0; long double sv = 0; double vmin = 1e300, vmax = -1e300; int64_t isum = 0;
               int imin = INT32_MAX, imax = INT32_MIN; std::vector<int> vals; };
  std::map<int64_t, Ref> ref;
  for (int64_t r = 0; r < n; ++r) {
    Ref& x = ref[kv[r] ? k[r] : INT64_MIN];
    x.n++;
    if (vv[r]) { x.cv++; x.sv += v[r]; x.vmin = std::min(x.vmin, v[r]); x.vmax = std::max(x.vmax, v[r]); }
    if (iv_ok[r]) { x.ci++; x.isum += iv[r]; x.imin = std::min(x.imin, iv[r]); x.imax = std::max(x.imax, iv[r]); x.vals.push_back(iv[r]); }
  }
  int64_t bad2 = 0;
  for (int64_t g = 0; g < G; ++g) {
    bool null = out[0].valid && !out[0].valid[g];
    Ref& x = ref[null ? INT64_MIN : ok_keys[g]];
    std::sort(x.vals.begin(), x.vals.end());
    int64_t nd = std::unique(x.vals.begin(), x.vals.end()) - x.vals.begin();
    x.vals.resize(nd);
    auto D = [&](int j) { return ((const double*)out[j].data)[g]; };
    auto I64 = [&](int j) { return ((const int64_t*)out[j].data)[g]; };
    auto I32 = [&](int j) { return ((const int32_t*)out[j].data)[g]; };
    auto V = [&](int j) { return out[j].valid ? out[j].valid[g] != 0 : true; };
    bool ok = true;
    ok &= V(1) == (x.cv > 0) && (x.cv == 0 || fabs(D(1) - (double)x.sv) <= 1e-9 * (fabsl(x.sv) + 1));
    ok &= V(2) == (x.cv > 0) && (x.cv == 0 || fabs(D(2) - (double)(x.sv / x.cv)) <= 1e-9);
    ok &= I64(3) == x.cv && I64(4) == x.n;
    ok &= x.cv == 0 || (D(5) == x.vmin && D(6) == x.vmax);
    ok &= x.ci == 0 || (I32(7) == x.imin && I32(8) == x.imax);
    ok &= I64(9) == nd;
    ok &= x.ci == 0 || I64(10) == x.isum;
    ok &= x.ci == 0 || fabs(D(11) - (double)x.isum / x.ci) <= 1e-9;
    ok &= I64(12) == nd + (x.n > x.ci ? 1 : 0);
    if (!ok && bad2 < 5) printf("group %lld (key %lld null %d) mismatch: n %lld/%lld cv %lld/%lld nd %lld/%lld\n", (long long)g, (long long)ok_keys[g], null, (long long)I64(4), (long long)x.n, (long long)I64(3), (long long)x.cv, (long long)I64(9), (long long)nd);
    bad2 += !ok;
  }
  printf("aggregate mismatches %lld of %lld groups\n", (long long)bad2, (long long)G);
  return 0;
}
