// Hash groupby aggregation: SUM, MIN, MAX, COUNT (valid / all / null),
// COUNT_ALL, MEAN, COUNT_DISTINCT (NUNIQUE).
//
// Reference semantics: Acero `aggregate` with hash_<kind> kernels
// (cpp/src/groupby_aggregation.cpp:41-94) and the cudf path
// (cpp/src/groupby_aggregation.cu:90-167) it must agree with:
//  * null keys form a group (cudf::null_policy::INCLUDE, .cu:143);
//  * SUM / MIN / MAX / MEAN skip nulls and are null for a group with no valid
//    value; COUNT counts valid values by default, CountOptions(mode) selects
//    all / only-null (.cu:33-44); COUNT_ALL counts rows; COUNT_DISTINCT counts
//    distinct valid values, plus one for null under mode "all".
//  * output types are the Arrow hash_<kind> result types (.cpp:100-132).
//
// Device plan:
//  1. estimate #groups (and #distinct (group, value) pairs) from a strided
//     sample with the GEE estimator  D = sqrt(N/n) f1 + sum_{j>=2} f_j; tables
//     are sized 3x the estimate (load <= 1/3); a probe sequence longer than
//     kMaxProbe flags overflow and the call re-runs with 4x the capacity.
//  2. one fused pass over the rows (persistent grid, 1 row per thread per
//     step, coalesced column reads):
//       global find-or-insert of the key -> group slot (L1/L2-resident for
//       heavy hitters, read-mostly);
//       per-CTA shared-memory table keyed by group slot absorbs the updates of
//       the groups a CTA sees (heavy hitters), so hot groups cost shared-memory
//       atomics and one flush per CTA instead of global same-address atomics;
//       float sums accumulate exactly in 192-bit two's-complement fixed point
//       (LSB 2^-96): integer adds are associative, so the result is
//       independent of thread order and bit-identical alone or in a batch;
//       NUNIQUE inserts (group slot, value) into a pair set and counts
//       first insertions.
//  3. compact occupied slots (look-back), 4. finalize each group into the
//     output columns (fixed point -> correctly rounded double).
#include "table_ops.cuh"

#include <cmath>

namespace ldf {
namespace {

constexpr int kMaxAggCols = 8;
constexpr int kMaxAggs    = 32;
constexpr int kMaxProbe   = 512;
constexpr uint64_t kEmpty = ~0ull;
// Empty marker of the 8-byte key table; a key equal to it lives in the extra
// slot `cap` (and a null single key in slot cap + 1).
constexpr uint64_t kSentinel64 = 0x7ff4dead7ff4beefull;
constexpr uint32_t kEmpty32    = 0xffffffffu;
constexpr int kGbThreads       = 256;

enum : uint32_t { ST_SUM = 1, ST_MIN = 2, ST_MAX = 4, ST_NDIST = 8 };
enum : uint32_t { SP_NAN = 1, SP_PINF = 2, SP_NINF = 4 };

struct ColPlan {
  DCol col;
  uint32_t states;
  int fixed;  // float sum in fixed point (3 limbs), else 1 limb integer sum
  int limbs;
  unsigned long long* vcount;
  unsigned long long* sum;  // [slot * limbs + l]
  double* fb;               // float values outside the fixed-point range
  unsigned int* special;    // NaN / +inf / -inf seen
  unsigned long long* mn;   // ~ordered(x), max-combined
  unsigned long long* mx;   // ordered(x), max-combined
  unsigned long long* ndist;
  // pair set for COUNT_DISTINCT
  unsigned long long* pairs;
  uint64_t pair_cap;
  int pair_packed;  // (slot << 32 | value32) keys when the value fits 32 bits
  // shared-memory offsets (bytes)
  int s_vcount, s_sum, s_mn, s_mx, s_ndist;
};

struct GbPlan {
  KeyCols k;
  int64_t n;
  void* slots;  // uint64_t[cap]
  uint64_t cap;
  int* overflow;
  unsigned long long* count_all;
  int ncols;
  ColPlan c[kMaxAggCols];
  int smem_slots;  // power of two
  int s_keys, s_count;
  int smem_bytes;
};

// ---- ordered encodings (min/max) ----------------------------------------
__device__ __forceinline__ uint64_t ordered_bits(const DCol& c, int64_t r)
{
  switch (c.type) {
    case LDF_INT8: return static_cast<uint64_t>(static_cast<int64_t>(static_cast<const int8_t*>(c.data)[r])) ^ (1ull << 63);
    case LDF_INT16: return static_cast<uint64_t>(static_cast<int64_t>(static_cast<const int16_t*>(c.data)[r])) ^ (1ull << 63);
    case LDF_INT32: return static_cast<uint64_t>(static_cast<int64_t>(static_cast<const int32_t*>(c.data)[r])) ^ (1ull << 63);
    case LDF_INT64:
    case LDF_TIMESTAMP_US: return static_cast<uint64_t>(static_cast<const int64_t*>(c.data)[r]) ^ (1ull << 63);
    case LDF_FLOAT32: {
      uint32_t b = static_cast<const uint32_t*>(c.data)[r];
      b          = (b & 0x80000000u) ? ~b : (b | 0x80000000u);
      return b;
    }
    case LDF_FLOAT64: {
      uint64_t b = static_cast<const uint64_t*>(c.data)[r];
      return (b & (1ull << 63)) ? ~b : (b | (1ull << 63));
    }
    default: return dbits(c, r);  // unsigned, bool
  }
}

// ---- 192-bit fixed point ------------------------------------------------
// x (finite double) -> m << s with LSB 2^-96; exact for 2^-44 <= |x| < 2^95.
__device__ __forceinline__ bool to_fixed192(double x, uint64_t& a0, uint64_t& a1, uint64_t& a2)
{
  uint64_t b = __double_as_longlong(x);
  int e      = static_cast<int>((b >> 52) & 0x7ff);
  if (e == 0 && (b << 1) == 0) {
    a0 = a1 = a2 = 0;
    return true;
  }
  int E = e - 1023;
  if (e == 0 || E < -44 || E >= 95) return false;
  uint64_t m = (b & ((1ull << 52) - 1)) | (1ull << 52);
  int s      = E + 44;  // 0 .. 138
  if (s < 64) {
    a0 = m << s;
    a1 = s == 0 ? 0 : (m >> (64 - s));
    a2 = 0;
  } else if (s < 128) {
    int t = s - 64;
    a0    = 0;
    a1    = m << t;
    a2    = t == 0 ? 0 : (m >> (64 - t));
  } else {
    a0 = 0;
    a1 = 0;
    a2 = m << (s - 128);
  }
  if (b >> 63) {  // two's complement negate
    a0 = ~a0;
    a1 = ~a1;
    a2 = ~a2;
    a0 += 1;
    if (a0 == 0) {
      a1 += 1;
      if (a1 == 0) a2 += 1;
    }
  }
  return true;
}

// Exact 192-bit add with atomics on three 64-bit limbs (global or shared):
// each limb add detects its own carry-out, so the total is exact mod 2^192
// whatever the interleaving.
__device__ __forceinline__ void atomic_add192(unsigned long long* p, uint64_t a0, uint64_t a1, uint64_t a2)
{
  unsigned long long o0 = atomicAdd(&p[0], static_cast<unsigned long long>(a0));
  uint64_t c0           = (o0 + a0 < o0) ? 1 : 0;
  uint64_t t1           = a1 + c0;
  uint64_t c1           = (t1 < a1) ? 1 : 0;
  if (t1 != 0) {
    unsigned long long o1 = atomicAdd(&p[1], static_cast<unsigned long long>(t1));
    c1 += (o1 + t1 < o1) ? 1 : 0;
  }
  uint64_t t2 = a2 + c1;
  if (t2 != 0) atomicAdd(&p[2], static_cast<unsigned long long>(t2));
}

__device__ __forceinline__ double fixed192_to_double(uint64_t l0, uint64_t l1, uint64_t l2)
{
  bool neg = static_cast<int64_t>(l2) < 0;
  if (neg) {
    l0 = ~l0;
    l1 = ~l1;
    l2 = ~l2;
    l0 += 1;
    if (l0 == 0) {
      l1 += 1;
      if (l1 == 0) l2 += 1;
    }
  }
  int msb;
  if (l2) msb = 128 + 63 - __clzll(l2);
  else if (l1) msb = 64 + 63 - __clzll(l1);
  else if (l0) msb = 63 - __clzll(l0);
  else return 0.0;
  // top 64 bits [msb-63, msb] plus a sticky bit for everything below
  uint64_t top, sticky = 0;
  int lo = msb - 63;
  if (lo <= 0) {
    int sh = -lo;  // value fits in 64 bits: l0 only (msb < 64)
    top    = l0 << sh;
  } else {
    // extract 64 bits starting at bit `lo` of the 192-bit number
    uint64_t w[3] = {l0, l1, l2};
    int li = lo >> 6, bi = lo & 63;
    top = w[li] >> bi;
    if (bi && li + 1 < 3) top |= w[li + 1] << (64 - bi);
    for (int i = 0; i < li; ++i) sticky |= w[i];
    if (bi) sticky |= w[li] & ((1ull << bi) - 1);
  }
  double d = __ull2double_rn(top | (sticky ? 1ull : 0ull));
  d        = scalbn(d, lo - 96);
  return neg ? -d : d;
}

// ---- global find-or-insert ----------------------------------------------
template <KeyMode M>
__device__ __forceinline__ int64_t find_or_insert(const GbPlan& p, int64_t r)
{
  if (M != KeyMode::GEN && !dvalid(p.k.c[0], r)) return static_cast<int64_t>(p.cap) + 1;
  uint64_t kb = key_bits<M>(p.k, r);
  uint64_t entry, h;
  if (M == KeyMode::K32) {
    entry = kb;
    h     = mix64(kb);
  } else if (M == KeyMode::K64) {
    if (kb == kSentinel64) return static_cast<int64_t>(p.cap);
    entry = kb;
    h     = mix64(kb);
  } else {
    h     = kb;
    entry = (static_cast<uint64_t>(r) << 32) | static_cast<uint32_t>(h);
  }
  const uint64_t empty = M == KeyMode::K64 ? kSentinel64 : kEmpty;
  unsigned long long* s = static_cast<unsigned long long*>(p.slots);
  uint64_t idx          = fastrange(h, p.cap);
  for (int probe = 0; probe < kMaxProbe; ++probe) {
    uint64_t v = s[idx];
    if (v == empty) {
      v = atomicCAS(&s[idx], empty, entry);
      if (v == empty) return static_cast<int64_t>(idx);
    }
    if (M == KeyMode::GEN) {
      if (static_cast<uint32_t>(v) == static_cast<uint32_t>(h) &&
          keys_equal(p.k, r, p.k, static_cast<int64_t>(v >> 32)))
        return static_cast<int64_t>(idx);
    } else if (v == entry) {
      return static_cast<int64_t>(idx);
    }
    idx = idx + 1 == p.cap ? 0 : idx + 1;
  }
  atomicExch(p.overflow, 1);
  return -1;
}

// Pair set insert for COUNT_DISTINCT; true when (group, value) is new.
__device__ __forceinline__ bool pair_insert(const GbPlan& p, const ColPlan& c, int64_t slot, int64_t r,
                                            int* overflow)
{
  uint64_t entry, h;
  if (c.pair_packed) {
    entry = (static_cast<uint64_t>(slot) << 32) | static_cast<uint32_t>(dbits(c.col, r));
    h     = mix64(entry);
  } else {
    h     = hash_combine64(mix64(static_cast<uint64_t>(slot)), hash_value(c.col, r));
    entry = (static_cast<uint64_t>(r) << 32) | static_cast<uint32_t>(h);
  }
  uint64_t idx = fastrange(h, c.pair_cap);
  for (int probe = 0; probe < kMaxProbe; ++probe) {
    uint64_t v = c.pairs[idx];
    if (v == kEmpty) {
      v = atomicCAS(&c.pairs[idx], kEmpty, entry);
      if (v == kEmpty) return true;
    }
    if (c.pair_packed) {
      if (v == entry) return false;
    } else if (static_cast<uint32_t>(v) == static_cast<uint32_t>(h)) {
      int64_t o = static_cast<int64_t>(v >> 32);
      if (keys_equal(p.k, r, p.k, o) && values_equal(c.col, r, c.col, o)) return false;
    }
    idx = idx + 1 == c.pair_cap ? 0 : idx + 1;
  }
  atomicExch(overflow, 1);
  return false;
}

// ---- the fused aggregation pass -----------------------------------------
template <KeyMode M>
__global__ void __launch_bounds__(kGbThreads) aggregate_kernel(GbPlan p)
{
  extern __shared__ __align__(16) unsigned char smem[];
  uint32_t* s_keys  = reinterpret_cast<uint32_t*>(smem + p.s_keys);
  uint32_t* s_count = reinterpret_cast<uint32_t*>(smem + p.s_count);
  const int S       = p.smem_slots;
  // init shared table
  for (int i = threadIdx.x; i < S; i += blockDim.x) {
    s_keys[i]  = kEmpty32;
    s_count[i] = 0;
  }
  for (int ci = 0; ci < p.ncols; ++ci) {
    const ColPlan& c = p.c[ci];
    uint32_t* vc     = reinterpret_cast<uint32_t*>(smem + c.s_vcount);
    for (int i = threadIdx.x; i < S; i += blockDim.x) vc[i] = 0;
    if (c.states & ST_SUM) {
      unsigned long long* sm = reinterpret_cast<unsigned long long*>(smem + c.s_sum);
      for (int i = threadIdx.x; i < S * c.limbs; i += blockDim.x) sm[i] = 0;
    }
    if (c.states & ST_MIN) {
      unsigned long long* a = reinterpret_cast<unsigned long long*>(smem + c.s_mn);
      for (int i = threadIdx.x; i < S; i += blockDim.x) a[i] = 0;
    }
    if (c.states & ST_MAX) {
      unsigned long long* a = reinterpret_cast<unsigned long long*>(smem + c.s_mx);
      for (int i = threadIdx.x; i < S; i += blockDim.x) a[i] = 0;
    }
    if (c.states & ST_NDIST) {
      uint32_t* a = reinterpret_cast<uint32_t*>(smem + c.s_ndist);
      for (int i = threadIdx.x; i < S; i += blockDim.x) a[i] = 0;
    }
  }
  __syncthreads();

  const int shift = 32 - (31 - __clz(S));  // S is a power of two
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < p.n;
       r += (int64_t)gridDim.x * blockDim.x) {
    const int64_t g = find_or_insert<M>(p, r);
    if (g < 0) continue;
    // shared-memory slot for g (bounded linear probe; -1 when full)
    int si       = -1;
    uint32_t key = static_cast<uint32_t>(g);
    uint32_t h   = (key * 0x9E3779B1u) >> shift;
#pragma unroll 1
    for (int t = 0; t < 8; ++t) {
      uint32_t v = s_keys[h];
      if (v == key) {
        si = static_cast<int>(h);
        break;
      }
      if (v == kEmpty32) {
        v = atomicCAS(&s_keys[h], kEmpty32, key);
        if (v == kEmpty32 || v == key) {
          si = static_cast<int>(h);
          break;
        }
      }
      h = (h + 1) & (S - 1);
    }
    if (si >= 0) atomicAdd(&s_count[si], 1u);
    else atomicAdd(&p.count_all[g], 1ull);

    for (int ci = 0; ci < p.ncols; ++ci) {
      const ColPlan& c = p.c[ci];
      if (!dvalid(c.col, r)) continue;
      if (si >= 0) atomicAdd(reinterpret_cast<uint32_t*>(smem + c.s_vcount) + si, 1u);
      else atomicAdd(&c.vcount[g], 1ull);
      if (c.states & ST_SUM) {
        if (c.fixed) {
          double x = c.col.type == LDF_FLOAT64 ? static_cast<const double*>(c.col.data)[r]
                                               : static_cast<double>(static_cast<const float*>(c.col.data)[r]);
          uint64_t a0, a1, a2;
          if (to_fixed192(x, a0, a1, a2)) {
            unsigned long long* dst = si >= 0
                                        ? reinterpret_cast<unsigned long long*>(smem + c.s_sum) + 3 * si
                                        : c.sum + 3 * g;
            atomic_add192(dst, a0, a1, a2);
          } else if (isnan(x)) {
            atomicOr(&c.special[g], SP_NAN);
          } else if (isinf(x)) {
            atomicOr(&c.special[g], x > 0 ? SP_PINF : SP_NINF);
          } else {
            atomicAdd(&c.fb[g], x);
          }
        } else {
          uint64_t v;
          if (is_signed_int_dev(c.col.type)) v = static_cast<uint64_t>(signed_value(c.col, r));
          else v = dbits(c.col, r);
          unsigned long long* dst = si >= 0 ? reinterpret_cast<unsigned long long*>(smem + c.s_sum) + si
                                            : c.sum + g;
          atomicAdd(dst, static_cast<unsigned long long>(v));
        }
      }
      if (c.states & (ST_MIN | ST_MAX)) {
        uint64_t o = ordered_bits(c.col, r);
        if (c.states & ST_MIN) {
          unsigned long long* dst = si >= 0 ? reinterpret_cast<unsigned long long*>(smem + c.s_mn) + si : c.mn + g;
          atomicMax(dst, static_cast<unsigned long long>(~o));
        }
        if (c.states & ST_MAX) {
          unsigned long long* dst = si >= 0 ? reinterpret_cast<unsigned long long*>(smem + c.s_mx) + si : c.mx + g;
          atomicMax(dst, static_cast<unsigned long long>(o));
        }
      }
      if (c.states & ST_NDIST) {
        if (pair_insert(p, c, g, r, p.overflow)) {
          if (si >= 0) atomicAdd(reinterpret_cast<uint32_t*>(smem + c.s_ndist) + si, 1u);
          else atomicAdd(&c.ndist[g], 1ull);
        }
      }
    }
  }
  __syncthreads();

  // flush the shared table into the global states
  for (int i = threadIdx.x; i < S; i += blockDim.x) {
    uint32_t key = s_keys[i];
    if (key == kEmpty32) continue;
    const int64_t g = key;
    if (s_count[i]) atomicAdd(&p.count_all[g], static_cast<unsigned long long>(s_count[i]));
    for (int ci = 0; ci < p.ncols; ++ci) {
      const ColPlan& c = p.c[ci];
      uint32_t vc      = reinterpret_cast<uint32_t*>(smem + c.s_vcount)[i];
      if (vc == 0) continue;
      atomicAdd(&c.vcount[g], static_cast<unsigned long long>(vc));
      if (c.states & ST_SUM) {
        const unsigned long long* sm = reinterpret_cast<unsigned long long*>(smem + c.s_sum);
        if (c.fixed) atomic_add192(c.sum + 3 * g, sm[3 * i], sm[3 * i + 1], sm[3 * i + 2]);
        else atomicAdd(c.sum + g, sm[i]);
      }
      if (c.states & ST_MIN) atomicMax(c.mn + g, reinterpret_cast<unsigned long long*>(smem + c.s_mn)[i]);
      if (c.states & ST_MAX) atomicMax(c.mx + g, reinterpret_cast<unsigned long long*>(smem + c.s_mx)[i]);
      if (c.states & ST_NDIST) {
        uint32_t nd = reinterpret_cast<uint32_t*>(smem + c.s_ndist)[i];
        if (nd) atomicAdd(c.ndist + g, static_cast<unsigned long long>(nd));
      }
    }
  }
}

// ---- cardinality estimate on a strided sample ----------------------------
// Counts sampled keys (and sampled (group, value) pairs of the first
// COUNT_DISTINCT column) in scratch tables; the GEE estimate is formed on the
// host from (occupied, singletons).
template <KeyMode M>
__global__ void sample_kernel(GbPlan sp, int64_t n_sample, int64_t stride, unsigned int* counts,
                              int pair_col, unsigned int* pair_counts)
{
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n_sample;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = i * stride;
    const int64_t g = find_or_insert<M>(sp, r);
    if (g < 0) continue;
    atomicAdd(&counts[g], 1u);
    if (pair_col >= 0) {
      const ColPlan& c = sp.c[pair_col];
      if (!dvalid(c.col, r)) continue;
      // pair set keyed by the sample slot; count every sampled pair
      uint64_t entry, h;
      if (c.pair_packed) {
        entry = (static_cast<uint64_t>(g) << 32) | static_cast<uint32_t>(dbits(c.col, r));
        h     = mix64(entry);
      } else {
        h     = hash_combine64(mix64(static_cast<uint64_t>(g)), hash_value(c.col, r));
        entry = (static_cast<uint64_t>(r) << 32) | static_cast<uint32_t>(h);
      }
      uint64_t idx = fastrange(h, c.pair_cap);
      for (int probe = 0; probe < kMaxProbe; ++probe) {
        uint64_t v = c.pairs[idx];
        if (v == kEmpty) {
          v = atomicCAS(&c.pairs[idx], kEmpty, entry);
          if (v == kEmpty) {
            atomicAdd(&pair_counts[idx], 1u);
            break;
          }
        }
        bool same;
        if (c.pair_packed) same = v == entry;
        else {
          int64_t o = static_cast<int64_t>(v >> 32);
          same = static_cast<uint32_t>(v) == static_cast<uint32_t>(h) && keys_equal(sp.k, r, sp.k, o) &&
                 values_equal(c.col, r, c.col, o);
        }
        if (same) {
          atomicAdd(&pair_counts[idx], 1u);
          break;
        }
        idx = idx + 1 == c.pair_cap ? 0 : idx + 1;
      }
    }
  }
}

// out[0] = occupied, out[1] = singletons
__global__ void freq_stats_kernel(const unsigned int* counts, int64_t n, unsigned long long* out)
{
  unsigned long long occ = 0, f1 = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    unsigned int c = counts[i];
    occ += c > 0;
    f1 += c == 1;
  }
  occ = warp_reduce_sum(occ);
  f1  = warp_reduce_sum(f1);
  if ((threadIdx.x & 31) == 0) {
    if (occ) atomicAdd(&out[0], occ);
    if (f1) atomicAdd(&out[1], f1);
  }
}

template <typename T>
__global__ void fill_kernel(T* p, int64_t n, T v)
{
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    p[i] = v;
}

// ---- compaction of occupied group slots ----------------------------------
template <KeyMode M>
__global__ void __launch_bounds__(kGbThreads)
  compact_groups_kernel(GbPlan p, int64_t nslots, int64_t* groups, uint64_t* status,
                        unsigned long long* counter, int64_t* total, int* err)
{
  constexpr int ITEMS = 4;
  __shared__ int64_t s_scan[kGbThreads / 32 + 1];
  __shared__ int64_t s_tile;
  __shared__ uint64_t s_prefix;
  const int64_t tile = next_tile_id(counter, &s_tile);
  const int64_t base = tile * (kGbThreads * ITEMS) + static_cast<int64_t>(threadIdx.x) * ITEMS;
  const unsigned long long* s = static_cast<const unsigned long long*>(p.slots);
  const uint64_t empty = M == KeyMode::K64 ? kSentinel64 : kEmpty;
  int f[ITEMS];
  int64_t c = 0;
#pragma unroll
  for (int i = 0; i < ITEMS; ++i) {
    int64_t j = base + i;
    f[i]      = 0;
    if (j < static_cast<int64_t>(p.cap)) f[i] = s[j] != empty;
    else if (j < nslots) f[i] = p.count_all[j] > 0;
    c += f[i];
  }
  int64_t tot;
  int64_t ex = block_exclusive_scan<int64_t, kGbThreads>(c, s_scan, &tot);
  if (threadIdx.x == 0) {
    s_prefix = lookback_exclusive(status, tile, static_cast<uint64_t>(tot), err);
    if (tile == static_cast<int64_t>(gridDim.x) - 1) *total = static_cast<int64_t>(s_prefix) + tot;
  }
  __syncthreads();
  int64_t pos = static_cast<int64_t>(s_prefix) + ex;
#pragma unroll
  for (int i = 0; i < ITEMS; ++i)
    if (f[i]) groups[pos++] = base + i;
}

// ---- finalize ------------------------------------------------------------
struct AggOut {
  int kind;
  int count_mode;
  int col;  // ColPlan index (-1 for COUNT_ALL)
  int in_type;
  OCol dst;
};
struct FinArgs {
  GbPlan p;
  int key_mode;
  const int64_t* groups;
  int64_t ngroups;
  int nkeys;
  OCol key_dst[kMaxKeys];
  int32_t* repr;  // GEN: representative row per output group
  int nagg;
  AggOut a[kMaxAggs];
};

__device__ __forceinline__ void store_double(const OCol& d, int64_t i, double v)
{
  if (d.type == LDF_FLOAT32) static_cast<float*>(d.data)[i] = static_cast<float>(v);
  else static_cast<double*>(d.data)[i] = v;
}
__device__ __forceinline__ void store_int(const OCol& d, int64_t i, uint64_t v)
{
  switch (d.width) {
    case 1: static_cast<uint8_t*>(d.data)[i] = static_cast<uint8_t>(v); break;
    case 2: static_cast<uint16_t*>(d.data)[i] = static_cast<uint16_t>(v); break;
    case 4:
      if (d.type == LDF_FLOAT32) static_cast<float*>(d.data)[i] = static_cast<float>(static_cast<int64_t>(v));
      else static_cast<uint32_t*>(d.data)[i] = static_cast<uint32_t>(v);
      break;
    default:
      if (d.type == LDF_FLOAT64) static_cast<double*>(d.data)[i] = static_cast<double>(static_cast<int64_t>(v));
      else static_cast<uint64_t*>(d.data)[i] = v;
      break;
  }
}
__device__ __forceinline__ uint64_t unordered_bits(int type, uint64_t o)
{
  switch (type) {
    case LDF_INT8:
    case LDF_INT16:
    case LDF_INT32:
    case LDF_INT64:
    case LDF_TIMESTAMP_US: return o ^ (1ull << 63);
    case LDF_FLOAT32: {
      uint32_t b = static_cast<uint32_t>(o);
      return (b & 0x80000000u) ? (b & 0x7fffffffu) : ~b;
    }
    case LDF_FLOAT64: return (o & (1ull << 63)) ? (o & ~(1ull << 63)) : ~o;
    default: return o;
  }
}

__device__ __forceinline__ double float_sum(const ColPlan& c, int64_t g, bool& special, double& sval)
{
  unsigned int sp = c.special[g];
  special         = sp != 0;
  if (special) {
    if ((sp & SP_NAN) || ((sp & SP_PINF) && (sp & SP_NINF))) sval = __longlong_as_double(0x7ff8000000000000ll);
    else sval = (sp & SP_PINF) ? __longlong_as_double(0x7ff0000000000000ll)
                               : __longlong_as_double(0xfff0000000000000ll);
  }
  return fixed192_to_double(c.sum[3 * g], c.sum[3 * g + 1], c.sum[3 * g + 2]) + c.fb[g];
}

__global__ void finalize_kernel(FinArgs f)
{
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < f.ngroups;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t g = f.groups[i];
    const GbPlan& p = f.p;
    // keys
    if (f.key_mode == static_cast<int>(KeyMode::GEN)) {
      uint64_t v = static_cast<const unsigned long long*>(p.slots)[g];
      int64_t rr = static_cast<int64_t>(v >> 32);
      f.repr[i]  = static_cast<int32_t>(rr);
      for (int j = 0; j < f.nkeys; ++j) {
        const OCol& d = f.key_dst[j];
        if (d.type == LDF_STRING) continue;
        copy_fixed(d.data, i, p.k.c[j].data, rr, d.width);
        if (d.valid) d.valid[i] = dvalid(p.k.c[j], rr) ? 1 : 0;
      }
    } else {
      const OCol& d = f.key_dst[0];
      bool is_null  = g == static_cast<int64_t>(p.cap) + 1;
      uint64_t kb   = g == static_cast<int64_t>(p.cap) ? kSentinel64
                      : is_null                        ? 0
                                                       : static_cast<const unsigned long long*>(p.slots)[g];
      store_int(OCol{d.data, nullptr, LDF_UINT64, d.width}, i, kb);
      if (d.valid) d.valid[i] = is_null ? 0 : 1;
    }
    const uint64_t call = p.count_all[g];
    for (int a = 0; a < f.nagg; ++a) {
      const AggOut& o = f.a[a];
      const OCol& d   = o.dst;
      if (o.kind == LDF_AGG_COUNT_ALL) {
        store_int(d, i, call);
        if (d.valid) d.valid[i] = 1;
        continue;
      }
      const ColPlan& c = p.c[o.col];
      const uint64_t vc = c.vcount[g];
      bool ok           = vc > 0;
      switch (o.kind) {
        case LDF_AGG_COUNT: {
          uint64_t v = o.count_mode == LDF_COUNT_ALL ? call : o.count_mode == LDF_COUNT_ONLY_NULL ? call - vc : vc;
          store_int(d, i, v);
          ok = true;
          break;
        }
        case LDF_AGG_COUNT_DISTINCT: {
          uint64_t has_null = call > vc ? 1 : 0;
          uint64_t nd       = c.ndist ? c.ndist[g] : 0;
          uint64_t v = o.count_mode == LDF_COUNT_ALL ? nd + has_null : o.count_mode == LDF_COUNT_ONLY_NULL ? has_null : nd;
          store_int(d, i, v);
          ok = true;
          break;
        }
        case LDF_AGG_SUM:
        case LDF_AGG_MEAN: {
          if (!ok) {
            store_int(d, i, 0);
            break;
          }
          double sv;
          if (c.fixed) {
            bool special;
            double sval;
            sv = float_sum(c, g, special, sval);
            if (special) sv = sval;
            if (o.kind == LDF_AGG_MEAN) sv = sv / static_cast<double>(vc);
            store_double(d, i, sv);
          } else {
            uint64_t s = c.sum[g];
            if (o.kind == LDF_AGG_MEAN) {
              double m = is_signed_int_dev(o.in_type) ? static_cast<double>(static_cast<int64_t>(s))
                                                      : static_cast<double>(s);
              store_double(d, i, m / static_cast<double>(vc));
            } else if (d.type == LDF_FLOAT64 || d.type == LDF_FLOAT32) {
              store_double(d, i, is_signed_int_dev(o.in_type) ? static_cast<double>(static_cast<int64_t>(s))
                                                              : static_cast<double>(s));
            } else {
              store_int(d, i, s);
            }
          }
          break;
        }
        case LDF_AGG_MIN:
        case LDF_AGG_MAX: {
          if (!ok) {
            store_int(d, i, 0);
            break;
          }
          uint64_t o64 = o.kind == LDF_AGG_MIN ? ~c.mn[g] : c.mx[g];
          uint64_t b   = unordered_bits(o.in_type, o64);
          if (d.type == o.in_type) {
            OCol raw{d.data, nullptr, LDF_UINT64, d.width};
            store_int(raw, i, b);
          } else if (o.in_type == LDF_FLOAT32) {
            store_double(d, i, static_cast<double>(__uint_as_float(static_cast<uint32_t>(b))));
          } else if (o.in_type == LDF_FLOAT64) {
            store_double(d, i, __longlong_as_double(static_cast<long long>(b)));
          } else {
            store_int(d, i, b);
          }
          break;
        }
        default: break;
      }
      if (d.valid) d.valid[i] = ok ? 1 : 0;
    }
  }
}

unsigned gs_blocks(int64_t n, int threads)
{
  int64_t b   = ceil_div(n, threads);
  int64_t cap = static_cast<int64_t>(num_sms()) * 8;
  return static_cast<unsigned>(b < 1 ? 1 : (b > cap ? cap : b));
}

template <KeyMode M>
void run_groupby(const OpContext& ctx, GbPlan p, const ldf_column* table, const int32_t* keys,
                 int nkeys, const ldf_aggregation* aggs, int naggs, const std::vector<int>& agg_col,
                 ldf_column* out)
{
  const Allocator& al = ctx.alloc();
  cudaStream_t s      = ctx.stream();
  const int64_t n     = p.n;

  int ndist_col = -1;
  for (int ci = 0; ci < p.ncols; ++ci)
    if (p.c[ci].states & ST_NDIST) {
      ndist_col = ci;
      break;
    }

  // ---- estimate groups / pairs ----------------------------------------------
  int64_t est_groups = n, est_pairs = n;
  const int64_t kSampleMax = int64_t(1) << 20;
  if (n > (int64_t(1) << 16)) {
    const int64_t ns     = std::min<int64_t>(n, kSampleMax);
    const int64_t stride = n / ns;
    GbPlan sp            = p;
    sp.cap               = static_cast<uint64_t>(2 * ns + 64);
    Buffer<unsigned long long> sslots(al, sp.cap + 2);
    Buffer<unsigned int> scounts(al, sp.cap + 2);
    Buffer<int> sover(al, 1);
    LDF_CUDA(cudaMemsetAsync(sslots.get(), 0xff, (sp.cap + 2) * 8, s));
    if (M == KeyMode::K64)
      launch("fill", fill_kernel<unsigned long long>, gs_blocks(sp.cap, 256), 256, 0, s, sslots.get(), sp.cap, kSentinel64);
    LDF_CUDA(cudaMemsetAsync(scounts.get(), 0, (sp.cap + 2) * 4, s));
    LDF_CUDA(cudaMemsetAsync(sover.get(), 0, 4, s));
    sp.slots    = sslots.get();
    sp.overflow = sover.get();
    Buffer<unsigned long long> spairs;
    Buffer<unsigned int> spcounts;
    if (ndist_col >= 0) {
      ColPlan& c  = sp.c[ndist_col];
      c.pair_cap  = static_cast<uint64_t>(2 * ns + 64);
      spairs      = Buffer<unsigned long long>(al, c.pair_cap);
      spcounts    = Buffer<unsigned int>(al, c.pair_cap);
      LDF_CUDA(cudaMemsetAsync(spairs.get(), 0xff, c.pair_cap * 8, s));
      LDF_CUDA(cudaMemsetAsync(spcounts.get(), 0, c.pair_cap * 4, s));
      c.pairs = spairs.get();
    }
    launch("sample", sample_kernel<M>, gs_blocks(ns, 256), 256, 0, s, sp, ns, stride, scounts.get(), ndist_col,
                                                         spcounts.get());
    LDF_CHECK_LAUNCH();
    Buffer<unsigned long long> stats(al, 4);
    LDF_CUDA(cudaMemsetAsync(stats.get(), 0, 32, s));
    launch("freq_stats", freq_stats_kernel, gs_blocks(sp.cap + 2, 256), 256, 0, s, scounts.get(), sp.cap + 2, stats.get());
    if (ndist_col >= 0)
      launch("freq_stats", freq_stats_kernel, gs_blocks(sp.c[ndist_col].pair_cap, 256), 256, 0, s, 
        spcounts.get(), sp.c[ndist_col].pair_cap, stats.get() + 2);
    LDF_CHECK_LAUNCH();
    unsigned long long h[4];
    LDF_CUDA(cudaMemcpyAsync(h, stats.get(), 32, cudaMemcpyDeviceToHost, s));
    ctx.finish();
    const double scale = std::sqrt(static_cast<double>(n) / static_cast<double>(ns));
    est_groups = static_cast<int64_t>(scale * h[1] + (h[0] - h[1])) + 1;
    est_pairs  = static_cast<int64_t>(scale * h[3] + (h[2] - h[3])) + 1;
    est_groups = std::min<int64_t>(est_groups, n);
    est_pairs  = std::min<int64_t>(est_pairs, n);
  }

  uint64_t cap      = static_cast<uint64_t>(std::max<int64_t>(3 * est_groups, 64));
  uint64_t pair_cap = static_cast<uint64_t>(std::max<int64_t>(3 * est_pairs, 64));

  // ---- shared-memory plan --------------------------------------------------
  int per_slot = 8;  // key + count_all
  for (int ci = 0; ci < p.ncols; ++ci) {
    const ColPlan& c = p.c[ci];
    per_slot += 4;
    if (c.states & ST_SUM) per_slot += 8 * c.limbs;
    if (c.states & ST_MIN) per_slot += 8;
    if (c.states & ST_MAX) per_slot += 8;
    if (c.states & ST_NDIST) per_slot += 4;
  }
  int S = 4096;
  const int kSmemBudget = 100 * 1024;
  while (S > 64 && S * per_slot + 64 * (p.ncols * 5 + 2) > kSmemBudget) S >>= 1;
  {
    int off      = 0;
    auto take    = [&](int bytes) {
      int o = off;
      off += (bytes + 15) & ~15;
      return o;
    };
    p.smem_slots = S;
    for (int ci = 0; ci < p.ncols; ++ci) {
      ColPlan& c = p.c[ci];
      c.s_sum    = (c.states & ST_SUM) ? take(8 * c.limbs * S) : 0;
      c.s_mn     = (c.states & ST_MIN) ? take(8 * S) : 0;
      c.s_mx     = (c.states & ST_MAX) ? take(8 * S) : 0;
    }
    p.s_keys  = take(4 * S);
    p.s_count = take(4 * S);
    for (int ci = 0; ci < p.ncols; ++ci) {
      ColPlan& c  = p.c[ci];
      c.s_vcount  = take(4 * S);
      c.s_ndist   = (c.states & ST_NDIST) ? take(4 * S) : 0;
    }
    p.smem_bytes = off;
  }
  LDF_CUDA(cudaFuncSetAttribute(aggregate_kernel<M>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                p.smem_bytes));
  int occ = 1;
  LDF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, aggregate_kernel<M>, kGbThreads,
                                                         p.smem_bytes));
  occ = std::max(occ, 1);

  for (int attempt = 0;; ++attempt) {
    // ---- allocate + init tables ------------------------------------------------
    const uint64_t nslots = cap + 2;
    Buffer<unsigned long long> slots(al, cap);
    if (M == KeyMode::K64)
      launch("fill", fill_kernel<unsigned long long>, gs_blocks(cap, 256), 256, 0, s, slots.get(), cap, kSentinel64);
    else
      LDF_CUDA(cudaMemsetAsync(slots.get(), 0xff, cap * 8, s));
    // one zeroed arena for every per-group state
    size_t words = nslots;  // count_all
    for (int ci = 0; ci < p.ncols; ++ci) {
      const ColPlan& c = p.c[ci];
      words += nslots;  // vcount
      if (c.states & ST_SUM) words += nslots * c.limbs + (c.fixed ? 2 * nslots : 0);
      if (c.states & ST_MIN) words += nslots;
      if (c.states & ST_MAX) words += nslots;
      if (c.states & ST_NDIST) words += nslots;
    }
    Buffer<unsigned long long> arena(al, words);
    LDF_CUDA(cudaMemsetAsync(arena.get(), 0, words * 8, s));
    unsigned long long* w = arena.get();
    p.slots               = slots.get();
    p.cap                 = cap;
    p.count_all           = w;
    w += nslots;
    std::vector<Buffer<unsigned long long>> pair_bufs;
    for (int ci = 0; ci < p.ncols; ++ci) {
      ColPlan& c = p.c[ci];
      c.vcount   = w;
      w += nslots;
      if (c.states & ST_SUM) {
        c.sum = w;
        w += nslots * c.limbs;
        if (c.fixed) {
          c.fb = reinterpret_cast<double*>(w);
          w += nslots;
          c.special = reinterpret_cast<unsigned int*>(w);
          w += nslots;
        }
      }
      if (c.states & ST_MIN) {
        c.mn = w;
        w += nslots;
      }
      if (c.states & ST_MAX) {
        c.mx = w;
        w += nslots;
      }
      if (c.states & ST_NDIST) {
        c.ndist = w;
        w += nslots;
        c.pair_cap = pair_cap;
        pair_bufs.emplace_back(al, pair_cap);
        c.pairs = pair_bufs.back().get();
        LDF_CUDA(cudaMemsetAsync(c.pairs, 0xff, pair_cap * 8, s));
      }
    }
    Buffer<int64_t> over(al, 1);
    LDF_CUDA(cudaMemsetAsync(over.get(), 0, 8, s));
    p.overflow = reinterpret_cast<int*>(over.get());

    // ---- aggregate ----------------------------------------------------------------
    if (n > 0) {
      int64_t blocks = std::min<int64_t>(static_cast<int64_t>(num_sms()) * occ, ceil_div(n, kGbThreads));
      launch("aggregate", aggregate_kernel<M>, static_cast<unsigned>(blocks), kGbThreads, p.smem_bytes, s, p);
      LDF_CHECK_LAUNCH();
    }
    if (ctx.read_i64(over.get()) != 0) {
      if (attempt >= 4) fail(LDF_ERR_INTERNAL, "groupby hash table overflow");
      cap *= 4;
      pair_cap *= 4;
      continue;
    }

    // ---- compact + finalize -------------------------------------------------------
    const int64_t tiles = ceil_div(static_cast<int64_t>(nslots), kGbThreads * 4);
    Buffer<int64_t> groups(al, nslots);
    Buffer<uint64_t> status(al, tiles + 2);
    Buffer<int64_t> total(al, 1);
    LDF_CUDA(cudaMemsetAsync(status.get(), 0, (tiles + 2) * 8, s));
    launch("compact_groups", compact_groups_kernel<M>, static_cast<unsigned>(tiles), kGbThreads, 0, s, 
      p, static_cast<int64_t>(nslots), groups.get(), status.get(),
      reinterpret_cast<unsigned long long*>(status.get() + tiles), total.get(), ctx.err());
    LDF_CHECK_LAUNCH();
    const int64_t G = ctx.read_i64(total.get());

    FinArgs f{};
    f.p        = p;
    f.key_mode = static_cast<int>(M);
    f.groups   = groups.get();
    f.ngroups  = G;
    f.nkeys    = nkeys;
    for (int j = 0; j < nkeys; ++j) {
      const ldf_column& kc = table[keys[j]];
      bool nullable        = kc.valid != nullptr;
      out[j]               = alloc_out_column(al, kc.type, G, nullable);
      f.key_dst[j]         = OCol{out[j].data, out[j].valid, kc.type, type_width(kc.type)};
    }
    Buffer<int32_t> repr;
    if (M == KeyMode::GEN) {
      repr   = Buffer<int32_t>(al, std::max<int64_t>(G, 1));
      f.repr = repr.get();
    }
    f.nagg = naggs;
    for (int a = 0; a < naggs; ++a) {
      const ldf_aggregation& ag = aggs[a];
      bool nullable = !(ag.kind == LDF_AGG_COUNT_ALL || ag.kind == LDF_AGG_COUNT_DISTINCT);
      out[nkeys + a] = alloc_out_column(al, ag.out_type, G, nullable);
      AggOut& o      = f.a[a];
      o.kind         = ag.kind;
      o.count_mode   = ag.count_mode;
      o.col          = agg_col[a];
      o.in_type      = ag.kind == LDF_AGG_COUNT_ALL ? LDF_INT64 : table[ag.in_col].type;
      o.dst = OCol{out[nkeys + a].data, out[nkeys + a].valid, ag.out_type, type_width(ag.out_type)};
    }
    if (G > 0) {
      launch("finalize", finalize_kernel, gs_blocks(G, 256), 256, 0, s, f);
      LDF_CHECK_LAUNCH();
    }
    for (int j = 0; j < nkeys; ++j)
      if (table[keys[j]].type == LDF_STRING)
        gather_strings(ctx, make_dcol(table[keys[j]]), repr.get(), G, out[j]);
    ctx.finish();
    return;
  }
}

}  // namespace

void groupby_aggregation(const ldf_column* table, int ncols, const int32_t* keys, int nkeys,
                         const ldf_aggregation* aggs, int naggs, ldf_column* out, const OpContext& ctx)
{
  if (nkeys < 1) fail(LDF_ERR_INVALID_ARGUMENT, "must pass at least one key column");
  LDF_REQUIRE(naggs <= kMaxAggs, "too many aggregations");
  KeyCols k = make_keys(table, ncols, keys, nkeys);
  const int64_t n = ncols > 0 ? table[0].size : 0;
  LDF_REQUIRE(n < (int64_t(1) << 31), "tables of 2^31 rows or more per task are not supported");
  GbPlan p{};
  p.k = k;
  p.n = n;
  std::vector<int> agg_col(naggs, -1);
  std::vector<int> col_of_plan;
  for (int a = 0; a < naggs; ++a) {
    const ldf_aggregation& ag = aggs[a];
    if (ag.kind == LDF_AGG_COUNT_ALL) continue;
    LDF_REQUIRE(ag.in_col >= 0 && ag.in_col < ncols, "aggregation input column out of range");
    const ldf_column& c = table[ag.in_col];
    int ci              = -1;
    for (size_t q = 0; q < col_of_plan.size(); ++q)
      if (col_of_plan[q] == ag.in_col) ci = static_cast<int>(q);
    if (ci < 0) {
      LDF_REQUIRE(p.ncols < kMaxAggCols, "too many distinct aggregation input columns");
      ci = p.ncols++;
      col_of_plan.push_back(ag.in_col);
      ColPlan& cp = p.c[ci];
      cp.col      = make_dcol(c);
      cp.fixed    = is_float(c.type) ? 1 : 0;
      cp.limbs    = cp.fixed ? 3 : 1;
      cp.pair_packed = type_width(c.type) <= 4 && c.type != LDF_STRING;
    }
    agg_col[a] = ci;
    ColPlan& cp = p.c[ci];
    switch (ag.kind) {
      case LDF_AGG_SUM:
      case LDF_AGG_MEAN:
        LDF_REQUIRE(c.type != LDF_STRING, "sum/mean of a string column is not supported");
        cp.states |= ST_SUM;
        break;
      case LDF_AGG_MIN: cp.states |= ST_MIN; break;
      case LDF_AGG_MAX: cp.states |= ST_MAX; break;
      case LDF_AGG_COUNT: break;
      case LDF_AGG_COUNT_DISTINCT: cp.states |= ST_NDIST; break;
      default: fail(LDF_ERR_UNSUPPORTED, "Unsupported groupby aggregation");
    }
    if ((ag.kind == LDF_AGG_MIN || ag.kind == LDF_AGG_MAX) && c.type == LDF_STRING)
      fail(LDF_ERR_UNSUPPORTED, "min/max of a string column is not supported");
  }
  switch (key_mode(k)) {
    case KeyMode::K32: run_groupby<KeyMode::K32>(ctx, p, table, keys, nkeys, aggs, naggs, agg_col, out); break;
    case KeyMode::K64: run_groupby<KeyMode::K64>(ctx, p, table, keys, nkeys, aggs, naggs, agg_col, out); break;
    default: run_groupby<KeyMode::GEN>(ctx, p, table, keys, nkeys, aggs, naggs, agg_col, out); break;
  }
}

}  // namespace ldf
