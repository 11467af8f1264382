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
// Device plan (stream ordered; the host reads back sizes between passes):
//  1. sample  2^20 strided rows into scratch tables: GEE estimates (Charikar et
//             al. 2000) of the groups (x4, heavy tails are underestimated) and
//             of the (group, value) pairs of the first NUNIQUE column.
//  2. assign  key -> dense id through an open-addressing key table (one word
//             {id, key32} for <= 4-byte keys, {key word, id} otherwise, the
//             word of multi-column / string keys being {representative row,
//             hash tag}); ids come from per-warp pools of 32; row counts per
//             id (the hottest ids in shared memory).  Warps take 1,024-row
//             chunks; multi-column and string keys go one row per lane (their
//             code is large).  A probe longer than kMaxProbe or too many ids
//             flags overflow and the call re-runs with a 4x table.
//  3. ranks   ids renumbered by descending row count (radix sort), so the
//             most frequent groups get the smallest ranks; the row count and
//             distinct counts live in field-major arrays by rank, each value
//             column's valid count / sum / min / max in its own rank-major
//             block (one row's updates share a cache line).
//  4. columns one pass per value column: the most frequent ranks accumulate
//             in shared memory (flushed once per CTA), the others with
//             red.add / red.max.  Float sums are exact fixed point (six 32-bit
//             chunks, LSB 2^-96): integer adds are associative, so a sum is
//             independent of thread order and bit-identical alone or in a
//             batch, and is rounded once at the end.
//  5. NUNIQUE <= 4-byte values: one bit per value of the column's range for
//             the most frequent ranks (96 MB of bitmaps), a pair set for the
//             next ranks, and per-rank segments deduplicated in shared memory
//             for the rest; wider values and strings: a generic pair set.
//  6. output  used ranks compacted; keys, aggregates and their Arrow result
//             types written in one finalize pass.
// Input columns in host memory are copied in by HostStaging (keys first) and
// each pass waits only for the columns it reads.
#include "radix.cuh"

#include <cmath>
#include <cstdio>
#include <cstdlib>

namespace ldf {
namespace {

constexpr int kMaxAggCols = 8;
constexpr int kMaxAggs    = 32;
constexpr int kMaxProbe   = 1024;
constexpr int kGbThreads  = 512;
// inputs of at most this many rows keep their assign-pass ids as ranks
constexpr int64_t kSmallPlanRows = int64_t(1) << 18;
constexpr uint64_t kEmpty = ~0ull;
// Empty marker of the 8-byte key table; a key equal to it is the group with
// the reserved id kIdSentinel, a null single key the group kIdNull.
constexpr uint64_t kSentinel64 = 0x7ff4dead7ff4beefull;
constexpr uint32_t kUnsetId    = 0xffffffffu;
constexpr uint32_t kIdNull     = 0;
constexpr uint32_t kIdSentinel = 1;
constexpr uint32_t kIdFirst    = 2;

enum : uint32_t { ST_SUM = 1, ST_MIN = 2, ST_MAX = 4, ST_NDIST = 8 };
enum : uint32_t { SP_NAN = 1, SP_PINF = 2, SP_NINF = 4 };

struct ColPlan {
  DCol col;
  uint32_t states;
  int nullable;     // the record has a valid-count word
  int fixed;        // float sum: 3 words of fixed point, else 1 word
  int pair_packed;  // (id << 32 | value32) pair keys
  // valid count / sum / min / max live in the column's own rank-major block
  // (word k of rank g at crec[g * cw + k], so one row's updates share a
  // cache line); the distinct count lives in the shared field-major record
  int off_vcount, off_sum, off_mn, off_mx;  // word offsets in the column block
  int off_nd;                               // field of the shared record
  int cw;                                   // words per rank in the column block
  unsigned long long* crec;
  // shared-memory hot records (byte offsets of typed arrays, [hot] entries)
  int sh_vcount, sh_sum, sh_mn, sh_mx, sh_nd;
  int sum_chunks;  // 32-bit chunks of a sum magnitude: 6 (float, 2^-96 LSB) or 2 (integers)
  int mm64;        // min/max kept as 64-bit words (8-byte types) instead of 32-bit
  unsigned long long* pairs;
  uint64_t pair_cap;
  unsigned long long* pair_buf;  // [n] (id << 32 | value32) per valid row, ~0 otherwise (packed pairs)
  double* fb;             // [id_cap] float values outside the fixed-point range
  unsigned int* special;  // [id_cap] NaN / +inf / -inf seen
};

struct GbPlan {
  KeyCols k;
  int64_t n;
  unsigned long long* slots;  // [cap] K32 words, or [2 * cap] {key word, id} pairs
  uint64_t cap;
  unsigned long long* id_counter;
  uint64_t id_cap;
  unsigned long long* states;  // [id_cap * stride] group records
  unsigned long long* id_key;  // [id_cap] key word (1-8 byte keys) or representative row
  int stride;                  // words per record
  int hot;                     // ids below `hot` aggregate in shared memory
  unsigned long long* chunk_counter;  // dynamic row-chunk scheduler
  int sh_count;                // byte offset of the hot count array
  int ncols;
  ColPlan c[kMaxAggCols];
  int* overflow;
  int* err;
};

// 32-bit ordered form of a <= 4-byte value -> its 64-bit ordered form (the
// one the global min/max words hold).
template <int W, bool SGN, bool FLT>
__device__ __forceinline__ uint64_t widen32(uint32_t o32)
{
  if (!FLT && SGN) {
    const int32_t v = static_cast<int32_t>(o32 ^ 0x80000000u);
    return static_cast<uint64_t>(static_cast<int64_t>(v)) ^ (1ull << 63);
  }
  return o32;
}

// ---- exact float sums: carry-save 32-bit chunks ------------------------------
// A finite double x with 2^-44 <= |x| < 2^95 is an integer multiple of 2^-96:
// x = +-m * 2^(s - 96) with m < 2^53 and 0 <= s <= 138.  Its 2^-96 fixed-point
// value is split into 32-bit chunks (bits [32j, 32j + 32), j = 0..5); each
// chunk is added, signed, into its own 64-bit accumulator with a
// fire-and-forget reduction.  A chunk is < 2^32 and a group has < 2^31 rows,
// so accumulators never overflow and the sum is exact whatever the order.
constexpr int kSumChunks = 6;

__device__ __forceinline__ bool fixed_parts(double x, uint64_t& m, int& s, bool& neg)
{
  const uint64_t b = __double_as_longlong(x);
  const int e      = static_cast<int>((b >> 52) & 0x7ff);
  neg              = (b >> 63) != 0;
  if (e == 0 && (b << 1) == 0) {
    m = 0;
    s = 0;
    return true;
  }
  const int E = e - 1023;
  if (e == 0 || E < -44 || E >= 95) return false;
  m = (b & ((1ull << 52) - 1)) | (1ull << 52);
  s = E + 44;
  return true;
}

// Fire-and-forget reductions on global memory (explicit global space: the
// record pointers live in the parameter struct, where the compiler cannot
// infer it).
__device__ __forceinline__ void red_add(unsigned long long* p, uint64_t v)
{
  asm volatile("red.relaxed.gpu.global.add.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ void red_max(unsigned long long* p, uint64_t v)
{
  asm volatile("red.relaxed.gpu.global.max.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Add +-m << s into the chunk accumulators acc[0..5].
__device__ __forceinline__ void add_fixed_chunks(unsigned long long* acc, uint64_t m, int s, bool neg,
                                                 uint64_t cstride = 1)
{
  if (m == 0) return;
  const int j0 = s >> 5, j1 = (s + 52) >> 5;
  for (int j = j0; j <= j1; ++j) {
    const int off   = 32 * j - s;  // bit of m that lands at chunk bit 0
    uint64_t chunk  = off >= 0 ? (m >> off) : (m << (-off));
    chunk &= 0xffffffffull;
    if (chunk) red_add(acc + j * cstride, neg ? (0ull - chunk) : chunk);
  }
}

// Exact value of sum_j acc_j * 2^(32j - 96), correctly rounded to double.
__device__ __forceinline__ double chunks_to_double(const unsigned long long* acc, uint64_t cstride = 1)
{
  // 256-bit two's complement accumulation of the signed partials
  uint64_t w[4] = {0, 0, 0, 0};
  for (int j = 0; j < kSumChunks; ++j) {
    const int64_t a = static_cast<int64_t>(acc[j * cstride]);
    uint64_t t[5]   = {0, 0, 0, 0, 0};
    const int sh = 32 * j, li = sh >> 6, bi = sh & 63;
    const uint64_t lo = static_cast<uint64_t>(a);
    const uint64_t ext = a < 0 ? ~0ull : 0ull;
    t[li] = lo << bi;
    t[li + 1] = bi ? (lo >> (64 - bi)) | (ext << bi) : ext;
    for (int q = li + 2; q < 5; ++q) t[q] = ext;
    uint64_t carry = 0;
    for (int q = 0; q < 4; ++q) {
      const uint64_t x = w[q] + t[q];
      const uint64_t c1 = x < w[q] ? 1 : 0;
      const uint64_t y = x + carry;
      const uint64_t c2 = y < x ? 1 : 0;
      w[q] = y;
      carry = c1 + c2;
    }
  }
  const bool neg = static_cast<int64_t>(w[3]) < 0;
  if (neg) {
    uint64_t c = 1;
    for (int q = 0; q < 4; ++q) {
      w[q] = ~w[q] + c;
      c    = (c && w[q] == 0) ? 1 : 0;
    }
  }
  int msb = -1;
  for (int q = 3; q >= 0; --q)
    if (w[q]) {
      msb = 64 * q + 63 - __clzll(w[q]);
      break;
    }
  if (msb < 0) return 0.0;
  const int lo = msb - 63;
  uint64_t top, sticky = 0;
  if (lo <= 0) {
    top = w[0] << (-lo);
  } else {
    const int li = lo >> 6, bi = lo & 63;
    top = w[li] >> bi;
    if (bi && li + 1 < 4) top |= w[li + 1] << (64 - bi);
    for (int i = 0; i < li; ++i) sticky |= w[i];
    if (bi) sticky |= w[li] & ((1ull << bi) - 1);
  }
  double d = __ull2double_rn(top | (sticky ? 1ull : 0ull));
  d        = scalbn(d, lo - 96);
  return neg ? -d : d;
}

// ---- group ids ------------------------------------------------------------
// Key table slots.  K32: one word (id << 32 | key32), published by one CAS.
// K64 / GEN: two words {key word, id}; the key word is claimed by CAS and the
// id stored right after, so a reader that sees the key before its id waits
// (bounded) for the id.  Empty key word: kEmpty, or kSentinel64 for K64.
template <KeyMode M>
__device__ __forceinline__ uint64_t empty_word()
{
  return M == KeyMode::K64 ? kSentinel64 : kEmpty;
}

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31; }

__device__ __forceinline__ uint32_t wait_id(const unsigned long long* slot_hi, int* err)
{
  for (uint32_t spin = 0; spin < kSpinLimit; ++spin) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(slot_hi) : "memory");
    if (v != kEmpty) return static_cast<uint32_t>(v);
    __nanosleep(64);
  }
  atomicExch(err, LDF_ERR_TIMEOUT);
  return kUnsetId;
}

template <KeyMode M>
__device__ __forceinline__ bool same_key(const GbPlan& p, uint64_t v, uint64_t word, uint64_t h, int64_t r)
{
  if (M == KeyMode::K32) return static_cast<uint32_t>(v) == static_cast<uint32_t>(word);
  if (M == KeyMode::K64) return v == word;
  return static_cast<uint32_t>(v) == static_cast<uint32_t>(h) &&
         keys_equal(p.k, r, p.k, static_cast<int64_t>(v >> 32));
}

// Per-warp pool of pre-zeroed group ids (warp-uniform state).
struct IdPool {
  uint64_t next, end;
};

// Take ids for the lanes with `need` set; refills the pool (32 ids, records
// zeroed, one fence) when it runs short.  All 32 lanes call it together.
__device__ __forceinline__ uint64_t pool_take(const GbPlan& p, IdPool& pool, bool need)
{
  const uint32_t want = __ballot_sync(0xffffffffu, need);
  if (want == 0) return kEmpty;
  const uint32_t k = __popc(want);
  if (pool.end - pool.next < k) {
    unsigned long long base = 0;
    if (lane_id() == 0) base = atomicAdd(p.id_counter, 32ull);
    base = __shfl_sync(0xffffffffu, base, 0);
    const uint64_t end = base + 32 < p.id_cap ? base + 32 : p.id_cap;
    if (base < end) {
      const uint64_t w0 = base * p.stride, w1 = end * p.stride;
      for (uint64_t w = w0 + lane_id(); w < w1; w += 32) p.states[w] = 0;
      __threadfence();
    }
    pool.next = base;
    pool.end  = end > base ? end : base;
    if (pool.end - pool.next < k) {
      if (lane_id() == 0) atomicExch(p.overflow, 1);
      return kEmpty;
    }
  }
  const uint64_t mine = pool.next + __popc(want & ((1u << lane_id()) - 1u));
  pool.next += k;
  return need ? mine : kEmpty;
}

constexpr int kRows = 4;  // rows per lane per step (memory-level parallelism)
// Rows per lane per step of the assign pass.  Multi-column and string keys
// (GEN) take one: their key hashing and comparison code is large, and four
// unrolled copies of it outgrow the instruction cache.
constexpr int kGenRows = 1;
template <KeyMode M>
__host__ __device__ constexpr int assign_rows()
{
  return M == KeyMode::GEN ? kGenRows : kRows;
}

// Group ids of the R rows of this lane (kUnsetId for rows past the end).
template <KeyMode M, int R>
__device__ void group_ids(const GbPlan& p, IdPool& pool, const int64_t (&r)[R], uint32_t (&id)[R])
{
  const uint64_t empty = empty_word<M>();
  uint64_t word[R], h[R], idx[R], hi[R];
  bool pending[R];
  unsigned long long* s = p.slots;
  const int sw          = M == KeyMode::K32 ? 1 : 2;  // words per slot
#pragma unroll
  for (int j = 0; j < R; ++j) {
    id[j]      = kUnsetId;
    pending[j] = false;
    word[j] = h[j] = idx[j] = hi[j] = 0;
    if (r[j] >= p.n) continue;
    if (M != KeyMode::GEN && !dvalid_stream(p.k.c[0], r[j])) {
      id[j] = kIdNull;
      continue;
    }
    const uint64_t kb = M == KeyMode::GEN ? key_bits<M>(p.k, r[j]) : dbits_stream(p.k.c[0], r[j]);
    if (M == KeyMode::GEN) {
      h[j]    = kb;
      word[j] = (static_cast<uint64_t>(r[j]) << 32) | static_cast<uint32_t>(kb);
    } else {
      h[j]    = mix64(kb);
      word[j] = kb;
    }
    if (M == KeyMode::K64 && kb == kSentinel64) {
      id[j] = kIdSentinel;
      continue;
    }
    idx[j]     = fastrange(h[j], p.cap);
    pending[j] = true;
  }
  // first probes of all rows in flight together
  uint64_t v[R];
#pragma unroll
  for (int j = 0; j < R; ++j) {
    v[j] = 0;
    if (!pending[j]) continue;
    if (M == KeyMode::K32) {
      v[j] = s[idx[j]];
    } else {
      const ulonglong2 t = *reinterpret_cast<const ulonglong2*>(s + 2 * idx[j]);
      v[j]               = t.x;
      hi[j]              = t.y;
    }
  }
  bool need[R];
#pragma unroll
  for (int j = 0; j < R; ++j) {
    need[j] = false;
    if (!pending[j]) continue;
    for (int probe = 0; probe < kMaxProbe; ++probe) {
      if (v[j] == empty) {
        need[j] = true;
        break;
      }
      if (same_key<M>(p, v[j], word[j], h[j], r[j])) {
        if (M == KeyMode::K32) id[j] = static_cast<uint32_t>(v[j] >> 32);
        else id[j] = hi[j] != kEmpty ? static_cast<uint32_t>(hi[j]) : wait_id(s + 2 * idx[j] + 1, p.err);
        break;
      }
      idx[j] = idx[j] + 1 == p.cap ? 0 : idx[j] + 1;
      if (M == KeyMode::K32) {
        v[j] = s[idx[j]];
      } else {
        const ulonglong2 t = *reinterpret_cast<const ulonglong2*>(s + 2 * idx[j]);
        v[j]               = t.x;
        hi[j]              = t.y;
      }
      if (probe + 1 == kMaxProbe) atomicExch(p.overflow, 1);
    }
  }
  // inserts: ids from the warp pool, then publish
#pragma unroll
  for (int j = 0; j < R; ++j) {
    const uint64_t mine = pool_take(p, pool, need[j]);
    if (!need[j] || mine == kEmpty) continue;
    p.id_key[mine]      = M == KeyMode::GEN ? static_cast<uint64_t>(r[j]) : word[j];
    const uint64_t full = M == KeyMode::K32 ? ((mine << 32) | (word[j] & 0xffffffffull)) : word[j];
    for (int probe = 0; probe < kMaxProbe; ++probe) {
      const uint64_t old = atomicCAS(s + sw * idx[j], empty, full);
      if (old == empty) {
        if (M != KeyMode::K32) s[2 * idx[j] + 1] = mine;
        id[j] = static_cast<uint32_t>(mine);
        break;
      }
      if (same_key<M>(p, old, word[j], h[j], r[j])) {  // lost the race: `mine` stays a zeroed hole
        id[j] = M == KeyMode::K32 ? static_cast<uint32_t>(old >> 32) : wait_id(s + 2 * idx[j] + 1, p.err);
        break;
      }
      // another key took the slot: probe on to the key or the next empty slot
      bool done = false;
      for (; probe < kMaxProbe; ++probe) {
        idx[j]           = idx[j] + 1 == p.cap ? 0 : idx[j] + 1;
        const uint64_t t = s[sw * idx[j]];
        if (t == empty) break;
        if (same_key<M>(p, t, word[j], h[j], r[j])) {
          id[j] = M == KeyMode::K32 ? static_cast<uint32_t>(t >> 32) : wait_id(s + 2 * idx[j] + 1, p.err);
          done  = true;
          break;
        }
      }
      if (done) break;
      if (probe >= kMaxProbe - 1) atomicExch(p.overflow, 1);
    }
  }
}

// Pair set insert for COUNT_DISTINCT; true when (group, value) is new.
__device__ __forceinline__ bool pair_insert(const GbPlan& p, const ColPlan& c, uint32_t id, int64_t r)
{
  uint64_t entry, h;
  if (c.pair_packed) {
    entry = (static_cast<uint64_t>(id) << 32) | static_cast<uint32_t>(dbits(c.col, r));
    h     = mix64(entry);
  } else {
    h     = hash_combine64(mix64(static_cast<uint64_t>(id)), hash_value(c.col, r));
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
  atomicExch(p.overflow, 1);
  return false;
}

// ---- shared-memory (hot) records ------------------------------------------------
// Shared-memory atomics are only fast at 32 bits (a 64-bit add is emulated and
// collapses under the same-address contention of heavy hitters), so hot
// records hold 32-bit counters, and sums as sign-magnitude 32-bit chunks, each
// with a 32-bit carry counter: chunk j of a sum = lo_j + 2^32 carry_j, exact.
// Layout of one hot sum: [chunk][sign][lo, carry] u32 words.
__device__ __forceinline__ void sh_add_chunk(uint32_t* base, uint32_t v)
{
  const uint32_t old = atomicAdd(base, v);
  if (old + v < old) atomicAdd(base + 1, 1u);
}

__device__ __forceinline__ void sh_add_magnitude(uint32_t* sum, int nchunks, int first_chunk, uint64_t m_lo,
                                                 uint64_t m_hi, bool neg)
{
  // m (up to 128 bits: m_hi:m_lo) placed at chunk `first_chunk` boundary already
  (void)nchunks;
  uint32_t c[4] = {static_cast<uint32_t>(m_lo), static_cast<uint32_t>(m_lo >> 32), static_cast<uint32_t>(m_hi),
                   static_cast<uint32_t>(m_hi >> 32)};
#pragma unroll
  for (int q = 0; q < 4; ++q)
    if (c[q]) sh_add_chunk(sum + ((first_chunk + q) * 2 + (neg ? 1 : 0)) * 2, c[q]);
}

// ---- pass 1: dense group id of every row ---------------------------------------
// gid[r] = group id (kUnsetId past an overflow); the row count of each group is
// accumulated here too (hot ids in shared memory).
template <KeyMode M>
__global__ void __launch_bounds__(kGbThreads) assign_kernel(GbPlan p, uint32_t* gid)
{
  extern __shared__ __align__(16) unsigned char smem[];
  uint32_t* cnt = reinterpret_cast<uint32_t*>(smem);
  const int H   = p.hot;
  for (int i = threadIdx.x; i < H; i += blockDim.x) cnt[i] = 0;
  __syncthreads();
  IdPool pool{0, 0};
  constexpr int R          = assign_rows<M>();
  constexpr int64_t kChunk = 32 * R * 8;  // rows per dynamically scheduled chunk
  for (;;) {
    unsigned long long chunk = 0;
    if (lane_id() == 0) chunk = atomicAdd(p.chunk_counter, 1ull);
    chunk = __shfl_sync(0xffffffffu, chunk, 0);
    const int64_t c0 = static_cast<int64_t>(chunk) * kChunk;
    if (c0 >= p.n) break;
    const int64_t c1 = c0 + kChunk < p.n ? c0 + kChunk : p.n;
    for (int64_t base = c0; base < c1; base += 32 * R) {
      int64_t r[R];
      uint32_t id[R];
#pragma unroll
      for (int j = 0; j < R; ++j) {
        r[j] = base + j * 32 + lane_id();
        if (r[j] >= c1) r[j] = p.n;  // past the chunk: no row
      }
      group_ids<M, R>(p, pool, r, id);
#pragma unroll
      for (int j = 0; j < R; ++j) {
        if (r[j] >= p.n) continue;
        __stcs(gid + r[j], id[j]);
        if (id[j] == kUnsetId) continue;
        if (id[j] < static_cast<uint32_t>(H)) atomicAdd(cnt + id[j], 1u);
        else red_add(p.states + static_cast<int64_t>(id[j]) * p.stride, 1);
      }
    }
  }
  __syncthreads();
  for (int g = threadIdx.x; g < H; g += blockDim.x)
    if (cnt[g]) red_add(p.states + static_cast<int64_t>(g) * p.stride, cnt[g]);
}

// Factor from the sampled group estimate to the key-table sizing estimate
// (LDF_B200_GB_EST_MULT, 1 to 8).
inline int64_t est_multiplier()
{
  static const int64_t m = [] {
    const char* e = std::getenv("LDF_B200_GB_EST_MULT");
    const int v   = e ? std::atoi(e) : 4;
    return static_cast<int64_t>(v >= 1 && v <= 8 ? v : 4);
  }();
  return m;
}

// ---- pass 2: one value column (valid count, sum, min, max) ---------------------
struct ColArgs {
  const uint32_t* gid;
  int64_t n;
  DCol col;
  int nullable;
  uint32_t states;
  int sum_chunks;  // 6 (float, fixed point) or 2 (integer magnitude)
  int off_vcount, off_sum, off_mn, off_mx;
  unsigned long long* rec;  // the column block: word k of rank g at rec[g * cw + k * ld]
  uint64_t ld;
  int cw;
  const uint32_t* newid;    // assign-pass id -> frequency rank
  double* fb;
  unsigned int* special;
  int hot;
  int sh_vcount, sh_sum, sh_mn, sh_mx, smem_bytes;
  unsigned int* vrange;  // != null: also record min/max of the (flipped) value bits of the rows (NUNIQUE range)
  uint32_t vflip;
};

// Value of row r as raw bits, and its order-preserving encoding (64-bit form,
// as in the global records).
template <int W, bool SGN, bool FLT>
__device__ __forceinline__ uint64_t load_raw(const void* data, int64_t r)
{
  if (W == 1) return __ldcs(static_cast<const unsigned char*>(data) + r);
  if (W == 2) return __ldcs(static_cast<const unsigned short*>(data) + r);
  if (W == 4) return __ldcs(static_cast<const unsigned int*>(data) + r);
  return __ldcs(static_cast<const unsigned long long*>(data) + r);
}
template <int W, bool SGN, bool FLT>
__device__ __forceinline__ uint64_t ordered64(uint64_t raw)
{
  if (FLT) {
    if (W == 4) {
      uint32_t b = static_cast<uint32_t>(raw);
      return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
    }
    return (raw & (1ull << 63)) ? ~raw : (raw | (1ull << 63));
  }
  if (SGN) {
    int64_t v = W == 1 ? static_cast<int8_t>(raw) : W == 2 ? static_cast<int16_t>(raw)
              : W == 4 ? static_cast<int32_t>(raw) : static_cast<int64_t>(raw);
    return static_cast<uint64_t>(v) ^ (1ull << 63);
  }
  return raw;
}
// 32-bit ordered form for <= 4-byte types (shared-memory min/max)
template <int W, bool SGN, bool FLT>
__device__ __forceinline__ uint32_t ordered32(uint64_t raw)
{
  if (FLT) {
    uint32_t b = static_cast<uint32_t>(raw);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
  }
  if (SGN) {
    int32_t v = W == 1 ? static_cast<int8_t>(raw) : W == 2 ? static_cast<int16_t>(raw) : static_cast<int32_t>(raw);
    return static_cast<uint32_t>(v) ^ 0x80000000u;
  }
  return static_cast<uint32_t>(raw);
}

template <int W, bool SGN, bool FLT>
__global__ void __launch_bounds__(kGbThreads) column_kernel(ColArgs a)
{
  extern __shared__ __align__(16) unsigned char smem[];
  {
    uint32_t* z = reinterpret_cast<uint32_t*>(smem);
    for (int i = threadIdx.x; i < a.smem_bytes / 4; i += blockDim.x) z[i] = 0;
  }
  __syncthreads();
  constexpr bool MM64 = W > 4;
  const int H         = a.hot;
  const int64_t step  = static_cast<int64_t>(gridDim.x) * blockDim.x * kRows;
  uint32_t vlo = 0xffffffffu, vhi = 0;
  for (int64_t base = (static_cast<int64_t>(blockIdx.x) * blockDim.x) * kRows; base < a.n; base += step) {
    uint32_t g[kRows];
    uint64_t raw[kRows];
    bool ok[kRows];
#pragma unroll
    for (int j = 0; j < kRows; ++j) {
      const int64_t r = base + static_cast<int64_t>(j) * blockDim.x + threadIdx.x;
      ok[j]           = r < a.n;
      g[j] = ok[j] ? __ldcs(a.gid + r) : kUnsetId;
      if (g[j] != kUnsetId) g[j] = __ldg(a.newid + g[j]);
      raw[j] = ok[j] ? load_raw<W, SGN, FLT>(a.col.data, r) : 0;
      if (ok[j] && a.nullable) ok[j] = __ldcs(a.col.valid + r) != 0;
      ok[j] = ok[j] && g[j] != kUnsetId;
    }
    if (W <= 4 && a.vrange) {
#pragma unroll
      for (int j = 0; j < kRows; ++j)
        if (ok[j]) {
          const uint32_t x = static_cast<uint32_t>(raw[j]) ^ a.vflip;
          vlo              = min(vlo, x);
          vhi              = max(vhi, x);
        }
    }
#pragma unroll
    for (int j = 0; j < kRows; ++j) {
      if (!ok[j]) continue;
      const uint32_t gg = g[j];
      if (gg < static_cast<uint32_t>(H)) {
        if (a.nullable) atomicAdd(reinterpret_cast<uint32_t*>(smem + a.sh_vcount) + gg, 1u);
        if (a.states & ST_SUM) {
          uint32_t* sum = reinterpret_cast<uint32_t*>(smem + a.sh_sum) + static_cast<int64_t>(gg) * a.sum_chunks * 4;
          if (FLT) {
            const double x = W == 8 ? __longlong_as_double(static_cast<long long>(raw[j]))
                                    : static_cast<double>(__uint_as_float(static_cast<uint32_t>(raw[j])));
            uint64_t m;
            int sh;
            bool neg;
            if (fixed_parts(x, m, sh, neg)) {
              if (m) {
                const int j0 = sh >> 5, b = sh & 31;
                sh_add_magnitude(sum, a.sum_chunks, j0, m << b, b ? (m >> (64 - b)) : 0, neg);
              }
            } else if (isnan(x)) {
              atomicOr(a.special + gg, SP_NAN);
            } else if (isinf(x)) {
              atomicOr(a.special + gg, x > 0 ? SP_PINF : SP_NINF);
            } else {
              atomicAdd(a.fb + gg, x);
            }
          } else {
            uint64_t mag = raw[j];
            bool neg     = false;
            if (SGN) {
              const int64_t v = W == 1 ? static_cast<int8_t>(raw[j]) : W == 2 ? static_cast<int16_t>(raw[j])
                              : W == 4 ? static_cast<int32_t>(raw[j]) : static_cast<int64_t>(raw[j]);
              neg = v < 0;
              mag = neg ? (0ull - static_cast<uint64_t>(v)) : static_cast<uint64_t>(v);
            }
            sh_add_magnitude(sum, a.sum_chunks, 0, mag, 0, neg);
          }
        }
        if (a.states & (ST_MIN | ST_MAX)) {
          if (MM64) {
            const uint64_t o = ordered64<W, SGN, FLT>(raw[j]);
            if (a.states & ST_MIN) atomicMax(reinterpret_cast<unsigned long long*>(smem + a.sh_mn) + gg, ~o);
            if (a.states & ST_MAX) atomicMax(reinterpret_cast<unsigned long long*>(smem + a.sh_mx) + gg, o);
          } else {
            const uint32_t o = ordered32<W, SGN, FLT>(raw[j]);
            if (a.states & ST_MIN) atomicMax(reinterpret_cast<uint32_t*>(smem + a.sh_mn) + gg, ~o);
            if (a.states & ST_MAX) atomicMax(reinterpret_cast<uint32_t*>(smem + a.sh_mx) + gg, o);
          }
        }
      } else {
        unsigned long long* rec = a.rec + static_cast<uint64_t>(gg) * a.cw;
        const uint64_t L        = a.ld;
        if (a.nullable) red_add(rec + a.off_vcount * L, 1);
        if (a.states & ST_SUM) {
          if (FLT) {
            const double x = W == 8 ? __longlong_as_double(static_cast<long long>(raw[j]))
                                    : static_cast<double>(__uint_as_float(static_cast<uint32_t>(raw[j])));
            uint64_t m;
            int sh;
            bool neg;
            if (fixed_parts(x, m, sh, neg)) add_fixed_chunks(rec + a.off_sum * L, m, sh, neg, L);
            else if (isnan(x)) atomicOr(a.special + gg, SP_NAN);
            else if (isinf(x)) atomicOr(a.special + gg, x > 0 ? SP_PINF : SP_NINF);
            else atomicAdd(a.fb + gg, x);
          } else {
            uint64_t v = raw[j];
            if (SGN) {
              const int64_t sv = W == 1 ? static_cast<int8_t>(raw[j]) : W == 2 ? static_cast<int16_t>(raw[j])
                               : W == 4 ? static_cast<int32_t>(raw[j]) : static_cast<int64_t>(raw[j]);
              v = static_cast<uint64_t>(sv);
            }
            red_add(rec + a.off_sum * L, v);
          }
        }
        if (a.states & (ST_MIN | ST_MAX)) {
          const uint64_t o = ordered64<W, SGN, FLT>(raw[j]);
          if (a.states & ST_MIN) red_max(rec + a.off_mn * L, ~o);
          if (a.states & ST_MAX) red_max(rec + a.off_mx * L, o);
        }
      }
    }
  }
  if (W <= 4 && a.vrange) {
    for (int o = 16; o > 0; o >>= 1) {
      vlo = min(vlo, __shfl_xor_sync(0xffffffffu, vlo, o));
      vhi = max(vhi, __shfl_xor_sync(0xffffffffu, vhi, o));
    }
    if ((threadIdx.x & 31) == 0 && vlo <= vhi) {
      atomicMin(a.vrange, vlo);
      atomicMax(a.vrange + 1, vhi);
    }
  }
  __syncthreads();
  for (int gg = threadIdx.x; gg < H; gg += blockDim.x) {
    unsigned long long* rec = a.rec + static_cast<uint64_t>(gg) * a.cw;
    const uint64_t L        = a.ld;
    if (a.nullable) {
      const uint32_t vc = reinterpret_cast<const uint32_t*>(smem + a.sh_vcount)[gg];
      if (vc == 0) continue;
      red_add(rec + a.off_vcount * L, vc);
    }
    if (a.states & ST_SUM) {
      const uint32_t* sum = reinterpret_cast<const uint32_t*>(smem + a.sh_sum) + static_cast<int64_t>(gg) * a.sum_chunks * 4;
      if (FLT) {
        for (int q = 0; q < a.sum_chunks; ++q) {
          const int64_t pos = static_cast<int64_t>(sum[q * 4 + 0]) + (static_cast<int64_t>(sum[q * 4 + 1]) << 32);
          const int64_t neg = static_cast<int64_t>(sum[q * 4 + 2]) + (static_cast<int64_t>(sum[q * 4 + 3]) << 32);
          if (pos != neg) red_add(rec + (a.off_sum + q) * L, static_cast<uint64_t>(pos - neg));
        }
      } else {
        uint64_t tot = 0;  // integer sum mod 2^64
        for (int q = 0; q < a.sum_chunks; ++q) {
          const uint64_t pos = static_cast<uint64_t>(sum[q * 4 + 0]) + (static_cast<uint64_t>(sum[q * 4 + 1]) << 32);
          const uint64_t neg = static_cast<uint64_t>(sum[q * 4 + 2]) + (static_cast<uint64_t>(sum[q * 4 + 3]) << 32);
          tot += (pos - neg) << (32 * q);
        }
        if (tot) red_add(rec + a.off_sum * L, tot);
      }
    }
    if (a.states & (ST_MIN | ST_MAX)) {
      // groups of a non-nullable column reach here with or without rows in
      // this CTA: an untouched max word 0 is the identity either way
      if (MM64) {
        if (a.states & ST_MIN) red_max(rec + a.off_mn * L, reinterpret_cast<const unsigned long long*>(smem + a.sh_mn)[gg]);
        if (a.states & ST_MAX) red_max(rec + a.off_mx * L, reinterpret_cast<const unsigned long long*>(smem + a.sh_mx)[gg]);
      } else {
        const uint32_t mn = reinterpret_cast<const uint32_t*>(smem + a.sh_mn)[gg];
        const uint32_t mx = reinterpret_cast<const uint32_t*>(smem + a.sh_mx)[gg];
        // an untouched word (no row of this group here) flushes the identity
        // of the opposite extreme, which never wins
        if (a.states & ST_MIN) red_max(rec + a.off_mn * L, ~widen32<W, SGN, FLT>(~mn));
        if (a.states & ST_MAX) red_max(rec + a.off_mx * L, widen32<W, SGN, FLT>(mx));
      }
    }
  }
}

// ---- NUNIQUE: dedupe the (group id, value) pairs -----------------------------
// The `hb` most frequent ranks keep one bit per value of the column's value
// range ([vbase, vbase + 32 * wpr) after the order-preserving flip): a row sets
// its bit with a fire-and-forget OR (the bitmaps stay L2-resident) and a
// popcount pass counts them.  Pairs (rank << 32 | value32) of the other ranks
// go into a pair set; first insertions count per rank (ranks below `hot` in
// shared memory first).  Eight rows per thread with their first probes in
// flight together.
constexpr int kPairsPerThread = 8;
struct NdArgs {
  const uint32_t* gid;
  const uint32_t* newid;
  DCol col;
  int64_t n;
  unsigned long long* set;
  uint64_t cap;
  unsigned long long* nd;  // distinct-count field (indexed by frequency rank)
  int hot;
  int* overflow;
  uint32_t* bits;  // hb x wpr bitmap words
  uint32_t hb;
  uint32_t wpr;
  uint32_t vbase;
  uint32_t flip;  // 0x80000000 for signed 32-bit values, else 0
  // ranks >= s0 scatter their values into per-rank segments
  uint32_t s0;
  unsigned long long* seg_cursor;  // [rank - s0]: next free position of the segment
  uint32_t* seg_vals;
};

__device__ __forceinline__ void red_or32(uint32_t* p, uint32_t v)
{
  asm volatile("red.relaxed.gpu.global.or.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Raw bits of a W-byte value (W known at compile time, so the loads of an
// unrolled loop issue together).
template <int W>
__device__ __forceinline__ uint32_t load_bits(const void* data, int64_t r)
{
  if (W == 1) return __ldcs(static_cast<const uint8_t*>(data) + r);
  if (W == 2) return __ldcs(static_cast<const uint16_t*>(data) + r);
  return __ldcs(static_cast<const uint32_t*>(data) + r);
}

template <int W>
__global__ void __launch_bounds__(kGbThreads, 2) nunique_kernel(NdArgs a)
{
  extern __shared__ __align__(16) unsigned char smem[];
  uint32_t* cnt = reinterpret_cast<uint32_t*>(smem);
  for (int i = threadIdx.x; i < a.hot; i += blockDim.x) cnt[i] = 0;
  __syncthreads();
  const int64_t per_block = static_cast<int64_t>(blockDim.x) * kPairsPerThread;
  for (int64_t base = blockIdx.x * per_block; base < a.n; base += static_cast<int64_t>(gridDim.x) * per_block) {
    uint64_t e[kPairsPerThread], v[kPairsPerThread];
    uint32_t g[kPairsPerThread], x[kPairsPerThread];
    // independent loads first: group id, value, validity of every row
#pragma unroll
    for (int j = 0; j < kPairsPerThread; ++j) {
      const int64_t r = base + j * blockDim.x + threadIdx.x;
      g[j]            = kUnsetId;
      x[j]            = 0;
      if (r < a.n) {
        g[j] = __ldcs(a.gid + r);
        x[j] = load_bits<W>(a.col.data, r);
        if (a.col.valid != nullptr && __ldcs(a.col.valid + r) == 0) g[j] = kUnsetId;
      }
    }
    // then the rank of each group (eight dependent loads in flight)
#pragma unroll
    for (int j = 0; j < kPairsPerThread; ++j) g[j] = g[j] != kUnsetId ? __ldg(a.newid + g[j]) : kUnsetId;
    // v[j] first holds the segment position of a scattered row (bit j of scat)
    uint32_t scat = 0;
#pragma unroll
    for (int j = 0; j < kPairsPerThread; ++j) {
      e[j] = kEmpty;
      if (g[j] != kUnsetId) {
        if (g[j] < a.hb) {
          const uint32_t off = (x[j] ^ a.flip) - a.vbase;
          red_or32(a.bits + static_cast<uint64_t>(g[j]) * a.wpr + (off >> 5), 1u << (off & 31));
        } else if (g[j] >= a.s0) {
          v[j] = atomicAdd(a.seg_cursor + (g[j] - a.s0), 1ull);  // eight in flight
          scat |= 1u << j;
        } else {
          e[j] = (static_cast<uint64_t>(g[j]) << 32) | x[j];
        }
      }
    }
#pragma unroll
    for (int j = 0; j < kPairsPerThread; ++j)
      if (scat & (1u << j)) a.seg_vals[v[j]] = x[j];
#pragma unroll
    for (int j = 0; j < kPairsPerThread; ++j)
      if (e[j] != kEmpty) v[j] = a.set[fastrange(mix64(e[j]), a.cap)];
#pragma unroll
    for (int j = 0; j < kPairsPerThread; ++j) {
      if (e[j] == kEmpty) continue;
      bool fresh = false;
      uint64_t xs = fastrange(mix64(e[j]), a.cap), cur = v[j];
      int probe   = 0;
      for (; probe < kMaxProbe; ++probe) {
        if (cur == e[j]) break;
        if (cur == kEmpty) {
          cur = atomicCAS(a.set + xs, kEmpty, e[j]);
          if (cur == kEmpty) {
            fresh = true;
            break;
          }
          if (cur == e[j]) break;
        }
        xs  = xs + 1 == a.cap ? 0 : xs + 1;
        cur = a.set[xs];
      }
      if (probe == kMaxProbe) atomicExch(a.overflow, 1);
      if (!fresh) continue;
      const uint32_t rk = static_cast<uint32_t>(e[j] >> 32);
      if (rk < static_cast<uint32_t>(a.hot)) atomicAdd(cnt + rk, 1u);
      else red_add(a.nd + rk, 1);
    }
  }
  __syncthreads();
  for (int gg = threadIdx.x; gg < a.hot; gg += blockDim.x)
    if (cnt[gg]) red_add(a.nd + gg, cnt[gg]);
}

// Range of the (flipped) W-byte values of the valid rows: out[0] = min,
// out[1] = max.  Eight strided rows per thread and step keep eight loads in
// flight.
template <int W>
__global__ void value_range_kernel(DCol col, int64_t n, uint32_t flip, unsigned int* out)
{
  constexpr int kU = 8;
  uint32_t lo = 0xffffffffu, hi = 0;
  const int64_t nth = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t base = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; base < n; base += kU * nth) {
    uint32_t x[kU];
    bool ok[kU];
#pragma unroll
    for (int j = 0; j < kU; ++j) {
      const int64_t r = base + j * nth;
      ok[j]           = r < n;
      x[j]            = ok[j] ? load_bits<W>(col.data, r) ^ flip : 0u;
      if (ok[j] && col.valid != nullptr) ok[j] = __ldg(col.valid + r) != 0;
    }
#pragma unroll
    for (int j = 0; j < kU; ++j)
      if (ok[j]) {
        lo = min(lo, x[j]);
        hi = max(hi, x[j]);
      }
  }
  for (int o = 16; o > 0; o >>= 1) {
    lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMin(out, lo);
    atomicMax(out + 1, hi);
  }
}

// ---- NUNIQUE of the per-rank segments ---------------------------------------
// Ranks are in descending row-count order, so each size tier is a contiguous
// rank range.  bounds[k] = first rank whose row count is <= seg_tier(k).
constexpr int kSegTiers                 = 3;
__host__ __device__ constexpr uint64_t seg_tier(int k) { return k == 0 ? 8192 : k == 1 ? 512 : 16; }
constexpr int kSegBlockThreads          = 256;
constexpr int kSegBlockSlots            = 16384;  // shared table of a block (64 KB)
constexpr int kSegWarpSlots             = 1024;   // shared table of a warp (4 KB)
constexpr uint32_t kSegEmpty            = 0xffffffffu;

__global__ void seg_bounds_kernel(const unsigned long long* count, int64_t nid, int64_t* bounds)
{
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < nid; g += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t c = count[g];
    for (int k = 0; k < kSegTiers; ++k)
      if (c <= seg_tier(k) && (g == 0 || count[g - 1] > seg_tier(k))) bounds[k] = g;
  }
}

__device__ __forceinline__ uint32_t seg_hash(uint32_t x, int log2cap)
{
  return (x * 0x9e3779b1u) >> (32 - log2cap);
}

// Insert into a shared open-addressing table; true if x was not there yet.
// The empty marker value itself is tracked by `saw_empty_value`.
__device__ __forceinline__ bool seg_insert(uint32_t* table, int log2cap, uint32_t x, int* saw_empty_value)
{
  if (x == kSegEmpty) return atomicExch(saw_empty_value, 1) == 0;
  const uint32_t mask = (1u << log2cap) - 1u;
  uint32_t i          = seg_hash(x, log2cap);
  for (uint32_t probe = 0; probe <= mask; ++probe) {
    const uint32_t cur = atomicCAS(table + i, kSegEmpty, x);
    if (cur == kSegEmpty) return true;
    if (cur == x) return false;
    i = (i + 1) & mask;
  }
  return false;  // unreachable: the table holds at most half its slots
}

__device__ __forceinline__ int seg_log2cap(uint64_t c, int max_log2)
{
  int l = 6;
  while (l < max_log2 && (1ull << l) < 2 * c) ++l;
  return l;
}

struct SegArgs {
  const unsigned long long* start;  // segment start (exclusive scan of row counts)
  const unsigned long long* end;    // segment end (the cursor after the scatter)
  const uint32_t* vals;
  unsigned long long* nd;           // distinct-count field, indexed by rank
  int64_t s0;                       // rank of segment 0
  int64_t r_begin, r_end;           // ranks of this tier
};

// 512 < rows <= 8192: one CTA per rank.
__global__ void __launch_bounds__(kSegBlockThreads) seg_block_kernel(SegArgs a)
{
  extern __shared__ __align__(16) uint32_t table[];  // kSegBlockSlots entries
  __shared__ int saw;
  __shared__ unsigned int fresh;
  for (int64_t g = a.r_begin + blockIdx.x; g < a.r_end; g += gridDim.x) {
    const uint64_t b = a.start[g - a.s0], e = a.end[g - a.s0];
    const int l2     = seg_log2cap(e - b, 14);
    for (int i = threadIdx.x; i < (1 << l2); i += blockDim.x) table[i] = kSegEmpty;
    if (threadIdx.x == 0) {
      saw   = 0;
      fresh = 0;
    }
    __syncthreads();
    unsigned int mine = 0;
    for (uint64_t i = b + threadIdx.x; i < e; i += blockDim.x) mine += seg_insert(table, l2, a.vals[i], &saw) ? 1u : 0u;
    for (int o = 16; o > 0; o >>= 1) mine += __shfl_xor_sync(0xffffffffu, mine, o);
    if ((threadIdx.x & 31) == 0 && mine) atomicAdd(&fresh, mine);
    __syncthreads();
    if (threadIdx.x == 0) a.nd[g] = fresh;
    __syncthreads();
  }
}

// 16 < rows <= 512: one warp per rank, a 1024-slot table per warp.
__global__ void __launch_bounds__(256) seg_warp_kernel(SegArgs a)
{
  __shared__ uint32_t tables[8][kSegWarpSlots];
  __shared__ int saw[8];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint32_t* table = tables[w];
  const int64_t nw = static_cast<int64_t>(gridDim.x) * 8;
  for (int64_t g = a.r_begin + blockIdx.x * 8 + w; g < a.r_end; g += nw) {
    const uint64_t b = a.start[g - a.s0], e = a.end[g - a.s0];
    const int l2     = seg_log2cap(e - b, 10);
    for (int i = lane; i < (1 << l2); i += 32) table[i] = kSegEmpty;
    if (lane == 0) saw[w] = 0;
    __syncwarp();
    unsigned int mine = 0;
    for (uint64_t i = b + lane; i < e; i += 32) mine += seg_insert(table, l2, a.vals[i], &saw[w]) ? 1u : 0u;
    for (int o = 16; o > 0; o >>= 1) mine += __shfl_xor_sync(0xffffffffu, mine, o);
    if (lane == 0) a.nd[g] = mine;
    __syncwarp();
  }
}

// rows <= 16: one thread per rank, pairwise comparison.
__global__ void seg_thread_kernel(SegArgs a)
{
  for (int64_t g = a.r_begin + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < a.r_end;
       g += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t b = a.start[g - a.s0], e = a.end[g - a.s0];
    unsigned int d   = 0;
    for (uint64_t i = b; i < e; ++i) {
      const uint32_t x = a.vals[i];
      bool dup         = false;
      for (uint64_t j = b; j < i && !dup; ++j) dup = a.vals[j] == x;
      d += dup ? 0u : 1u;
    }
    a.nd[g] = d;
  }
}

// Distinct counts of the bitmap ranks: one CTA per rank (grid-stride).
__global__ void bitmap_count_kernel(const uint32_t* bits, uint32_t hb, uint32_t wpr, unsigned long long* nd)
{
  __shared__ unsigned long long part[32];
  for (uint32_t g = blockIdx.x; g < hb; g += gridDim.x) {
    const uint4* w4 = reinterpret_cast<const uint4*>(bits + static_cast<uint64_t>(g) * wpr);
    unsigned long long c = 0;
    for (uint32_t i = threadIdx.x; i < wpr / 4; i += blockDim.x) {
      const uint4 q = w4[i];
      c += __popc(q.x) + __popc(q.y) + __popc(q.z) + __popc(q.w);
    }
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
      unsigned long long t = 0;
      for (int i = 0; i < static_cast<int>(blockDim.x >> 5); ++i) t += part[i];
      if (t) red_add(nd + g, t);
    }
    __syncthreads();
  }
}

// NUNIQUE of 8-byte or string values: pairs hashed on (group, value) with the
// representative row in the set (generic, slower path).
template <KeyMode M>
__global__ void nunique_generic_kernel(GbPlan p, ColPlan c, const uint32_t* gid, const uint32_t* newid,
                                       unsigned long long* nd)
{
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < p.n; r += (int64_t)gridDim.x * blockDim.x) {
    if (!dvalid(c.col, r)) continue;
    uint32_t g = gid[r];
    if (g == kUnsetId) continue;
    g = newid[g];
    if (pair_insert(p, c, g, r)) red_add(nd + g, 1);
  }
}

// ---- cardinality estimate on a strided sample -------------------------------
// Keys (and (key slot, value) pairs of the first COUNT_DISTINCT column) of a
// strided sample are counted in scratch tables; (occupied, singletons) feed
// the estimates.
template <KeyMode M>
__global__ void sample_kernel(KeyCols k, int64_t n_sample, int64_t stride, unsigned long long* slots, uint64_t cap,
                              unsigned int* counts, ColPlan pc, int with_pairs, unsigned int* pair_counts)
{
  const uint64_t empty = M == KeyMode::K64 ? kSentinel64 : kEmpty;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n_sample;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = i * stride;
    int64_t g       = -1;
    if (M != KeyMode::GEN && !dvalid(k.c[0], r)) {
      g = static_cast<int64_t>(cap);
    } else {
      const uint64_t kb = key_bits<M>(k, r);
      uint64_t word, h;
      if (M == KeyMode::GEN) {
        h    = kb;
        word = (static_cast<uint64_t>(r) << 32) | static_cast<uint32_t>(h);
      } else {
        h    = mix64(kb);
        word = M == KeyMode::K32 ? (kb | (1ull << 32)) : kb;
      }
      if (M == KeyMode::K64 && kb == kSentinel64) {
        g = static_cast<int64_t>(cap) + 1;
      } else {
        uint64_t idx = fastrange(h, cap);
        for (int probe = 0; probe < kMaxProbe; ++probe) {
          uint64_t v = slots[idx];
          if (v == empty) {
            v = atomicCAS(&slots[idx], empty, word);
            if (v == empty) {
              g = static_cast<int64_t>(idx);
              break;
            }
          }
          bool same = M == KeyMode::GEN ? (static_cast<uint32_t>(v) == static_cast<uint32_t>(h) &&
                                           keys_equal(k, r, k, static_cast<int64_t>(v >> 32)))
                                        : v == word;
          if (same) {
            g = static_cast<int64_t>(idx);
            break;
          }
          idx = idx + 1 == cap ? 0 : idx + 1;
        }
      }
    }
    if (g < 0) continue;
    {
      // lanes of the warp that sampled the same key add once (the most
      // frequent keys would otherwise serialize on one counter)
      const uint32_t active = __activemask();
      const uint32_t peers  = __match_any_sync(active, static_cast<unsigned long long>(g));
      if ((threadIdx.x & 31) == static_cast<unsigned>(__ffs(peers) - 1))
        atomicAdd(&counts[g], static_cast<unsigned>(__popc(peers)));
    }
    if (with_pairs && dvalid(pc.col, r)) {
      uint64_t entry, h;
      if (pc.pair_packed) {
        entry = (static_cast<uint64_t>(g) << 32) | static_cast<uint32_t>(dbits(pc.col, r));
        h     = mix64(entry);
      } else {
        h     = hash_combine64(mix64(static_cast<uint64_t>(g)), hash_value(pc.col, r));
        entry = (static_cast<uint64_t>(r) << 32) | static_cast<uint32_t>(h);
      }
      uint64_t idx = fastrange(h, pc.pair_cap);
      for (int probe = 0; probe < kMaxProbe; ++probe) {
        uint64_t v = pc.pairs[idx];
        if (v == kEmpty) {
          v = atomicCAS(&pc.pairs[idx], kEmpty, entry);
          if (v == kEmpty) {
            atomicAdd(&pair_counts[idx], 1u);
            break;
          }
        }
        bool same;
        if (pc.pair_packed) same = v == entry;
        else {
          int64_t o = static_cast<int64_t>(v >> 32);
          same = static_cast<uint32_t>(v) == static_cast<uint32_t>(h) && keys_equal(k, r, k, o) &&
                 values_equal(pc.col, r, pc.col, o);
        }
        if (same) {
          atomicAdd(&pair_counts[idx], 1u);
          break;
        }
        idx = idx + 1 == pc.pair_cap ? 0 : idx + 1;
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

// p[i] = {a, b} for i < n (16-byte stores)
__global__ void fill_pairs_kernel(ulonglong2* p, int64_t n, unsigned long long a, unsigned long long b)
{
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    p[i] = make_ulonglong2(a, b);
}

template <typename T>
__global__ void fill_kernel(T* p, int64_t n, T v)
{
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    p[i] = v;
}

// p[i] = i (ranks of a small input: its assign-pass ids)
__global__ void iota_kernel(int32_t* p, int64_t n)
{
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    p[i] = static_cast<int32_t>(i);
}

// ---- frequency ranks --------------------------------------------------------
// key = ~count: an ascending stable sort puts the most frequent ids first and
// unused ids (holes, count 0) last.
__global__ void rank_keys_kernel(const unsigned long long* counts, int64_t nid, uint32_t* key)
{
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nid; i += (int64_t)gridDim.x * blockDim.x)
    key[i] = ~static_cast<uint32_t>(counts[i]);
}
// newid[perm[i]] = i; the count field (field 0) of rank i
__global__ void rank_scatter_kernel(const int32_t* perm, int64_t nid, const unsigned long long* counts,
                                    uint32_t* newid, unsigned long long* count_field)
{
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nid; i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t old = perm[i];
    newid[old]        = static_cast<uint32_t>(i);
    count_field[i]    = counts[old];
  }
}

// ---- compaction of the used ids (record count > 0) ---------------------------
__global__ void __launch_bounds__(256)
  compact_groups_kernel(const unsigned long long* states, int stride, int64_t nid, int64_t* groups,
                        uint64_t* status, unsigned long long* counter, int64_t* total, int* err)
{
  constexpr int ITEMS = 4;
  __shared__ int64_t s_scan[256 / 32 + 1];
  __shared__ int64_t s_tile;
  __shared__ uint64_t s_prefix;
  const int64_t tile = next_tile_id(counter, &s_tile);
  const int64_t base = tile * (256 * ITEMS) + static_cast<int64_t>(threadIdx.x) * ITEMS;
  int f[ITEMS];
  int64_t c = 0;
#pragma unroll
  for (int i = 0; i < ITEMS; ++i) {
    const int64_t j = base + i;
    f[i]            = (j < nid && states[j * stride] > 0) ? 1 : 0;
    c += f[i];
  }
  int64_t tot;
  int64_t ex = block_exclusive_scan<int64_t, 256>(c, s_scan, &tot);
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

// ---- finalize --------------------------------------------------------------
struct AggOut {
  int kind;
  int count_mode;
  int col;  // ColPlan index (-1 for COUNT_ALL)
  int in_type;
  OCol dst;
};
struct FinArgs {
  GbPlan p;
  const unsigned long long* rec;  // field-major records of the frequency ranks
  uint64_t ld;
  const int32_t* perm;            // rank -> assign-pass id
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

__device__ __forceinline__ double float_sum(const ColPlan& c, const unsigned long long* rec, uint64_t L, int64_t id,
                                            bool& special, double& sval)
{
  unsigned int sp = c.special[id];
  special         = sp != 0;
  if (special) {
    if ((sp & SP_NAN) || ((sp & SP_PINF) && (sp & SP_NINF))) sval = __longlong_as_double(0x7ff8000000000000ll);
    else sval = (sp & SP_PINF) ? __longlong_as_double(0x7ff0000000000000ll)
                               : __longlong_as_double(0xfff0000000000000ll);
  }
  return chunks_to_double(rec + c.off_sum * L, L) + c.fb[id];
}

__global__ void finalize_kernel(FinArgs f)
{
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < f.ngroups;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t id              = f.groups[i];  // frequency rank
    const GbPlan& p               = f.p;
    const uint64_t L              = f.ld;
    const unsigned long long* rec = f.rec + id;
    const int64_t old             = f.perm[id];  // assign-pass id
    // keys
    if (f.key_mode == static_cast<int>(KeyMode::GEN)) {
      const int64_t rr = static_cast<int64_t>(p.id_key[old]);
      f.repr[i]        = static_cast<int32_t>(rr);
      for (int j = 0; j < f.nkeys; ++j) {
        const OCol& d = f.key_dst[j];
        if (d.type == LDF_STRING) continue;
        copy_fixed(d.data, i, p.k.c[j].data, rr, d.width);
        if (d.valid) d.valid[i] = dvalid(p.k.c[j], rr) ? 1 : 0;
      }
    } else {
      const OCol& d      = f.key_dst[0];
      const bool is_null = old == kIdNull;
      const uint64_t kb  = old == kIdSentinel ? kSentinel64 : is_null ? 0 : p.id_key[old];
      store_int(OCol{d.data, nullptr, LDF_UINT64, d.width}, i, kb);
      if (d.valid) d.valid[i] = is_null ? 0 : 1;
    }
    const uint64_t call = rec[0];
    // the exact float sum of a column, rounded once, is shared by its SUM and MEAN
    int sum_col      = -1;
    double sum_val   = 0.0;
    bool sum_special = false;
    double sum_sval  = 0.0;
    for (int a = 0; a < f.nagg; ++a) {
      const AggOut& o = f.a[a];
      const OCol& d   = o.dst;
      if (o.kind == LDF_AGG_COUNT_ALL) {
        store_int(d, i, call);
        if (d.valid) d.valid[i] = 1;
        continue;
      }
      const ColPlan& c               = p.c[o.col];
      const unsigned long long* crec = c.crec + static_cast<uint64_t>(id) * c.cw;
      const uint64_t vc              = c.nullable ? crec[c.off_vcount] : call;
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
          uint64_t nd       = (c.states & ST_NDIST) ? rec[c.off_nd * L] : 0;
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
          if (c.fixed) {
            if (sum_col != o.col) {
              sum_val = float_sum(c, crec, 1, id, sum_special, sum_sval);
              sum_col = o.col;
            }
            double sv = sum_special ? sum_sval : sum_val;
            if (o.kind == LDF_AGG_MEAN) sv = sv / static_cast<double>(vc);
            store_double(d, i, sv);
          } else {
            const uint64_t s = crec[c.off_sum];
            const double sd  = is_signed_int_dev(o.in_type) ? static_cast<double>(static_cast<int64_t>(s))
                                                            : static_cast<double>(s);
            if (o.kind == LDF_AGG_MEAN) store_double(d, i, sd / static_cast<double>(vc));
            else if (d.type == LDF_FLOAT64 || d.type == LDF_FLOAT32) store_double(d, i, sd);
            else store_int(d, i, s);
          }
          break;
        }
        case LDF_AGG_MIN:
        case LDF_AGG_MAX: {
          if (!ok) {
            store_int(d, i, 0);
            break;
          }
          const uint64_t o64 = o.kind == LDF_AGG_MIN ? ~crec[c.off_mn] : crec[c.off_mx];
          const uint64_t b   = unordered_bits(o.in_type, o64);
          if (d.type == o.in_type) {
            store_int(OCol{d.data, nullptr, LDF_UINT64, d.width}, i, b);
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

void launch_column(ColArgs& a, int type, cudaStream_t s)
{
  auto go = [&](auto kernel) {
    LDF_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024));
    int occ = 1;
    LDF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, kGbThreads, a.smem_bytes));
    const int64_t blocks = std::min<int64_t>(static_cast<int64_t>(num_sms()) * std::max(occ, 1),
                                             ceil_div(a.n, int64_t(kGbThreads) * kRows));
    launch("column", kernel, static_cast<unsigned>(blocks), kGbThreads, static_cast<size_t>(a.smem_bytes), s, a);
  };
  switch (type) {
    case LDF_BOOL8:
    case LDF_UINT8: go(column_kernel<1, false, false>); break;
    case LDF_INT8: go(column_kernel<1, true, false>); break;
    case LDF_UINT16: go(column_kernel<2, false, false>); break;
    case LDF_INT16: go(column_kernel<2, true, false>); break;
    case LDF_UINT32: go(column_kernel<4, false, false>); break;
    case LDF_INT32: go(column_kernel<4, true, false>); break;
    case LDF_FLOAT32: go(column_kernel<4, false, true>); break;
    case LDF_UINT64: go(column_kernel<8, false, false>); break;
    case LDF_INT64:
    case LDF_TIMESTAMP_US: go(column_kernel<8, true, false>); break;
    case LDF_FLOAT64: go(column_kernel<8, false, true>); break;
    default: fail(LDF_ERR_UNSUPPORTED, "unsupported aggregation column type");
  }
}

template <KeyMode M>
void run_groupby(const OpContext& ctx, GbPlan p, const ldf_column* table, const int32_t* keys, int nkeys,
                 const ldf_aggregation* aggs, int naggs, const std::vector<int>& agg_col, ldf_column* out,
                 const HostStaging& hs, const std::vector<int>& col_of_plan)
{
  // host-resident inputs: wait for a column's copy right before its first reader
  auto wait_keys = [&]() {
    for (int j = 0; j < nkeys; ++j) hs.wait(keys[j]);
  };
  auto wait_plan_col = [&](int ci) { hs.wait(col_of_plan[ci]); };
  const Allocator& al = ctx.alloc();
  cudaStream_t s      = ctx.stream();
  const int64_t n     = p.n;

  int ndist_col = -1;
  for (int ci = 0; ci < p.ncols; ++ci)
    if (p.c[ci].states & ST_NDIST) {
      ndist_col = ci;
      break;
    }

  // ---- estimate #groups and #(group, value) pairs ----------------------------
  int64_t est_groups = n, est_pairs = n;
  const int64_t kSampleMax = int64_t(1) << 20;
  if (n > (int64_t(1) << 16)) {
    const int64_t ns     = std::min<int64_t>(n, kSampleMax);
    const int64_t stride = n / ns;
    const uint64_t scap  = static_cast<uint64_t>(2 * ns + 64);
    Buffer<unsigned long long> sslots(al, scap);
    Buffer<unsigned int> scounts(al, scap + 2);
    if (M == KeyMode::K64)
      launch("fill", fill_kernel<unsigned long long>, gs_blocks(scap, 256), 256, 0, s, sslots.get(),
             static_cast<int64_t>(scap), kSentinel64);
    else
      LDF_CUDA(cudaMemsetAsync(sslots.get(), 0xff, scap * 8, s));
    LDF_CUDA(cudaMemsetAsync(scounts.get(), 0, (scap + 2) * 4, s));
    ColPlan pc{};
    Buffer<unsigned long long> spairs;
    Buffer<unsigned int> spcounts;
    if (ndist_col >= 0) {
      pc          = p.c[ndist_col];
      pc.pair_cap = static_cast<uint64_t>(2 * ns + 64);
      spairs      = Buffer<unsigned long long>(al, pc.pair_cap);
      spcounts    = Buffer<unsigned int>(al, pc.pair_cap);
      LDF_CUDA(cudaMemsetAsync(spairs.get(), 0xff, pc.pair_cap * 8, s));
      LDF_CUDA(cudaMemsetAsync(spcounts.get(), 0, pc.pair_cap * 4, s));
      pc.pairs = spairs.get();
    }
    wait_keys();
    if (ndist_col >= 0) wait_plan_col(ndist_col);
    launch("sample", sample_kernel<M>, gs_blocks(ns, 256), 256, 0, s, p.k, ns, stride, sslots.get(), scap,
           scounts.get(), pc, ndist_col >= 0 ? 1 : 0, spcounts.get());
    Buffer<unsigned long long> stats(al, 4);
    LDF_CUDA(cudaMemsetAsync(stats.get(), 0, 32, s));
    launch("freq_stats", freq_stats_kernel, gs_blocks(scap + 2, 256), 256, 0, s, scounts.get(),
           static_cast<int64_t>(scap + 2), stats.get());
    if (ndist_col >= 0)
      launch("freq_stats", freq_stats_kernel, gs_blocks(pc.pair_cap, 256), 256, 0, s, spcounts.get(),
             static_cast<int64_t>(pc.pair_cap), stats.get() + 2);
    unsigned long long h[4];
    LDF_CUDA(cudaMemcpyAsync(h, stats.get(), 32, cudaMemcpyDeviceToHost, s));
    ctx.finish();
    // GEE (Charikar et al. 2000) for the groups, taken x4 below because it
    // underestimates heavy tails (a table that turns out too small overflows
    // and the pass re-runs with 4x the slots); (group, value) pairs are mostly unique in a
    // sample, where GEE fails, so they use the scale-up d * N / n, an
    // overestimate whenever pairs repeat.
    const double scale = std::sqrt(static_cast<double>(n) / static_cast<double>(ns));
    est_groups         = static_cast<int64_t>(scale * h[1] + (h[0] - h[1])) + 1;
    est_pairs          = static_cast<int64_t>(static_cast<double>(h[2]) * n / ns) + 1;
    est_groups         = std::min<int64_t>(est_multiplier() * est_groups, n);
    est_pairs          = std::min<int64_t>(est_pairs, n);
  }
  if (std::getenv("LDF_B200_DEBUG"))
    std::fprintf(stderr, "[ldf_b200] groupby n=%lld est_groups=%lld est_pairs=%lld\n", static_cast<long long>(n),
                 static_cast<long long>(est_groups), static_cast<long long>(est_pairs));

  uint64_t cap      = static_cast<uint64_t>(std::max<int64_t>(2 * est_groups, 64));
  uint64_t pair_cap = static_cast<uint64_t>(std::max<int64_t>(est_pairs + est_pairs / 2, 64));

  // ---- record layout and shared-memory hot set -------------------------------
  int w = 1;  // shared record: count_all, then the distinct counts
  for (int ci = 0; ci < p.ncols; ++ci) {
    ColPlan& c   = p.c[ci];
    c.sum_chunks = c.fixed ? kSumChunks : 2;
    c.mm64       = type_width(c.col.type) > 4 ? 1 : 0;
    int cw       = 0;  // the column block
    c.off_vcount = c.nullable ? cw++ : 0;
    if (c.states & ST_SUM) {
      c.off_sum = cw;
      cw += c.fixed ? kSumChunks : 1;
    }
    if (c.states & ST_MIN) c.off_mn = cw++;
    if (c.states & ST_MAX) c.off_mx = cw++;
    c.cw = cw;
    if (c.states & ST_NDIST) c.off_nd = w++;
  }
  p.stride = w;
  const int kSmemBudget = 96 * 1024;
  LDF_CUDA(cudaFuncSetAttribute(assign_kernel<M>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBudget));
  int hot_limit = 1 << 30;
  if (const char* e = std::getenv("LDF_B200_GB_HOT")) hot_limit = std::max(0, std::atoi(e));
  // bytes of NUNIQUE value bitmaps (mostly L2-resident; more bitmap ranks
  // beat sending ranks of more than seg_tier(0) rows to the pair set)
  uint64_t bitmap_budget = 96ull << 20;
  if (const char* e = std::getenv("LDF_B200_ND_BITMAP_MB")) bitmap_budget = std::max(0ll, std::atoll(e)) << 20;
  // per-rank segments for the less frequent ranks (LDF_B200_ND_SEGMENTS=0 keeps them in the pair set)
  bool seg_enabled = true;
  if (const char* e = std::getenv("LDF_B200_ND_SEGMENTS")) seg_enabled = std::atoi(e) != 0;
  // Small inputs skip the frequency ranking (ranks = assign-pass ids), so
  // NUNIQUE cannot use the rank-ordered bitmap and segment tiers: every
  // (group, value) pair goes to the pair set.
  const bool small = n <= kSmallPlanRows;
  if (small) {
    bitmap_budget = 0;
    seg_enabled   = false;
  }

  for (int attempt = 0;; ++attempt) {
    const uint64_t id_cap = cap + kIdFirst;
    const int sw          = M == KeyMode::K32 ? 1 : 2;
    Buffer<unsigned long long> slots(al, cap * sw);
    Buffer<unsigned long long> counts(al, id_cap);  // rows per assign-pass id
    Buffer<unsigned long long> id_key(al, id_cap);
    Buffer<unsigned long long> misc(al, 4);  // id counter, overflow, chunk counter
    Buffer<uint32_t> gid(al, std::max<int64_t>(n, 1));
    if (M == KeyMode::K64)  // empty slot: {sentinel key word, no id}
      launch("fill_slots", fill_pairs_kernel, gs_blocks(cap, 256), 256, 0, s,
             reinterpret_cast<ulonglong2*>(slots.get()), static_cast<int64_t>(cap), kSentinel64, kEmpty);
    else
      LDF_CUDA(cudaMemsetAsync(slots.get(), 0xff, cap * sw * 8, s));
    LDF_CUDA(cudaMemsetAsync(counts.get(), 0, static_cast<size_t>(kIdFirst) * 8, s));  // reserved ids
    const unsigned long long first = kIdFirst;
    LDF_CUDA(cudaMemsetAsync(misc.get(), 0, 32, s));
    LDF_CUDA(cudaMemcpyAsync(misc.get(), &first, 8, cudaMemcpyHostToDevice, s));
    p.slots         = slots.get();
    p.cap           = cap;
    p.id_counter    = misc.get();
    p.id_cap        = id_cap;
    p.states        = counts.get();
    p.id_key        = id_key.get();
    p.overflow      = reinterpret_cast<int*>(misc.get() + 1);
    p.chunk_counter = misc.get() + 2;
    p.err           = ctx.err();
    const int hot_cap = static_cast<int>(std::min<uint64_t>(id_cap, static_cast<uint64_t>(hot_limit)));

    std::vector<Buffer<unsigned long long>> pair_bufs;
    std::vector<Buffer<double>> fb_bufs;
    std::vector<Buffer<unsigned int>> sp_bufs;
    for (int ci = 0; ci < p.ncols; ++ci) {
      ColPlan& c = p.c[ci];
      if ((c.states & ST_SUM) && c.fixed) {
        fb_bufs.emplace_back(al, id_cap);
        sp_bufs.emplace_back(al, id_cap);
        LDF_CUDA(cudaMemsetAsync(fb_bufs.back().get(), 0, id_cap * 8, s));
        LDF_CUDA(cudaMemsetAsync(sp_bufs.back().get(), 0, id_cap * 4, s));
        c.fb      = fb_bufs.back().get();
        c.special = sp_bufs.back().get();
      }
      if ((c.states & ST_NDIST) && !c.pair_packed) {  // packed pair sets are sized exactly in pass 3
        c.pair_cap = pair_cap;
        pair_bufs.emplace_back(al, pair_cap);
        c.pairs = pair_bufs.back().get();
        LDF_CUDA(cudaMemsetAsync(c.pairs, 0xff, pair_cap * 8, s));
      }
    }

    Buffer<int32_t> perm;
    Buffer<uint32_t> newid;
    Buffer<unsigned long long> rec;
    std::vector<Buffer<unsigned long long>> col_blocks(p.ncols);
    uint64_t L  = 1;
    int64_t nid = 0;
    if (n > 0) {
      // pass 1: group ids + row counts (per assign-pass id)
      GbPlan pa             = p;
      pa.states             = counts.get();
      pa.stride             = 1;
      pa.hot                = std::min(hot_cap, (kSmemBudget - 64) / 4);
      const size_t a_smem   = static_cast<size_t>(pa.hot) * 4;
      int occ               = 1;
      LDF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, assign_kernel<M>, kGbThreads, a_smem));
      const int64_t ablocks = std::min<int64_t>(static_cast<int64_t>(num_sms()) * std::max(occ, 1),
                                                ceil_div(n, int64_t(kGbThreads) * assign_rows<M>()));
      wait_keys();
      launch("assign", assign_kernel<M>, static_cast<unsigned>(ablocks), kGbThreads, a_smem, s, pa, gid.get());
      unsigned long long hm[2];
      LDF_CUDA(cudaMemcpyAsync(hm, misc.get(), 16, cudaMemcpyDeviceToHost, s));
      ctx.finish();
      if (static_cast<int>(hm[1]) != 0) {
        if (attempt >= 4) fail(LDF_ERR_INTERNAL, "groupby hash table overflow");
        cap      = cap * 4;
        pair_cap = pair_cap * 4;
        continue;
      }
      // the id counter may pass id_cap (pool refills are clipped to it)
      nid = static_cast<int64_t>(std::min<unsigned long long>(hm[0], id_cap));

      // frequency ranks: sort ids by descending row count (stable radix
      // sort).  Small inputs keep the assign-pass ids as ranks: the ranking
      // only decides which groups get shared-memory records, which matters
      // for heavy hitters in large inputs, while its passes and read-back
      // cost more than they save here.
      perm = Buffer<int32_t>(al, nid);
      if (small) {
        launch("iota", iota_kernel, gs_blocks(nid, 256), 256, 0, s, perm.get(), nid);
      } else {
        Buffer<uint32_t> rkey(al, nid);
        launch("rank_keys", rank_keys_kernel, gs_blocks(nid, 256), 256, 0, s,
               static_cast<const unsigned long long*>(counts.get()), nid, rkey.get());
        DCol kc{};
        kc.data  = rkey.get();
        kc.type  = LDF_UINT32;
        kc.width = 4;
        std::vector<RadixPass> passes;
        for (int b = 0; b < 4; ++b) {
          RadixPass rp{};
          rp.src   = DigitSrc::COLUMN;
          rp.shift = 8 * b;
          rp.key   = SortKeyDesc{kc, 0, 1, 4};
          passes.push_back(rp);
        }
        radix_sort_rows(ctx, passes, nid, perm.get());
      }
      newid = Buffer<uint32_t>(al, nid);
      L     = static_cast<uint64_t>(nid);
      rec   = Buffer<unsigned long long>(al, L * p.stride);
      LDF_CUDA(cudaMemsetAsync(rec.get(), 0, L * p.stride * 8, s));
      for (int ci = 0; ci < p.ncols; ++ci) {
        ColPlan& c = p.c[ci];
        if (c.cw == 0) continue;
        col_blocks[ci] = Buffer<unsigned long long>(al, L * c.cw);
        LDF_CUDA(cudaMemsetAsync(col_blocks[ci].get(), 0, L * c.cw * 8, s));
        c.crec = col_blocks[ci].get();
      }
      launch("rank_scatter", rank_scatter_kernel, gs_blocks(nid, 256), 256, 0, s,
             static_cast<const int32_t*>(perm.get()), nid, static_cast<const unsigned long long*>(counts.get()),
             newid.get(), rec.get());

      // pass 2: one kernel per value column that needs valid counts / sums / min / max
      // (a NUNIQUE column of <= 4-byte values also gets its value range here).
      // NUNIQUE columns first: host-resident inputs are copied in that order.
      std::vector<Buffer<unsigned int>> vranges(p.ncols);
      std::vector<int> pass_order;
      for (int ci = 0; ci < p.ncols; ++ci)
        if (p.c[ci].states & ST_NDIST) pass_order.push_back(ci);
      for (int ci = 0; ci < p.ncols; ++ci)
        if (!(p.c[ci].states & ST_NDIST)) pass_order.push_back(ci);
      auto column_pass = [&](int ci) {
        ColPlan& c = p.c[ci];
        if (!c.nullable && !(c.states & (ST_SUM | ST_MIN | ST_MAX))) return;
        ColArgs a{};
        if ((c.states & ST_NDIST) && c.pair_packed) {
          vranges[ci]                  = Buffer<unsigned int>(al, 2);
          const unsigned int init[2]   = {0xffffffffu, 0u};
          LDF_CUDA(cudaMemcpyAsync(vranges[ci].get(), init, 8, cudaMemcpyHostToDevice, s));
          a.vrange = vranges[ci].get();
          a.vflip  = (c.col.width == 4 && is_signed_int(c.col.type)) ? 0x80000000u : 0u;
        }
        a.gid        = gid.get();
        a.newid      = newid.get();
        a.n          = n;
        a.col        = c.col;
        a.nullable   = c.nullable;
        a.states     = c.states & (ST_SUM | ST_MIN | ST_MAX);
        a.sum_chunks = c.sum_chunks;
        a.off_vcount = c.off_vcount;
        a.off_sum    = c.off_sum;
        a.off_mn     = c.off_mn;
        a.off_mx     = c.off_mx;
        a.rec        = c.crec;
        a.ld         = 1;
        a.cw         = c.cw;
        a.fb         = c.fb;
        a.special    = c.special;
        const int mmw = c.mm64 ? 8 : 4;
        const int per = (c.nullable ? 4 : 0) + ((a.states & ST_SUM) ? 16 * c.sum_chunks : 0) +
                        ((a.states & ST_MIN) ? mmw : 0) + ((a.states & ST_MAX) ? mmw : 0);
        a.hot         = static_cast<int>(std::min<int64_t>(std::min(hot_cap, (kSmemBudget - 256) / std::max(per, 1)), nid));
        int off       = 0;
        auto take     = [&](int bytes_per) {
          const int o = off;
          off += (bytes_per * a.hot + 15) & ~15;
          return o;
        };
        a.sh_mn      = (a.states & ST_MIN) && c.mm64 ? take(8) : 0;
        a.sh_mx      = (a.states & ST_MAX) && c.mm64 ? take(8) : 0;
        a.sh_sum     = (a.states & ST_SUM) ? take(16 * c.sum_chunks) : 0;
        a.sh_vcount  = c.nullable ? take(4) : 0;
        if ((a.states & ST_MIN) && !c.mm64) a.sh_mn = take(4);
        if ((a.states & ST_MAX) && !c.mm64) a.sh_mx = take(4);
        a.smem_bytes = off;
        wait_plan_col(ci);
        launch_column(a, c.col.type, s);
      };
      // pass 3: NUNIQUE of one column (after its column pass, which records
      // the value range).  With host-resident inputs it runs right after that
      // pass, before the other columns' passes, so a column still being
      // copied holds back as little work as possible.
      auto nunique_pass = [&](int ci) {
        ColPlan& c = p.c[ci];
        wait_plan_col(ci);
        if (c.pair_packed) {
          NdArgs na{gid.get(), newid.get(), c.col, n, c.pairs, c.pair_cap, rec.get() + c.off_nd * L,
                    static_cast<int>(std::min<int64_t>(std::min(hot_cap, 12 * 1024), nid)), p.overflow};
          // value bitmaps for the most frequent ranks when the value range is small
          na.flip = (c.col.width == 4 && is_signed_int(c.col.type)) ? 0x80000000u : 0u;
          Buffer<unsigned int> vr_own;
          unsigned int* vr = vranges[ci].get();  // set by the column pass when the column had one
          if (vr == nullptr) {
            vr_own                        = Buffer<unsigned int>(al, 2);
            vr                            = vr_own.get();
            const unsigned int vr_init[2] = {0xffffffffu, 0u};
            LDF_CUDA(cudaMemcpyAsync(vr, vr_init, 8, cudaMemcpyHostToDevice, s));
            auto vk = c.col.width == 1 ? value_range_kernel<1> : c.col.width == 2 ? value_range_kernel<2>
                                                                                   : value_range_kernel<4>;
            launch("value_range", vk, static_cast<unsigned>(4 * num_sms()), 256, 0, s, c.col, n, na.flip, vr);
          }
          // size tiers of the ranks (row counts are field 0 of the records)
          Buffer<int64_t> tb(al, kSegTiers);
          {
            const int64_t init[kSegTiers] = {nid, nid, nid};
            LDF_CUDA(cudaMemcpyAsync(tb.get(), init, sizeof(init), cudaMemcpyHostToDevice, s));
            launch("seg_bounds", seg_bounds_kernel, gs_blocks(nid, 256), 256, 0, s,
                   static_cast<const unsigned long long*>(rec.get()), nid, tb.get());
          }
          unsigned int hv[2];
          int64_t tier[kSegTiers];
          LDF_CUDA(cudaMemcpyAsync(hv, vr, 8, cudaMemcpyDeviceToHost, s));
          LDF_CUDA(cudaMemcpyAsync(tier, tb.get(), sizeof(tier), cudaMemcpyDeviceToHost, s));
          ctx.finish();
          Buffer<uint32_t> bits;
          if (hv[0] <= hv[1] && bitmap_budget > 0) {
            const uint64_t range = static_cast<uint64_t>(hv[1]) - hv[0] + 1;
            const uint64_t wpr   = (((range + 31) / 32) + 3) / 4 * 4;  // 16-byte rows
            const uint64_t hb    = std::min<uint64_t>(static_cast<uint64_t>(nid), bitmap_budget / (4 * wpr));
            if (hb >= 8) {
              bits = Buffer<uint32_t>(al, hb * wpr);
              LDF_CUDA(cudaMemsetAsync(bits.get(), 0, hb * wpr * 4, s));
              na.bits  = bits.get();
              na.hb    = static_cast<uint32_t>(hb);
              na.wpr   = static_cast<uint32_t>(wpr);
              na.vbase = hv[0];
            }
          }
          // Ranks [hb, s0) go to the pair set, ranks [s0, nid) (at most
          // seg_tier(0) rows each) to per-rank segments.  The prefix sums of
          // the row counts from hb on give both the exact pair-set bound and
          // the segment offsets.
          na.s0            = 0xffffffffu;
          const int64_t hb = static_cast<int64_t>(na.hb);
          const int64_t s0 = (seg_enabled && n < (int64_t(1) << 32))
                               ? std::min<int64_t>(std::max<int64_t>(hb, tier[0]), nid) : nid;
          Buffer<unsigned long long> seg_start, seg_cursor;
          Buffer<uint32_t> seg_vals;
          Buffer<unsigned long long> pairs;
          int64_t pair_rows = 0;
          if (nid > hb) {
            const int64_t T = nid - hb;
            seg_start       = Buffer<unsigned long long>(al, T);
            Buffer<int64_t> seg_total(al, 1);
            exclusive_scan_i64(reinterpret_cast<const int64_t*>(rec.get() + hb),
                               reinterpret_cast<int64_t*>(seg_start.get()), T, seg_total.get(), ctx);
            int64_t hv2[2] = {0, 0};  // total rows of ranks >= hb, rows of ranks [hb, s0)
            LDF_CUDA(cudaMemcpyAsync(&hv2[0], seg_total.get(), 8, cudaMemcpyDeviceToHost, s));
            if (s0 < nid)
              LDF_CUDA(cudaMemcpyAsync(&hv2[1], seg_start.get() + (s0 - hb), 8, cudaMemcpyDeviceToHost, s));
            ctx.finish();
            const int64_t total = hv2[0];
            pair_rows           = s0 < nid ? hv2[1] : total;
            if (s0 < nid) {
              seg_cursor = Buffer<unsigned long long>(al, nid - s0);
              LDF_CUDA(cudaMemcpyAsync(seg_cursor.get(), seg_start.get() + (s0 - hb), (nid - s0) * 8,
                                       cudaMemcpyDeviceToDevice, s));
              seg_vals      = Buffer<uint32_t>(al, std::max<int64_t>(total, 1));  // indexed by the prefix sums
              na.s0         = static_cast<uint32_t>(s0);
              na.seg_cursor = seg_cursor.get();
              na.seg_vals   = seg_vals.get();
            }
          }
          // distinct pairs of ranks [hb, s0) <= their rows: load factor <= 0.5
          const uint64_t pcap = static_cast<uint64_t>(std::max<int64_t>(64, 2 * pair_rows)) << attempt;
          pairs   = Buffer<unsigned long long>(al, pcap);
          LDF_CUDA(cudaMemsetAsync(pairs.get(), 0xff, pcap * 8, s));
          na.set = pairs.get();
          na.cap = pcap;
          const size_t nd_smem = static_cast<size_t>(na.hot) * 4;
          int nocc             = 1;
          auto ndk = c.col.width == 1 ? nunique_kernel<1> : c.col.width == 2 ? nunique_kernel<2> : nunique_kernel<4>;
          LDF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nocc, ndk, kGbThreads, nd_smem));
          const int64_t nblocks = std::min<int64_t>(static_cast<int64_t>(num_sms()) * std::max(nocc, 1),
                                                    ceil_div(n, int64_t(kGbThreads) * kPairsPerThread));
          launch("nunique", ndk, static_cast<unsigned>(nblocks), kGbThreads, nd_smem, s, na);
          if (na.hb > 0)
            launch("bitmap_count", bitmap_count_kernel, std::min<unsigned>(na.hb, 4u * num_sms()), 256u, 0, s,
                   static_cast<const uint32_t*>(na.bits), na.hb, na.wpr, na.nd);
          if (na.s0 != 0xffffffffu) {
            SegArgs sa{seg_start.get() + (s0 - hb), seg_cursor.get(), seg_vals.get(), na.nd, s0, 0, 0};
            const int64_t m1 = std::max(s0, tier[1]), m2 = std::max(m1, tier[2]);
            sa.r_begin = s0;
            sa.r_end   = m1;
            if (m1 > s0) {
              LDF_CUDA(cudaFuncSetAttribute(seg_block_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            kSegBlockSlots * 4));
              launch("seg_block", seg_block_kernel, static_cast<unsigned>(std::min<int64_t>(m1 - s0, 3 * num_sms())),
                     static_cast<unsigned>(kSegBlockThreads), static_cast<size_t>(kSegBlockSlots) * 4, s, sa);
            }
            sa.r_begin = m1;
            sa.r_end   = m2;
            if (m2 > m1)
              launch("seg_warp", seg_warp_kernel,
                     static_cast<unsigned>(std::min<int64_t>(ceil_div(m2 - m1, 8), 8 * num_sms())), 256u, 0, s, sa);
            sa.r_begin = m2;
            sa.r_end   = nid;
            if (nid > m2) launch("seg_thread", seg_thread_kernel, gs_blocks(nid - m2, 256), 256u, 0, s, sa);
          }
        } else {
          launch("nunique_generic", nunique_generic_kernel<M>, gs_blocks(n, 256), 256, 0, s, p, c,
                 static_cast<const uint32_t*>(gid.get()), static_cast<const uint32_t*>(newid.get()),
                 rec.get() + c.off_nd * L);
        }
      };
      if (hs.staged_bytes() > 0) {
        for (int ci : pass_order) {
          column_pass(ci);
          if (p.c[ci].states & ST_NDIST) nunique_pass(ci);
        }
      } else {  // all inputs on the device: every column pass, then the NUNIQUE passes
        for (int ci : pass_order) column_pass(ci);
        for (int ci : pass_order)
          if (p.c[ci].states & ST_NDIST) nunique_pass(ci);
      }
      if (ndist_col >= 0) {  // only pair-set inserts can overflow after the assign pass
        LDF_CUDA(cudaMemcpyAsync(hm, misc.get(), 16, cudaMemcpyDeviceToHost, s));
        ctx.finish();
      }
      if (ndist_col >= 0 && static_cast<int>(hm[1]) != 0) {  // the pair set overflowed
        if (attempt >= 4) fail(LDF_ERR_INTERNAL, "groupby hash table overflow");
        cap      = cap * 4;
        pair_cap = pair_cap * 4;
        continue;
      }
    }

    // ---- used ranks (count > 0; holes sort last) + finalize ---------------------
    const int64_t tiles = std::max<int64_t>(1, ceil_div(nid, 256 * 4));
    Buffer<int64_t> groups(al, std::max<int64_t>(nid, 1));
    Buffer<uint64_t> status(al, tiles + 2);
    Buffer<int64_t> total(al, 1);
    LDF_CUDA(cudaMemsetAsync(status.get(), 0, (tiles + 2) * 8, s));
    launch("compact_groups", compact_groups_kernel, static_cast<unsigned>(tiles), 256, 0, s,
           static_cast<const unsigned long long*>(rec.get()), 1, nid, groups.get(), status.get(),
           reinterpret_cast<unsigned long long*>(status.get() + tiles), total.get(), ctx.err());
    const int64_t G = ctx.read_i64(total.get());

    FinArgs f{};
    f.p        = p;
    f.rec      = rec.get();
    f.ld       = L;
    f.perm     = perm.get();
    f.key_mode = static_cast<int>(M);
    f.groups   = groups.get();
    f.ngroups  = G;
    f.nkeys    = nkeys;
    for (int j = 0; j < nkeys; ++j) {
      const ldf_column& kc = table[keys[j]];
      out[j]               = alloc_out_column(al, kc.type, G, kc.valid != nullptr);
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
      const bool nullable       = !(ag.kind == LDF_AGG_COUNT_ALL || ag.kind == LDF_AGG_COUNT_DISTINCT);
      out[nkeys + a]            = alloc_out_column(al, ag.out_type, G, nullable);
      AggOut& o                 = f.a[a];
      o.kind                    = ag.kind;
      o.count_mode              = ag.count_mode;
      o.col                     = agg_col[a];
      o.in_type                 = ag.kind == LDF_AGG_COUNT_ALL ? LDF_INT64 : table[ag.in_col].type;
      o.dst = OCol{out[nkeys + a].data, out[nkeys + a].valid, ag.out_type, type_width(ag.out_type)};
    }
    if (G > 0) launch("finalize", finalize_kernel, gs_blocks(G, 256), 256, 0, s, f);
    for (int j = 0; j < nkeys; ++j)
      if (table[keys[j]].type == LDF_STRING) gather_strings(ctx, make_dcol(table[keys[j]]), repr.get(), G, out[j]);
    ctx.finish();
    return;
  }
}


// ===========================================================================
// Partitioned plan: one fixed-width key, at most two fixed-width value
// columns (the second at most 4 bytes wide), NUNIQUE of at most one column
// of <= 4-byte values.  Every row is read once by a routing pass:
//  * the keys the sample saw most often ("hot", at most kPartHotMax, plus the
//    null key) are aggregated in shared memory (flushed once per CTA) and
//    their NUNIQUE values set bits of per-group value bitmaps;
//  * every other row is written as one 24-byte record {key, value 0,
//    value 1 | validity bits} into the hash bucket of its key (2^logP
//    buckets, sized by a counting pre-pass over the keys).
// A bucket pass then aggregates each bucket in shared memory (a CTA per
// bucket: local key table, records, then a pair set for NUNIQUE) and writes
// its groups' output rows; buckets too large for shared memory take the same
// code on per-CTA global scratch.  No per-row group id is ever written.
// Float sums are the exact fixed-point sums of the general plan; a float
// SUM/MEAN value outside the fixed-point range (NaN, inf, |x| < 2^-44 or
// >= 2^95) makes the call fall back to the general plan.
// ===========================================================================
constexpr int kPartThreads    = 512;   // routing pass
constexpr int kCountThreads   = 1024;  // counting pre-pass
constexpr int kPartHotMax     = 1024;  // hot keys (the null key takes one more record)
constexpr int kPartHotSlots   = 2048;  // shared hot key table (power of two)
constexpr uint32_t kPartNoId  = 0xffffffffu;
constexpr uint32_t kPartBusy  = 0xfffffffeu;
constexpr int kBucketThreads  = 512;   // bucket pass (two CTAs per SM)
constexpr int kBucketKeySlots = 1024;  // shared local key table (power of two)
constexpr int kBucketRecBytes = 96 * 1024;  // shared records, then the pair set
constexpr int kBucketGroupsMax = 768;

struct PVal {  // one value column of the partitioned plan
  DCol col;
  int nullable;
  uint32_t states;  // ST_SUM | ST_MIN | ST_MAX | ST_NDIST
  int fixed;        // float sum: six fixed-point chunks
  int chunks;       // sum chunks (6 float, 2 integer)
  int mm64;         // min/max as 64-bit ordered words
  // shared (32-bit) record: byte offsets of the fields
  int b_vc, b_sum, b_mn, b_mx;
  // global hot record (64-bit words): word offsets of the fields
  int w_vc, w_sum, w_mn, w_mx;
};

struct PartOut {
  OCol key;
  int nagg;
  AggOut a[kMaxAggs];  // AggOut::col = value column (0 / 1), -1 for COUNT_ALL
};

struct PartArgs {
  DCol key;
  int64_t n;
  int ncol;
  PVal c[2];
  int nd;  // value column with NUNIQUE, -1 for none
  // hot keys
  const unsigned long long* hot_keys;
  int H;       // hot keys; record H is the null key's
  int rb;      // bytes of a shared record
  int rw;      // words of a global hot record
  unsigned long long* hot_rec;  // [(H + 1) * rw]
  uint32_t* bits;               // [(H + 1) * wpr] NUNIQUE value bitmaps
  uint32_t wpr, vbase, vflip;
  // buckets
  int logP;
  const int64_t* bstart;     // [P + 1] first record of each bucket
  unsigned int* hist;        // [P] cold rows per bucket (counting pre-pass)
  unsigned int* bcursor;     // [P] records written so far (routing pass)
  unsigned long long* recs;  // 3 words per cold row
  int* flag;                 // a float sum value outside the fixed-point range
};

__device__ __forceinline__ uint64_t part_ord64(uint64_t raw, int type)
{
  switch (type) {
    case LDF_FLOAT32: {
      const uint32_t b = static_cast<uint32_t>(raw);
      return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
    }
    case LDF_FLOAT64: return (raw >> 63) ? ~raw : (raw | (1ull << 63));
    case LDF_INT8: return static_cast<uint64_t>(static_cast<int64_t>(static_cast<int8_t>(raw))) ^ (1ull << 63);
    case LDF_INT16: return static_cast<uint64_t>(static_cast<int64_t>(static_cast<int16_t>(raw))) ^ (1ull << 63);
    case LDF_INT32: return static_cast<uint64_t>(static_cast<int64_t>(static_cast<int32_t>(raw))) ^ (1ull << 63);
    case LDF_INT64:
    case LDF_TIMESTAMP_US: return raw ^ (1ull << 63);
    default: return raw;
  }
}
__device__ __forceinline__ uint32_t part_ord32(uint64_t raw, int type)
{
  switch (type) {
    case LDF_FLOAT32: {
      const uint32_t b = static_cast<uint32_t>(raw);
      return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
    }
    case LDF_INT8: return static_cast<uint32_t>(static_cast<int32_t>(static_cast<int8_t>(raw))) ^ 0x80000000u;
    case LDF_INT16: return static_cast<uint32_t>(static_cast<int32_t>(static_cast<int16_t>(raw))) ^ 0x80000000u;
    case LDF_INT32: return static_cast<uint32_t>(raw) ^ 0x80000000u;
    default: return static_cast<uint32_t>(raw);
  }
}
// 32-bit ordered form -> the 64-bit ordered form of the same value
__device__ __forceinline__ uint64_t part_widen32(uint32_t o32, int type)
{
  if (type == LDF_INT8 || type == LDF_INT16 || type == LDF_INT32) {
    const int32_t v = static_cast<int32_t>(o32 ^ 0x80000000u);
    return static_cast<uint64_t>(static_cast<int64_t>(v)) ^ (1ull << 63);
  }
  return o32;
}

// Column kinds the routing pass is compiled for: a known kind turns the
// per-row type dispatch into straight-line code (the generic kind's switches
// made the kernel outgrow the instruction cache).
enum : int { PK_GEN = 0, PK_F64 = 1, PK_I32 = 2, PK_NONE = 3 };
template <int K>
__device__ __forceinline__ int pk_width(const PVal& c)
{
  return K == PK_F64 ? 8 : K == PK_I32 ? 4 : c.col.width;
}
template <int K>
__device__ __forceinline__ int pk_type(const PVal& c)
{
  return K == PK_F64 ? LDF_FLOAT64 : K == PK_I32 ? LDF_INT32 : c.col.type;
}

__device__ __forceinline__ uint64_t load_width(const void* data, int w, int64_t r)
{
  switch (w) {
    case 1: return __ldg(static_cast<const uint8_t*>(data) + r);
    case 2: return __ldg(static_cast<const uint16_t*>(data) + r);
    case 4: return __ldg(static_cast<const uint32_t*>(data) + r);
    default: return __ldg(static_cast<const unsigned long long*>(data) + r);
  }
}
__device__ __forceinline__ uint64_t part_load(const DCol& c, int64_t r) { return load_width(c.data, c.width, r); }
template <int K>
__device__ __forceinline__ uint64_t part_load_k(const PVal& c, int64_t r)
{
  return load_width(c.col.data, pk_width<K>(c), r);
}

// Add one valid value of column `c` into a 32-bit record (shared memory or
// per-CTA global scratch; generic addresses).  Returns false for a float sum
// value outside the fixed-point range.
template <int K = PK_GEN>
__device__ __forceinline__ bool part_add(const PVal& c, unsigned char* rec, uint64_t raw)
{
  const int W      = pk_width<K>(c);
  const int T      = pk_type<K>(c);
  const bool fixed = K == PK_F64 ? true : K == PK_I32 ? false : c.fixed != 0;
  const bool mm64  = K == PK_F64 ? true : K == PK_I32 ? false : c.mm64 != 0;
  const int chunks = K == PK_F64 ? kSumChunks : K == PK_I32 ? 2 : c.chunks;
  bool ok          = true;
  if (c.nullable) atomicAdd(reinterpret_cast<uint32_t*>(rec + c.b_vc), 1u);
  if (c.states & ST_SUM) {
    uint32_t* sum = reinterpret_cast<uint32_t*>(rec + c.b_sum);
    if (fixed) {
      const double x = W == 8 ? __longlong_as_double(static_cast<long long>(raw))
                              : static_cast<double>(__uint_as_float(static_cast<uint32_t>(raw)));
      uint64_t m;
      int sh;
      bool neg;
      if (fixed_parts(x, m, sh, neg)) {
        if (m) {
          const int j0 = sh >> 5, b = sh & 31;
          sh_add_magnitude(sum, chunks, j0, m << b, b ? (m >> (64 - b)) : 0, neg);
        }
      } else {
        ok = false;
      }
    } else {
      uint64_t mag = raw;
      bool neg     = false;
      if (is_signed_int_dev(T)) {
        const int64_t v = W == 1 ? static_cast<int8_t>(raw) : W == 2 ? static_cast<int16_t>(raw)
                        : W == 4 ? static_cast<int32_t>(raw) : static_cast<int64_t>(raw);
        neg = v < 0;
        mag = neg ? (0ull - static_cast<uint64_t>(v)) : static_cast<uint64_t>(v);
      }
      sh_add_magnitude(sum, chunks, 0, mag, 0, neg);
    }
  }
  if (c.states & (ST_MIN | ST_MAX)) {
    if (mm64) {
      const uint64_t o = part_ord64(raw, T);
      if (c.states & ST_MIN) atomicMax(reinterpret_cast<unsigned long long*>(rec + c.b_mn), ~o);
      if (c.states & ST_MAX) atomicMax(reinterpret_cast<unsigned long long*>(rec + c.b_mx), o);
    } else {
      const uint32_t o = part_ord32(raw, T);
      if (c.states & ST_MIN) atomicMax(reinterpret_cast<uint32_t*>(rec + c.b_mn), ~o);
      if (c.states & ST_MAX) atomicMax(reinterpret_cast<uint32_t*>(rec + c.b_mx), o);
    }
  }
  return ok;
}

// The aggregates of one group, unpacked from either record form.
struct PartVals {
  uint64_t call;
  uint64_t vc[2];
  unsigned long long acc[2][kSumChunks];  // signed chunk sums (float) / acc[c][0] = sum mod 2^64 (integer)
  uint64_t omn[2], omx[2];                // 64-bit ordered min / max
};

// from a 32-bit record (bucket pass)
__device__ __forceinline__ void part_unpack32(const PartArgs& a, const unsigned char* rec, PartVals& v)
{
  v.call = *reinterpret_cast<const uint32_t*>(rec + 8);
  for (int ci = 0; ci < a.ncol; ++ci) {
    const PVal& c = a.c[ci];
    v.vc[ci]      = c.nullable ? *reinterpret_cast<const uint32_t*>(rec + c.b_vc) : v.call;
    if (c.states & ST_SUM) {
      const uint32_t* sum = reinterpret_cast<const uint32_t*>(rec + c.b_sum);
      uint64_t tot        = 0;
      for (int q = 0; q < c.chunks; ++q) {
        const int64_t pos = static_cast<int64_t>(sum[q * 4 + 0]) + (static_cast<int64_t>(sum[q * 4 + 1]) << 32);
        const int64_t neg = static_cast<int64_t>(sum[q * 4 + 2]) + (static_cast<int64_t>(sum[q * 4 + 3]) << 32);
        v.acc[ci][q]      = static_cast<unsigned long long>(pos - neg);
        tot += static_cast<uint64_t>(pos - neg) << (32 * q);
      }
      if (!c.fixed) v.acc[ci][0] = tot;
    }
    if (c.states & (ST_MIN | ST_MAX)) {
      if (c.mm64) {
        v.omn[ci] = ~*reinterpret_cast<const unsigned long long*>(rec + c.b_mn);
        v.omx[ci] = *reinterpret_cast<const unsigned long long*>(rec + c.b_mx);
      } else {
        v.omn[ci] = part_widen32(~*reinterpret_cast<const uint32_t*>(rec + c.b_mn), c.col.type);
        v.omx[ci] = part_widen32(*reinterpret_cast<const uint32_t*>(rec + c.b_mx), c.col.type);
      }
    }
  }
}

// from a global 64-bit hot record (after every CTA flushed into it)
__device__ __forceinline__ void part_unpack64(const PartArgs& a, const unsigned long long* w, PartVals& v)
{
  v.call = w[0];
  for (int ci = 0; ci < a.ncol; ++ci) {
    const PVal& c = a.c[ci];
    v.vc[ci]      = c.nullable ? w[c.w_vc] : v.call;
    if (c.states & ST_SUM)
      for (int q = 0; q < (c.fixed ? c.chunks : 1); ++q) v.acc[ci][q] = w[c.w_sum + q];
    if (c.states & ST_MIN) v.omn[ci] = ~w[c.w_mn];
    if (c.states & ST_MAX) v.omx[ci] = w[c.w_mx];
  }
}

// Output row i of one group: key and every aggregation but NUNIQUE.
__device__ __forceinline__ void part_emit(const PartArgs& a, const PartOut& o, int64_t i, uint64_t kb, bool knull,
                                          const PartVals& v)
{
  store_int(OCol{o.key.data, nullptr, LDF_UINT64, o.key.width}, i, knull ? 0 : kb);
  if (o.key.valid) o.key.valid[i] = knull ? 0 : 1;
  double fsum[2];
  bool fsum_done[2] = {false, false};
  for (int k = 0; k < o.nagg; ++k) {
    const AggOut& g = o.a[k];
    const OCol& d   = g.dst;
    if (g.kind == LDF_AGG_COUNT_ALL) {
      store_int(d, i, v.call);
      if (d.valid) d.valid[i] = 1;
      continue;
    }
    if (g.kind == LDF_AGG_COUNT_DISTINCT) continue;
    const int ci  = g.col;
    const PVal& c = a.c[ci];
    const uint64_t vc = v.vc[ci];
    bool ok           = vc > 0;
    switch (g.kind) {
      case LDF_AGG_COUNT: {
        store_int(d, i, g.count_mode == LDF_COUNT_ALL ? v.call : g.count_mode == LDF_COUNT_ONLY_NULL ? v.call - vc : vc);
        ok = true;
        break;
      }
      case LDF_AGG_SUM:
      case LDF_AGG_MEAN: {
        if (!ok) {
          store_int(d, i, 0);
          break;
        }
        if (c.fixed) {
          if (!fsum_done[ci]) {
            fsum[ci]      = chunks_to_double(v.acc[ci], 1);
            fsum_done[ci] = true;
          }
          store_double(d, i, g.kind == LDF_AGG_MEAN ? fsum[ci] / static_cast<double>(vc) : fsum[ci]);
        } else {
          const uint64_t s = v.acc[ci][0];
          const double sd  = is_signed_int_dev(g.in_type) ? static_cast<double>(static_cast<int64_t>(s))
                                                          : static_cast<double>(s);
          if (g.kind == LDF_AGG_MEAN) store_double(d, i, sd / static_cast<double>(vc));
          else if (d.type == LDF_FLOAT64 || d.type == LDF_FLOAT32) store_double(d, i, sd);
          else store_int(d, i, s);
        }
        break;
      }
      case LDF_AGG_MIN:
      case LDF_AGG_MAX: {
        if (!ok) {
          store_int(d, i, 0);
          break;
        }
        const uint64_t b = unordered_bits(g.in_type, g.kind == LDF_AGG_MIN ? v.omn[ci] : v.omx[ci]);
        if (d.type == g.in_type) store_int(OCol{d.data, nullptr, LDF_UINT64, d.width}, i, b);
        else if (g.in_type == LDF_FLOAT32) store_double(d, i, static_cast<double>(__uint_as_float(static_cast<uint32_t>(b))));
        else if (g.in_type == LDF_FLOAT64) store_double(d, i, __longlong_as_double(static_cast<long long>(b)));
        else store_int(d, i, b);
        break;
      }
      default: break;
    }
    if (d.valid) d.valid[i] = ok ? 1 : 0;
  }
}

// NUNIQUE outputs of output row i: nd distinct valid values; has_null: the
// group has a null in the column.
__device__ __forceinline__ void part_emit_nd(const PartOut& o, int64_t i, uint64_t nd, bool has_null)
{
  for (int k = 0; k < o.nagg; ++k) {
    const AggOut& g = o.a[k];
    if (g.kind != LDF_AGG_COUNT_DISTINCT) continue;
    const uint64_t hn = has_null ? 1 : 0;
    store_int(g.dst, i, g.count_mode == LDF_COUNT_ALL ? nd + hn : g.count_mode == LDF_COUNT_ONLY_NULL ? hn : nd);
    if (g.dst.valid) g.dst.valid[i] = 1;
  }
}

// Shared hot key table: slot -> hot id (kPartNoId empty) and key.
__device__ __forceinline__ void hot_table_build(const PartArgs& a, uint32_t* ids, unsigned long long* keys)
{
  for (int i = threadIdx.x; i < kPartHotSlots; i += blockDim.x) ids[i] = kPartNoId;
  __syncthreads();
  for (int i = threadIdx.x; i < a.H; i += blockDim.x) {
    const uint64_t kb = a.hot_keys[i];
    uint32_t idx      = static_cast<uint32_t>(mix64(kb)) & (kPartHotSlots - 1);
    for (int probe = 0; probe < kPartHotSlots; ++probe) {
      if (atomicCAS(ids + idx, kPartNoId, static_cast<uint32_t>(i)) == kPartNoId) {
        keys[idx] = kb;
        break;
      }
      idx = (idx + 1) & (kPartHotSlots - 1);
    }
  }
  __syncthreads();
}

__device__ __forceinline__ uint32_t hot_lookup(const uint32_t* ids, const unsigned long long* keys, uint64_t kb,
                                               uint64_t h)
{
  uint32_t idx = static_cast<uint32_t>(h) & (kPartHotSlots - 1);
  for (int probe = 0; probe < kPartHotSlots; ++probe) {
    const uint32_t id = ids[idx];
    if (id == kPartNoId) return kPartNoId;
    if (keys[idx] == kb) return id;
    idx = (idx + 1) & (kPartHotSlots - 1);
  }
  return kPartNoId;
}

__device__ __forceinline__ uint32_t bucket_of(uint64_t h, int logP)
{
  return logP == 0 ? 0u : static_cast<uint32_t>(h >> (64 - logP));
}

// ---- counting pre-pass: cold rows per bucket ---------------------------------
__global__ void __launch_bounds__(kCountThreads, 1) part_count_kernel(PartArgs a)
{
  extern __shared__ __align__(16) unsigned char smem[];
  uint32_t* ids            = reinterpret_cast<uint32_t*>(smem);
  unsigned long long* keys = reinterpret_cast<unsigned long long*>(smem + kPartHotSlots * 4);
  uint32_t* hist           = reinterpret_cast<uint32_t*>(smem + kPartHotSlots * 12);
  const uint32_t P         = 1u << a.logP;
  for (uint32_t i = threadIdx.x; i < P; i += blockDim.x) hist[i] = 0;
  hot_table_build(a, ids, keys);
  const int64_t step = static_cast<int64_t>(gridDim.x) * blockDim.x * kRows;
  for (int64_t base = static_cast<int64_t>(blockIdx.x) * blockDim.x * kRows; base < a.n; base += step) {
    uint64_t kb[kRows];
    bool ok[kRows];
#pragma unroll
    for (int j = 0; j < kRows; ++j) {
      const int64_t r = base + static_cast<int64_t>(j) * blockDim.x + threadIdx.x;
      ok[j]           = r < a.n && dvalid(a.key, r);
      kb[j]           = ok[j] ? part_load(a.key, r) : 0;
    }
#pragma unroll
    for (int j = 0; j < kRows; ++j) {
      if (!ok[j]) continue;
      const uint64_t h = mix64(kb[j]);
      if (hot_lookup(ids, keys, kb[j], h) == kPartNoId) atomicAdd(hist + bucket_of(h, a.logP), 1u);
    }
  }
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < P; i += blockDim.x)
    if (hist[i]) atomicAdd(a.hist + i, hist[i]);
}

// ---- routing pass -----------------------------------------------------------
template <int K0, int K1>
__global__ void __launch_bounds__(kPartThreads) part_route_kernel(PartArgs a)
{
  // the second value column: none, or its kind (generic: decided at run time)
  const bool two = K1 == PK_NONE ? false : (K1 == PK_GEN ? a.ncol > 1 : true);
  extern __shared__ __align__(16) unsigned char smem[];
  uint32_t* ids            = reinterpret_cast<uint32_t*>(smem);
  unsigned long long* keys = reinterpret_cast<unsigned long long*>(smem + kPartHotSlots * 4);
  unsigned char* recs      = smem + kPartHotSlots * 12;
  const int nrec           = a.H + 1;
  {
    uint4* z       = reinterpret_cast<uint4*>(recs);
    const int n16  = nrec * a.rb / 16;
    for (int i = threadIdx.x; i < n16; i += blockDim.x) z[i] = make_uint4(0, 0, 0, 0);
  }
  hot_table_build(a, ids, keys);
  bool range_ok      = true;
  const int64_t step = static_cast<int64_t>(gridDim.x) * blockDim.x * kRows;
  for (int64_t base = static_cast<int64_t>(blockIdx.x) * blockDim.x * kRows; base < a.n; base += step) {
    uint64_t kb[kRows], v0[kRows], v1[kRows];
    uint32_t fl[kRows];  // bit 0: row exists, 1: key valid, 2: value 0 valid, 3: value 1 valid
#pragma unroll
    for (int j = 0; j < kRows; ++j) {
      const int64_t r = base + static_cast<int64_t>(j) * blockDim.x + threadIdx.x;
      fl[j]           = 0;
      kb[j] = v0[j] = v1[j] = 0;
      if (r < a.n) {
        fl[j] = 1;
        if (dvalid(a.key, r)) {
          fl[j] |= 2;
          kb[j] = part_load(a.key, r);
        }
        v0[j] = part_load_k<K0>(a.c[0], r);
        if (dvalid(a.c[0].col, r)) fl[j] |= 4;
        if (two) {
          v1[j] = part_load_k<K1>(a.c[1], r);
          if (dvalid(a.c[1].col, r)) fl[j] |= 8;
        }
      }
    }
#pragma unroll
    for (int j = 0; j < kRows; ++j) {
      if (!(fl[j] & 1)) continue;
      const uint64_t h = mix64(kb[j]);
      const uint32_t hid = (fl[j] & 2) ? hot_lookup(ids, keys, kb[j], h) : static_cast<uint32_t>(a.H);
      if (hid != kPartNoId) {
        unsigned char* rec = recs + static_cast<int64_t>(hid) * a.rb;
        atomicAdd(reinterpret_cast<uint32_t*>(rec + 8), 1u);
        if (fl[j] & 4) range_ok &= part_add<K0>(a.c[0], rec, v0[j]);
        if (two && (fl[j] & 8)) range_ok &= part_add<K1 == PK_NONE ? PK_GEN : K1>(a.c[1], rec, v1[j]);
        if (a.nd >= 0 && (fl[j] & (a.nd == 0 ? 4 : 8))) {
          const uint32_t off = (static_cast<uint32_t>(a.nd == 0 ? v0[j] : v1[j]) ^ a.vflip) - a.vbase;
          red_or32(a.bits + static_cast<uint64_t>(hid) * a.wpr + (off >> 5), 1u << (off & 31));
        }
      } else {
        // a cold row: the validity bits ride in the top of the third word
        // (value 1 is at most 4 bytes)
        const bool fixed0 = K0 == PK_F64 ? true : K0 == PK_I32 ? false : a.c[0].fixed != 0;
        const bool fixed1 = K1 == PK_F64 ? true : (K1 == PK_I32 || K1 == PK_NONE) ? false : a.c[1].fixed != 0;
        if (fixed0 && (a.c[0].states & ST_SUM) && (fl[j] & 4)) {
          const double x = pk_width<K0>(a.c[0]) == 8 ? __longlong_as_double(static_cast<long long>(v0[j]))
                                                 : static_cast<double>(__uint_as_float(static_cast<uint32_t>(v0[j])));
          uint64_t m;
          int sh;
          bool neg;
          range_ok &= fixed_parts(x, m, sh, neg);
        }
        if (two && fixed1 && (a.c[1].states & ST_SUM) && (fl[j] & 8)) {
          const double x = static_cast<double>(__uint_as_float(static_cast<uint32_t>(v1[j])));
          uint64_t m;
          int sh;
          bool neg;
          range_ok &= fixed_parts(x, m, sh, neg);
        }
        const uint32_t b    = bucket_of(h, a.logP);
        const int64_t pos   = a.bstart[b] + atomicAdd(a.bcursor + b, 1u);
        unsigned long long* d = a.recs + 3 * pos;
        d[0] = kb[j];
        d[1] = v0[j];
        d[2] = (v1[j] & 0xffffffffull) | (static_cast<uint64_t>((fl[j] >> 2) & 3) << 32);
      }
    }
  }
  if (!range_ok) atomicExch(a.flag, 1);
  __syncthreads();
  // flush the hot records
  for (int g = threadIdx.x; g < nrec; g += blockDim.x) {
    const unsigned char* rec = recs + static_cast<int64_t>(g) * a.rb;
    const uint32_t call      = *reinterpret_cast<const uint32_t*>(rec + 8);
    if (call == 0) continue;
    unsigned long long* w = a.hot_rec + static_cast<int64_t>(g) * a.rw;
    red_add(w, call);
    for (int ci = 0; ci < a.ncol; ++ci) {
      const PVal& c = a.c[ci];
      if (c.nullable) red_add(w + c.w_vc, *reinterpret_cast<const uint32_t*>(rec + c.b_vc));
      if (c.states & ST_SUM) {
        const uint32_t* sum = reinterpret_cast<const uint32_t*>(rec + c.b_sum);
        uint64_t tot        = 0;
        for (int q = 0; q < c.chunks; ++q) {
          const int64_t pos = static_cast<int64_t>(sum[q * 4 + 0]) + (static_cast<int64_t>(sum[q * 4 + 1]) << 32);
          const int64_t neg = static_cast<int64_t>(sum[q * 4 + 2]) + (static_cast<int64_t>(sum[q * 4 + 3]) << 32);
          if (c.fixed) {
            if (pos != neg) red_add(w + c.w_sum + q, static_cast<uint64_t>(pos - neg));
          } else {
            tot += static_cast<uint64_t>(pos - neg) << (32 * q);
          }
        }
        if (!c.fixed && tot) red_add(w + c.w_sum, tot);
      }
      if (c.states & (ST_MIN | ST_MAX)) {
        if (c.mm64) {
          if (c.states & ST_MIN) red_max(w + c.w_mn, *reinterpret_cast<const unsigned long long*>(rec + c.b_mn));
          if (c.states & ST_MAX) red_max(w + c.w_mx, *reinterpret_cast<const unsigned long long*>(rec + c.b_mx));
        } else {
          // an untouched word flushes the identity of the opposite extreme
          if (c.states & ST_MIN)
            red_max(w + c.w_mn, ~part_widen32(~*reinterpret_cast<const uint32_t*>(rec + c.b_mn), c.col.type));
          if (c.states & ST_MAX)
            red_max(w + c.w_mx, part_widen32(*reinterpret_cast<const uint32_t*>(rec + c.b_mx), c.col.type));
        }
      }
    }
  }
}

// ---- hot groups: one output row each (a CTA per hot record) ----------------
__global__ void __launch_bounds__(256) part_hot_emit_kernel(PartArgs a, PartOut o, unsigned long long* out_count,
                                                            int64_t out_cap)
{
  __shared__ unsigned long long part[8];
  __shared__ int64_t s_pos;
  for (int g = blockIdx.x; g <= a.H; g += gridDim.x) {
    const unsigned long long* w = a.hot_rec + static_cast<int64_t>(g) * a.rw;
    if (w[0] == 0) continue;  // uniform across the block
    unsigned long long c = 0;
    if (a.nd >= 0) {
      const uint4* w4 = reinterpret_cast<const uint4*>(a.bits + static_cast<uint64_t>(g) * a.wpr);
      for (uint32_t i = threadIdx.x; i < a.wpr / 4; i += blockDim.x) {
        const uint4 q = w4[i];
        c += __popc(q.x) + __popc(q.y) + __popc(q.z) + __popc(q.w);
      }
      for (int off = 16; off > 0; off >>= 1) c += __shfl_xor_sync(0xffffffffu, c, off);
      if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = c;
    }
    if (threadIdx.x == 0) s_pos = static_cast<int64_t>(atomicAdd(out_count, 1ull));
    __syncthreads();
    const int64_t pos = s_pos;
    if (threadIdx.x == 0 && pos < out_cap) {
      PartVals v;
      part_unpack64(a, w, v);
      const bool knull = g == a.H;
      part_emit(a, o, pos, knull ? 0 : a.hot_keys[g], knull, v);
      if (a.nd >= 0) {
        unsigned long long t = 0;
        for (int i = 0; i < static_cast<int>((blockDim.x + 31) >> 5); ++i) t += part[i];
        part_emit_nd(o, pos, t, v.call > v.vc[a.nd]);
      }
    }
    __syncthreads();
  }
}

// ---- bucket pass ---------------------------------------------------------------
// Work memory of one bucket: local key table (ids + keys, `ks` slots, a power
// of two), records (`gc` groups of a.rb bytes; key word at offset 0, the
// group's row count at 8), NUNIQUE counts and null flags per group, and a
// pair set of `ps` 8-byte slots that reuses the record space once the
// records have been written out.
struct BucketMem {
  uint32_t* ids;
  unsigned long long* keys;
  unsigned char* recs;
  uint32_t* nd;
  uint8_t* hasnull;
  unsigned long long* pairs;
  int ks;
  int gc;
  int64_t ps;
};

struct BucketArgs {
  PartArgs a;
  PartOut o;
  unsigned long long* out_count;
  int64_t out_cap;
  const int32_t* list;         // large pass: bucket ids to take (nullptr: every bucket)
  int64_t nlist;
  unsigned long long* next;    // bucket counter
  int32_t* deferred;           // shared-memory pass: buckets that did not fit
  unsigned int* ndeferred;
  int64_t small_rows;          // shared-memory pass: buckets above this many rows are skipped
  int pair32;                  // NUNIQUE pairs as 32-bit words (local id < 4096, value offset < 2^20)
  // large pass: per-CTA global work memory
  unsigned char* scratch;
  int64_t scratch_stride;
  int ks, gc;
  int64_t ps;
  int* err;
};

// Local id of key kb in the bucket's key table, inserting it when new (the
// inserting thread claims the slot, then publishes the key and the id; a
// reader that finds the slot claimed waits for the id, bounded).  *fresh is
// set for the inserting thread.
__device__ __forceinline__ uint32_t local_id(const BucketMem& m, uint32_t* nlocal, uint64_t kb, uint64_t h,
                                             int* err, bool* fresh)
{
  uint32_t idx = static_cast<uint32_t>(h) & (m.ks - 1);
  *fresh       = false;
  for (int probe = 0; probe < m.ks; ++probe) {
    uint32_t id = *reinterpret_cast<volatile uint32_t*>(m.ids + idx);
    if (id == kPartNoId) {
      id = atomicCAS(m.ids + idx, kPartNoId, kPartBusy);
      if (id == kPartNoId) {  // claimed: publish key, then id
        const uint32_t lid = atomicAdd(nlocal, 1u);
        m.keys[idx]        = kb;
        __threadfence_block();
        atomicExch(m.ids + idx, lid);
        *fresh = true;
        return lid;
      }
    }
    if (id == kPartBusy) {  // another thread of the CTA is publishing this slot
      uint32_t spin = 0;
      do {
        id = *reinterpret_cast<volatile uint32_t*>(m.ids + idx);
        if (++spin > kSpinLimit) {
          atomicExch(err, LDF_ERR_TIMEOUT);
          return kPartNoId;
        }
      } while (id == kPartBusy);
      __threadfence_block();
    }
    if (reinterpret_cast<volatile unsigned long long*>(m.keys)[idx] == kb) return id;
    idx = (idx + 1) & (m.ks - 1);
  }
  return kPartNoId;  // the table is sized above the rows: not reached
}

// Aggregates one bucket: rows [r0, r1) of a.recs.  Returns false (nothing
// written) when the bucket has more groups than m.gc.
__device__ bool process_bucket(const BucketArgs& B, const BucketMem& m, int64_t r0, int64_t r1, uint32_t* sh_nlocal,
                               int64_t* sh_base)
{
  const PartArgs& a = B.a;
  const int64_t rows = r1 - r0;
  // clear the work memory
  for (int i = threadIdx.x; i < m.ks; i += blockDim.x) m.ids[i] = kPartNoId;
  {
    const int64_t n16 = static_cast<int64_t>(m.gc) * a.rb / 16;
    uint4* z          = reinterpret_cast<uint4*>(m.recs);
    for (int64_t i = threadIdx.x; i < n16; i += blockDim.x) z[i] = make_uint4(0, 0, 0, 0);
  }
  if (threadIdx.x == 0) *sh_nlocal = 0;
  __syncthreads();
  // records into the local groups
  for (int64_t i = threadIdx.x; i < rows; i += blockDim.x) {
    const unsigned long long* s = a.recs + 3 * (r0 + i);
    const uint64_t kb = s[0], w1 = s[1], w2 = s[2];
    bool fresh;
    const uint32_t lid = local_id(m, sh_nlocal, kb, mix64(kb), B.err, &fresh);
    if (lid >= static_cast<uint32_t>(m.gc)) continue;
    unsigned char* rec = m.recs + static_cast<int64_t>(lid) * a.rb;
    if (fresh) *reinterpret_cast<unsigned long long*>(rec) = kb;
    atomicAdd(reinterpret_cast<uint32_t*>(rec + 8), 1u);
    if ((w2 >> 32) & 1) part_add(a.c[0], rec, w1);
    if (a.ncol > 1 && ((w2 >> 33) & 1)) part_add(a.c[1], rec, w2 & 0xffffffffull);
  }
  __syncthreads();
  const uint32_t ng = *sh_nlocal;
  if (ng > static_cast<uint32_t>(m.gc)) return false;
  if (threadIdx.x == 0) *sh_base = static_cast<int64_t>(atomicAdd(B.out_count, static_cast<unsigned long long>(ng)));
  __syncthreads();
  const int64_t base = *sh_base;
  for (uint32_t g = threadIdx.x; g < ng; g += blockDim.x) {
    const unsigned char* rec = m.recs + static_cast<int64_t>(g) * a.rb;
    PartVals v;
    part_unpack32(a, rec, v);
    if (a.nd >= 0) {
      m.nd[g]      = 0;
      m.hasnull[g] = v.call > v.vc[a.nd] ? 1 : 0;
    }
    if (base + g < B.out_cap) part_emit(a, B.o, base + g, *reinterpret_cast<const unsigned long long*>(rec), false, v);
  }
  if (a.nd < 0) {
    __syncthreads();
    return true;
  }
  // NUNIQUE: (local id, value) pairs of the valid rows, counted when new
  __syncthreads();
  const int64_t cap = B.pair32 ? 2 * m.ps : m.ps;  // slots of the pair set
  const int64_t ps  = cap < 2 * rows + 64 ? cap : 2 * rows + 64;
  uint32_t* pairs32 = reinterpret_cast<uint32_t*>(m.pairs);
  if (B.pair32)
    for (int64_t i = threadIdx.x; i < ps; i += blockDim.x) pairs32[i] = kPartNoId;
  else
    for (int64_t i = threadIdx.x; i < ps; i += blockDim.x) m.pairs[i] = kEmpty;
  __syncthreads();
  const uint64_t vbit = a.nd == 0 ? (1ull << 32) : (2ull << 32);
  for (int64_t i = threadIdx.x; i < rows; i += blockDim.x) {
    const unsigned long long* s = a.recs + 3 * (r0 + i);
    const uint64_t kb = s[0], w2 = s[2];
    if (!(w2 & vbit)) continue;
    const uint32_t x   = static_cast<uint32_t>(a.nd == 0 ? s[1] : w2);
    bool fresh;
    const uint32_t lid = local_id(m, sh_nlocal, kb, mix64(kb), B.err, &fresh);  // present: a pure lookup
    if (lid >= ng) continue;  // only after an expired wait (reported through B.err)
    if (B.pair32) {
      const uint32_t e32 = (lid << 20) | ((x ^ a.vflip) - a.vbase);
      uint64_t idx       = fastrange(mix64(e32), static_cast<uint64_t>(ps));
      for (int64_t probe = 0; probe < ps; ++probe) {
        const uint32_t cur = atomicCAS(pairs32 + idx, kPartNoId, e32);
        if (cur == kPartNoId) {
          atomicAdd(m.nd + lid, 1u);
          break;
        }
        if (cur == e32) break;
        idx = idx + 1 == static_cast<uint64_t>(ps) ? 0 : idx + 1;
      }
      continue;
    }
    const uint64_t e   = (static_cast<uint64_t>(lid) << 32) | x;
    uint64_t idx       = fastrange(mix64(e), static_cast<uint64_t>(ps));
    for (int64_t probe = 0; probe < ps; ++probe) {
      const unsigned long long cur = atomicCAS(m.pairs + idx, kEmpty, e);
      if (cur == kEmpty) {
        atomicAdd(m.nd + lid, 1u);
        break;
      }
      if (cur == e) break;
      idx = idx + 1 == static_cast<uint64_t>(ps) ? 0 : idx + 1;
    }
  }
  __syncthreads();
  for (uint32_t g = threadIdx.x; g < ng; g += blockDim.x)
    if (base + g < B.out_cap) part_emit_nd(B.o, base + g, m.nd[g], m.hasnull[g] != 0);
  __syncthreads();
  return true;
}

// Shared-memory bucket pass: persistent CTAs take buckets in order; a bucket
// above `small_rows` rows is left to the large pass, one with more groups
// than the shared records hold is deferred to it.
__global__ void __launch_bounds__(kBucketThreads, 2) part_bucket_kernel(BucketArgs B)
{
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ uint32_t s_nlocal;
  __shared__ int64_t s_base;
  __shared__ int64_t s_bucket;
  BucketMem m;
  m.ids     = reinterpret_cast<uint32_t*>(smem);
  m.keys    = reinterpret_cast<unsigned long long*>(smem + kBucketKeySlots * 4);
  m.recs    = smem + kBucketKeySlots * 12;
  m.pairs   = reinterpret_cast<unsigned long long*>(m.recs);
  m.nd      = reinterpret_cast<uint32_t*>(m.recs + kBucketRecBytes);
  m.hasnull = reinterpret_cast<uint8_t*>(m.nd + kBucketGroupsMax);
  m.ks      = kBucketKeySlots;
  m.gc      = min(kBucketGroupsMax, kBucketRecBytes / B.a.rb);
  m.ps      = kBucketRecBytes / 8;
  const uint32_t P = 1u << B.a.logP;
  for (;;) {
    if (threadIdx.x == 0) s_bucket = static_cast<int64_t>(atomicAdd(B.next, 1ull));
    __syncthreads();
    const int64_t b = s_bucket;
    __syncthreads();
    if (b >= P) break;
    const int64_t r0 = B.a.bstart[b], r1 = B.a.bstart[b + 1];
    if (r1 == r0 || r1 - r0 > B.small_rows) continue;
    if (!process_bucket(B, m, r0, r1, &s_nlocal, &s_base)) {
      if (threadIdx.x == 0) B.deferred[atomicAdd(B.ndeferred, 1u)] = static_cast<int32_t>(b);
      __syncthreads();
    }
  }
}

// Large bucket pass: the same work on per-CTA global memory sized for the
// largest of the listed buckets.
__global__ void __launch_bounds__(kBucketThreads, 1) part_bucket_large_kernel(BucketArgs B)
{
  __shared__ uint32_t s_nlocal;
  __shared__ int64_t s_base;
  __shared__ int64_t s_item;
  unsigned char* w = B.scratch + static_cast<int64_t>(blockIdx.x) * B.scratch_stride;
  BucketMem m;
  m.ids     = reinterpret_cast<uint32_t*>(w);
  m.keys    = reinterpret_cast<unsigned long long*>(w + static_cast<int64_t>(B.ks) * 4);
  m.recs    = w + static_cast<int64_t>(B.ks) * 12;
  m.pairs   = reinterpret_cast<unsigned long long*>(m.recs);
  const int64_t rbytes = static_cast<int64_t>(B.gc) * B.a.rb > B.ps * 8 ? static_cast<int64_t>(B.gc) * B.a.rb : B.ps * 8;
  m.nd      = reinterpret_cast<uint32_t*>(m.recs + rbytes);
  m.hasnull = reinterpret_cast<uint8_t*>(m.nd + B.gc);
  m.ks      = B.ks;
  m.gc      = B.gc;
  m.ps      = B.ps;
  for (;;) {
    if (threadIdx.x == 0) s_item = static_cast<int64_t>(atomicAdd(B.next, 1ull));
    __syncthreads();
    const int64_t it = s_item;
    __syncthreads();
    if (it >= B.nlist) break;
    const int32_t b = B.list[it];
    process_bucket(B, m, B.a.bstart[b], B.a.bstart[b + 1], &s_nlocal, &s_base);
  }
}

// ---- sample: the most frequent keys -------------------------------------------
// Strided sample of the keys into an open-addressing table {key, count}
// (slot taken when its count word leaves 0), counts warp-aggregated.
__global__ void part_sample_kernel(DCol key, int64_t n_sample, int64_t stride, unsigned long long* keys,
                                   unsigned int* counts, uint64_t cap)
{
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n_sample;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = i * stride;
    int64_t g       = -1;
    if (dvalid(key, r)) {
      const uint64_t kb = part_load(key, r);
      uint64_t idx      = fastrange(mix64(kb), cap);
      for (int probe = 0; probe < kMaxProbe; ++probe) {
        const unsigned long long v = atomicCAS(keys + idx, kEmpty, kb);
        if (v == kEmpty || v == kb) {
          g = static_cast<int64_t>(idx);
          break;
        }
        idx = idx + 1 == cap ? 0 : idx + 1;
      }
    }
    const uint32_t active = __activemask();
    const uint32_t peers  = __match_any_sync(active, static_cast<unsigned long long>(g));
    if (g >= 0 && (threadIdx.x & 31) == static_cast<unsigned>(__ffs(peers) - 1))
      atomicAdd(&counts[g], static_cast<unsigned>(__popc(peers)));
  }
}

// hist[min(count, 4095)] over the occupied slots; out[0] occupied, out[1] singletons
__global__ void part_sample_stats_kernel(const unsigned int* counts, uint64_t cap, unsigned int* hist,
                                         unsigned long long* out)
{
  unsigned long long occ = 0, f1 = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < static_cast<int64_t>(cap);
       i += (int64_t)gridDim.x * blockDim.x) {
    const unsigned int c = counts[i];
    if (c == 0) continue;
    ++occ;
    f1 += c == 1;
    atomicAdd(hist + min(c, 4095u), 1u);
  }
  occ = warp_reduce_sum(occ);
  f1  = warp_reduce_sum(f1);
  if ((threadIdx.x & 31) == 0) {
    if (occ) atomicAdd(&out[0], occ);
    if (f1) atomicAdd(&out[1], f1);
  }
}

// keys with count >= threshold -> hot list (at most hmax)
__global__ void part_hot_select_kernel(const unsigned long long* keys, const unsigned int* counts, uint64_t cap,
                                       unsigned int threshold, unsigned long long* hot, unsigned int* nhot, int hmax)
{
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < static_cast<int64_t>(cap);
       i += (int64_t)gridDim.x * blockDim.x) {
    if (counts[i] < threshold || counts[i] == 0) continue;
    const unsigned int at = atomicAdd(nhot, 1u);
    if (at < static_cast<unsigned>(hmax)) hot[at] = keys[i];
  }
}

// ---- host ----------------------------------------------------------------------
// Runs the partitioned plan when it applies; false (nothing written to `out`)
// when it does not, or when a float sum value fell outside the fixed-point
// range, so the caller runs the general plan.
bool try_partitioned(const OpContext& ctx, const GbPlan& p, const ldf_column* table, const int32_t* keys, int nkeys,
                     const ldf_aggregation* aggs, int naggs, const std::vector<int>& agg_col, ldf_column* out,
                     const HostStaging& hs, const std::vector<int>& col_of_plan)
{
  // Opt-in (LDF_B200_GB_PART=1): on the 200M-row Zipf(1.1) workload this
  // plan measured slower than the general one (21.8 ms a call: routing pass
  // 6.0 ms, bucket passes 4.5 + 1.7 ms, counting pass 1.0 ms, against 13.5 ms
  // for the whole general plan).  The shared-memory atomics of the hot rows
  // are the same work as the general plan's column passes.
  const char* on = std::getenv("LDF_B200_GB_PART");
  if (on == nullptr || std::atoi(on) == 0) return false;
  int64_t min_rows = int64_t(1) << 22;
  if (const char* e = std::getenv("LDF_B200_GB_PART_MIN_ROWS")) min_rows = std::max(0ll, std::atoll(e));
  const int64_t n = p.n;
  if (nkeys != 1 || n < std::max<int64_t>(min_rows, 1) || p.ncols < 1 || p.ncols > 2) return false;
  const ldf_column& kc = table[keys[0]];
  if (kc.type == LDF_STRING) return false;
  // value columns: the one of at most 4 bytes second
  int order[2] = {0, 1};
  if (p.ncols == 2 && type_width(p.c[1].col.type) > 4) std::swap(order[0], order[1]);
  if (p.ncols == 2 && type_width(p.c[order[1]].col.type) > 4) return false;
  int nd = -1;
  for (int q = 0; q < p.ncols; ++q) {
    const ColPlan& c = p.c[order[q]];
    if (c.col.type == LDF_STRING) return false;
    if (c.states & ST_NDIST) {
      if (nd >= 0 || type_width(c.col.type) > 4) return false;
      nd = q;
    }
  }
  const Allocator& al = ctx.alloc();
  cudaStream_t s      = ctx.stream();
  const int nsm       = num_sms();

  PartArgs a{};
  a.key  = make_dcol(kc);
  a.n    = n;
  a.ncol = p.ncols;
  a.nd   = nd;
  // record layouts
  int b = 12, w = 1;
  for (int q = 0; q < a.ncol; ++q) {
    PVal& v     = a.c[q];
    const ColPlan& c = p.c[order[q]];
    v.col       = c.col;
    v.nullable  = c.nullable;
    v.states    = c.states;
    v.fixed     = c.fixed;
    v.chunks    = c.fixed ? kSumChunks : 2;
    v.mm64      = type_width(c.col.type) > 4 ? 1 : 0;
    if (v.nullable) {
      v.b_vc = b;
      b += 4;
      v.w_vc = w++;
    }
  }
  b = (b + 15) & ~15;
  for (int q = 0; q < a.ncol; ++q) {
    PVal& v = a.c[q];
    if (v.states & ST_SUM) {
      v.b_sum = b;
      b += 16 * v.chunks;
      v.w_sum = w;
      w += v.fixed ? v.chunks : 1;
    }
  }
  for (int q = 0; q < a.ncol; ++q) {
    PVal& v       = a.c[q];
    const int mmw = v.mm64 ? 8 : 4;
    if (v.states & ST_MIN) {
      b = (b + mmw - 1) & ~(mmw - 1);
      v.b_mn = b;
      b += mmw;
      v.w_mn = w++;
    }
    if (v.states & ST_MAX) {
      b = (b + mmw - 1) & ~(mmw - 1);
      v.b_mx = b;
      b += mmw;
      v.w_mx = w++;
    }
  }
  a.rb = (b + 15) & ~15;
  a.rw = w;

  for (int j = 0; j < nkeys; ++j) hs.wait(keys[j]);
  // ---- sample: key frequencies (+ the NUNIQUE column's value range) ------------
  const int64_t ns     = std::min<int64_t>(n, int64_t(1) << 20);
  const int64_t stride = n / ns;
  const uint64_t scap  = static_cast<uint64_t>(2 * ns + 64);
  Buffer<unsigned long long> skeys(al, scap);
  Buffer<unsigned int> scounts(al, scap);
  Buffer<unsigned int> shist(al, 4096 + 4 + 2);  // count histogram, {occupied, singletons} (u64), value range
  LDF_CUDA(cudaMemsetAsync(skeys.get(), 0xff, scap * 8, s));
  LDF_CUDA(cudaMemsetAsync(scounts.get(), 0, scap * 4, s));
  LDF_CUDA(cudaMemsetAsync(shist.get(), 0, (4096 + 4) * 4, s));
  unsigned int* vr = shist.get() + 4096 + 4;
  const unsigned int vr_init[2] = {0xffffffffu, 0u};
  LDF_CUDA(cudaMemcpyAsync(vr, vr_init, 8, cudaMemcpyHostToDevice, s));
  launch("sample", part_sample_kernel, gs_blocks(ns, 256), 256, 0, s, a.key, ns, stride, skeys.get(), scounts.get(),
         scap);
  launch("freq_stats", part_sample_stats_kernel, gs_blocks(scap, 256), 256, 0, s,
         static_cast<const unsigned int*>(scounts.get()), scap, shist.get(),
         reinterpret_cast<unsigned long long*>(shist.get() + 4096));
  if (nd >= 0) {
    a.vflip = (a.c[nd].col.width == 4 && is_signed_int(a.c[nd].col.type)) ? 0x80000000u : 0u;
    hs.wait(col_of_plan[order[nd]]);
    const int wd = a.c[nd].col.width;
    auto vk      = wd == 1 ? value_range_kernel<1> : wd == 2 ? value_range_kernel<2> : value_range_kernel<4>;
    launch("value_range", vk, static_cast<unsigned>(4 * nsm), 256, 0, s, a.c[nd].col, n, a.vflip, vr);
  }
  std::vector<unsigned int> hh(4096 + 4 + 2);
  LDF_CUDA(cudaMemcpyAsync(hh.data(), shist.get(), hh.size() * 4, cudaMemcpyDeviceToHost, s));
  ctx.finish();
  unsigned long long occ_f1[2];
  std::memcpy(occ_f1, hh.data() + 4096, 16);
  const double scale       = std::sqrt(static_cast<double>(n) / static_cast<double>(ns));
  const int64_t est_groups = std::min<int64_t>(
    n, static_cast<int64_t>(scale * occ_f1[1] + (occ_f1[0] - occ_f1[1])) + 1);
  // hot set: bounded by shared memory (two routing CTAs per SM) and, with
  // NUNIQUE, by the value bitmaps' budget
  const int smem_route_budget = 110 * 1024;
  int hmax = std::min(kPartHotMax, (smem_route_budget - kPartHotSlots * 12) / a.rb - 1);
  if (nd >= 0) {
    if (hh[4096 + 4] > hh[4096 + 5]) {  // no valid value: a one-word range
      hh[4096 + 4] = 0;
      hh[4096 + 5] = 0;
    }
    a.vbase              = hh[4096 + 4];
    const uint64_t range = static_cast<uint64_t>(hh[4096 + 5]) - hh[4096 + 4] + 1;
    a.wpr                = static_cast<uint32_t>((((range + 31) / 32) + 3) / 4 * 4);
    uint64_t budget      = 96ull << 20;
    if (const char* e = std::getenv("LDF_B200_ND_BITMAP_MB")) budget = std::max(0ll, std::atoll(e)) << 20;
    const int64_t hb = static_cast<int64_t>(budget / (4ull * a.wpr)) - 1;
    if (hb < 16) return false;  // value range too wide for the bitmaps
    hmax = static_cast<int>(std::min<int64_t>(hmax, hb));
  }
  // smallest count threshold (>= 2) whose keys fit the hot set
  int64_t above = 0;
  unsigned int thr = 4096;
  for (int c = 4095; c >= 2; --c) {
    if (above + hh[c] > hmax) break;
    above += hh[c];
    thr = static_cast<unsigned int>(c);
  }
  a.H = static_cast<int>(above);
  Buffer<unsigned long long> hot_keys(al, std::max(a.H, 1));
  if (a.H > 0) {
    Buffer<unsigned int> nhot(al, 1);
    LDF_CUDA(cudaMemsetAsync(nhot.get(), 0, 4, s));
    launch("hot_select", part_hot_select_kernel, gs_blocks(scap, 256), 256, 0, s,
           static_cast<const unsigned long long*>(skeys.get()), static_cast<const unsigned int*>(scounts.get()),
           scap, thr, hot_keys.get(), nhot.get(), a.H);
  }
  a.hot_keys = hot_keys.get();
  // buckets: about 200 groups each
  int logP = 0;
  // (the sampled estimate undercounts a heavy-tailed key distribution: 2.2M
  // for the 6.7M groups of Zipf(1.1) over 10M keys at 200M rows)
  while (logP < 15 && (int64_t(200) << logP) < 3 * est_groups) ++logP;
  a.logP          = logP;
  const int64_t P = int64_t(1) << logP;

  // ---- counting pre-pass ---------------------------------------------------------
  Buffer<unsigned int> hist(al, P);
  LDF_CUDA(cudaMemsetAsync(hist.get(), 0, P * 4, s));
  a.hist = hist.get();
  const size_t count_smem = kPartHotSlots * 12 + P * 4;
  LDF_CUDA(cudaFuncSetAttribute(part_count_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(count_smem)));
  int occ = 1;
  LDF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, part_count_kernel, kCountThreads, count_smem));
  launch("part_count", part_count_kernel, static_cast<unsigned>(std::max(occ, 1) * nsm), kCountThreads, count_smem, s,
         a);
  std::vector<unsigned int> hist_h(P);
  LDF_CUDA(cudaMemcpyAsync(hist_h.data(), hist.get(), P * 4, cudaMemcpyDeviceToHost, s));
  ctx.finish();
  std::vector<int64_t> bstart_h(P + 1);
  int64_t cold = 0;
  for (int64_t q = 0; q < P; ++q) {
    bstart_h[q] = cold;
    cold += hist_h[q];
  }
  bstart_h[P] = cold;
  // 32-bit NUNIQUE pairs (local id << 20 | value offset) when the values
  // span at most 2^20: twice the rows fit the shared pair set
  const bool pair32        = nd >= 0 && a.wpr <= (1u << 20) / 32;
  const int64_t small_rows = kBucketRecBytes / (pair32 ? 4 : 8) / 2 - 64;
  std::vector<int32_t> large_h;
  int64_t large_max = 0;
  for (int64_t q = 0; q < P; ++q)
    if (hist_h[q] > small_rows) {
      large_h.push_back(static_cast<int32_t>(q));
      large_max = std::max<int64_t>(large_max, hist_h[q]);
    }
  Buffer<int64_t> bstart(al, P + 1);
  LDF_CUDA(cudaMemcpyAsync(bstart.get(), bstart_h.data(), (P + 1) * 8, cudaMemcpyHostToDevice, s));
  a.bstart = bstart.get();

  // ---- routing pass ----------------------------------------------------------------
  Buffer<unsigned int> bcursor(al, P);
  Buffer<unsigned long long> recs(al, std::max<int64_t>(3 * cold, 1));
  Buffer<unsigned long long> hot_rec(al, static_cast<int64_t>(a.H + 1) * a.rw);
  Buffer<uint32_t> bits;
  Buffer<int> flag(al, 1);
  LDF_CUDA(cudaMemsetAsync(bcursor.get(), 0, P * 4, s));
  LDF_CUDA(cudaMemsetAsync(hot_rec.get(), 0, static_cast<size_t>(a.H + 1) * a.rw * 8, s));
  LDF_CUDA(cudaMemsetAsync(flag.get(), 0, 4, s));
  if (nd >= 0) {
    bits = Buffer<uint32_t>(al, static_cast<int64_t>(a.H + 1) * a.wpr);
    LDF_CUDA(cudaMemsetAsync(bits.get(), 0, static_cast<size_t>(a.H + 1) * a.wpr * 4, s));
    a.bits = bits.get();
  }
  a.bcursor = bcursor.get();
  a.recs    = recs.get();
  a.hot_rec = hot_rec.get();
  a.flag    = flag.get();
  for (int q = 0; q < a.ncol; ++q) hs.wait(col_of_plan[order[q]]);
  const size_t route_smem = kPartHotSlots * 12 + static_cast<size_t>(a.H + 1) * a.rb;
  auto kind = [&](int q) {
    return a.c[q].col.type == LDF_FLOAT64 ? PK_F64 : a.c[q].col.type == LDF_INT32 ? PK_I32 : PK_GEN;
  };
  const int k0 = kind(0), k1 = a.ncol > 1 ? kind(1) : PK_NONE;
  auto route = k0 == PK_F64 && k1 == PK_I32    ? part_route_kernel<PK_F64, PK_I32>
               : k0 == PK_F64 && k1 == PK_NONE ? part_route_kernel<PK_F64, PK_NONE>
                                               : part_route_kernel<PK_GEN, PK_GEN>;
  LDF_CUDA(cudaFuncSetAttribute(route, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(route_smem)));
  LDF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, route, kPartThreads, route_smem));
  launch("part_route", route,
         static_cast<unsigned>(std::min<int64_t>(std::max(occ, 1) * nsm, ceil_div(n, int64_t(kPartThreads) * kRows))),
         kPartThreads, route_smem, s, a);

  // ---- outputs, bucket passes, hot groups ---------------------------------------
  PartOut o{};
  o.nagg = naggs;
  int64_t cap_out = std::min<int64_t>(cold + a.H + 1, 2 * est_groups + a.H + 4096);
  std::vector<ldf_column> big(nkeys + naggs);
  auto alloc_outputs = [&](int64_t rows) {
    big[0] = alloc_out_column(al, kc.type, rows, kc.valid != nullptr);
    o.key  = OCol{big[0].data, big[0].valid, kc.type, type_width(kc.type)};
    for (int g = 0; g < naggs; ++g) {
      const ldf_aggregation& ag = aggs[g];
      const bool nullable       = !(ag.kind == LDF_AGG_COUNT_ALL || ag.kind == LDF_AGG_COUNT_DISTINCT);
      big[1 + g]                = alloc_out_column(al, ag.out_type, rows, nullable);
      AggOut& x                 = o.a[g];
      x.kind                    = ag.kind;
      x.count_mode              = ag.count_mode;
      x.col                     = -1;
      if (agg_col[g] >= 0) x.col = agg_col[g] == order[0] ? 0 : 1;
      x.in_type = ag.kind == LDF_AGG_COUNT_ALL ? LDF_INT64 : table[ag.in_col].type;
      x.dst     = OCol{big[1 + g].data, big[1 + g].valid, ag.out_type, type_width(ag.out_type)};
    }
  };
  auto free_outputs = [&]() {
    for (auto& c : big) free_out_column(al, c);
  };
  Buffer<unsigned long long> counters(al, 4);  // out rows, bucket counter, large counter, deferred count
  Buffer<int32_t> deferred(al, P);
  BucketArgs B{};
  B.a          = a;
  B.out_count  = counters.get();
  B.small_rows = small_rows;
  B.pair32     = pair32 ? 1 : 0;
  B.err        = ctx.err();
  B.deferred   = deferred.get();
  B.ndeferred  = reinterpret_cast<unsigned int*>(counters.get() + 3);
  Buffer<int32_t> large(al, std::max<int64_t>(static_cast<int64_t>(large_h.size()), 1));
  if (!large_h.empty())
    LDF_CUDA(cudaMemcpyAsync(large.get(), large_h.data(), large_h.size() * 4, cudaMemcpyHostToDevice, s));
  const size_t bucket_smem = kBucketKeySlots * 12 + kBucketRecBytes + kBucketGroupsMax * 5;
  LDF_CUDA(cudaFuncSetAttribute(part_bucket_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(bucket_smem)));
  // per-CTA global work memory of the large pass, sized for `rows` rows
  auto large_pass = [&](const int32_t* list, int64_t nlist, int64_t rows) {
    if (nlist == 0) return;
    int ks = 64;
    while (ks < 2 * rows + 64) ks *= 2;
    const int64_t gc  = rows;
    const int64_t ps  = 2 * rows + 64;
    const int64_t rbytes = std::max<int64_t>(gc * a.rb, ps * 8);
    const int64_t stride = ((static_cast<int64_t>(ks) * 12 + rbytes + gc * 5) + 255) / 256 * 256;
    const int64_t grid   = std::min<int64_t>(nlist, nsm);
    Buffer<unsigned char> scratch(al, grid * stride);
    BucketArgs L = B;
    L.list           = list;
    L.nlist          = nlist;
    L.next           = counters.get() + 2;
    L.scratch        = scratch.get();
    L.scratch_stride = stride;
    L.ks             = ks;
    L.gc             = static_cast<int>(gc);
    L.ps             = ps;
    L.pair32         = 0;  // local ids may pass 4096 here
    LDF_CUDA(cudaMemsetAsync(counters.get() + 2, 0, 8, s));
    launch("part_bucket_large", part_bucket_large_kernel, static_cast<unsigned>(grid), kBucketThreads, 0, s, L);
  };
  for (int attempt = 0;; ++attempt) {
    alloc_outputs(cap_out);
    B.o       = o;
    B.out_cap = cap_out;
    B.next    = counters.get() + 1;
    LDF_CUDA(cudaMemsetAsync(counters.get(), 0, 32, s));
    launch("part_bucket", part_bucket_kernel, static_cast<unsigned>(2 * nsm), kBucketThreads, bucket_smem, s, B);
    large_pass(large.get(), static_cast<int64_t>(large_h.size()), large_max);
    launch("part_hot_emit", part_hot_emit_kernel, static_cast<unsigned>(std::min(a.H + 1, 4 * nsm)), 256, 0, s, a,
           o, counters.get(), cap_out);
    unsigned long long cnt[4];
    int fl = 0;
    LDF_CUDA(cudaMemcpyAsync(cnt, counters.get(), 32, cudaMemcpyDeviceToHost, s));
    LDF_CUDA(cudaMemcpyAsync(&fl, flag.get(), 4, cudaMemcpyDeviceToHost, s));
    ctx.finish();
    if (fl != 0) {  // a float sum value outside the fixed-point range: the general plan
      free_outputs();
      return false;
    }
    const int64_t ndef = static_cast<int64_t>(cnt[3] & 0xffffffffull);
    if (ndef > 0) {  // buckets with more groups than the shared records hold
      std::vector<int32_t> dh(ndef);
      LDF_CUDA(cudaMemcpyAsync(dh.data(), deferred.get(), ndef * 4, cudaMemcpyDeviceToHost, s));
      ctx.finish();
      int64_t rows = 0;
      for (int32_t q : dh) rows = std::max<int64_t>(rows, hist_h[q]);
      large_pass(deferred.get(), ndef, rows);
      LDF_CUDA(cudaMemcpyAsync(cnt, counters.get(), 8, cudaMemcpyDeviceToHost, s));
      ctx.finish();
    }
    const int64_t G = static_cast<int64_t>(cnt[0]);
    if (G > cap_out) {  // more groups than the estimate allowed for: once more with room for all
      if (attempt >= 2) fail(LDF_ERR_INTERNAL, "groupby output overflow");
      free_outputs();
      cap_out = G;
      continue;
    }
    // outputs of exactly G rows
    for (int j = 0; j < nkeys + naggs; ++j) {
      const ldf_column& c = big[j];
      ldf_column e        = alloc_out_column(al, c.type, G, c.valid != nullptr);
      const int wdt       = type_width(c.type);
      if (G > 0) {
        LDF_CUDA(cudaMemcpyAsync(e.data, c.data, static_cast<size_t>(G) * wdt, cudaMemcpyDeviceToDevice, s));
        if (c.valid) LDF_CUDA(cudaMemcpyAsync(e.valid, c.valid, static_cast<size_t>(G), cudaMemcpyDeviceToDevice, s));
      }
      out[j] = e;
    }
    ctx.finish();
    free_outputs();
    return true;
  }
}

}  // namespace

void groupby_aggregation(const ldf_column* table, int ncols, const int32_t* keys, int nkeys,
                         const ldf_aggregation* aggs, int naggs, ldf_column* out, const OpContext& ctx)
{
  if (nkeys < 1) fail(LDF_ERR_INVALID_ARGUMENT, "must pass at least one key column");
  LDF_REQUIRE(naggs <= kMaxAggs, "too many aggregations");
  // Host-resident inputs are copied in the order the passes read them: the
  // keys, then NUNIQUE inputs, then the other aggregated columns.
  std::vector<int> order(keys, keys + nkeys);
  for (int pass = 0; pass < 2; ++pass)
    for (int a = 0; a < naggs; ++a)
      if (aggs[a].kind != LDF_AGG_COUNT_ALL && (aggs[a].kind == LDF_AGG_COUNT_DISTINCT) == (pass == 0))
        order.push_back(aggs[a].in_col);
  for (int j = 0; j < nkeys; ++j) LDF_REQUIRE(keys[j] >= 0 && keys[j] < ncols, "key column index out of range");
  HostStaging hs(ctx, table, ncols, order);
  table = hs.table();
  KeyCols k       = make_keys(table, ncols, keys, nkeys);
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
      ColPlan& cp    = p.c[ci];
      cp.col         = make_dcol(c);
      cp.nullable    = c.valid != nullptr;
      cp.fixed       = is_float(c.type) ? 1 : 0;
      cp.pair_packed = type_width(c.type) <= 4 && c.type != LDF_STRING;
    }
    agg_col[a]  = ci;
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
  if (try_partitioned(ctx, p, table, keys, nkeys, aggs, naggs, agg_col, out, hs, col_of_plan)) return;
  switch (key_mode(k)) {
    case KeyMode::K32:
      run_groupby<KeyMode::K32>(ctx, p, table, keys, nkeys, aggs, naggs, agg_col, out, hs, col_of_plan);
      break;
    case KeyMode::K64:
      run_groupby<KeyMode::K64>(ctx, p, table, keys, nkeys, aggs, naggs, agg_col, out, hs, col_of_plan);
      break;
    default: run_groupby<KeyMode::GEN>(ctx, p, table, keys, nkeys, aggs, naggs, agg_col, out, hs, col_of_plan); break;
  }
}

}  // namespace ldf
