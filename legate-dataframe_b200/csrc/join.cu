// Hash join (inner / left / full / semi / anti), build on rhs, probe with lhs.
//
// Reference semantics: JoinTask::cpu_variant -> arrow_join_and_gather
// (cpp/src/join.cpp:168-228) and JoinTask::gpu_variant -> cudf_join +
// cudf::gather (cpp/src/join.cu:32-155):
//  * nulls_equal: a null key matches a null key and nothing else (join.cpp:117-162
//    coalesces nullable keys and adds the validity column as an extra key).
//  * !nulls_equal: rows with a null in any key never match.
//  * LEFT: unmatched lhs rows emit nulls for the rhs columns; FULL additionally
//    emits unmatched rhs rows with nulls for the lhs columns (NULLIFY gather,
//    join.cu:79-101).  SEMI/ANTI emit lhs rows with / without a match.
//
// Device plan (one GPU, stream ordered):
//  1. build   a single integer key whose build values span at most twice the
//             build rows gets a direct-address table (row of key - min; a
//             repeated key falls back to hashing).  Otherwise an
//             open-addressing table over the rhs keys, linear probing, load
//             factor 0.5, 8-byte slots {row, key32 | hash tag} (16-byte
//             {key64, row} for 8-byte keys).  Nullable single keys with
//             nulls_equal keep their null rows in a separate "null list".
//  2. unique? one self-probe over the build keys.  Unique build keys bound
//             the output by the probe size, so the probe runs ONCE and each
//             tile claims its output range with one atomic on the running
//             total (no tile waits on another; output rows come in tile
//             completion order); otherwise a count pass sizes every tile's
//             output exactly first.
//  3. probe   tiles of 256 threads x 4 rows: the items' first lookups are
//             prefetched together, matches resolved, the block scan counts
//             output rows, then the fixed-width output columns are written
//             directly from the probe kernel, column by column with the
//             items' loads issued together (the gather is fused: no gather
//             maps for fixed-width columns).  The build key column is
//             written from the equal probe key, and two other build columns
//             can come packed in one 16-byte record per build row.  String
//             output columns go through int32 gather maps and a string
//             gather.
//  4. FULL    unmatched rhs rows (never touched by a probe) are compacted and
//             appended after the probe output.
// Optional (LDF_B200_JOIN_PARTITION=1): both sides are first scattered into
// 256 hash partitions so that the build partitions being probed stay in L2.
// On the 200M x 20M int32-key workload on B200 it probed faster than the
// hash table (5.6 vs 7.9 ms) but the partitioning cost more than it saved,
// so it is off by default (and dense keys take the direct table instead).
#include "table_ops.cuh"

namespace ldf {
namespace {

constexpr int kProbeThreads = 256;
constexpr int kProbeItems   = 4;
constexpr int kProbeTile    = kProbeThreads * kProbeItems;
constexpr uint64_t kEmpty64 = ~0ull;

struct Slot16 {
  uint64_t key;
  uint64_t row;
};

template <int W>
__device__ __forceinline__ uint64_t load_w(const void* data, int64_t r)
{
  if (W == 1) return __ldg(static_cast<const uint8_t*>(data) + r);
  if (W == 2) return __ldg(static_cast<const uint16_t*>(data) + r);
  if (W == 4) return __ldg(static_cast<const uint32_t*>(data) + r);
  return __ldg(static_cast<const unsigned long long*>(data) + r);
}
template <int W>
__device__ __forceinline__ void store_w(void* data, int64_t i, uint64_t v)
{
  if (W == 1) static_cast<uint8_t*>(data)[i] = static_cast<uint8_t>(v);
  else if (W == 2) static_cast<uint16_t*>(data)[i] = static_cast<uint16_t>(v);
  else if (W == 4) static_cast<uint32_t*>(data)[i] = static_cast<uint32_t>(v);
  else static_cast<unsigned long long*>(data)[i] = v;
}

// Streaming (evict-first) forms for the probe side and the output rows, which
// are touched once: they then leave L2 before the build-side table and
// payload records that the probe rows hit repeatedly.
template <int W>
__device__ __forceinline__ uint64_t load_w_stream(const void* data, int64_t r)
{
  if (W == 1) return __ldcs(static_cast<const unsigned char*>(data) + r);
  if (W == 2) return __ldcs(static_cast<const unsigned short*>(data) + r);
  if (W == 4) return __ldcs(static_cast<const unsigned int*>(data) + r);
  return __ldcs(static_cast<const unsigned long long*>(data) + r);
}
template <int W>
__device__ __forceinline__ void store_w_stream(void* data, int64_t i, uint64_t v)
{
  if (W == 1) __stcs(static_cast<unsigned char*>(data) + i, static_cast<unsigned char>(v));
  else if (W == 2) __stcs(static_cast<unsigned short*>(data) + i, static_cast<unsigned short>(v));
  else if (W == 4) __stcs(static_cast<unsigned int*>(data) + i, static_cast<unsigned int>(v));
  else __stcs(static_cast<unsigned long long*>(data) + i, static_cast<unsigned long long>(v));
}

// Device-side view of the build table.
struct BuildTable {
  KeyCols bk;             // build keys (rhs)
  void* slots;            // uint64_t[cap] (K32, GEN) or Slot16[cap] (K64)
  uint64_t cap;
  const int32_t* null_list;  // rows with a null single key (nulls_equal, K32/K64)
  const int64_t* null_count;
  int nulls_equal;
  // Radix-partitioned tables (K32/K64): partition b = top 8 bits of the key
  // hash owns slots [part_base[b], part_base[b] + part_cap[b]); the slot
  // inside it comes from the remaining hash bits.
  int parts;
  const uint64_t* part_base;
  const uint64_t* part_cap;
  int* dup;  // K32: set by the build when a key occurs twice
  // Dense integer keys (K32/K64): direct[key - dmin] = the build row with
  // that key (-1 none) for the drange values from dmin on, instead of slots.
  const int32_t* direct;
  int64_t dmin, dmax;
  uint64_t drange;
};

// Slot of key value k in a direct-address table, or drange when k is outside
// [dmin, dmax] (compared as values, so no wrap-around can alias a slot).
__device__ __forceinline__ uint64_t direct_slot(const BuildTable& t, int64_t k)
{
  return (k >= t.dmin && k <= t.dmax) ? static_cast<uint64_t>(k - t.dmin) : t.drange;
}

// Integer value of a single fixed-width key (sign-extended for signed types).
__device__ __forceinline__ int64_t key_value(const DCol& c, int64_t r)
{
  switch (c.type) {
    case LDF_INT8: return static_cast<const int8_t*>(c.data)[r];
    case LDF_INT16: return static_cast<const int16_t*>(c.data)[r];
    case LDF_INT32: return static_cast<const int32_t*>(c.data)[r];
    case LDF_INT64:
    case LDF_TIMESTAMP_US: return static_cast<const int64_t*>(c.data)[r];
    default: return static_cast<int64_t>(dbits(c, r));  // unsigned, bool
  }
}

// First slot and slot range [lo, hi) of hash h.
__device__ __forceinline__ uint64_t first_slot(const BuildTable& t, uint64_t h, uint64_t& lo, uint64_t& hi)
{
  if (t.parts) {
    const uint32_t b = static_cast<uint32_t>(h >> 56);
    lo               = t.part_base[b];
    const uint64_t c = t.part_cap[b];
    hi               = lo + c;
    return lo + fastrange(h << 8, c);
  }
  lo = 0;
  hi = t.cap;
  return fastrange(h, t.cap);
}
__device__ __forceinline__ uint64_t next_slot(uint64_t i, uint64_t lo, uint64_t hi) { return i + 1 == hi ? lo : i + 1; }

template <KeyMode M>
__global__ void build_kernel(BuildTable t, int64_t n)
{
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n;
       r += (int64_t)gridDim.x * blockDim.x) {
    if (M == KeyMode::GEN) {
      if (!t.nulls_equal && key_has_null(t.bk, r)) continue;
    } else {
      if (!dvalid(t.bk.c[0], r)) continue;  // null rows: null list or excluded
    }
    uint64_t kb  = key_bits<M>(t.bk, r);
    uint64_t h   = M == KeyMode::GEN ? kb : mix64(kb);
    uint64_t lo, hi;
    uint64_t idx = first_slot(t, h, lo, hi);
    if (M == KeyMode::K64) {
      Slot16* s = static_cast<Slot16*>(t.slots);
      while (true) {
        unsigned long long old = atomicCAS(reinterpret_cast<unsigned long long*>(&s[idx].row),
                                           kEmpty64, static_cast<unsigned long long>(r));
        if (old == kEmpty64) {
          s[idx].key = kb;
          break;
        }
        idx = next_slot(idx, lo, hi);
      }
    } else {
      uint32_t tag   = M == KeyMode::GEN ? static_cast<uint32_t>(h) : static_cast<uint32_t>(kb);
      uint64_t entry = (static_cast<uint64_t>(r) << 32) | tag;
      uint64_t* s    = static_cast<uint64_t*>(t.slots);
      while (true) {
        const unsigned long long old = atomicCAS(reinterpret_cast<unsigned long long*>(&s[idx]), kEmpty64,
                                                 static_cast<unsigned long long>(entry));
        if (old == kEmpty64) break;
        // K32: the tag is the whole key, and an equal key inserted earlier
        // (or concurrently) always lies on this probe path
        if (M == KeyMode::K32 && t.dup && static_cast<uint32_t>(old) == tag) *t.dup = 1;
        idx = next_slot(idx, lo, hi);
      }
    }
  }
}

// Range of the valid build keys' values: mm[0] = min, mm[1] = max (as
// order-preserving unsigned words), mm[2] = 1 when an unsigned 64-bit key
// does not fit int64.
__global__ void key_range_kernel(DCol key, int64_t n, unsigned long long* mm)
{
  unsigned long long lo = ~0ull, hi = 0;
  int wide              = 0;
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
    if (!dvalid(key, r)) continue;
    const int64_t v = key_value(key, r);
    if (key.type == LDF_UINT64 && v < 0) wide = 1;
    const unsigned long long o = static_cast<unsigned long long>(v) ^ (1ull << 63);
    lo                         = o < lo ? o : lo;
    hi                         = o > hi ? o : hi;
  }
  for (int d = 16; d > 0; d >>= 1) {
    const unsigned long long l2 = __shfl_xor_sync(0xffffffffu, lo, d), h2 = __shfl_xor_sync(0xffffffffu, hi, d);
    lo                          = l2 < lo ? l2 : lo;
    hi                          = h2 > hi ? h2 : hi;
  }
  wide = __any_sync(0xffffffffu, wide);
  if ((threadIdx.x & 31) == 0) {
    atomicMin(mm, lo);
    atomicMax(mm + 1, hi);
    if (wide) atomicExch(mm + 2, 1ull);
  }
}

// Direct-address build: a second row with the same key sets *dup.
__global__ void direct_build_kernel(DCol key, int64_t n, int64_t dmin, int32_t* direct, int* dup)
{
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
    if (!dvalid(key, r)) continue;  // null rows: null list or excluded
    const uint64_t u = static_cast<uint64_t>(key_value(key, r) - dmin);  // every valid key lies in [dmin, dmax]
    if (atomicCAS(direct + u, -1, static_cast<int32_t>(r)) != -1) *dup = 1;
  }
}

// Enumerate the build rows matching probe row r of `pk`; f(build_row) returns
// false to stop early.
template <KeyMode M, typename F>
__device__ __forceinline__ void for_each_match(const BuildTable& t, const KeyCols& pk, int64_t r, F f)
{
  if (M == KeyMode::GEN) {
    if (!t.nulls_equal && key_has_null(pk, r)) return;
  } else if (!dvalid(pk.c[0], r)) {
    if (t.nulls_equal && t.null_list) {
      int64_t nn = *t.null_count;
      for (int64_t i = 0; i < nn; ++i)
        if (!f(static_cast<int64_t>(t.null_list[i]))) return;
    }
    return;
  }
  if (M != KeyMode::GEN && t.direct) {
    const uint64_t u = direct_slot(t, key_value(pk.c[0], r));
    if (u < t.drange) {
      const int32_t br = __ldg(t.direct + u);
      if (br >= 0) f(static_cast<int64_t>(br));
    }
    return;
  }
  uint64_t kb  = key_bits<M>(pk, r);
  uint64_t h   = M == KeyMode::GEN ? kb : mix64(kb);
  uint64_t lo, hi;
  uint64_t idx = first_slot(t, h, lo, hi);
  if (M == KeyMode::K64) {
    const Slot16* s = static_cast<const Slot16*>(t.slots);
    while (true) {
      Slot16 v = s[idx];
      if (v.row == kEmpty64) return;
      if (v.key == kb && !f(static_cast<int64_t>(v.row))) return;
      idx = next_slot(idx, lo, hi);
    }
  } else {
    const uint64_t* s = static_cast<const uint64_t*>(t.slots);
    uint32_t tag      = M == KeyMode::GEN ? static_cast<uint32_t>(h) : static_cast<uint32_t>(kb);
    while (true) {
      uint64_t v = __ldg(reinterpret_cast<const unsigned long long*>(&s[idx]));
      if (v == kEmpty64) return;
      if (static_cast<uint32_t>(v) == tag) {
        int64_t br = static_cast<int64_t>(v >> 32);
        if (M != KeyMode::GEN || keys_equal(pk, r, t.bk, br)) {
          if (!f(br)) return;
        }
      }
      idx = next_slot(idx, lo, hi);
    }
  }
}

// Self-probe of the build rows: sets *dup when some key occurs twice.
template <KeyMode M>
__global__ void dup_check_kernel(BuildTable t, int64_t n, int* dup)
{
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n;
       r += (int64_t)gridDim.x * blockDim.x) {
    if (M == KeyMode::GEN) {
      if (!t.nulls_equal && key_has_null(t.bk, r)) continue;
    } else if (!dvalid(t.bk.c[0], r)) {
      continue;
    }
    int c = 0;
    for_each_match<M>(t, t.bk, r, [&](int64_t) { return ++c < 2; });
    if (c > 1) atomicExch(dup, 1);
  }
  // Null rows with nulls_equal all match one another.
  if (M != KeyMode::GEN && t.nulls_equal && t.null_list && blockIdx.x == 0 && threadIdx.x == 0) {
    if (*t.null_count > 1) atomicExch(dup, 1);
  }
}

// Null list of a nullable single build key: rows with a null key, in row order.
__global__ void null_list_kernel(DCol key, int64_t n, int32_t* list, uint64_t* status,
                                 unsigned long long* counter, int64_t* count, int* err)
{
  __shared__ int64_t s_scan[kProbeThreads / 32 + 1];
  __shared__ int64_t s_tile;
  __shared__ uint64_t s_prefix;
  const int64_t tile = next_tile_id(counter, &s_tile);
  const int64_t base = tile * kProbeTile + static_cast<int64_t>(threadIdx.x) * kProbeItems;
  int f[kProbeItems];
  int64_t c = 0;
#pragma unroll
  for (int i = 0; i < kProbeItems; ++i) {
    int64_t r = base + i;
    f[i]      = (r < n && !dvalid(key, r)) ? 1 : 0;
    c += f[i];
  }
  int64_t tot;
  int64_t ex = block_exclusive_scan<int64_t, kProbeThreads>(c, s_scan, &tot);
  if (threadIdx.x == 0) {
    s_prefix = lookback_exclusive(status, tile, static_cast<uint64_t>(tot), err);
    if (tile == static_cast<int64_t>(gridDim.x) - 1) *count = static_cast<int64_t>(s_prefix) + tot;
  }
  __syncthreads();
  int64_t pos = static_cast<int64_t>(s_prefix) + ex;
#pragma unroll
  for (int i = 0; i < kProbeItems; ++i)
    if (f[i]) list[pos++] = static_cast<int32_t>(base + i);
}

struct ProbeArgs {
  BuildTable t;
  KeyCols pk;
  int64_t n_probe;
  int join_type;
  OutSpec lo;  // lhs output columns
  OutSpec ro;  // rhs output columns
  int32_t* lmap;  // gather maps (string outputs), may be null
  int32_t* rmap;
  uint8_t* matched;  // FULL: per build row
  uint32_t* tile_counts;        // count pass output
  const int64_t* tile_offsets;  // write pass with known offsets (null -> claim with an atomic)
  int64_t* total;  // device: number of rows written by the probe
  // Build-side outputs.  rkey: the column of `ro` that is the build key
  // (-1 none): a matched row takes it from its own probe key, which is equal.
  // rpack: two other columns (ro indices pcol[0], pcol[1]) packed per build
  // row as two 8-byte words, read with one 16-byte load (null: none packed).
  int rkey;
  const ulonglong2* rpack;
  int pcol[2];
  int* err;
};

// Output rows produced by one probe row with m matches.
__device__ __forceinline__ int out_rows(int jt, int m)
{
  switch (jt) {
    case LDF_JOIN_INNER: return m;
    case LDF_JOIN_LEFT:
    case LDF_JOIN_FULL: return m > 0 ? m : 1;
    case LDF_JOIN_SEMI: return m > 0 ? 1 : 0;
    default: return m > 0 ? 0 : 1;  // ANTI
  }
}

__device__ __forceinline__ void emit(const ProbeArgs& a, int64_t pos, int64_t lrow, int64_t brow)
{
  write_out_row(a.lo, pos, lrow);
  write_out_row(a.ro, pos, brow);
  if (a.lmap) a.lmap[pos] = static_cast<int32_t>(lrow);
  if (a.rmap) a.rmap[pos] = static_cast<int32_t>(brow);
}

// Write output column set `o` for the kProbeItems rows of a thread at once:
// for each column, the items' source values are loaded together, then
// stored (row[i] < 0 -> null / zero; pos[i] < 0 -> no output row).  STREAM:
// the source is the probe side (rows in order, read once); otherwise the
// build side (random rows, kept in L2).
template <int W, bool STREAM>
__device__ __forceinline__ void emit_column_batch(const DCol& src, const OCol& d, const int64_t* pos,
                                                  const int64_t* row)
{
  uint64_t v[kProbeItems];
  bool ok[kProbeItems];
#pragma unroll
  for (int i = 0; i < kProbeItems; ++i) {
    ok[i] = row[i] >= 0;
    v[i]  = 0;
    if (pos[i] >= 0 && ok[i]) v[i] = STREAM ? load_w_stream<W>(src.data, row[i]) : load_w<W>(src.data, row[i]);
    if (d.valid && pos[i] >= 0 && ok[i] && src.valid)
      ok[i] = (STREAM ? __ldcs(src.valid + row[i]) : __ldg(src.valid + row[i])) != 0;
  }
#pragma unroll
  for (int i = 0; i < kProbeItems; ++i) {
    if (pos[i] < 0) continue;
    store_w_stream<W>(d.data, pos[i], v[i]);
    if (d.valid) __stcs(d.valid + pos[i], static_cast<uint8_t>(ok[i] ? 1 : 0));
  }
}

// One output column of `o` from source rows row[i] (see emit_column_batch).
template <bool STREAM>
__device__ __forceinline__ void emit_one(const DCol& src, const OCol& d, const int64_t* pos, const int64_t* row)
{
  switch (d.width) {
    case 1: emit_column_batch<1, STREAM>(src, d, pos, row); break;
    case 2: emit_column_batch<2, STREAM>(src, d, pos, row); break;
    case 4: emit_column_batch<4, STREAM>(src, d, pos, row); break;
    default: emit_column_batch<8, STREAM>(src, d, pos, row); break;
  }
}

// Build-side output columns of the thread's items (brow[i] < 0: no match).
__device__ __forceinline__ void emit_build_batch(const ProbeArgs& a, const int64_t* pos, const int64_t* lrow,
                                                 const int64_t* brow)
{
  const OutSpec& o = a.ro;
  if (a.rpack) {
    ulonglong2 w[kProbeItems];
#pragma unroll
    for (int i = 0; i < kProbeItems; ++i)
      w[i] = (pos[i] >= 0 && brow[i] >= 0) ? __ldg(a.rpack + brow[i]) : make_ulonglong2(0, 0);
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const OCol& d = o.dst[a.pcol[q]];
#pragma unroll
      for (int i = 0; i < kProbeItems; ++i) {
        if (pos[i] < 0) continue;
        const uint64_t v = q == 0 ? w[i].x : w[i].y;
        switch (d.width) {
          case 1: store_w_stream<1>(d.data, pos[i], v); break;
          case 2: store_w_stream<2>(d.data, pos[i], v); break;
          case 4: store_w_stream<4>(d.data, pos[i], v); break;
          default: store_w_stream<8>(d.data, pos[i], v); break;
        }
        if (d.valid) __stcs(d.valid + pos[i], static_cast<uint8_t>(brow[i] >= 0 ? 1 : 0));
      }
    }
  }
  for (int j = 0; j < o.n; ++j) {
    if (a.rpack && (j == a.pcol[0] || j == a.pcol[1])) continue;
    if (j == a.rkey) {
      // the probe key of a matched row (its validity too: null keys match
      // only null keys)
      int64_t krow[kProbeItems];
#pragma unroll
      for (int i = 0; i < kProbeItems; ++i) krow[i] = brow[i] >= 0 ? lrow[i] : -1;
      emit_one<true>(a.pk.c[0], o.dst[j], pos, krow);
    } else {
      emit_one<false>(o.src[j], o.dst[j], pos, brow);
    }
  }
}

// The probe-side output columns (rows in order, streamed).
__device__ __forceinline__ void emit_batch(const OutSpec& o, const int64_t* pos, const int64_t* row)
{
  for (int j = 0; j < o.n; ++j) emit_one<true>(o.src[j], o.dst[j], pos, row);
}

// COUNT: per-tile output counts.  WRITE: probe again (or use the single match
// of a unique build side) and write output rows at the tile's offset.
//
// Resident CTAs per SM asked of the compiler for each variant.  The one-pass
// probe of 4-byte keys waits on one random load per matched row: at six CTAs
// (40 registers, a few spilled bytes that stay in L1) instead of five it runs
// 2-4 % faster on B200.  The other values pin the register budgets the
// compiler picks for those variants by itself (64 for multi-column keys, 48
// for the other unique writes, 32 for the rest).
template <KeyMode M, bool WRITE, bool UNIQUE>
constexpr int probe_min_blocks()
{
  if (M == KeyMode::GEN) return 4;
  if (WRITE && UNIQUE) return M == KeyMode::K32 ? 6 : 5;
  return 8;
}

template <KeyMode M, bool WRITE, bool UNIQUE>
__global__ void __launch_bounds__(kProbeThreads, (probe_min_blocks<M, WRITE, UNIQUE>()))
probe_kernel(ProbeArgs a)
{
  __shared__ int64_t s_scan[kProbeThreads / 32 + 1];
  __shared__ uint64_t s_prefix;
  // Without precomputed tile offsets (unique build keys) a tile claims its
  // output range with one atomic on the running total: no tile waits on
  // another, and output rows come in tile completion order.
  const bool claim   = WRITE && a.tile_offsets == nullptr;
  const int64_t tile = static_cast<int64_t>(blockIdx.x);
  const int64_t base = tile * kProbeTile;

  int m[kProbeItems];
  int64_t first[kProbeItems];
  int64_t cnt = 0;
  if (M != KeyMode::GEN) {
    // touch every item's first slot before resolving any: the loads overlap
    // and the resolving walks below mostly hit L1
#pragma unroll
    for (int i = 0; i < kProbeItems; ++i) {
      const int64_t r = base + i * kProbeThreads + threadIdx.x;
      if (r < a.n_probe && dvalid(a.pk.c[0], r)) {
        const void* p;
        if (a.t.direct) {
          const uint64_t u = direct_slot(a.t, key_value(a.pk.c[0], r));
          if (u >= a.t.drange) continue;
          p = a.t.direct + u;
        } else {
          uint64_t lo, hi;
          const uint64_t idx = first_slot(a.t, mix64(key_bits<M>(a.pk, r)), lo, hi);
          p = M == KeyMode::K64 ? static_cast<const void*>(static_cast<const Slot16*>(a.t.slots) + idx)
                                : static_cast<const void*>(static_cast<const uint64_t*>(a.t.slots) + idx);
        }
        asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
      }
    }
  }
#pragma unroll
  for (int i = 0; i < kProbeItems; ++i) {
    const int64_t r = base + i * kProbeThreads + threadIdx.x;
    m[i]            = 0;
    first[i]        = -1;
    if (r < a.n_probe) {
      int c      = 0;
      int64_t fr = -1;
      for_each_match<M>(a.t, a.pk, r, [&](int64_t b) {
        if (c == 0) fr = b;
        ++c;
        return !UNIQUE;  // a unique build side has at most one match
      });
      m[i]     = c;
      first[i] = fr;
      cnt += out_rows(a.join_type, c);
    }
  }
  int64_t tile_total;
  int64_t excl = block_exclusive_scan<int64_t, kProbeThreads>(cnt, s_scan, &tile_total);
  if (!WRITE) {
    if (threadIdx.x == 0) a.tile_counts[tile] = static_cast<uint32_t>(tile_total);
    return;
  }
  if (threadIdx.x == 0) {
    if (claim) {
      s_prefix = tile_total > 0 ? atomicAdd(reinterpret_cast<unsigned long long*>(a.total),
                                            static_cast<unsigned long long>(tile_total))
                                : 0;
    } else {
      s_prefix = static_cast<uint64_t>(a.tile_offsets[tile]);
    }
  }
  __syncthreads();
  int64_t pos = static_cast<int64_t>(s_prefix) + excl;
  const int jt = a.join_type;
  if (UNIQUE && M != KeyMode::GEN && a.lmap == nullptr) {
    // at most one output row per probe row: batched, column-wise emit
    int64_t opos[kProbeItems], lrow[kProbeItems], brow[kProbeItems];
#pragma unroll
    for (int i = 0; i < kProbeItems; ++i) {
      const int64_t r = base + i * kProbeThreads + threadIdx.x;
      opos[i]         = -1;
      lrow[i]         = r;
      brow[i]         = -1;
      if (r >= a.n_probe) continue;
      bool out;
      if (jt == LDF_JOIN_SEMI) out = m[i] > 0;
      else if (jt == LDF_JOIN_ANTI) out = m[i] == 0;
      else if (jt == LDF_JOIN_INNER) out = m[i] > 0;
      else out = true;
      if (jt != LDF_JOIN_SEMI && jt != LDF_JOIN_ANTI && m[i] > 0) {
        brow[i] = first[i];
        if (a.matched && !a.matched[first[i]]) a.matched[first[i]] = 1;  // hot rows: read, no write
      }
      if (out) opos[i] = pos++;
    }
    emit_batch(a.lo, opos, lrow);
    emit_build_batch(a, opos, lrow, brow);
    return;
  }
#pragma unroll
  for (int i = 0; i < kProbeItems; ++i) {
    const int64_t r = base + i * kProbeThreads + threadIdx.x;
    if (r >= a.n_probe) continue;
    if (jt == LDF_JOIN_SEMI) {
      if (m[i] > 0) emit(a, pos++, r, -1);
      continue;
    }
    if (jt == LDF_JOIN_ANTI) {
      if (m[i] == 0) emit(a, pos++, r, -1);
      continue;
    }
    if (m[i] == 0) {
      if (jt != LDF_JOIN_INNER) emit(a, pos++, r, -1);
      continue;
    }
    if (UNIQUE || m[i] == 1) {
      emit(a, pos++, r, first[i]);
      if (a.matched && !a.matched[first[i]]) a.matched[first[i]] = 1;  // hot rows: read, no write
    } else {
      for_each_match<M>(a.t, a.pk, r, [&](int64_t b) {
        emit(a, pos++, r, b);
        if (a.matched && !a.matched[b]) a.matched[b] = 1;
        return true;
      });
    }
  }
}

// Two build-side output columns packed per row (see ProbeArgs::rpack).
template <int W0, int W1>
__global__ void pack_rows_kernel(DCol c0, DCol c1, int64_t n, ulonglong2* out)
{
  for (int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; b < n; b += (int64_t)gridDim.x * blockDim.x)
    out[b] = make_ulonglong2(load_w<W0>(c0.data, b), load_w<W1>(c1.data, b));
}

template <int W0>
void launch_pack(const DCol& c0, const DCol& c1, int64_t n, ulonglong2* out, cudaStream_t s, unsigned grid)
{
  switch (c1.width) {
    case 1: launch("pack_rows", pack_rows_kernel<W0, 1>, grid, 256, 0, s, c0, c1, n, out); break;
    case 2: launch("pack_rows", pack_rows_kernel<W0, 2>, grid, 256, 0, s, c0, c1, n, out); break;
    case 4: launch("pack_rows", pack_rows_kernel<W0, 4>, grid, 256, 0, s, c0, c1, n, out); break;
    default: launch("pack_rows", pack_rows_kernel<W0, 8>, grid, 256, 0, s, c0, c1, n, out); break;
  }
}

// FULL join tail: rhs rows never matched, appended after the probe rows.
struct TailArgs {
  const uint8_t* matched;
  int64_t n_build;
  const int64_t* base_pos;  // device: probe output rows
  OutSpec lo, ro;
  int32_t* lmap;
  int32_t* rmap;
  int64_t* total;
  int* err;
};

__global__ void __launch_bounds__(kProbeThreads) full_tail_kernel(TailArgs a)
{
  __shared__ int64_t s_scan[kProbeThreads / 32 + 1];
  __shared__ uint64_t s_prefix;
  // the tile claims its output range with one atomic on the tail total
  const int64_t tile = static_cast<int64_t>(blockIdx.x);
  const int64_t base = tile * kProbeTile + static_cast<int64_t>(threadIdx.x) * kProbeItems;
  int f[kProbeItems];
  int64_t c = 0;
#pragma unroll
  for (int i = 0; i < kProbeItems; ++i) {
    int64_t r = base + i;
    f[i]      = (r < a.n_build && !a.matched[r]) ? 1 : 0;
    c += f[i];
  }
  int64_t tot;
  int64_t ex = block_exclusive_scan<int64_t, kProbeThreads>(c, s_scan, &tot);
  if (threadIdx.x == 0)
    s_prefix = tot > 0 ? atomicAdd(reinterpret_cast<unsigned long long*>(a.total), static_cast<unsigned long long>(tot))
                       : 0;
  __syncthreads();
  int64_t pos = *a.base_pos + static_cast<int64_t>(s_prefix) + ex;
#pragma unroll
  for (int i = 0; i < kProbeItems; ++i) {
    if (!f[i]) continue;
    int64_t r = base + i;
    write_out_row(a.lo, pos, -1);
    write_out_row(a.ro, pos, r);
    if (a.lmap) a.lmap[pos] = -1;
    if (a.rmap) a.rmap[pos] = static_cast<int32_t>(r);
    ++pos;
  }
}

unsigned grid_stride_blocks(int64_t n, int threads)
{
  int64_t b   = ceil_div(n, threads);
  int64_t cap = static_cast<int64_t>(num_sms()) * 8;
  return static_cast<unsigned>(b < 1 ? 1 : (b > cap ? cap : b));
}

struct StatusBuf {
  Buffer<uint64_t> buf;
  uint64_t* status;
  unsigned long long* counter;
  StatusBuf(const OpContext& ctx, int64_t tiles)
  {
    buf     = Buffer<uint64_t>(ctx.alloc(), tiles + 2);
    status  = buf.get();
    counter = reinterpret_cast<unsigned long long*>(buf.get() + tiles);
    LDF_CUDA(cudaMemsetAsync(buf.get(), 0, (tiles + 2) * sizeof(uint64_t), ctx.stream()));
  }
};

// ---- radix partitioning (single fixed-width key) ----------------------------
// Both sides are scattered into kParts hash partitions (+ one partition for
// null keys), carrying the key and the output columns.  The build table gets
// one region per partition; the probe then walks the partitioned probe rows in
// order, so the partitions being probed at any moment (table + rhs outputs)
// stay in L2 instead of every probe costing random HBM accesses.
constexpr int kParts        = 256;
constexpr int kPartBuckets  = kParts + 1;
constexpr int kPartThreads  = 512;
constexpr int kPartPerThr   = 16;
constexpr int kPartTile     = kPartThreads * kPartPerThr;  // 8192 rows
constexpr int kMaxCarry     = kMaxOut + 1;

// Partition of row r: top 8 bits of the key hash (the table hash of K32/K64
// keys), kParts for a null key.
template <int W>
__device__ __forceinline__ uint32_t part_of(const DCol& key, int64_t r)
{
  if (key.valid != nullptr && __ldg(key.valid + r) == 0) return kParts;
  return static_cast<uint32_t>(mix64(load_w<W>(key.data, r)) >> 56);
}

// hist[b * ntiles + tile]: rows of partition b in the tile; totals[b] += them.
template <int W>
__global__ void __launch_bounds__(kPartThreads) part_hist_kernel(DCol key, int64_t n, int64_t ntiles, uint32_t* hist,
                                                                 unsigned long long* totals)
{
  __shared__ uint32_t cnt[kPartBuckets];
  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    for (int b = threadIdx.x; b < kPartBuckets; b += blockDim.x) cnt[b] = 0;
    __syncthreads();
    const int64_t t0 = tile * kPartTile;
    uint32_t pb[kPartPerThr];
#pragma unroll
    for (int i = 0; i < kPartPerThr; ++i) {
      const int64_t r = t0 + i * kPartThreads + threadIdx.x;
      pb[i]           = r < n ? part_of<W>(key, r) : 0xffffffffu;
    }
#pragma unroll
    for (int i = 0; i < kPartPerThr; ++i)
      if (pb[i] != 0xffffffffu) atomicAdd(&cnt[pb[i]], 1u);
    __syncthreads();
    for (int b = threadIdx.x; b < kPartBuckets; b += blockDim.x) {
      hist[b * ntiles + tile] = cnt[b];
      if (cnt[b]) atomicAdd(&totals[b], static_cast<unsigned long long>(cnt[b]));
    }
    __syncthreads();
  }
}

// offs[b * ntiles + t] = base[b] + rows of partition b in tiles < t (one CTA per partition).
__global__ void __launch_bounds__(256) part_offsets_kernel(const uint32_t* hist, int64_t ntiles, const int64_t* base,
                                                           int64_t* offs)
{
  __shared__ int64_t s_scan[256 / 32 + 1];
  const int b = blockIdx.x;
  int64_t run = base[b];
  for (int64_t t0 = 0; t0 < ntiles; t0 += blockDim.x) {
    const int64_t t = t0 + threadIdx.x;
    const int64_t v = t < ntiles ? hist[b * ntiles + t] : 0;
    int64_t tot;
    const int64_t ex = block_exclusive_scan<int64_t, 256>(v, s_scan, &tot);
    if (t < ntiles) offs[b * ntiles + t] = run + ex;
    run += tot;
    __syncthreads();
  }
}

struct PartCols {
  int n;
  DCol src[kMaxCarry];
  void* dst[kMaxCarry];
  uint8_t* dst_valid[kMaxCarry];
};

// Scatter every row to its partition, one tile at a time: the tile's rows
// are ranked inside their partition (order inside a partition is
// unspecified), staged in shared memory grouped by partition, and every
// column is written out as contiguous runs per partition.
template <int WC>
__device__ __forceinline__ void stage_column(unsigned long long* stage, const uint32_t* slot, const DCol& c, int64_t t0,
                                             bool validity)
{
#pragma unroll
  for (int i = 0; i < kPartPerThr; ++i) {
    if (slot[i] == 0xffffffffu) continue;
    const int64_t r = t0 + i * kPartThreads + threadIdx.x;
    stage[slot[i]]  = validity ? static_cast<unsigned long long>(__ldg(c.valid + r) != 0) : load_w<WC>(c.data, r);
  }
}
template <int WC>
__device__ __forceinline__ void write_column(const unsigned long long* stage, const uint16_t* slot_part,
                                             const uint32_t* toff, const int64_t* gbase, int rows, void* dst)
{
  for (int sl = threadIdx.x; sl < rows; sl += blockDim.x) {
    const uint32_t b = slot_part[sl];
    store_w<WC>(dst, gbase[b] + (sl - static_cast<int>(toff[b])), stage[sl]);
  }
}

template <int W>
__global__ void __launch_bounds__(kPartThreads) part_scatter_kernel(DCol key, int64_t n, int64_t ntiles,
                                                                    const int64_t* offs, PartCols pc)
{
  extern __shared__ __align__(16) unsigned char smem[];
  unsigned long long* stage = reinterpret_cast<unsigned long long*>(smem);        // kPartTile values
  int64_t* gbase            = reinterpret_cast<int64_t*>(stage + kPartTile);      // global start of the tile's run
  uint16_t* slot_part       = reinterpret_cast<uint16_t*>(gbase + kPartBuckets);  // partition of a staged slot
  uint32_t* cnt             = reinterpret_cast<uint32_t*>(slot_part + kPartTile); // kPartBuckets
  uint32_t* toff            = cnt + kPartBuckets;                                  // tile-local start of a partition
  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    for (int b = threadIdx.x; b < kPartBuckets; b += blockDim.x) {
      cnt[b]   = 0;
      gbase[b] = offs[b * ntiles + tile];
    }
    __syncthreads();
    const int64_t t0   = tile * kPartTile;
    const int rows     = static_cast<int>(n - t0 < kPartTile ? n - t0 : kPartTile);
    uint32_t slot[kPartPerThr];  // partition << 16 | local rank, then the staged slot
#pragma unroll
    for (int i = 0; i < kPartPerThr; ++i) {
      const int lr = i * kPartThreads + threadIdx.x;
      slot[i]      = 0xffffffffu;
      if (lr < rows) {
        const uint32_t b = part_of<W>(key, t0 + lr);
        slot[i]          = (b << 16) | atomicAdd(&cnt[b], 1u);
      }
    }
    __syncthreads();
    if (threadIdx.x < 32) {  // exclusive scan of the 257 partition counts by one warp
      uint32_t run = 0;
      for (int c0 = 0; c0 < kPartBuckets; c0 += 32) {
        const int b     = c0 + threadIdx.x;
        uint32_t v      = b < kPartBuckets ? cnt[b] : 0u;
        uint32_t incl   = v;
        for (int o = 1; o < 32; o <<= 1) {
          const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
          if (threadIdx.x >= o) incl += y;
        }
        if (b < kPartBuckets) toff[b] = run + incl - v;
        run += __shfl_sync(0xffffffffu, incl, 31);
      }
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < kPartPerThr; ++i)
      if (slot[i] != 0xffffffffu) {
        const uint32_t b = slot[i] >> 16;
        slot[i]          = toff[b] + (slot[i] & 0xffffu);
        slot_part[slot[i]] = static_cast<uint16_t>(b);
      }
    __syncthreads();
    for (int j = 0; j < pc.n; ++j) {
      const DCol& c = pc.src[j];
      for (int pass = 0; pass < (pc.dst_valid[j] ? 2 : 1); ++pass) {
        const int w = pass == 0 ? c.width : 1;
        switch (w) {  // uniform over the CTA
          case 1: stage_column<1>(stage, slot, c, t0, pass == 1); break;
          case 2: stage_column<2>(stage, slot, c, t0, false); break;
          case 4: stage_column<4>(stage, slot, c, t0, false); break;
          default: stage_column<8>(stage, slot, c, t0, false); break;
        }
        __syncthreads();
        void* dst = pass == 0 ? pc.dst[j] : static_cast<void*>(pc.dst_valid[j]);
        switch (w) {
          case 1: write_column<1>(stage, slot_part, toff, gbase, rows, dst); break;
          case 2: write_column<2>(stage, slot_part, toff, gbase, rows, dst); break;
          case 4: write_column<4>(stage, slot_part, toff, gbase, rows, dst); break;
          default: write_column<8>(stage, slot_part, toff, gbase, rows, dst); break;
        }
        __syncthreads();
      }
    }
  }
}
constexpr size_t kPartScatterSmem =
  static_cast<size_t>(kPartTile) * 8 + kPartBuckets * 8 + kPartTile * 2 + kPartBuckets * 4 + (kPartBuckets + 1) * 4;
static_assert((static_cast<size_t>(kPartTile) * 8 + kPartBuckets * 8 + kPartTile * 2) % 4 == 0, "u32 alignment");

// A table scattered into partitions: partitioned copies of the carried
// columns (key first) and the row count of every partition.
struct PartitionedTable {
  std::vector<Buffer<uint8_t>> data, valid;
  std::vector<DCol> cols;
  int64_t counts[kPartBuckets];
};

void partition_table(const OpContext& ctx, const DCol& key, int64_t n, const std::vector<DCol>& carry,
                     PartitionedTable& out)
{
  const Allocator& al = ctx.alloc();
  cudaStream_t s      = ctx.stream();
  LDF_REQUIRE(static_cast<int>(carry.size()) <= kMaxCarry, "too many partitioned columns");
  const int64_t ntiles = std::max<int64_t>(1, ceil_div(n, kPartTile));
  Buffer<uint32_t> hist(al, kPartBuckets * ntiles);
  Buffer<unsigned long long> totals(al, kPartBuckets);
  Buffer<int64_t> offs(al, kPartBuckets * ntiles);
  Buffer<int64_t> base(al, kPartBuckets);
  LDF_CUDA(cudaMemsetAsync(totals.get(), 0, kPartBuckets * 8, s));
  const unsigned grid = static_cast<unsigned>(std::min<int64_t>(ntiles, 2 * num_sms()));
  LDF_REQUIRE(key.width == 1 || key.width == 2 || key.width == 4 || key.width == 8, "partition key width");
  auto hk = key.width == 8 ? part_hist_kernel<8> : key.width == 4 ? part_hist_kernel<4>
          : key.width == 2 ? part_hist_kernel<2> : part_hist_kernel<1>;
  launch("part_hist", hk, grid, kPartThreads, 0, s, key, n, ntiles, hist.get(), totals.get());
  unsigned long long h[kPartBuckets];
  LDF_CUDA(cudaMemcpyAsync(h, totals.get(), sizeof(h), cudaMemcpyDeviceToHost, s));
  ctx.finish();
  int64_t hb[kPartBuckets], acc = 0;
  for (int b = 0; b < kPartBuckets; ++b) {
    out.counts[b] = static_cast<int64_t>(h[b]);
    hb[b]         = acc;
    acc += out.counts[b];
  }
  LDF_CUDA(cudaMemcpyAsync(base.get(), hb, sizeof(hb), cudaMemcpyHostToDevice, s));
  launch("part_offsets", part_offsets_kernel, static_cast<unsigned>(kPartBuckets), 256u, 0, s,
         static_cast<const uint32_t*>(hist.get()), ntiles, static_cast<const int64_t*>(base.get()), offs.get());
  PartCols pc{};
  pc.n = static_cast<int>(carry.size());
  for (size_t j = 0; j < carry.size(); ++j) {
    const DCol& c = carry[j];
    out.data.emplace_back(al, static_cast<size_t>(std::max<int64_t>(n, 1)) * c.width);
    out.valid.emplace_back();
    if (c.valid) out.valid.back() = Buffer<uint8_t>(al, std::max<int64_t>(n, 1));
    pc.src[j]       = c;
    pc.dst[j]       = out.data.back().get();
    pc.dst_valid[j] = c.valid ? out.valid.back().get() : nullptr;
    DCol d          = c;
    d.data          = out.data.back().get();
    d.valid         = pc.dst_valid[j];
    out.cols.push_back(d);
  }
  auto sk = key.width == 8 ? part_scatter_kernel<8> : key.width == 4 ? part_scatter_kernel<4>
          : key.width == 2 ? part_scatter_kernel<2> : part_scatter_kernel<1>;
  LDF_CUDA(cudaFuncSetAttribute(sk, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(kPartScatterSmem)));
  launch("part_scatter", sk, grid, kPartThreads, kPartScatterSmem, s, key, n, ntiles,
         static_cast<const int64_t*>(offs.get()), pc);
  // the Buffers above are released stream-ordered once the scatter has run
}

// Slot regions of a partitioned build table: 2 x rows of each partition.
struct PartPlan {
  const uint64_t* base;  // device, kParts entries
  const uint64_t* cap;
  uint64_t total;
};

template <KeyMode M>
void run_join(const OpContext& ctx, const KeyCols& pk, int64_t n_probe, const KeyCols& bk,
              int64_t n_build, int join_type, bool nulls_equal, OutSpec lo, OutSpec ro,
              const std::vector<ldf_column*>& out_cols, const std::vector<int>& out_is_lhs,
              const std::vector<DCol>& out_src, const std::vector<int>& out_types,
              const std::vector<int>& out_nullable, const PartPlan* plan = nullptr)
{
  const Allocator& al = ctx.alloc();
  cudaStream_t s      = ctx.stream();

  // ---- build ---------------------------------------------------------------
  BuildTable t{};
  t.bk          = bk;
  t.nulls_equal = nulls_equal ? 1 : 0;
  t.cap         = static_cast<uint64_t>(std::max<int64_t>(2 * n_build, 64));
  if (plan) {
    t.parts     = kParts;
    t.part_base = plan->base;
    t.part_cap  = plan->cap;
    t.cap       = plan->total;
  }
  // Dense integer keys: when the build keys' value range is at most twice the
  // build rows (and 2^31), a direct-address table of build rows replaces the
  // hash table if no key repeats (a repeat falls back to the hash table).
  // The table is 4 bytes per key value, so the probe's lookups mostly stay in
  // L2, and probe keys outside the range need no lookup at all.
  Buffer<int32_t> direct;
  if (M != KeyMode::GEN && !plan && n_build > 0 && !is_float(bk.c[0].type)) {
    Buffer<unsigned long long> mm(al, 4);
    const unsigned long long init[4] = {~0ull, 0ull, 0ull, 0ull};
    LDF_CUDA(cudaMemcpyAsync(mm.get(), init, sizeof(init), cudaMemcpyHostToDevice, s));
    launch("key_range", key_range_kernel, grid_stride_blocks(n_build, 256), 256, 0, s, bk.c[0], n_build, mm.get());
    unsigned long long h[3];
    LDF_CUDA(cudaMemcpyAsync(h, mm.get(), sizeof(h), cudaMemcpyDeviceToHost, s));
    ctx.finish();
    const uint64_t span  = h[0] <= h[1] ? (h[1] - h[0]) : ~0ull;  // max - min (order-preserving words)
    const uint64_t limit = static_cast<uint64_t>(std::max<int64_t>(2 * n_build, int64_t(1) << 16));
    if (h[2] == 0 && span < limit && span < (uint64_t(1) << 31)) {
      const int64_t dmin = static_cast<int64_t>(h[0] ^ (1ull << 63));
      direct             = Buffer<int32_t>(al, span + 1);
      LDF_CUDA(cudaMemsetAsync(direct.get(), 0xff, (span + 1) * sizeof(int32_t), s));
      LDF_CUDA(cudaMemsetAsync(mm.get() + 3, 0, sizeof(unsigned long long), s));
      launch("direct_build", direct_build_kernel, grid_stride_blocks(n_build, 256), 256, 0, s, bk.c[0], n_build,
             dmin, direct.get(), reinterpret_cast<int*>(mm.get() + 3));
      unsigned long long dup = 0;
      LDF_CUDA(cudaMemcpyAsync(&dup, mm.get() + 3, sizeof(dup), cudaMemcpyDeviceToHost, s));
      ctx.finish();
      if (dup == 0) {
        t.direct = direct.get();
        t.dmin   = dmin;
        t.dmax   = static_cast<int64_t>(h[1] ^ (1ull << 63));
        t.drange = span + 1;
      } else {
        direct.reset();
      }
    }
  }
  const size_t slot_bytes = M == KeyMode::K64 ? sizeof(Slot16) : sizeof(uint64_t);
  Buffer<uint8_t> slots;
  if (t.direct == nullptr) {
    slots = Buffer<uint8_t>(al, t.cap * slot_bytes);
    LDF_CUDA(cudaMemsetAsync(slots.get(), 0xff, t.cap * slot_bytes, s));
    t.slots = slots.get();
  }

  Buffer<int32_t> null_list;
  Buffer<int64_t> null_count;
  if (M != KeyMode::GEN && nulls_equal && bk.c[0].valid != nullptr && n_build > 0) {
    null_list  = Buffer<int32_t>(al, n_build);
    null_count = Buffer<int64_t>(al, 1);
    const int64_t tiles = ceil_div(n_build, kProbeTile);
    StatusBuf sb(ctx, tiles);
    launch("null_list", null_list_kernel, static_cast<unsigned>(tiles), kProbeThreads, 0, s, 
      bk.c[0], n_build, null_list.get(), sb.status, sb.counter, null_count.get(), ctx.err());
    LDF_CHECK_LAUNCH();
    t.null_list  = null_list.get();
    t.null_count = null_count.get();
  }
  // K32 builds flag duplicate keys themselves (the slot word holds the key)
  Buffer<int64_t> dupflag;
  if (M == KeyMode::K32 && t.direct == nullptr) {
    dupflag = Buffer<int64_t>(al, 1);
    LDF_CUDA(cudaMemsetAsync(dupflag.get(), 0, sizeof(int64_t), s));
    t.dup = reinterpret_cast<int*>(dupflag.get());
  }
  if (n_build > 0 && t.direct == nullptr) {
    launch("build", build_kernel<M>, grid_stride_blocks(n_build, 256), 256, 0, s, t, n_build);
    LDF_CHECK_LAUNCH();
  }

  // ---- uniqueness ----------------------------------------------------------
  bool unique = true;
  if (t.direct != nullptr) {  // no key repeats; null keys match each other with nulls_equal
    if (t.null_count) unique = ctx.read_i64(t.null_count) <= 1;
  } else if (M == KeyMode::K32 && n_build > 1) {
    int64_t h[2] = {0, 0};  // duplicate flag, null-key rows (all equal with nulls_equal)
    LDF_CUDA(cudaMemcpyAsync(&h[0], dupflag.get(), sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    if (t.null_count) LDF_CUDA(cudaMemcpyAsync(&h[1], t.null_count, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    ctx.finish();
    unique = static_cast<int>(h[0]) == 0 && h[1] <= 1;
  } else if (n_build > 1) {
    Buffer<int64_t> dup(al, 1);
    LDF_CUDA(cudaMemsetAsync(dup.get(), 0, sizeof(int64_t), s));
    launch("dup_check", dup_check_kernel<M>, grid_stride_blocks(n_build, 256), 256, 0, s, 
      t, n_build, reinterpret_cast<int*>(dup.get()));
    LDF_CHECK_LAUNCH();
    unique = ctx.read_i64(dup.get()) == 0;
  }

  // ---- probe ---------------------------------------------------------------
  const int64_t tiles = ceil_div(n_probe, kProbeTile);
  ProbeArgs a{};
  a.t         = t;
  a.pk        = pk;
  a.n_probe   = n_probe;
  a.join_type = join_type;
  a.lo        = lo;
  a.ro        = ro;
  a.err       = ctx.err();

  const bool full = join_type == LDF_JOIN_FULL;
  Buffer<int64_t> d_total(al, 2);
  LDF_CUDA(cudaMemsetAsync(d_total.get(), 0, 2 * sizeof(int64_t), s));
  Buffer<int64_t> tile_offsets;
  int64_t capacity = 0;
  if (unique) {
    capacity = (join_type == LDF_JOIN_INNER || join_type == LDF_JOIN_SEMI ||
                join_type == LDF_JOIN_ANTI || join_type == LDF_JOIN_LEFT)
                 ? n_probe
                 : n_probe + n_build;
  } else if (tiles > 0) {
    Buffer<uint32_t> counts(al, tiles);
    tile_offsets = Buffer<int64_t>(al, tiles);
    a.tile_counts = counts.get();
    launch("probe", probe_kernel<M, false, false>, static_cast<unsigned>(tiles), kProbeThreads, 0, s, a);
    LDF_CHECK_LAUNCH();
    exclusive_scan_u32(counts.get(), tile_offsets.get(), tiles, d_total.get(), ctx);
    capacity = ctx.read_i64(d_total.get()) + (full ? n_build : 0);
    a.tile_counts = nullptr;
  } else {
    capacity = full ? n_build : 0;
  }

  // ---- allocate outputs ----------------------------------------------------
  bool need_maps = false;
  for (size_t j = 0; j < out_cols.size(); ++j) {
    *out_cols[j] = alloc_out_column(al, out_types[j], capacity, out_nullable[j] != 0);
    if (out_types[j] == LDF_STRING) need_maps = true;
  }
  // Bind output pointers into the specs (lhs columns first, then rhs).
  {
    int li = 0, ri = 0;
    for (size_t j = 0; j < out_cols.size(); ++j) {
      OCol d{out_cols[j]->data, out_cols[j]->valid, out_types[j], type_width(out_types[j])};
      if (out_is_lhs[j]) a.lo.dst[li++] = d;
      else a.ro.dst[ri++] = d;
    }
  }
  Buffer<int32_t> lmap, rmap;
  if (need_maps) {
    lmap   = Buffer<int32_t>(al, std::max<int64_t>(capacity, 1));
    rmap   = Buffer<int32_t>(al, std::max<int64_t>(capacity, 1));
    a.lmap = lmap.get();
    a.rmap = rmap.get();
  }
  Buffer<uint8_t> matched;
  if (full && n_build > 0) {
    matched = Buffer<uint8_t>(al, n_build);
    LDF_CUDA(cudaMemsetAsync(matched.get(), 0, n_build, s));
    a.matched = matched.get();
  }

  // Build-side outputs of the one-pass probe: the build key column comes from
  // the probe key, and two other non-nullable fixed-width columns are packed
  // into one 16-byte record per build row, so a matched probe row reads them
  // with one random access.
  a.rkey = -1;
  Buffer<ulonglong2> rpack;
  if (unique && M != KeyMode::GEN && !need_maps && tiles > 0 && n_build > 0) {
    std::vector<int> rest;
    for (int j = 0; j < ro.n; ++j) {
      if (a.rkey < 0 && ro.src[j].data == bk.c[0].data && ro.src[j].type == bk.c[0].type) a.rkey = j;
      else rest.push_back(j);
    }
    bool packable = rest.size() == 2;
    for (int j : rest) packable = packable && ro.src[j].valid == nullptr && ro.src[j].type != LDF_STRING;
    if (packable) {
      const DCol& c0 = ro.src[rest[0]];
      const DCol& c1 = ro.src[rest[1]];
      rpack          = Buffer<ulonglong2>(al, n_build);
      const unsigned g = grid_stride_blocks(n_build, 256);
      switch (c0.width) {
        case 1: launch_pack<1>(c0, c1, n_build, rpack.get(), s, g); break;
        case 2: launch_pack<2>(c0, c1, n_build, rpack.get(), s, g); break;
        case 4: launch_pack<4>(c0, c1, n_build, rpack.get(), s, g); break;
        default: launch_pack<8>(c0, c1, n_build, rpack.get(), s, g); break;
      }
      a.rpack   = rpack.get();
      a.pcol[0] = rest[0];
      a.pcol[1] = rest[1];
    }
  }

  if (tiles > 0) {
    if (unique) {
      a.total = d_total.get();
      launch("probe", probe_kernel<M, true, true>, static_cast<unsigned>(tiles), kProbeThreads, 0, s, a);
      LDF_CHECK_LAUNCH();
    } else {
      a.tile_offsets = tile_offsets.get();
      launch("probe", probe_kernel<M, true, false>, static_cast<unsigned>(tiles), kProbeThreads, 0, s, a);
      LDF_CHECK_LAUNCH();
    }
  }
  int64_t rows = 0;
  if (full && n_build > 0) {
    const int64_t btiles = ceil_div(n_build, kProbeTile);
    TailArgs ta{};
    ta.matched  = matched.get();
    ta.n_build  = n_build;
    ta.base_pos = d_total.get();
    ta.lo       = a.lo;
    ta.ro       = a.ro;
    ta.lmap     = a.lmap;
    ta.rmap     = a.rmap;
    ta.total    = d_total.get() + 1;
    ta.err      = ctx.err();
    launch("full_tail", full_tail_kernel, static_cast<unsigned>(btiles), kProbeThreads, 0, s, ta);
    LDF_CHECK_LAUNCH();
    int64_t h[2];
    LDF_CUDA(cudaMemcpyAsync(h, d_total.get(), 2 * sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    ctx.finish();
    rows = h[0] + h[1];
  } else {
    rows = ctx.read_i64(d_total.get());
  }

  // ---- string outputs through gather maps ---------------------------------
  for (size_t j = 0; j < out_cols.size(); ++j) {
    out_cols[j]->size = rows;
    if (out_types[j] == LDF_STRING)
      gather_strings(ctx, out_src[j], out_is_lhs[j] ? lmap.get() : rmap.get(), rows, *out_cols[j]);
  }
}

}  // namespace

void join(const ldf_column* lhs, int lhs_ncols, const ldf_column* rhs, int rhs_ncols,
          const int32_t* lhs_keys, const int32_t* rhs_keys, int nkeys, int join_type,
          bool nulls_equal, const int32_t* lhs_out, int n_lhs_out, const int32_t* rhs_out,
          int n_rhs_out, ldf_column* out, const OpContext& ctx)
{
  LDF_REQUIRE(join_type >= LDF_JOIN_INNER && join_type <= LDF_JOIN_ANTI, "Unknown JoinType");
  LDF_REQUIRE(nkeys >= 1, "The size of `lhs_keys` and `rhs_keys` must be equal and non-zero");
  if ((join_type == LDF_JOIN_SEMI || join_type == LDF_JOIN_ANTI) && n_rhs_out > 0)
    fail(LDF_ERR_INVALID_ARGUMENT, "rhs must have no output columns for SEMI and ANTI join");
  LDF_REQUIRE(n_lhs_out <= kMaxOut && n_rhs_out <= kMaxOut, "too many output columns");
  KeyCols pk = make_keys(lhs, lhs_ncols, lhs_keys, nkeys);
  KeyCols bk = make_keys(rhs, rhs_ncols, rhs_keys, nkeys);
  for (int j = 0; j < nkeys; ++j)
    LDF_REQUIRE(pk.c[j].type == bk.c[j].type, "join key types of lhs and rhs must match");
  const int64_t n_probe = lhs_ncols > 0 ? lhs[0].size : 0;
  const int64_t n_build = rhs_ncols > 0 ? rhs[0].size : 0;
  LDF_REQUIRE(n_build < (int64_t(1) << 31) && n_probe < (int64_t(1) << 31),
              "tables of 2^31 rows or more per task are not supported");

  // Output schema and nullability (join.cpp:348-383).
  OutSpec lo{}, ro{};
  std::vector<ldf_column*> out_cols;
  std::vector<int> out_is_lhs, out_types, out_nullable;
  std::vector<DCol> out_src;
  for (int j = 0; j < n_lhs_out; ++j) {
    LDF_REQUIRE(lhs_out[j] >= 0 && lhs_out[j] < lhs_ncols, "lhs output column out of range");
    const ldf_column& c = lhs[lhs_out[j]];
    bool nullable = join_type == LDF_JOIN_FULL || c.valid != nullptr;
    lo.src[lo.n++] = make_dcol(c);
    out_cols.push_back(&out[out_cols.size()]);
    out_is_lhs.push_back(1);
    out_types.push_back(c.type);
    out_nullable.push_back(nullable);
    out_src.push_back(make_dcol(c));
  }
  for (int j = 0; j < n_rhs_out; ++j) {
    LDF_REQUIRE(rhs_out[j] >= 0 && rhs_out[j] < rhs_ncols, "rhs output column out of range");
    const ldf_column& c = rhs[rhs_out[j]];
    bool nullable = join_type == LDF_JOIN_FULL || join_type == LDF_JOIN_LEFT || c.valid != nullptr;
    ro.src[ro.n++] = make_dcol(c);
    out_cols.push_back(&out[out_cols.size()]);
    out_is_lhs.push_back(0);
    out_types.push_back(c.type);
    out_nullable.push_back(nullable);
    out_src.push_back(make_dcol(c));
  }

  const KeyMode mode = key_mode(bk);
  // Radix-partitioned path (opt-in, LDF_B200_JOIN_PARTITION=1): one
  // fixed-width key and fixed-width outputs.
  bool partitioned = false;
  if (const char* e = std::getenv("LDF_B200_JOIN_PARTITION")) {
    bool all_fixed = true;
    for (int ty : out_types)
      if (ty == LDF_STRING) all_fixed = false;
    partitioned = std::atoi(e) != 0 && all_fixed && (mode == KeyMode::K32 || mode == KeyMode::K64);
  }
  if (partitioned) {
    // carried columns: the key, then the output columns of the side
    // carried columns: the key, then each distinct output column of the side
    PartitionedTable lp, rp;
    auto carry = [](const DCol& key, const OutSpec& o, std::vector<DCol>& cols, int* where) {
      cols.push_back(key);
      for (int j = 0; j < o.n; ++j) {
        where[j] = -1;
        for (size_t k = 0; k < cols.size(); ++k)
          if (cols[k].data == o.src[j].data && cols[k].valid == o.src[j].valid && cols[k].width == o.src[j].width)
            where[j] = static_cast<int>(k);
        if (where[j] < 0) {
          where[j] = static_cast<int>(cols.size());
          cols.push_back(o.src[j]);
        }
      }
    };
    std::vector<DCol> lc, rc;
    int lw[kMaxOut], rw[kMaxOut];
    carry(pk.c[0], lo, lc, lw);
    carry(bk.c[0], ro, rc, rw);
    partition_table(ctx, bk.c[0], n_build, rc, rp);
    partition_table(ctx, pk.c[0], n_probe, lc, lp);
    KeyCols pk2 = pk, bk2 = bk;
    pk2.c[0]    = lp.cols[0];
    bk2.c[0]    = rp.cols[0];
    OutSpec lo2 = lo, ro2 = ro;
    for (int j = 0; j < lo.n; ++j) {
      lo2.src[j]      = lp.cols[lw[j]];
      lo2.src[j].type = lo.src[j].type;
    }
    for (int j = 0; j < ro.n; ++j) {
      ro2.src[j]      = rp.cols[rw[j]];
      ro2.src[j].type = ro.src[j].type;
    }
    uint64_t hb[kParts], hc[kParts], acc = 0;
    for (int b = 0; b < kParts; ++b) {
      hc[b] = static_cast<uint64_t>(std::max<int64_t>(2 * rp.counts[b], 2));
      hb[b] = acc;
      acc += hc[b];
    }
    Buffer<uint64_t> pb(ctx.alloc(), 2 * kParts);
    LDF_CUDA(cudaMemcpyAsync(pb.get(), hb, sizeof(hb), cudaMemcpyHostToDevice, ctx.stream()));
    LDF_CUDA(cudaMemcpyAsync(pb.get() + kParts, hc, sizeof(hc), cudaMemcpyHostToDevice, ctx.stream()));
    PartPlan plan{pb.get(), pb.get() + kParts, acc};
    if (mode == KeyMode::K32)
      run_join<KeyMode::K32>(ctx, pk2, n_probe, bk2, n_build, join_type, nulls_equal, lo2, ro2, out_cols,
                             out_is_lhs, out_src, out_types, out_nullable, &plan);
    else
      run_join<KeyMode::K64>(ctx, pk2, n_probe, bk2, n_build, join_type, nulls_equal, lo2, ro2, out_cols,
                             out_is_lhs, out_src, out_types, out_nullable, &plan);
    return;
  }
  switch (mode) {
    case KeyMode::K32:
      run_join<KeyMode::K32>(ctx, pk, n_probe, bk, n_build, join_type, nulls_equal, lo, ro,
                             out_cols, out_is_lhs, out_src, out_types, out_nullable);
      break;
    case KeyMode::K64:
      run_join<KeyMode::K64>(ctx, pk, n_probe, bk, n_build, join_type, nulls_equal, lo, ro,
                             out_cols, out_is_lhs, out_src, out_types, out_nullable);
      break;
    default:
      run_join<KeyMode::GEN>(ctx, pk, n_probe, bk, n_build, join_type, nulls_equal, lo, ro,
                             out_cols, out_is_lhs, out_src, out_types, out_nullable);
      break;
  }
}

}  // namespace ldf
