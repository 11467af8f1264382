// Onesweep LSD radix sort (Adinets & Merrill, "Onesweep", 2022) of row ids by
// 8-bit digits, stable.  One upfront kernel builds the digit histograms of all
// passes from the unpermuted columns (histograms do not depend on order); each
// pass is then ONE kernel: tile load -> warp-level stable ranking (peer lanes
// from one ballot per digit bit) -> per-digit decoupled look-back across
// tiles -> tile staged in shared memory in digit order -> coalesced runs
// written out.  Passes whose digit is constant over all rows are skipped from
// the histograms.
#include "radix.cuh"

namespace ldf {
namespace {

constexpr int RT    = kRadixThreads;
constexpr int RI    = kRadixItems;
constexpr int RTILE = kRadixTile;
constexpr int RW    = RT / 32;

// Order-preserving word of a sort key from the value's raw bits (zero for a
// null or a NaN: those rows are placed by the CLASS pass).
__device__ __forceinline__ uint64_t sort_word_of(const SortKeyDesc& k, uint64_t raw, bool valid)
{
  if (!valid) return 0;
  uint64_t o;
  switch (k.col.type) {
    case LDF_INT8: o = (raw & 0xffu) ^ 0x80u; break;
    case LDF_INT16: o = (raw & 0xffffu) ^ 0x8000u; break;
    case LDF_INT32: o = (raw & 0xffffffffu) ^ 0x80000000u; break;
    case LDF_INT64:
    case LDF_TIMESTAMP_US: o = raw ^ (1ull << 63); break;
    case LDF_FLOAT32: {
      uint32_t b = static_cast<uint32_t>(raw);
      if ((b & 0x7f800000u) == 0x7f800000u && (b & 0x007fffffu)) return 0;  // NaN: CLASS pass
      if ((b & 0x7fffffffu) == 0) b = 0;                                    // -0.0 == 0.0
      o = (b & 0x80000000u) ? ~b : (b | 0x80000000u);
      o &= 0xffffffffull;
      break;
    }
    case LDF_FLOAT64: {
      uint64_t b = raw;
      if ((b & 0x7ff0000000000000ull) == 0x7ff0000000000000ull && (b & 0x000fffffffffffffull)) return 0;
      if ((b & 0x7fffffffffffffffull) == 0) b = 0;
      o = (b & (1ull << 63)) ? ~b : (b | (1ull << 63));
      break;
    }
    default: o = raw; break;  // unsigned, bool, string ranks (uint32)
  }
  if (k.descending) {
    const uint64_t mask = k.key_bytes >= 8 ? ~0ull : ((1ull << (8 * k.key_bytes)) - 1);
    o                   = ~o & mask;
  }
  return o;
}

__device__ __forceinline__ uint64_t sort_word(const SortKeyDesc& k, int64_t row)
{
  return sort_word_of(k, dbits(k.col, row), dvalid(k.col, row));
}

// 0 = value, 1 = NaN, 2 = null when nulls_at_end; reversed otherwise
// (Arrow places NaN next to the values and nulls outermost, either direction).
__device__ __forceinline__ uint32_t class_digit(const SortKeyDesc& k, int64_t row)
{
  const DCol& c = k.col;
  uint32_t cls  = 0;
  if (!dvalid(c, row)) cls = 2;
  else if (c.type == LDF_FLOAT64) {
    uint64_t b = static_cast<const uint64_t*>(c.data)[row];
    if ((b & 0x7ff0000000000000ull) == 0x7ff0000000000000ull && (b & 0x000fffffffffffffull)) cls = 1;
  } else if (c.type == LDF_FLOAT32) {
    uint32_t b = static_cast<const uint32_t*>(c.data)[row];
    if ((b & 0x7f800000u) == 0x7f800000u && (b & 0x007fffffu)) cls = 1;
  }
  return k.nulls_at_end ? cls : 2 - cls;
}

__device__ __forceinline__ uint64_t bucket_word(const RadixPass& p, int64_t row)
{
  return key_bits<KeyMode::GEN>(p.hash_keys, row) % p.nparts;
}

__device__ __forceinline__ uint64_t pass_word(const RadixPass& p, int64_t row)
{
  if (p.src == DigitSrc::BUCKET) return bucket_word(p, row);
  return sort_word(p.key, row);
}

// Adds a fused-word component v placed at bit `off` of W to C = W >> 8 and
// to W's low byte (components do not overlap, so OR adds them).  Since W has
// at most 72 bits, v << (off - 8) fits C.
__device__ __forceinline__ void fused_add(uint64_t v, int off, uint64_t& c, uint32_t& low)
{
  if (v == 0) return;  // also every component of no bits, whose `off` may reach 72
  if (off >= 8) {
    c |= v << (off - 8);
  } else {
    c |= v >> (8 - off);
    low |= static_cast<uint32_t>(v << off) & 0xffu;
  }
}

// C = W >> 8 of the fused word W of a row (FusedKey); *low = W's low byte.
__device__ __forceinline__ uint64_t fused_word(const FusedKey& f, int64_t row, uint32_t& low)
{
  uint64_t c = 0;
  low        = 0;
#pragma unroll
  for (int k = 0; k < kFuseMax; ++k)
    if (k < f.n) fused_add(sort_word(f.key[k], row) - f.min[k], f.off[k], c, low);
  return c;
}

constexpr int kHistPassesPerLaunch = 16;
struct HistArgs {
  int npasses;
  uint32_t reuse;  // bit q: pass q reads the same key word as pass q - 1
  RadixPass p[kHistPassesPerLaunch];
  FusedKey fused;
  int64_t n;
  uint32_t* hist;  // [npasses][256]
};

// Raw bits of kHR rows of a column of width W, all loads in flight together.
constexpr int kHR = 4;
template <int W>
__device__ __forceinline__ void load_raw_rows(const DCol& c, const int64_t (&r)[kHR], int64_t n, uint64_t (&raw)[kHR],
                                              bool (&ok)[kHR])
{
#pragma unroll
  for (int j = 0; j < kHR; ++j) {
    raw[j] = 0;
    ok[j]  = false;
    if (r[j] >= n) continue;
    if (W == 1) raw[j] = __ldg(static_cast<const uint8_t*>(c.data) + r[j]);
    else if (W == 2) raw[j] = __ldg(static_cast<const uint16_t*>(c.data) + r[j]);
    else if (W == 4) raw[j] = __ldg(static_cast<const uint32_t*>(c.data) + r[j]);
    else raw[j] = __ldg(static_cast<const unsigned long long*>(c.data) + r[j]);
    ok[j] = c.valid == nullptr || __ldg(c.valid + r[j]) != 0;
  }
}

// All digit histograms of up to kHistPassesPerLaunch passes in one read of the
// columns: kHR rows per thread, each key word loaded once for all the passes
// over it (their loads in flight together), shared-memory counts.
template <bool FUSED>
__global__ void __launch_bounds__(RT) histogram_kernel(HistArgs a)
{
  __shared__ uint32_t sh[kHistPassesPerLaunch * 256];
  for (int i = threadIdx.x; i < a.npasses * 256; i += RT) sh[i] = 0;
  __syncthreads();
  const int64_t per_iter = static_cast<int64_t>(RT) * kHR;
  for (int64_t base = blockIdx.x * per_iter; base < a.n; base += static_cast<int64_t>(gridDim.x) * per_iter) {
    int64_t r[kHR];
#pragma unroll
    for (int j = 0; j < kHR; ++j) r[j] = base + j * RT + threadIdx.x;
    uint64_t w[kHR];
    uint32_t low[kHR];
#pragma unroll
    for (int j = 0; j < kHR; ++j) w[j] = 0, low[j] = 0;
    for (int q = 0; q < a.npasses; ++q) {
      const RadixPass& p = a.p[q];
      uint32_t d[kHR];
      if (p.src == DigitSrc::CLASS) {
#pragma unroll
        for (int j = 0; j < kHR; ++j) d[j] = r[j] < a.n ? class_digit(p.key, r[j]) : 256u;
      } else {
        if (!((a.reuse >> q) & 1u)) {
          if (p.src == DigitSrc::BUCKET) {
#pragma unroll
            for (int j = 0; j < kHR; ++j) w[j] = r[j] < a.n ? bucket_word(p, r[j]) : 0;
          } else if (FUSED && p.src == DigitSrc::FUSED) {
#pragma unroll
            for (int j = 0; j < kHR; ++j) w[j] = r[j] < a.n ? fused_word(a.fused, r[j], low[j]) : 0;
          } else {
            uint64_t raw[kHR];
            bool ok[kHR];
            switch (p.key.col.width) {
              case 1: load_raw_rows<1>(p.key.col, r, a.n, raw, ok); break;
              case 2: load_raw_rows<2>(p.key.col, r, a.n, raw, ok); break;
              case 4: load_raw_rows<4>(p.key.col, r, a.n, raw, ok); break;
              default: load_raw_rows<8>(p.key.col, r, a.n, raw, ok); break;
            }
#pragma unroll
            for (int j = 0; j < kHR; ++j) w[j] = sort_word_of(p.key, raw[j], ok[j]);
          }
        }
#pragma unroll
        for (int j = 0; j < kHR; ++j)
          d[j] = r[j] < a.n ? ((FUSED && p.fused_low) ? low[j] : static_cast<uint32_t>(w[j] >> p.shift) & 0xffu)
                            : 256u;
      }
#pragma unroll
      for (int j = 0; j < kHR; ++j)
        if (d[j] < 256) atomicAdd(&sh[q * 256 + d[j]], 1u);
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < a.npasses * 256; i += RT)
    if (sh[i]) atomicAdd(&a.hist[i], sh[i]);
}

struct PassArgs {
  RadixPass p;
  int64_t n;
  const uint64_t* keys_in;
  uint64_t* keys_out;
  const int32_t* vals_in;  // null: identity
  int32_t* vals_out;
  const uint64_t* digit_base;  // [256]
  uint64_t* status;            // [tiles * 256]
  unsigned long long* counter;
  int32_t* inv_out;  // != null: inv_out[row] = the row's output position
  RadixPayload pay;  // columns moved by this pass (payload_empty: none)
  FusedKey fused;    // FUSED passes
  int* err;
  // > 0: each tile stages in L2, by bulk prefetches, the rows of the tile
  // this many tiles ahead (about one wave of resident CTAs; tiles are taken
  // in order): the row ids and carried words of a pass on the carried word,
  // and the key columns of a first pass over rows in input order
  // (pf_columns).
  int64_t pf_ahead;
  int pf_columns;
};

// L2 prefetch of rows [lo, hi) of a fixed-width column and its validity.
__device__ __forceinline__ void prefetch_column(const DCol& c, int64_t lo, int64_t hi)
{
  if (c.type == LDF_STRING || c.data == nullptr) return;
  l2_prefetch_bulk(c.data, lo * c.width, hi * c.width);
  if (c.valid) l2_prefetch_bulk(c.valid, lo, hi);
}

// Rows of a thread whose payload loads are issued together in a pass that
// moves columns.
constexpr int kMoveBatch = 3;

// dst[pos[k]] = src[row[k]] for 16-byte string ranges (8-byte aligned at the
// source: two 8-byte loads; the scratch destination is 16-byte aligned), every
// load issued before the first store.  pos < 0: no row.
__device__ __forceinline__ void move_ranges(const void* src, void* dst, const int32_t (&pos)[kMoveBatch],
                                            const int32_t (&row)[kMoveBatch])
{
  const unsigned long long* sp = static_cast<const unsigned long long*>(src);
  ulonglong2 v[kMoveBatch];
#pragma unroll
  for (int k = 0; k < kMoveBatch; ++k)
    if (pos[k] >= 0) v[k] = make_ulonglong2(__ldg(sp + 2 * row[k]), __ldg(sp + 2 * row[k] + 1));
#pragma unroll
  for (int k = 0; k < kMoveBatch; ++k)
    if (pos[k] >= 0) static_cast<ulonglong2*>(dst)[pos[k]] = v[k];
}

__device__ __forceinline__ unsigned long long ld_fixed(const DCol& c, int32_t row)
{
  switch (c.width) {
    case 1: return __ldg(static_cast<const uint8_t*>(c.data) + row);
    case 2: return __ldg(static_cast<const uint16_t*>(c.data) + row);
    case 4: return __ldg(static_cast<const uint32_t*>(c.data) + row);
    default: return __ldg(static_cast<const unsigned long long*>(c.data) + row);
  }
}

__device__ __forceinline__ void st_fixed(void* dst, int width, int64_t pos, unsigned long long v)
{
  switch (width) {
    case 1: static_cast<uint8_t*>(dst)[pos] = static_cast<uint8_t>(v); break;
    case 2: static_cast<uint16_t*>(dst)[pos] = static_cast<uint16_t>(v); break;
    case 4: static_cast<uint32_t*>(dst)[pos] = static_cast<uint32_t>(v); break;
    default: static_cast<unsigned long long*>(dst)[pos] = v; break;
  }
}

// Part of a packed payload record at byte offset `off` (the store truncates it
// to the part's width).
__device__ __forceinline__ unsigned long long record_part(const ulonglong2& r, int off)
{
  return (off < 8 ? r.x : r.y) >> ((off & 7) * 8);
}

// dst[pos] = src[row] for every payload column (one row: the identity copy).
__device__ __forceinline__ void move_payload(const RadixPayload& p, int64_t pos, int64_t row)
{
  if (p.nparts) {
    const ulonglong2 r = __ldg(p.packed + row);
    for (int k = 0; k < p.nparts; ++k) st_fixed(p.pdst[k], p.pwidth[k], pos, record_part(r, p.poff[k]));
  }
  for (int c = 0; c < p.n; ++c) {
    const DCol& sc = p.src[c];
    if (sc.width <= 8) {
      st_fixed(p.dst[c], sc.width, pos, ld_fixed(sc, static_cast<int32_t>(row)));
    } else {  // 16: string ranges (8-byte aligned at the source; the scratch is 16-byte aligned)
      const unsigned long long* r = static_cast<const unsigned long long*>(sc.data) + 2 * row;
      static_cast<ulonglong2*>(p.dst[c])[pos] = make_ulonglong2(__ldg(r), __ldg(r + 1));
    }
    if (p.dst_valid[c]) p.dst_valid[c][pos] = dvalid(sc, row) ? 1 : 0;
  }
}

// Every payload column's values (and masks) of kMoveBatch rows: the packed
// records first (one load per row for all their parts), then the other
// fixed-width columns with all their loads issued before the first store, so
// that their random rows are in flight together, then string ranges.
__device__ __forceinline__ void move_payload_rows(const RadixPayload& p, const int32_t (&pos)[kMoveBatch],
                                                  const int32_t (&row)[kMoveBatch])
{
  if (p.nparts) {
    ulonglong2 rv[kMoveBatch];
#pragma unroll
    for (int k = 0; k < kMoveBatch; ++k)
      if (pos[k] >= 0) rv[k] = __ldg(p.packed + row[k]);
#pragma unroll
    for (int k = 0; k < kMoveBatch; ++k)
      if (pos[k] >= 0)
        for (int q = 0; q < p.nparts; ++q) st_fixed(p.pdst[q], p.pwidth[q], pos[k], record_part(rv[k], p.poff[q]));
  }
  unsigned long long v[kPassPayload][kMoveBatch];
#pragma unroll
  for (int c = 0; c < kPassPayload; ++c)
    if (c < p.n && p.src[c].width <= 8) {
#pragma unroll
      for (int k = 0; k < kMoveBatch; ++k) v[c][k] = pos[k] >= 0 ? ld_fixed(p.src[c], row[k]) : 0;
    }
#pragma unroll
  for (int c = 0; c < kPassPayload; ++c)
    if (c < p.n && p.src[c].width <= 8) {
#pragma unroll
      for (int k = 0; k < kMoveBatch; ++k)
        if (pos[k] >= 0) st_fixed(p.dst[c], p.src[c].width, pos[k], v[c][k]);
    }
  for (int c = 0; c < p.n; ++c) {
    const DCol& sc = p.src[c];
    if (sc.width > 8) move_ranges(sc.data, p.dst[c], pos, row);
    if (p.dst_valid[c]) {
      uint8_t m[kMoveBatch];
#pragma unroll
      for (int k = 0; k < kMoveBatch; ++k) m[k] = pos[k] >= 0 && dvalid(sc, row[k]) ? 1 : 0;
#pragma unroll
      for (int k = 0; k < kMoveBatch; ++k)
        if (pos[k] >= 0) p.dst_valid[c][pos[k]] = m[k];
    }
  }
}

// Predecessor tiles whose status words one look-back round trip loads.
constexpr int kLookback = 8;

// Shared state of one onesweep tile.
struct OsShared {
  uint32_t whist[RW][256];  // per-warp digit counts, then per-warp digit prefixes
  uint32_t tile_start[256];  // tile-local start of each digit
  int32_t delta[256];        // output position of staged row j of digit d: delta[d] + j
  uint32_t scan[RW + 1];
  int64_t tile[2];
};

// Lanes of the warp whose digit equals this lane's (d <= 256; 256 marks an
// item without a row): one ballot per digit bit, each lane keeping the lanes
// that agree with it on that bit.
__device__ __forceinline__ uint32_t digit_peers(uint32_t d)
{
  uint32_t peers = 0xffffffffu;
#pragma unroll
  for (int b = 0; b < 9; ++b) {
    const uint32_t bit = (d >> b) & 1u;
    const uint32_t set = __ballot_sync(0xffffffffu, bit);
    peers &= bit ? set : ~set;
  }
  return peers;
}

// Everything of one pass over one tile after its rows are in registers:
// key[i] / val[i] / dr[i] (digit, 256 = no row) of item i of this thread,
// item order (warp, i, lane).  Stable warp-level ranking, tile-local scan, the
// tile's digit counts published at once, rows staged in digit order into
// s_keys / s_vals / s_dig (tile-local positions need no look-back), per-digit
// decoupled look-back, then coalesced runs written out.  sh.whist must be zero
// on entry.  Ends with every thread past its reads of the staging arrays.
template <bool WRITE_KEYS, bool MOVE>
__device__ __forceinline__ void rank_and_scatter(const PassArgs& a, int64_t tile, uint64_t (&key)[RI],
                                                 int32_t (&val)[RI], uint32_t (&dr)[RI], OsShared& sh,
                                                 uint64_t* s_keys, int32_t* s_vals, uint8_t* s_dig)
{
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t lt_mask = (1u << lane) - 1u;
  // stable warp-level ranking, items in (i, lane) order
#pragma unroll
  for (int i = 0; i < RI; ++i) {
    const uint32_t d     = dr[i];
    const uint32_t peers = digit_peers(d);
    const uint32_t rank  = __popc(peers & lt_mask);
    uint32_t base        = 0;
    if (d < 256) base = sh.whist[warp][d];
    __syncwarp();
    if (d < 256 && rank == 0) sh.whist[warp][d] = base + __popc(peers);
    __syncwarp();
    dr[i] = d | ((base + rank) << 9);
  }
  __syncthreads();
  // per-digit warp prefixes and tile counts (thread t owns digit t)
  const int t = threadIdx.x;
  uint32_t run = 0;
#pragma unroll
  for (int w = 0; w < RW; ++w) {
    uint32_t c       = sh.whist[w][t];
    sh.whist[w][t]   = run;
    run += c;
  }
  uint32_t tile_total;
  const uint32_t start = block_exclusive_scan<uint32_t, RT>(run, sh.scan, &tile_total);
  sh.tile_start[t]     = start;
  // publish this tile's digit counts before anything else, so the tiles
  // after it can finish their look-back while this one stages its rows
  uint64_t* st = a.status;
  if (tile == 0) st_release_u64(&st[t], kFlagPrefix | run);
  else st_release_u64(&st[tile * 256 + t], kFlagAgg | run);
  __syncthreads();
  // stage the tile in digit order
#pragma unroll
  for (int i = 0; i < RI; ++i) {
    const uint32_t d = dr[i] & 0x1ffu;
    if (d < 256) {
      const uint32_t lp = sh.tile_start[d] + sh.whist[warp][d] + (dr[i] >> 9);
      if (WRITE_KEYS) s_keys[lp] = key[i];
      s_vals[lp] = val[i];
      s_dig[lp]  = static_cast<uint8_t>(d);
    }
  }
  // per-digit decoupled look-back, kLookback predecessors' status words
  // loaded together per round trip
  {
    uint64_t excl = 0;
    if (tile > 0) {
      int64_t j      = tile - 1;  // next predecessor to fold in
      uint32_t spins = 0;
      while (j >= 0) {
        uint64_t sv[kLookback];
#pragma unroll
        for (int w = 0; w < kLookback; ++w) sv[w] = j - w >= 0 ? ld_volatile_u64(&st[(j - w) * 256 + t]) : kFlagPrefix;
        int used  = 0;
        bool done = false, stall = false;
#pragma unroll
        for (int w = 0; w < kLookback; ++w) {
          if (done || stall) continue;
          const uint64_t f = sv[w] & ~kValueMask;
          if (f == 0) {
            stall = true;
            continue;
          }
          excl += sv[w] & kValueMask;
          ++used;
          if (f == kFlagPrefix) done = true;
        }
        if (done) break;
        j -= used;
        if (stall) {
          if (++spins > kSpinLimit) {
            atomicExch(a.err, LDF_ERR_TIMEOUT);
            break;
          }
          __nanosleep(32);
        }
      }
      st_release_u64(&st[tile * 256 + t], kFlagPrefix | (excl + run));
    }
    // positions fit 32 bits (fewer than 2^31 rows)
    sh.delta[t] = static_cast<int32_t>(a.digit_base[t] + excl) - static_cast<int32_t>(start);
  }
  __syncthreads();
  const int64_t tbase = tile * RTILE;
  const int cnt       = static_cast<int>(a.n - tbase < RTILE ? a.n - tbase : RTILE);
  if constexpr (!MOVE) {
    for (int j = threadIdx.x; j < cnt; j += RT) {
      const int32_t pos = sh.delta[s_dig[j]] + j;
      if (WRITE_KEYS) a.keys_out[pos] = s_keys[j];
      a.vals_out[pos] = s_vals[j];
      if (a.inv_out) a.inv_out[s_vals[j]] = static_cast<int32_t>(pos);
    }
  } else {
    // a pass that moves columns: kMoveBatch rows of a thread at a time, so the
    // payload's loads (random rows after the first pass) overlap.  Positions
    // and rows fit 32 bits (fewer than 2^31 rows).
    for (int j0 = threadIdx.x; j0 < cnt; j0 += RT * kMoveBatch) {
      int32_t pos[kMoveBatch], row[kMoveBatch];
#pragma unroll
      for (int k = 0; k < kMoveBatch; ++k) {
        const int j = j0 + k * RT;
        pos[k]      = -1;
        row[k]      = 0;
        if (j < cnt) {
          pos[k]           = sh.delta[s_dig[j]] + j;
          row[k]           = s_vals[j];
          a.vals_out[pos[k]] = row[k];
          if (a.inv_out) a.inv_out[row[k]] = pos[k];
        }
      }
      move_payload_rows(a.pay, pos, row);
    }
  }
}

// Rows of a tile straight from global memory (GATHER: the word is loaded from
// the columns at the row, the first pass of a word; otherwise the carried key).
// In a pass on the carried word, all row ids and then all words are loaded
// before any digit is taken, so that the thread's loads are in flight together.
template <bool GATHER, bool FUSEDG = false>
__device__ __forceinline__ void load_tile_rows(const PassArgs& a, int64_t tile, uint64_t (&key)[RI],
                                               int32_t (&val)[RI], uint32_t (&dr)[RI])
{
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t wbase = tile * RTILE + warp * (32 * RI) + lane;
  if (!GATHER && a.p.src != DigitSrc::CLASS) {
#pragma unroll
    for (int i = 0; i < RI; ++i) {
      const int64_t idx = wbase + i * 32;
      val[i] = idx < a.n ? (a.vals_in ? __ldg(a.vals_in + idx) : static_cast<int32_t>(idx)) : 0;
    }
#pragma unroll
    for (int i = 0; i < RI; ++i) {
      const int64_t idx = wbase + i * 32;
      key[i] = idx < a.n ? __ldg(reinterpret_cast<const unsigned long long*>(a.keys_in) + idx) : 0ull;
    }
#pragma unroll
    for (int i = 0; i < RI; ++i)
      dr[i] = wbase + i * 32 < a.n ? static_cast<uint32_t>(key[i] >> a.p.shift) & 0xffu : 256u;
    return;
  }
  if (FUSEDG) {
    // the fused word from its key columns, one column at a time with the
    // items' loads in flight together; dr[i] gathers W's low byte
#pragma unroll
    for (int i = 0; i < RI; ++i) {
      const int64_t idx = wbase + i * 32;
      val[i] = idx < a.n ? (a.vals_in ? __ldg(a.vals_in + idx) : static_cast<int32_t>(idx)) : -1;
      key[i] = 0;
      dr[i]  = 0;
    }
    for (int k = 0; k < a.fused.n; ++k) {
      const SortKeyDesc& kk = a.fused.key[k];
      uint64_t raw[RI];
#pragma unroll
      for (int i = 0; i < RI; ++i) {
        raw[i] = 0;
        if (val[i] < 0) continue;
        switch (kk.col.width) {
          case 1: raw[i] = __ldg(static_cast<const uint8_t*>(kk.col.data) + val[i]); break;
          case 2: raw[i] = __ldg(static_cast<const uint16_t*>(kk.col.data) + val[i]); break;
          case 4: raw[i] = __ldg(static_cast<const uint32_t*>(kk.col.data) + val[i]); break;
          default: raw[i] = __ldg(static_cast<const unsigned long long*>(kk.col.data) + val[i]); break;
        }
      }
#pragma unroll
      for (int i = 0; i < RI; ++i)
        if (val[i] >= 0) fused_add(sort_word_of(kk, raw[i], true) - a.fused.min[k], a.fused.off[k], key[i], dr[i]);
    }
#pragma unroll
    for (int i = 0; i < RI; ++i) {
      if (val[i] < 0) {
        val[i] = 0;
        dr[i]  = 256;
      } else if (!a.p.fused_low) {
        dr[i] = static_cast<uint32_t>(key[i] >> a.p.shift) & 0xffu;
      }
    }
    return;
  }
#pragma unroll
  for (int i = 0; i < RI; ++i) {
    const int64_t idx = wbase + i * 32;
    key[i]            = 0;
    val[i]            = 0;
    dr[i]             = 256;
    if (idx < a.n) {
      const int64_t row = a.vals_in ? a.vals_in[idx] : idx;
      val[i]            = static_cast<int32_t>(row);
      if (a.p.src == DigitSrc::CLASS) {
        dr[i] = class_digit(a.p.key, row);
      } else {
        key[i] = GATHER ? pass_word(a.p, row) : a.keys_in[idx];
        dr[i]  = static_cast<uint32_t>(key[i] >> a.p.shift) & 0xffu;
      }
    }
  }
}

// Tiles ahead that a onesweep tile prefetches into L2 (one wave of resident
// CTAs); LDF_B200_L2_PREFETCH=0 turns the prefetch off.
int64_t prefetch_tiles()
{
  static const bool off = [] {
    const char* e = std::getenv("LDF_B200_L2_PREFETCH");
    return e != nullptr && std::atoi(e) == 0;
  }();
  return off ? 0 : static_cast<int64_t>(num_sms()) * kRadixMinBlocks;
}
// Whether a first pass over rows in input order prefetches its key columns
// (LDF_B200_L2_PREFETCH_FIRST=0 turns it off).
int prefetch_first_pass()
{
  static const bool off = [] {
    const char* e = std::getenv("LDF_B200_L2_PREFETCH_FIRST");
    return e != nullptr && std::atoi(e) == 0;
  }();
  return off ? 0 : 1;
}

// Whether p points into device memory (not pinned host or managed memory, as
// a zero-copy legate store would be): the first pass prefetches only columns
// held there.
bool on_device(const void* p)
{
  if (p == nullptr) return true;
  cudaPointerAttributes at{};
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeDevice;
}
bool column_on_device(const DCol& c) { return on_device(c.data) && on_device(c.valid); }

// The key columns the first pass of `p` reads in row order are all in
// device memory.
bool pass_columns_on_device(const RadixPass& p, const FusedKey* fused)
{
  if (p.src == DigitSrc::FUSED) {
    if (fused == nullptr) return false;
    for (int k = 0; k < fused->n; ++k)
      if (!column_on_device(fused->key[k].col)) return false;
    return true;
  }
  if (p.src == DigitSrc::BUCKET) {
    for (int k = 0; k < p.hash_keys.n; ++k)
      if (!column_on_device(p.hash_keys.c[k])) return false;
    return true;
  }
  return column_on_device(p.key.col);
}

// One tile per CTA.  WRITE_KEYS: later passes of the same word follow, so
// carry the word along.  MOVE: the pass also moves a.pay's columns (the last
// pass only, which carries no word).
template <bool GATHER, bool WRITE_KEYS, bool MOVE = false, bool FUSEDG = false>
__global__ void __launch_bounds__(RT, kRadixMinBlocks) onesweep_kernel(PassArgs a)
{
  __shared__ OsShared sh;
  // staged tile (dynamic): [keys u64 x RTILE when carried][rows i32 x RTILE][digits u8 x RTILE]
  extern __shared__ __align__(16) unsigned char s_stage[];
  uint64_t* s_keys = reinterpret_cast<uint64_t*>(s_stage);
  int32_t* s_vals  = reinterpret_cast<int32_t*>(s_stage + (WRITE_KEYS ? RTILE * sizeof(uint64_t) : 0));
  uint8_t* s_dig   = reinterpret_cast<uint8_t*>(s_vals + RTILE);

  const int64_t tile = next_tile_id(a.counter, &sh.tile[0]);
  for (int i = threadIdx.x; i < RW * 256; i += RT) (&sh.whist[0][0])[i] = 0;
  __syncthreads();
  uint64_t key[RI];
  int32_t val[RI];
  uint32_t dr[RI];
  if (a.pf_ahead > 0 && threadIdx.x == 0 && (tile + a.pf_ahead) * RTILE < a.n) {
    const int64_t lo = (tile + a.pf_ahead) * RTILE;
    const int64_t hi = min(lo + static_cast<int64_t>(RTILE), a.n);
    if (!GATHER) {
      if (a.vals_in) l2_prefetch_bulk(a.vals_in, lo * 4, hi * 4);
      if (a.p.src != DigitSrc::CLASS) l2_prefetch_bulk(a.keys_in, lo * 8, hi * 8);
    } else if (a.pf_columns && a.vals_in == nullptr) {  // rows in input order: the key columns are read in order
      if (FUSEDG) {
        for (int k = 0; k < a.fused.n; ++k) prefetch_column(a.fused.key[k].col, lo, hi);
      } else if (a.p.src == DigitSrc::BUCKET) {
        for (int k = 0; k < a.p.hash_keys.n; ++k) prefetch_column(a.p.hash_keys.c[k], lo, hi);
      } else {
        prefetch_column(a.p.key.col, lo, hi);
      }
    }
  }
  load_tile_rows<GATHER, FUSEDG>(a, tile, key, val, dr);
  rank_and_scatter<WRITE_KEYS, MOVE>(a, tile, key, val, dr, sh, s_keys, s_vals, s_dig);
}

constexpr size_t onesweep_smem(bool write_keys)
{
  return (write_keys ? RTILE * sizeof(uint64_t) : 0) + RTILE * (sizeof(int32_t) + 1);
}

template <bool GATHER, bool WRITE_KEYS, bool MOVE = false, bool FUSEDG = false>
void launch_onesweep(cudaStream_t s, unsigned tiles, const PassArgs& a)
{
  static_assert(!(MOVE && WRITE_KEYS), "the pass that moves columns is the last one");
  constexpr size_t smem = onesweep_smem(WRITE_KEYS);
  LDF_CUDA(cudaFuncSetAttribute(onesweep_kernel<GATHER, WRITE_KEYS, MOVE, FUSEDG>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(smem)));
  // profile names: a pass that loads its word from the columns, one that
  // moves the payload columns, the others
  const char* name = MOVE ? "onesweep_move" : (GATHER ? "onesweep_gather" : "onesweep");
  launch(name, onesweep_kernel<GATHER, WRITE_KEYS, MOVE, FUSEDG>, tiles, RT, smem, s, a);
}

// Identity order: the payload columns copied as they are.
__global__ void copy_payload_kernel(RadixPayload p, int64_t n)
{
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    move_payload(p, i, i);
}

__global__ void iota_kernel(int32_t* p, int64_t n)
{
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    p[i] = static_cast<int32_t>(i);
}

unsigned hblocks(int64_t n)
{
  int64_t b   = ceil_div(n, RT);
  int64_t cap = static_cast<int64_t>(num_sms()) * 4;
  return static_cast<unsigned>(b < 1 ? 1 : (b > cap ? cap : b));
}

// Histogram grid: one block per RT * kHR rows, at most five resident per SM.
unsigned hist_blocks(int64_t n)
{
  int64_t b   = ceil_div(n, static_cast<int64_t>(RT) * kHR);
  int64_t cap = static_cast<int64_t>(num_sms()) * 5;
  return static_cast<unsigned>(b < 1 ? 1 : (b > cap ? cap : b));
}

// Two passes belong to the same carried word when they read the same column
// transform (or bucket) and differ only in shift.
bool same_word(const RadixPass& a, const RadixPass& b)
{
  if (a.src != b.src || a.src == DigitSrc::CLASS) return false;
  if (a.src == DigitSrc::BUCKET || a.src == DigitSrc::FUSED) return true;
  return a.key.col.data == b.key.col.data && a.key.descending == b.key.descending;
}

struct WordRangeArgs {
  int n;
  SortKeyDesc key[kFuseMax];
};

// mm[2k] = min, mm[2k + 1] = max of key k's words (init ~0 and 0).  Eight
// rows per thread, one key column at a time, loads in flight together.
constexpr int kRangeRows = 8;
__global__ void __launch_bounds__(256) word_range_kernel(WordRangeArgs a, int64_t n, unsigned long long* mm)
{
  unsigned long long lo[kFuseMax], hi[kFuseMax];
#pragma unroll
  for (int k = 0; k < kFuseMax; ++k) lo[k] = ~0ull, hi[k] = 0;
  const int64_t per_iter = static_cast<int64_t>(blockDim.x) * kRangeRows;
  for (int64_t base = blockIdx.x * per_iter; base < n; base += static_cast<int64_t>(gridDim.x) * per_iter) {
#pragma unroll
    for (int k = 0; k < kFuseMax; ++k) {
      if (k >= a.n) continue;
      const DCol& c = a.key[k].col;
      uint64_t raw[kRangeRows];
#pragma unroll
      for (int j = 0; j < kRangeRows; ++j) {
        const int64_t r = base + j * blockDim.x + threadIdx.x;
        raw[j]          = 0;
        if (r >= n) continue;
        switch (c.width) {
          case 1: raw[j] = __ldg(static_cast<const uint8_t*>(c.data) + r); break;
          case 2: raw[j] = __ldg(static_cast<const uint16_t*>(c.data) + r); break;
          case 4: raw[j] = __ldg(static_cast<const uint32_t*>(c.data) + r); break;
          default: raw[j] = __ldg(static_cast<const unsigned long long*>(c.data) + r); break;
        }
      }
#pragma unroll
      for (int j = 0; j < kRangeRows; ++j) {
        if (base + j * blockDim.x + threadIdx.x >= n) continue;
        const unsigned long long w = sort_word_of(a.key[k], raw[j], true);
        lo[k]                      = w < lo[k] ? w : lo[k];
        hi[k]                      = w > hi[k] ? w : hi[k];
      }
    }
  }
#pragma unroll
  for (int k = 0; k < kFuseMax; ++k) {
    if (k >= a.n) continue;
    for (int d = 16; d > 0; d >>= 1) {
      const unsigned long long l = __shfl_xor_sync(0xffffffffu, lo[k], d);
      const unsigned long long h = __shfl_xor_sync(0xffffffffu, hi[k], d);
      lo[k]                      = l < lo[k] ? l : lo[k];
      hi[k]                      = h > hi[k] ? h : hi[k];
    }
    if ((threadIdx.x & 31) == 0) {
      atomicMin(mm + 2 * k, lo[k]);
      atomicMax(mm + 2 * k + 1, hi[k]);
    }
  }
}

}  // namespace

void sort_word_ranges(const OpContext& ctx, const SortKeyDesc* keys, int nkeys, int64_t n, uint64_t* mn,
                      uint64_t* mx)
{
  LDF_REQUIRE(nkeys >= 1 && nkeys <= kFuseMax, "sort_word_ranges: too many keys");
  cudaStream_t s = ctx.stream();
  Buffer<unsigned long long> mm(ctx.alloc(), 2 * kFuseMax);
  std::vector<unsigned long long> h(2 * kFuseMax);
  for (int k = 0; k < kFuseMax; ++k) h[2 * k] = ~0ull, h[2 * k + 1] = 0;
  LDF_CUDA(cudaMemcpyAsync(mm.get(), h.data(), h.size() * 8, cudaMemcpyHostToDevice, s));
  WordRangeArgs a{};
  a.n = nkeys;
  for (int k = 0; k < nkeys; ++k) a.key[k] = keys[k];
  if (n > 0) launch("word_range", word_range_kernel, hblocks(n), 256, 0, s, a, n, mm.get());
  LDF_CUDA(cudaMemcpyAsync(h.data(), mm.get(), h.size() * 8, cudaMemcpyDeviceToHost, s));
  ctx.finish();
  for (int k = 0; k < nkeys; ++k) {
    mn[k] = h[2 * k];
    mx[k] = h[2 * k + 1];
  }
}

void radix_histograms(const OpContext& ctx, const std::vector<RadixPass>& passes, int64_t n,
                      uint32_t* d_hist, const FusedKey* fused)
{
  cudaStream_t s = ctx.stream();
  LDF_CUDA(cudaMemsetAsync(d_hist, 0, passes.size() * 256 * sizeof(uint32_t), s));
  for (size_t b = 0; b < passes.size(); b += kHistPassesPerLaunch) {
    HistArgs h{};
    h.npasses = static_cast<int>(std::min<size_t>(kHistPassesPerLaunch, passes.size() - b));
    for (int q = 0; q < h.npasses; ++q) {
      h.p[q] = passes[b + q];
      if (q > 0 && same_word(passes[b + q - 1], passes[b + q])) h.reuse |= 1u << q;
    }
    if (fused) h.fused = *fused;
    h.n    = n;
    h.hist = d_hist + b * 256;
    if (n > 0 && fused) launch("histogram", histogram_kernel<true>, hist_blocks(n), RT, 0, s, h);
    else if (n > 0) launch("histogram", histogram_kernel<false>, hist_blocks(n), RT, 0, s, h);
    LDF_CHECK_LAUNCH();
  }
}

void radix_sort_rows(const OpContext& ctx, const std::vector<RadixPass>& passes, int64_t n,
                     int32_t* perm, std::vector<uint32_t>* hist_out, int32_t* inv, const RadixPayload* payload,
                     const FusedKey* fused)
{
  const Allocator& al = ctx.alloc();
  cudaStream_t s      = ctx.stream();
  const size_t P      = passes.size();
  std::vector<uint32_t> hist(P * 256, 0);
  if (P > 0 && n > 0) {
    Buffer<uint32_t> d_hist(al, P * 256);
    radix_histograms(ctx, passes, n, d_hist.get(), fused);
    LDF_CUDA(cudaMemcpyAsync(hist.data(), d_hist.get(), P * 256 * sizeof(uint32_t),
                             cudaMemcpyDeviceToHost, s));
    ctx.finish();
  }
  if (hist_out) *hist_out = hist;
  // schedule: skip constant-digit passes; the first executed pass of a word
  // gathers it, later passes of the same word read it carried
  std::vector<int> run;
  for (size_t q = 0; q < P; ++q) {
    bool constant = false;
    for (int d = 0; d < 256; ++d)
      if (hist[q * 256 + d] == static_cast<uint32_t>(n)) constant = true;
    if (!constant && n > 0) run.push_back(static_cast<int>(q));
  }
  if (run.empty()) {
    if (n > 0) launch("iota", iota_kernel, hblocks(n), RT, 0, s, perm, n);
    if (n > 0 && inv) launch("iota", iota_kernel, hblocks(n), RT, 0, s, inv, n);
    if (n > 0 && payload && !payload_empty(*payload))
      launch("copy_payload", copy_payload_kernel, hblocks(n), RT, 0, s, *payload, n);
    LDF_CHECK_LAUNCH();
    return;
  }
  std::vector<uint64_t> bases(run.size() * 256);
  for (size_t k = 0; k < run.size(); ++k) {
    uint64_t acc = 0;
    for (int d = 0; d < 256; ++d) {
      bases[k * 256 + d] = acc;
      acc += hist[run[k] * 256 + d];
    }
  }
  Buffer<uint64_t> d_bases(al, bases.size());
  LDF_CUDA(cudaMemcpyAsync(d_bases.get(), bases.data(), bases.size() * 8, cudaMemcpyHostToDevice, s));

  const int64_t tiles = ceil_div(n, RTILE);
  Buffer<uint64_t> status(al, tiles * 256 + 2);
  Buffer<uint64_t> keys[2] = {Buffer<uint64_t>(al, n), Buffer<uint64_t>(al, n)};
  Buffer<int32_t> vals_tmp(al, n);
  // ping-pong so that the last pass writes into `perm`
  int32_t* vbuf[2];
  const bool odd = run.size() % 2 == 1;
  vbuf[0]        = odd ? perm : vals_tmp.get();
  vbuf[1]        = odd ? vals_tmp.get() : perm;
  const int32_t* vin = nullptr;
  const uint64_t* kin = nullptr;
  for (size_t k = 0; k < run.size(); ++k) {
    const RadixPass& p = passes[run[k]];
    const bool gather  = k == 0 || !same_word(passes[run[k - 1]], p);
    const bool write_keys = p.src != DigitSrc::CLASS && k + 1 < run.size() && same_word(p, passes[run[k + 1]]);
    LDF_CUDA(cudaMemsetAsync(status.get(), 0, (tiles * 256 + 2) * 8, s));
    PassArgs a{};
    a.p          = p;
    a.n          = n;
    a.keys_in    = kin;
    a.keys_out   = keys[k % 2].get();
    a.vals_in    = vin;
    a.vals_out   = vbuf[k % 2];
    a.digit_base = d_bases.get() + k * 256;
    a.status     = status.get();
    a.counter    = reinterpret_cast<unsigned long long*>(status.get() + tiles * 256);
    a.inv_out    = k + 1 == run.size() ? inv : nullptr;
    if (k + 1 == run.size() && payload) a.pay = *payload;
    if (fused) a.fused = *fused;
    a.err        = ctx.err();
    a.pf_ahead   = prefetch_tiles();
    a.pf_columns = gather && k == 0 && prefetch_first_pass() && pass_columns_on_device(p, fused) ? 1 : 0;
    const unsigned g = static_cast<unsigned>(tiles);
    const bool move = !payload_empty(a.pay);
    if (gather && p.src == DigitSrc::FUSED) {  // the fused word's first pass
      if (move) launch_onesweep<true, false, true, true>(s, g, a);
      else if (write_keys) launch_onesweep<true, true, false, true>(s, g, a);
      else launch_onesweep<true, false, false, true>(s, g, a);
    } else if (move && gather) launch_onesweep<true, false, true>(s, g, a);
    else if (move) launch_onesweep<false, false, true>(s, g, a);
    else if (gather && write_keys) launch_onesweep<true, true>(s, g, a);
    else if (gather) launch_onesweep<true, false>(s, g, a);
    else if (write_keys) launch_onesweep<false, true>(s, g, a);
    else launch_onesweep<false, false>(s, g, a);
    LDF_CHECK_LAUNCH();
    vin = vbuf[k % 2];
    kin = keys[k % 2].get();
  }
}

}  // namespace ldf

// ---- raw-pointer helpers for the no-allocation hash partition ---------------
namespace ldf {

void radix_histogram_raw(cudaStream_t s, const RadixPass& p, int64_t n, uint32_t* d_hist)
{
  LDF_CUDA(cudaMemsetAsync(d_hist, 0, 256 * sizeof(uint32_t), s));
  if (n <= 0) return;
  HistArgs h{};
  h.npasses = 1;
  h.p[0]    = p;
  h.n       = n;
  h.hist    = d_hist;
  launch("histogram", histogram_kernel<false>, hist_blocks(n), RT, 0, s, h);
}

int64_t radix_status_words(int64_t n) { return ceil_div(n, RTILE) * 256 + 2; }

void onesweep_gather_pass_raw(cudaStream_t s, const RadixPass& p, int64_t n, int32_t* rows_out,
                              const uint64_t* d_bases, uint64_t* status, int* err)
{
  if (n <= 0) return;
  const int64_t tiles = ceil_div(n, RTILE);
  PassArgs a{};
  a.p          = p;
  a.n          = n;
  a.keys_in    = nullptr;
  a.keys_out   = nullptr;
  a.vals_in    = nullptr;
  a.vals_out   = rows_out;
  a.digit_base = d_bases;
  a.status     = status;
  a.counter    = reinterpret_cast<unsigned long long*>(status + tiles * 256);
  a.err        = err;
  launch_onesweep<true, false>(s, static_cast<unsigned>(tiles), a);
}

}  // namespace ldf
