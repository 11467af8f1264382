// CSV text in device memory -> columns in the legate layout, parsed on the
// device.  Replaces cudf::io::read_csv in CSVRead::gpu_variant (csv.cu:53-139)
// and follows the conversions of the reference's Arrow reader
// (CSVRead::cpu_variant, csv.cpp:58-130, with the Arrow defaults it keeps).
//
// 1. Records.  Quotes make the record boundaries depend on everything before
//    them, so the text is cut into 256-byte chunks and each chunk is run
//    through the 4-state quoting automaton from all four start states at once
//    (end state and terminator count per start state).  The chunk maps are
//    composed with a block scan and a one-block pass over the block
//    aggregates, which gives every chunk its true start state; the chunks
//    then write the positions of their terminators (after a scan of their
//    counts).
// 2. Rows.  One thread per record: empty records are skipped (a scan gives
//    each kept record its output row), the first record's field count is the
//    expected one.
// 3. Fields.  One thread per record runs the automaton over the record,
//    converts the requested fields and writes the outputs; string fields
//    record their source and unescaped length, and after a scan of the
//    lengths a copy kernel writes the characters and the ranges.
// Errors (a wrong field count, a value that does not convert) are recorded
// as the smallest (line, column, code) and reported after the parse.
#include "scan.cuh"
#include "table_ops.cuh"

#include "pow5_table.inc"

namespace ldf {
namespace {

constexpr int kCsvMaxCols   = 64;
constexpr int kCsvMaxFields = 1024;
constexpr int kCsvMaxNulls  = 32;
constexpr int kCsvNullBytes = 256;
constexpr int kCsvChunk     = 256;   // bytes per thread in the record split
constexpr int kCsvScanBlock = 1024;  // chunks per block in the map scan
constexpr int kCsvNumBuf    = 96;    // longest quoted numeric field converted

struct CsvParams {
  const uint8_t* text;
  int64_t n;
  int32_t delim;
  int32_t ncols;
  int32_t nfield_map;  // entries of col_of_field in use
  int32_t n_null;      // null spellings (0: no nulls)
  int32_t types[kCsvMaxCols];
  int32_t widths[kCsvMaxCols];
  int16_t col_of_field[kCsvMaxFields];  // output column of a field, -1: not read
  int32_t null_off[kCsvMaxNulls + 1];
  uint8_t null_chars[kCsvNullBytes];
};

// ---- the quoting automaton ---------------------------------------------------
// States: at a field start, in an unquoted field, in a quoted field, in a
// quoted field right after a quote (the end of the quotes or half of "").
enum : uint32_t { kFs = 0, kUq = 1, kQ = 2, kQq = 3 };
// Byte classes: other, quote, delimiter, terminator ('\n', or '\r' not
// followed by '\n'), '\r' followed by '\n'.
enum : uint32_t { kOther = 0, kQuote = 1, kDelim = 2, kTerm = 3, kCrLf = 4 };

// Next state (2 bits) and "a record ended" (bit 2) of (state, class), three
// bits per entry at 3 * (state * 5 + class).
constexpr uint64_t fsm_entry(uint32_t next, bool eol) { return next | (eol ? 4u : 0u); }
constexpr uint64_t kFsmTable =
  // field start: other -> unquoted, quote -> quoted, delim -> field start,
  // terminator -> field start + record end, CR before LF -> unchanged
  (fsm_entry(kUq, false) << 0) | (fsm_entry(kQ, false) << 3) | (fsm_entry(kFs, false) << 6) |
  (fsm_entry(kFs, true) << 9) | (fsm_entry(kFs, false) << 12) |
  // unquoted: a quote is an ordinary byte
  (fsm_entry(kUq, false) << 15) | (fsm_entry(kUq, false) << 18) | (fsm_entry(kFs, false) << 21) |
  (fsm_entry(kFs, true) << 24) | (fsm_entry(kUq, false) << 27) |
  // quoted: everything but a quote belongs to the field
  (fsm_entry(kQ, false) << 30) | (fsm_entry(kQq, false) << 33) | (fsm_entry(kQ, false) << 36) |
  (fsm_entry(kQ, false) << 39) | (fsm_entry(kQ, false) << 42) |
  // after a quote inside quotes: "" -> quoted again; other bytes are kept
  // as in an unquoted field
  (fsm_entry(kUq, false) << 45) | (fsm_entry(kQ, false) << 48) | (fsm_entry(kFs, false) << 51) |
  (fsm_entry(kFs, true) << 54) | (fsm_entry(kQq, false) << 57);

__device__ __forceinline__ uint32_t fsm_step(uint32_t st, uint32_t cls, uint32_t& eol)
{
  const uint32_t e = static_cast<uint32_t>(kFsmTable >> (3 * (st * 5 + cls))) & 7u;
  eol              = e >> 2;
  return e & 3u;
}

__device__ __forceinline__ uint32_t byte_class(uint8_t c, uint8_t next_c, bool has_next, uint8_t delim)
{
  if (c == '"') return kQuote;
  if (c == delim) return kDelim;
  if (c == '\n') return kTerm;
  if (c == '\r') return (has_next && next_c == '\n') ? kCrLf : kTerm;
  return kOther;
}

// A chunk's map: end state of each of the four start states, 2 bits each.
constexpr uint32_t kIdentityMap = 0xE4u;  // 3 2 1 0
__device__ __forceinline__ uint32_t map_apply(uint32_t m, uint32_t s) { return (m >> (2 * s)) & 3u; }
// f then g
__device__ __forceinline__ uint32_t map_compose(uint32_t f, uint32_t g)
{
  uint32_t h = 0;
#pragma unroll
  for (uint32_t s = 0; s < 4; ++s) h |= map_apply(g, map_apply(f, s)) << (2 * s);
  return h;
}

// ---- 1. records -------------------------------------------------------------------
// Bytes [b, e) of chunk c (e exclusive), 16 at a time where the text allows;
// `visit(i, cls)` for every byte with its class.
template <typename F>
__device__ __forceinline__ void scan_chunk(const uint8_t* text, int64_t n, int64_t b, int64_t e, uint8_t delim,
                                           F&& visit)
{
  for (int64_t i = b; i < e; i += 16) {
    uint8_t v[17];
    if (i + 16 < n) {  // 16 bytes plus the next one (CR-LF lookahead)
      const uint4 q = *reinterpret_cast<const uint4*>(text + i);
      const uint32_t w[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
      for (int k = 0; k < 16; ++k) v[k] = static_cast<uint8_t>(w[k >> 2] >> (8 * (k & 3)));
      v[16] = text[i + 16];
    } else {
#pragma unroll
      for (int k = 0; k < 17; ++k) v[k] = i + k < n ? text[i + k] : 0;
    }
    const int m = static_cast<int>(e - i < 16 ? e - i : 16);
    for (int k = 0; k < m; ++k) visit(i + k, byte_class(v[k], v[k + 1], i + k + 1 < n, delim));
  }
}

// Chunk c run from the four start states: maps[c] (end states) and
// counts[4c + s] (records ended when starting in state s).
__global__ void __launch_bounds__(256) csv_chunk_kernel(const uint8_t* text, int64_t n, int64_t nchunks, uint8_t delim,
                                                        uint8_t* maps, uint32_t* counts)
{
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < nchunks; c += (int64_t)gridDim.x * blockDim.x) {
    const int64_t b = c * kCsvChunk, e = b + kCsvChunk < n ? b + kCsvChunk : n;
    uint32_t st[4] = {kFs, kUq, kQ, kQq}, cnt[4] = {0, 0, 0, 0};
    scan_chunk(text, n, b, e, delim, [&](int64_t, uint32_t cls) {
#pragma unroll
      for (int s = 0; s < 4; ++s) {
        uint32_t eol;
        st[s] = fsm_step(st[s], cls, eol);
        cnt[s] += eol;
      }
    });
    maps[c] = static_cast<uint8_t>(st[0] | (st[1] << 2) | (st[2] << 4) | (st[3] << 6));
#pragma unroll
    for (int s = 0; s < 4; ++s) counts[4 * c + s] = cnt[s];
  }
}

// Block-local exclusive composition of the chunk maps (kCsvScanBlock chunks
// per block, four per thread): prefix[c] maps the block's start state to
// chunk c's; agg[block] is the whole block's map.
__global__ void __launch_bounds__(256) csv_map_scan_kernel(const uint8_t* maps, int64_t nchunks, uint8_t* prefix,
                                                           uint8_t* agg)
{
  __shared__ uint32_t s_warp[8];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t c0 = blockIdx.x * static_cast<int64_t>(kCsvScanBlock) + threadIdx.x * 4;
  uint32_t m[4], own = kIdentityMap;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    m[k] = c0 + k < nchunks ? maps[c0 + k] : kIdentityMap;
    own  = map_compose(own, m[k]);
  }
  uint32_t inc = own;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t other = __shfl_up_sync(0xffffffffu, inc, d);
    if (lane >= d) inc = map_compose(other, inc);
  }
  if (lane == 31) s_warp[warp] = inc;
  __syncthreads();
  uint32_t wpre = kIdentityMap;
  for (int w = 0; w < warp; ++w) wpre = map_compose(wpre, s_warp[w]);
  const uint32_t before = __shfl_up_sync(0xffffffffu, inc, 1);
  uint32_t run          = map_compose(wpre, lane > 0 ? before : kIdentityMap);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    if (c0 + k < nchunks) prefix[c0 + k] = static_cast<uint8_t>(run);
    run = map_compose(run, m[k]);
  }
  if (threadIdx.x == blockDim.x - 1) agg[blockIdx.x] = static_cast<uint8_t>(run);
}

// Start state of every block (one thread; a few thousand blocks per GB).
__global__ void csv_block_start_kernel(const uint8_t* agg, int64_t nblocks, uint8_t* start)
{
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  uint32_t st = kFs;
  for (int64_t b = 0; b < nblocks; ++b) {
    start[b] = static_cast<uint8_t>(st);
    st       = map_apply(agg[b], st);
  }
}

// Start state of every chunk and the number of records it ends.
__global__ void csv_chunk_start_kernel(const uint8_t* prefix, const uint8_t* block_start, const uint32_t* counts,
                                       int64_t nchunks, uint8_t* start, uint32_t* ends)
{
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < nchunks; c += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t s = map_apply(prefix[c], block_start[c / kCsvScanBlock]);
    start[c]         = static_cast<uint8_t>(s);
    ends[c]          = counts[4 * c + s];
  }
}

// Positions of the record terminators (outside quotes), in text order.
__global__ void __launch_bounds__(256) csv_terms_kernel(const uint8_t* text, int64_t n, int64_t nchunks, uint8_t delim,
                                                        const uint8_t* start, const int64_t* base, int64_t* term)
{
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < nchunks; c += (int64_t)gridDim.x * blockDim.x) {
    const int64_t b = c * kCsvChunk, e = b + kCsvChunk < n ? b + kCsvChunk : n;
    uint32_t st = start[c];
    int64_t out = base[c];
    scan_chunk(text, n, b, e, delim, [&](int64_t i, uint32_t cls) {
      uint32_t eol;
      st = fsm_step(st, cls, eol);
      if (eol) term[out++] = i;
    });
  }
}

// Record i: bytes [lstart, lend) (the terminator, and the '\r' of a "\r\n",
// excluded); flag = the record is not empty; *first = the first non-empty
// record (one atomic per block).
__global__ void __launch_bounds__(256) csv_records_kernel(const uint8_t* text, int64_t n, const int64_t* term,
                                                          int64_t nterm, int64_t nrec, int64_t* lstart, int64_t* lend,
                                                          uint32_t* flag, unsigned long long* first)
{
  __shared__ unsigned long long s_first;
  if (threadIdx.x == 0) s_first = ~0ull;
  __syncthreads();
  unsigned long long mine = ~0ull;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nrec; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t s = i == 0 ? 0 : term[i - 1] + 1;
    int64_t e       = i < nterm ? term[i] : n;
    if (i < nterm && text[e] == '\n' && e > s && text[e - 1] == '\r') --e;
    lstart[i]            = s;
    lend[i]              = e;
    const bool non_empty = e > s;
    flag[i]              = non_empty ? 1u : 0u;
    if (non_empty && static_cast<unsigned long long>(i) < mine) mine = static_cast<unsigned long long>(i);
  }
  if (mine != ~0ull) atomicMin(&s_first, mine);
  __syncthreads();
  if (threadIdx.x == 0 && s_first != ~0ull) atomicMin(first, s_first);
}

// ---- 3. field conversions ------------------------------------------------------------
enum : uint32_t { kErrFields = 1, kErrConvert = 2, kErrUtf8 = 3, kErrUnsupported = 4 };

__device__ __forceinline__ void csv_error(unsigned long long* err, int64_t line, int col, uint32_t code)
{
  atomicMin(err, (static_cast<unsigned long long>(line) << 16) | (static_cast<unsigned long long>(col) << 8) | code);
}

__device__ __forceinline__ bool is_blank(uint8_t c) { return c == ' ' || c == '\t'; }

__device__ __forceinline__ void trim(const uint8_t*& p, int& len)
{
  while (len > 0 && is_blank(p[0])) ++p, --len;
  while (len > 0 && is_blank(p[len - 1])) --len;
}

// Integer of `width` bytes: optional '-' (signed types), decimal digits; or
// 0x / 0X and at most 2 * width hex digits, taken as the value's bits.
// Returns false for anything else or a value out of range.
__device__ bool parse_integer(const uint8_t* p, int len, int width, bool is_signed, uint64_t& out)
{
  trim(p, len);
  if (len == 0) return false;
  int i    = 0;
  bool neg = false;
  if (is_signed && p[0] == '-') {
    neg = true;
    i   = 1;
    if (len == 1) return false;
  }
  if (!neg && len > 2 && p[0] == '0' && (p[1] | 0x20) == 'x') {
    const int nd = len - 2;
    if (nd > 2 * width) return false;
    uint64_t v = 0;
    for (int k = 2; k < len; ++k) {
      const uint8_t c = p[k];
      uint32_t d;
      if (c >= '0' && c <= '9') d = c - '0';
      else if ((c | 0x20) >= 'a' && (c | 0x20) <= 'f') d = (c | 0x20) - 'a' + 10;
      else return false;
      v = (v << 4) | d;
    }
    out = v;
    return true;
  }
  uint64_t v = 0;
  for (; i < len; ++i) {
    const uint32_t d = static_cast<uint32_t>(p[i]) - '0';
    if (d > 9) return false;
    if (v > (~0ull - d) / 10) return false;
    v = v * 10 + d;
  }
  const int bits = 8 * width;
  if (!is_signed) {
    if (bits < 64 && v > (1ull << bits) - 1) return false;
    out = v;
    return true;
  }
  const uint64_t lim = 1ull << (bits - 1);
  if (neg ? v > lim : v > lim - 1) return false;
  out = neg ? 0ull - v : v;
  return true;
}

__device__ __forceinline__ bool bytes_are(const uint8_t* p, int len, const char* s)
{
  int k = 0;
  for (; s[k] != 0; ++k)
    if (k >= len || p[k] != static_cast<uint8_t>(s[k])) return false;
  return k == len;
}

// Arrow's default true / false spellings, exactly.
__device__ bool parse_bool(const uint8_t* p, int len, uint64_t& out)
{
  if (bytes_are(p, len, "1") || bytes_are(p, len, "True") || bytes_are(p, len, "TRUE") || bytes_are(p, len, "true")) {
    out = 1;
    return true;
  }
  if (bytes_are(p, len, "0") || bytes_are(p, len, "False") || bytes_are(p, len, "FALSE") ||
      bytes_are(p, len, "false")) {
    out = 0;
    return true;
  }
  return false;
}

// Binary float bits (sign excluded) nearest to w * 10^q, w != 0, ties to
// even: the Eisel-Lemire method (Lemire 2021) with 128-bit powers of five,
// exact for w below 10^19 (Mushtak & Lemire 2023).  F64: binary64, else
// binary32.
template <bool F64>
__device__ uint64_t decimal_to_binary(uint64_t w, int64_t q)
{
  constexpr int kMant   = F64 ? 52 : 23;
  constexpr int kMinExp = F64 ? -1023 : -127;
  constexpr int kInf    = F64 ? 0x7FF : 0xFF;
  constexpr int kLo10   = F64 ? -342 : -64;
  constexpr int kHi10   = F64 ? 308 : 38;
  constexpr int kEvenLo = F64 ? -4 : -17;  // powers of ten whose products can be exact halfway cases
  constexpr int kEvenHi = F64 ? 23 : 10;
  if (q < kLo10) return 0;
  if (q > kHi10) return static_cast<uint64_t>(kInf) << kMant;
  const int lz = __clzll(static_cast<long long>(w));
  w <<= lz;
  const int idx = 2 * static_cast<int>(q - kPow5Smallest);
  uint64_t hi   = __umul64hi(w, kPow5Table[idx]);
  uint64_t lo   = w * kPow5Table[idx];
  constexpr uint64_t kPrecMask = ~0ull >> (kMant + 3);
  if ((hi & kPrecMask) == kPrecMask) {  // the low bits may be inexact: add the next 64 bits of the power
    const uint64_t hi2 = __umul64hi(w, kPow5Table[idx + 1]);
    lo += hi2;
    if (hi2 > lo) ++hi;
  }
  const int upper = static_cast<int>(hi >> 63);
  const int shift = upper + 64 - kMant - 3;
  uint64_t m      = hi >> shift;
  // floor(q * log2(10)) + 63 as a fixed-point product
  int64_t p2 = ((217706 * q) >> 16) + 63 + upper - lz - kMinExp;
  if (p2 <= 0) {  // subnormal
    if (-p2 + 1 >= 64) return 0;
    m >>= -p2 + 1;
    m += m & 1;
    m >>= 1;
    p2 = m < (1ull << kMant) ? 0 : 1;
    return (static_cast<uint64_t>(p2) << kMant) | (m & ((1ull << kMant) - 1));
  }
  if (lo <= 1 && q >= kEvenLo && q <= kEvenHi && (m & 3) == 1 && (m << shift) == hi) m &= ~1ull;  // exact tie
  m += m & 1;
  m >>= 1;
  if (m >= (2ull << kMant)) {
    m = 1ull << kMant;
    ++p2;
  }
  m &= ~(1ull << kMant);
  if (p2 >= kInf) return static_cast<uint64_t>(kInf) << kMant;
  return (static_cast<uint64_t>(p2) << kMant) | m;
}

__device__ __forceinline__ bool word_is(const uint8_t* p, int len, const char* lower)
{
  int k = 0;
  for (; lower[k] != 0; ++k)
    if (k >= len || (p[k] | 0x20) != static_cast<uint8_t>(lower[k])) return false;
  return k == len;
}

// Decimal text -> binary float bits with the sign: [+-] digits [. digits]
// [(e|E) [+-] digits], or inf / infinity / nan in any case; spaces and tabs
// trimmed.  0: converted; 1: not a number; 2: more than 19 significant
// digits that the 19-digit conversion cannot round (not supported).
template <bool F64>
__device__ int parse_real(const uint8_t* p, int len, uint64_t& out)
{
  constexpr int kBits   = F64 ? 64 : 32;
  constexpr int kMant   = F64 ? 52 : 23;
  trim(p, len);
  if (len == 0) return 1;
  int i    = 0;
  bool neg = false;
  if (p[0] == '+' || p[0] == '-') {
    neg = p[0] == '-';
    i   = 1;
  }
  const uint64_t sign = neg ? 1ull << (kBits - 1) : 0;
  const int rest      = len - i;
  if (word_is(p + i, rest, "inf") || word_is(p + i, rest, "infinity")) {
    out = sign | ((F64 ? 0x7FFull : 0xFFull) << kMant);
    return 0;
  }
  if (word_is(p + i, rest, "nan")) {
    out = sign | ((F64 ? 0xFFFull : 0x1FFull) << (kMant - 1));
    return 0;
  }
  uint64_t w     = 0;
  int kept       = 0;     // significant digits in w (at most 19)
  int64_t adj    = 0;     // decimal exponent of w's last digit
  bool truncated = false;  // a non-zero digit was dropped
  int ndig       = 0;
  for (; i < len && p[i] >= '0' && p[i] <= '9'; ++i, ++ndig) {
    const uint32_t d = p[i] - '0';
    if (kept == 0 && d == 0) continue;
    if (kept < 19) {
      w = w * 10 + d;
      ++kept;
    } else {
      ++adj;
      truncated |= d != 0;
    }
  }
  if (i < len && p[i] == '.') {
    for (++i; i < len && p[i] >= '0' && p[i] <= '9'; ++i, ++ndig) {
      const uint32_t d = p[i] - '0';
      if (kept == 0 && d == 0) {
        --adj;
        continue;
      }
      if (kept < 19) {
        w = w * 10 + d;
        ++kept;
        --adj;
      } else {
        truncated |= d != 0;
      }
    }
  }
  if (ndig == 0) return 1;
  int64_t e10 = 0;
  if (i < len && (p[i] | 0x20) == 'e') {
    ++i;
    bool eneg = false;
    if (i < len && (p[i] == '+' || p[i] == '-')) {
      eneg = p[i] == '-';
      ++i;
    }
    int edig = 0;
    for (; i < len && p[i] >= '0' && p[i] <= '9'; ++i, ++edig)
      if (e10 < 100000) e10 = e10 * 10 + (p[i] - '0');
    if (edig == 0) return 1;
    if (eneg) e10 = -e10;
  }
  if (i != len) return 1;
  if (w == 0) {
    out = sign;
    return 0;
  }
  const int64_t q = e10 + adj;
  const uint64_t b = decimal_to_binary<F64>(w, q);
  if (truncated && decimal_to_binary<F64>(w + 1, q) != b) return 2;
  out = sign | b;
  return 0;
}

// Streaming UTF-8 check: no overlong forms, no surrogates, at most U+10FFFF.
struct Utf8Check {
  int need    = 0;
  uint8_t lo  = 0x80, hi = 0xBF;
  bool bad    = false;
  __device__ __forceinline__ void put(uint8_t c)
  {
    if (need) {
      if (c < lo || c > hi) bad = true;
      lo = 0x80;
      hi = 0xBF;
      --need;
      return;
    }
    if (c < 0x80) return;
    if (c >= 0xC2 && c <= 0xDF) need = 1;
    else if (c == 0xE0) need = 2, lo = 0xA0;
    else if ((c >= 0xE1 && c <= 0xEC) || c == 0xEE || c == 0xEF) need = 2;
    else if (c == 0xED) need = 2, hi = 0x9F;
    else if (c == 0xF0) need = 3, lo = 0x90;
    else if (c >= 0xF1 && c <= 0xF3) need = 3;
    else if (c == 0xF4) need = 3, hi = 0x8F;
    else bad = true;
  }
  __device__ __forceinline__ bool ok() const { return !bad && need == 0; }
};

// The content of a quoted field that starts at t[b] == '"', byte by byte:
// "" inside the quotes is one quote, the first lone quote closes them, and
// bytes after it are kept as they are.  `e` bounds the walk (the field's end,
// or the text's end when the caller stops after a known length).
struct Unquote {
  const uint8_t* t;
  int64_t i, e;
  bool inq;
  __device__ Unquote(const uint8_t* t_, int64_t b, int64_t e_) : t(t_), i(b + 1), e(e_), inq(true) {}
  __device__ __forceinline__ bool next(uint8_t& c)
  {
    while (i < e) {
      const uint8_t x = t[i];
      if (inq && x == '"') {
        if (i + 1 < e && t[i + 1] == '"') {
          c = '"';
          i += 2;
          return true;
        }
        inq = false;
        ++i;
        continue;
      }
      c = x;
      ++i;
      return true;
    }
    return false;
  }
};

// A field's content as bytes: unquoted fields in place, quoted ones unescaped
// into `buf` (len = -1 when longer than kCsvNumBuf).
__device__ __forceinline__ const uint8_t* field_bytes(const uint8_t* t, int64_t b, int64_t e, bool quoted, uint8_t* buf,
                                                     int& len)
{
  if (!quoted) {
    len = static_cast<int>(e - b);
    return t + b;
  }
  Unquote u(t, b, e);
  uint8_t c;
  len = 0;
  while (u.next(c)) {
    if (len == kCsvNumBuf) {
      len = -1;
      return buf;
    }
    buf[len++] = c;
  }
  return buf;
}

__device__ __forceinline__ bool is_null_spelling(const CsvParams& P, const uint8_t* p, int len)
{
  for (int k = 0; k < P.n_null; ++k) {
    const int o = P.null_off[k], l = P.null_off[k + 1] - o - 1;  // spellings are NUL-terminated
    if (l != len) continue;
    bool eq = true;
    for (int j = 0; j < l && eq; ++j) eq = p[j] == P.null_chars[o + j];
    if (eq) return true;
  }
  return false;
}

// A float field that the 19-digit conversion cannot round (or a quoted one
// too long for the buffer), converted afterwards by csv_exact_float_kernel.
struct DeferredFloat {
  int64_t line, row, b, e;
  int32_t col;
};
constexpr int kCsvMaxDeferred = 1 << 16;

struct CsvOut {
  void* data[kCsvMaxCols];
  uint8_t* valid[kCsvMaxCols];      // null when the columns have no masks
  int64_t* str_src[kCsvMaxCols];    // strings: source offset (bit 62: quoted)
  int64_t* str_len[kCsvMaxCols];    // strings: unescaped length (0 for null)
  DeferredFloat* deferred;          // kCsvMaxDeferred entries
  unsigned int* ndeferred;
};

constexpr int64_t kQuotedBit = int64_t(1) << 62;

// Converts field t[b, e) of record `line` into output column k, row `row`;
// `off` turns positions in t into positions in the text (t may be a staged
// copy of part of it).
__device__ void convert_field(const CsvParams& P, const CsvOut& O, const uint8_t* t, int64_t off, int64_t line,
                              int64_t row, int k, int64_t b, int64_t e, unsigned long long* err)
{
  const bool quoted = e > b && t[b] == '"';
  const int type    = P.types[k];
  uint8_t buf[kCsvNumBuf];
  int len;
  const uint8_t* p = field_bytes(t, b, e, quoted, buf, len);
  const bool null  = P.n_null > 0 && len >= 0 && is_null_spelling(P, p, len);
  if (O.valid[k]) O.valid[k][row] = null ? 0 : 1;
  if (type == LDF_STRING) {
    int64_t n = 0;
    if (!null) {
      Utf8Check u8;
      if (quoted) {
        Unquote u(t, b, e);
        uint8_t c;
        while (u.next(c)) u8.put(c), ++n;
      } else {
        for (int64_t i = b; i < e; ++i) u8.put(t[i]);
        n = e - b;
      }
      if (!u8.ok()) csv_error(err, line, k, kErrUtf8);
    }
    O.str_src[k][row] = (b + off) | (quoted ? kQuotedBit : 0);
    O.str_len[k][row] = n;
    return;
  }
  uint64_t v = 0;
  if (!null) {
    if (type == LDF_FLOAT64 || type == LDF_FLOAT32) {
      int r = 2;
      if (len >= 0) r = type == LDF_FLOAT64 ? parse_real<true>(p, len, v) : parse_real<false>(p, len, v);
      if (r == 1) {
        csv_error(err, line, k, kErrConvert);
      } else if (r == 2) {
        const unsigned int d = atomicAdd(O.ndeferred, 1u);
        if (d < kCsvMaxDeferred) O.deferred[d] = DeferredFloat{line, row, b + off, e + off, k};
        else csv_error(err, line, k, kErrUnsupported);
      }
    } else if (len < 0) {
      csv_error(err, line, k, kErrUnsupported);
    } else if (type == LDF_BOOL8) {
      if (!parse_bool(p, len, v)) csv_error(err, line, k, kErrConvert);
    } else {
      const bool sgn  = type == LDF_INT8 || type == LDF_INT16 || type == LDF_INT32 || type == LDF_INT64;
      if (!parse_integer(p, len, P.widths[k], sgn, v)) csv_error(err, line, k, kErrConvert);
    }
  }
  switch (P.widths[k]) {
    case 1: static_cast<uint8_t*>(O.data[k])[row] = static_cast<uint8_t>(v); break;
    case 2: static_cast<uint16_t*>(O.data[k])[row] = static_cast<uint16_t>(v); break;
    case 4: static_cast<uint32_t*>(O.data[k])[row] = static_cast<uint32_t>(v); break;
    default: static_cast<unsigned long long*>(O.data[k])[row] = v; break;
  }
}

// ---- exact conversion of the deferred floats ----------------------------------------
// Big unsigned integers of 32-bit limbs (little-endian), enough for 800
// decimal digits times the powers of two and five that the comparison below
// needs (about 4,800 bits).
constexpr int kBigLimbs   = 224;
constexpr int kExactDigits = 800;
struct BigNum {
  uint32_t w[kBigLimbs];
  int n;
  bool ok;
  __device__ __forceinline__ void set(uint64_t v)
  {
    n  = 0;
    ok = true;
    while (v) {
      w[n++] = static_cast<uint32_t>(v);
      v >>= 32;
    }
  }
  __device__ void mul_add(uint32_t m, uint32_t a)
  {
    uint64_t c = a;
    for (int i = 0; i < n; ++i) {
      const uint64_t t = static_cast<uint64_t>(w[i]) * m + c;
      w[i]             = static_cast<uint32_t>(t);
      c                = t >> 32;
    }
    if (c) {
      if (n == kBigLimbs) ok = false;
      else w[n++] = static_cast<uint32_t>(c);
    }
  }
  __device__ void mul_pow5(int64_t k)
  {
    for (; k >= 13; k -= 13) mul_add(1220703125u, 0);  // 5^13
    uint32_t m = 1;
    for (; k > 0; --k) m *= 5;
    if (m != 1) mul_add(m, 0);
  }
  __device__ void shl(int64_t s)
  {
    if (n == 0 || s == 0) return;
    const int64_t limbs = s >> 5;
    const int bits      = static_cast<int>(s & 31);
    if (n + limbs + 1 > kBigLimbs) {
      ok = false;
      return;
    }
    uint32_t carry = 0;
    if (bits) {
      for (int i = 0; i < n; ++i) {
        const uint32_t x = w[i];
        w[i]             = (x << bits) | carry;
        carry            = x >> (32 - bits);
      }
    }
    if (carry) w[n++] = carry;
    for (int i = n - 1; i >= 0; --i) w[i + limbs] = w[i];
    for (int64_t i = 0; i < limbs; ++i) w[i] = 0;
    n += static_cast<int>(limbs);
  }
};

__device__ int big_cmp(const BigNum& a, const BigNum& b)
{
  int na = a.n, nb = b.n;
  while (na > 0 && a.w[na - 1] == 0) --na;
  while (nb > 0 && b.w[nb - 1] == 0) --nb;
  if (na != nb) return na < nb ? -1 : 1;
  for (int i = na - 1; i >= 0; --i)
    if (a.w[i] != b.w[i]) return a.w[i] < b.w[i] ? -1 : 1;
  return 0;
}

// A field's content, byte by byte (quoted fields unescaped).
struct FieldCursor {
  const uint8_t* t;
  int64_t i, e;
  bool quoted;
  Unquote u;
  __device__ FieldCursor(const uint8_t* t_, int64_t b, int64_t e_)
    : t(t_), i(b), e(e_), quoted(e_ > b && t_[b] == '"'), u(t_, b, e_)
  {
  }
  __device__ __forceinline__ bool next(uint8_t& c)
  {
    if (quoted) return u.next(c);
    if (i >= e) return false;
    c = t[i++];
    return true;
  }
};

// The nearest binary float to the field's decimal value, ties to even, for
// any number of digits: the 19-digit conversions of w and w + 1 give the two
// candidates, and the exact decimal (its first kExactDigits significant
// digits; any non-zero digit after them only breaks a tie upwards) is
// compared with their midpoint (2m + 1) * 2^(e - 1) in big integers.
// Returns 0 (bits set, sign included), 1 (not a number), 2 (too large for
// the big integers).
template <bool F64>
__device__ int exact_real(const uint8_t* t, int64_t b, int64_t e, uint64_t& out, BigNum& A, BigNum& B)
{
  constexpr int kBits = F64 ? 64 : 32;
  constexpr int kMant = F64 ? 52 : 23;
  constexpr int kBias = F64 ? 1023 : 127;
  FieldCursor cur(t, b, e);
  uint8_t c;
  bool have = cur.next(c);
  while (have && is_blank(c)) have = cur.next(c);
  bool neg = false;
  if (have && (c == '+' || c == '-')) {
    neg  = c == '-';
    have = cur.next(c);
  }
  const uint64_t sign = neg ? 1ull << (kBits - 1) : 0;
  if (have && ((c | 0x20) == 'i' || (c | 0x20) == 'n')) {  // inf / infinity / nan, possibly padded
    uint8_t word[9];
    int nw = 0;
    while (have && !is_blank(c)) {
      if (nw == 8) return 1;
      word[nw++] = c;
      have       = cur.next(c);
    }
    while (have && is_blank(c)) have = cur.next(c);
    if (have) return 1;
    if (word_is(word, nw, "inf") || word_is(word, nw, "infinity")) {
      out = sign | ((F64 ? 0x7FFull : 0xFFull) << kMant);
      return 0;
    }
    if (word_is(word, nw, "nan")) {
      out = sign | ((F64 ? 0xFFFull : 0x1FFull) << (kMant - 1));
      return 0;
    }
    return 1;
  }
  uint64_t w = 0;
  int kept19 = 0, kept = 0, ndig = 0;
  int64_t adj19 = 0, adj = 0;
  bool trunc19 = false, sticky = false;
  A.set(0);
  auto digit = [&](uint32_t d, bool frac) {
    ++ndig;
    if (kept == 0 && d == 0) {
      if (frac) --adj, --adj19;
      return;
    }
    if (kept19 < 19) {
      w = w * 10 + d;
      ++kept19;
      if (frac) --adj19;
    } else {
      if (!frac) ++adj19;
      trunc19 |= d != 0;
    }
    if (kept < kExactDigits) {
      A.mul_add(10, d);
      ++kept;
      if (frac) --adj;
    } else {
      if (!frac) ++adj;
      sticky |= d != 0;
    }
  };
  while (have && c >= '0' && c <= '9') {
    digit(c - '0', false);
    have = cur.next(c);
  }
  if (have && c == '.') {
    have = cur.next(c);
    while (have && c >= '0' && c <= '9') {
      digit(c - '0', true);
      have = cur.next(c);
    }
  }
  if (ndig == 0) return 1;
  int64_t e10 = 0;
  if (have && (c | 0x20) == 'e') {
    have      = cur.next(c);
    bool eneg = false;
    if (have && (c == '+' || c == '-')) {
      eneg = c == '-';
      have = cur.next(c);
    }
    int edig = 0;
    while (have && c >= '0' && c <= '9') {
      if (e10 < 100000) e10 = e10 * 10 + (c - '0');
      ++edig;
      have = cur.next(c);
    }
    if (edig == 0) return 1;
    if (eneg) e10 = -e10;
  }
  while (have && is_blank(c)) have = cur.next(c);
  if (have) return 1;
  if (w == 0) {
    out = sign;
    return 0;
  }
  const uint64_t lo = decimal_to_binary<F64>(w, e10 + adj19);
  if (!trunc19) {
    out = sign | lo;
    return 0;
  }
  const uint64_t hi = decimal_to_binary<F64>(w + 1, e10 + adj19);
  if (hi == lo) {
    out = sign | lo;
    return 0;
  }
  // midpoint of lo and the next float up: (2m + 1) * 2^(ex - 1)
  const uint64_t E  = lo >> kMant;
  const uint64_t fr = lo & ((1ull << kMant) - 1);
  const uint64_t m  = E ? (fr | (1ull << kMant)) : fr;
  const int64_t ex  = (E ? static_cast<int64_t>(E) : 1) - kBias - kMant;
  B.set(2 * m + 1);
  const int64_t qd = e10 + adj;  // decimal = A * 10^qd
  int64_t s;
  if (qd >= 0) {
    A.mul_pow5(qd);
    s = qd - (ex - 1);
  } else {
    B.mul_pow5(-qd);
    s = qd - (ex - 1);
  }
  if (s >= 0) A.shl(s);
  else B.shl(-s);
  if (!A.ok || !B.ok) return 2;
  int cmp = big_cmp(A, B);
  if (cmp == 0 && sticky) cmp = 1;
  const uint64_t r = cmp < 0 ? lo : (cmp > 0 ? hi : ((m & 1) ? hi : lo));
  out              = sign | r;
  return 0;
}

// One thread per deferred float field: the exact conversion, written over
// the placeholder of the parse.
__global__ void __launch_bounds__(64) csv_exact_float_kernel(CsvParams P, CsvOut O, unsigned int count,
                                                             unsigned long long* err)
{
  BigNum A, B;
  for (unsigned int d = blockIdx.x * blockDim.x + threadIdx.x; d < count; d += gridDim.x * blockDim.x) {
    const DeferredFloat f = O.deferred[d];
    uint64_t v            = 0;
    const int r = P.types[f.col] == LDF_FLOAT64 ? exact_real<true>(P.text, f.b, f.e, v, A, B)
                                                 : exact_real<false>(P.text, f.b, f.e, v, A, B);
    if (r) {
      csv_error(err, f.line, f.col, r == 1 ? kErrConvert : kErrUnsupported);
      continue;
    }
    if (P.widths[f.col] == 8) static_cast<unsigned long long*>(O.data[f.col])[f.row] = v;
    else static_cast<uint32_t*>(O.data[f.col])[f.row] = static_cast<uint32_t>(v);
  }
}

// Fields of record [s, e): calls on_field(f, b, e) for each, returns the count.
template <typename F>
__device__ __forceinline__ int walk_fields(const uint8_t* t, int64_t s, int64_t e, uint8_t delim, F&& on_field)
{
  int f       = 0;
  int64_t fb  = s;
  uint32_t st = kFs;
  for (int64_t i = s; i < e; ++i) {
    const uint8_t c     = t[i];
    const uint32_t cls  = c == '"' ? kQuote : (c == delim ? kDelim : kOther);
    if (cls == kDelim && st != kQ) {
      on_field(f++, fb, i);
      fb = i + 1;
      st = kFs;
      continue;
    }
    uint32_t eol;
    st = fsm_step(st, cls, eol);
  }
  on_field(f++, fb, e);
  return f;
}

// Field count of the first non-empty record (one thread).
__global__ void csv_first_fields_kernel(CsvParams P, const int64_t* lstart, const int64_t* lend,
                                        const unsigned long long* first, int64_t nrec, int* nfields)
{
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  const int64_t r = static_cast<int64_t>(*first);
  *nfields        = r < nrec ? walk_fields(P.text, lstart[r], lend[r], static_cast<uint8_t>(P.delim),
                                           [](int, int64_t, int64_t) {})
                             : 0;
}

// One thread per record: output row, field walk, conversions, field count.
// A block takes kParseRecords consecutive records at a time; their bytes
// (contiguous in the text) are first staged in shared memory with 16-byte
// loads (a group longer than the stage is read from global memory).  Each
// thread then walks its record once per batch of kColBatch output columns,
// noting the bounds of those columns' fields, and the batch's columns are
// converted one after another by all threads together: the conversion code
// of one type runs in lockstep across the warp instead of each thread being
// at a different field of its record.
constexpr int kParseRecords = 128;
constexpr int kParseStage   = 24 * 1024;
constexpr int kColBatch     = 16;
__global__ void __launch_bounds__(kParseRecords) csv_parse_kernel(CsvParams P, CsvOut O, const int64_t* lstart,
                                                                  const int64_t* lend, const int64_t* rowidx,
                                                                  int64_t nrec, int64_t first, int skip_first,
                                                                  int nfields, unsigned long long* err)
{
  __shared__ __align__(16) uint8_t stage[kParseStage];
  __shared__ int32_t s_fb[kColBatch][kParseRecords];  // field bounds relative to the record's start
  __shared__ int32_t s_fe[kColBatch][kParseRecords];
  const uint8_t delim = static_cast<uint8_t>(P.delim);
  const int tid       = threadIdx.x;
  for (int64_t g = static_cast<int64_t>(blockIdx.x) * kParseRecords; g < nrec;
       g += static_cast<int64_t>(gridDim.x) * kParseRecords) {
    const int64_t last = g + kParseRecords < nrec ? g + kParseRecords - 1 : nrec - 1;
    const int64_t gs   = lstart[g] & ~int64_t(15);
    const int64_t ge   = lend[last];
    const bool staged  = ge - gs <= kParseStage;
    if (staged) {
      const int64_t full = (ge - gs) >> 4;  // 16-byte blocks inside [gs, ge)
      for (int64_t q = tid; q < full; q += blockDim.x)
        reinterpret_cast<uint4*>(stage)[q] = *reinterpret_cast<const uint4*>(P.text + gs + 16 * q);
      for (int64_t i = gs + 16 * full + tid; i < ge; i += blockDim.x) stage[i - gs] = P.text[i];
    }
    __syncthreads();
    const uint8_t* t = staged ? stage : P.text;
    const int64_t off = staged ? gs : 0;
    const int64_t r   = g + tid;
    bool active       = false;
    int64_t s = 0, e = 0, row = 0;
    if (r < nrec) {
      s      = lstart[r] - off;
      e      = lend[r] - off;
      active = e > s && !(skip_first && r == first);
      if (active) row = rowidx[r] - (skip_first && r > first ? 1 : 0);
    }
    for (int k0 = 0; k0 < P.ncols; k0 += kColBatch) {
      const int k1 = k0 + kColBatch < P.ncols ? k0 + kColBatch : P.ncols;
      bool ok      = false;
      if (active) {
        const int got = walk_fields(t, s, e, delim, [&](int f, int64_t b, int64_t fe) {
          if (f >= P.nfield_map) return;
          const int k = P.col_of_field[f];
          if (k >= k0 && k < k1) {
            s_fb[k - k0][tid] = static_cast<int32_t>(b - s);
            s_fe[k - k0][tid] = static_cast<int32_t>(fe - s);
          }
        });
        ok = got == nfields;  // otherwise some fields were never found: reported, not converted
        if (!ok && k0 == 0) csv_error(err, r, 0, kErrFields);
      }
      for (int k = k0; k < k1; ++k)
        if (ok) convert_field(P, O, t, off, r, row, k, s + s_fb[k - k0][tid], s + s_fe[k - k0][tid], err);
    }
    __syncthreads();
  }
}

// Characters of one string column: row i's content at offs[i] (ranges
// written as local offsets, chars_base = 0).
// A block takes kCsvStrRows rows a thread: unquoted strings are read eight
// bytes at a time with the loads in flight together, quoted ones unescaped,
// into a shared stage laid out at the output's 16-byte phase, which the block
// writes with 16-byte stores (the range's two end chunks byte by byte).  A
// tile whose characters exceed the stage writes them directly.
constexpr int kCsvStrRows  = 2;
constexpr int kCsvStrStage = 16 * 1024;

__global__ void __launch_bounds__(256) csv_copy_strings_kernel(const uint8_t* text, int64_t ntext, const int64_t* src,
                                                               const int64_t* len, const int64_t* offs, int64_t rows,
                                                               int64_t nchars, uint8_t* chars, ldf_range* ranges)
{
  __shared__ __align__(16) uint8_t stage[kCsvStrStage];
  const int64_t per_tile = static_cast<int64_t>(blockDim.x) * kCsvStrRows;
  for (int64_t tile = blockIdx.x; tile * per_tile < rows; tile += gridDim.x) {
    const int64_t i0    = tile * per_tile;
    const int64_t lo    = offs[i0];
    const int64_t hi    = i0 + per_tile < rows ? offs[i0 + per_tile] : nchars;
    const int64_t abase = lo - static_cast<int64_t>(reinterpret_cast<uintptr_t>(chars + lo) & 15);
    const bool staged   = hi - abase <= kCsvStrStage;
    for (int j = 0; j < kCsvStrRows; ++j) {
      const int64_t i = i0 + j * blockDim.x + threadIdx.x;
      if (i >= rows) continue;
      const int64_t o = offs[i], n = len[i], sp = src[i];
      ranges[i]  = ldf_range{o, o + n - 1};
      uint8_t* q = staged ? stage + (o - abase) : chars + o;
      if (n == 0) continue;
      if (sp & kQuotedBit) {
        Unquote u(text, sp & ~kQuotedBit, ntext);
        uint8_t c;
        for (int64_t k = 0; k < n && u.next(c); ++k) q[k] = c;
      } else {
        for (int64_t k = 0; k < n; k += 8) {
          uint8_t b[8];
#pragma unroll
          for (int v = 0; v < 8; ++v) b[v] = k + v < n ? text[sp + k + v] : 0;
#pragma unroll
          for (int v = 0; v < 8; ++v)
            if (k + v < n) q[k + v] = b[v];
        }
      }
    }
    if (staged) {
      __syncthreads();
      const int64_t nchunks = (hi - abase + 15) >> 4;  // chunk c: chars [abase + 16c, abase + 16c + 16)
      for (int64_t c = threadIdx.x; c < nchunks; c += blockDim.x) {
        const int64_t a0 = abase + 16 * c;
        if (a0 >= lo && a0 + 16 <= hi) {
          *reinterpret_cast<uint4*>(chars + a0) = *reinterpret_cast<const uint4*>(stage + 16 * c);
        } else {
          for (int k = 0; k < 16; ++k)
            if (a0 + k >= lo && a0 + k < hi) chars[a0 + k] = stage[16 * c + k];
        }
      }
      __syncthreads();
    }
  }
}

unsigned csv_blocks(int64_t work, int threads)
{
  const int64_t b   = ceil_div(work, threads);
  const int64_t cap = static_cast<int64_t>(num_sms()) * 16;
  return static_cast<unsigned>(b < 1 ? 1 : (b > cap ? cap : b));
}

}  // namespace

void csv_read(const uint8_t* text, int64_t n, char delimiter, int skip_first, const int32_t* fields,
              const int32_t* types, int ncols, const char* nulls, int nulls_bytes, int n_nulls, ldf_column* out,
              int64_t* nrows, const OpContext& ctx)
{
  LDF_REQUIRE(ncols >= 1 && ncols <= kCsvMaxCols, "csv_read: between 1 and 64 columns");
  LDF_REQUIRE(fields != nullptr && types != nullptr && out != nullptr && nrows != nullptr, "csv_read: null argument");
  LDF_REQUIRE(delimiter != '"' && delimiter != '\n' && delimiter != '\r', "csv_read: invalid delimiter");
  LDF_REQUIRE(n >= 0 && (n == 0 || text != nullptr), "csv_read: no text");
  LDF_REQUIRE((reinterpret_cast<uintptr_t>(text) & 15) == 0, "csv_read: the text must be 16-byte aligned");
  CsvParams P{};
  P.text  = text;
  P.n     = n;
  P.delim = static_cast<uint8_t>(delimiter);
  P.ncols = ncols;
  for (int f = 0; f < kCsvMaxFields; ++f) P.col_of_field[f] = -1;
  for (int j = 0; j < ncols; ++j) {
    LDF_REQUIRE(fields[j] >= 0 && fields[j] < kCsvMaxFields, "csv_read: field index out of range");
    LDF_REQUIRE(P.col_of_field[fields[j]] < 0, "csv_read: a field is read twice");
    const int t = types[j];
    LDF_REQUIRE(t == LDF_BOOL8 || (t >= LDF_INT8 && t <= LDF_FLOAT64) || t == LDF_STRING,
                "csv_read: unsupported column type");
    P.col_of_field[fields[j]] = static_cast<int16_t>(j);
    P.nfield_map              = std::max(P.nfield_map, fields[j] + 1);
    P.types[j]                = t;
    P.widths[j]               = type_width(t);
  }
  LDF_REQUIRE(n_nulls >= 0 && n_nulls <= kCsvMaxNulls && nulls_bytes >= 0 && nulls_bytes <= kCsvNullBytes,
              "csv_read: too many null spellings");
  P.n_null = n_nulls;
  {
    int o = 0;
    for (int k = 0; k < n_nulls; ++k) {
      P.null_off[k] = o;
      while (o < nulls_bytes && nulls[o] != 0) ++o;
      LDF_REQUIRE(o < nulls_bytes, "csv_read: null spellings must be NUL-terminated");
      LDF_REQUIRE(o - P.null_off[k] <= 64, "csv_read: null spellings of at most 64 bytes");
      ++o;
    }
    P.null_off[n_nulls] = o;
    for (int b = 0; b < o; ++b) P.null_chars[b] = static_cast<uint8_t>(nulls[b]);
  }
  const Allocator& al = ctx.alloc();
  cudaStream_t s      = ctx.stream();
  int64_t rows        = 0;
  if (n > 0) {
    // 1. records
    const int64_t nchunks = ceil_div(n, kCsvChunk);
    const int64_t nblocks = ceil_div(nchunks, kCsvScanBlock);
    Buffer<uint8_t> maps(al, nchunks), prefix(al, nchunks), start(al, nchunks), agg(al, nblocks),
      bstart(al, nblocks);
    Buffer<uint32_t> counts(al, 4 * nchunks), ends(al, nchunks);
    Buffer<int64_t> base(al, nchunks), misc(al, 4);
    launch("csv_chunks", csv_chunk_kernel, csv_blocks(nchunks, 256), 256, 0, s, text, n, nchunks,
           static_cast<uint8_t>(P.delim), maps.get(), counts.get());
    launch("csv_map_scan", csv_map_scan_kernel, static_cast<unsigned>(nblocks), 256, 0, s,
           static_cast<const uint8_t*>(maps.get()), nchunks, prefix.get(), agg.get());
    launch("csv_block_start", csv_block_start_kernel, 1u, 32, 0, s, static_cast<const uint8_t*>(agg.get()), nblocks,
           bstart.get());
    launch("csv_chunk_start", csv_chunk_start_kernel, csv_blocks(nchunks, 256), 256, 0, s,
           static_cast<const uint8_t*>(prefix.get()), static_cast<const uint8_t*>(bstart.get()),
           static_cast<const uint32_t*>(counts.get()), nchunks, start.get(), ends.get());
    exclusive_scan_u32(ends.get(), base.get(), nchunks, misc.get(), ctx);
    const int64_t nterm = ctx.read_i64(misc.get());
    Buffer<int64_t> term(al, std::max<int64_t>(nterm, 1));
    launch("csv_terms", csv_terms_kernel, csv_blocks(nchunks, 256), 256, 0, s, text, n, nchunks,
           static_cast<uint8_t>(P.delim), static_cast<const uint8_t*>(start.get()),
           static_cast<const int64_t*>(base.get()), term.get());
    // 2. rows: nterm + 1 records (the last one empty when the text ends with a terminator)
    const int64_t nrec = nterm + 1;
    Buffer<int64_t> lstart(al, nrec), lend(al, nrec), rowidx(al, nrec);
    Buffer<uint32_t> flag(al, nrec);
    Buffer<unsigned long long> first(al, 2);  // first non-empty record; error record
    Buffer<int> nfields(al, 1);
    LDF_CUDA(cudaMemsetAsync(first.get(), 0xff, 2 * sizeof(unsigned long long), s));
    launch("csv_records", csv_records_kernel, csv_blocks(nrec, 256), 256, 0, s, text, n,
           static_cast<const int64_t*>(term.get()), nterm, nrec, lstart.get(), lend.get(), flag.get(), first.get());
    launch("csv_first_fields", csv_first_fields_kernel, 1u, 32, 0, s, P, static_cast<const int64_t*>(lstart.get()),
           static_cast<const int64_t*>(lend.get()), static_cast<const unsigned long long*>(first.get()), nrec,
           nfields.get());
    exclusive_scan_u32(flag.get(), rowidx.get(), nrec, misc.get(), ctx);
    int64_t h_total = 0;
    unsigned long long h_first = 0;
    int h_nfields = 0;
    LDF_CUDA(cudaMemcpyAsync(&h_total, misc.get(), sizeof(h_total), cudaMemcpyDeviceToHost, s));
    LDF_CUDA(cudaMemcpyAsync(&h_first, first.get(), sizeof(h_first), cudaMemcpyDeviceToHost, s));
    LDF_CUDA(cudaMemcpyAsync(&h_nfields, nfields.get(), sizeof(h_nfields), cudaMemcpyDeviceToHost, s));
    ctx.finish();
    const bool has_first = h_first < static_cast<unsigned long long>(nrec);
    rows                 = h_total - (skip_first && has_first ? 1 : 0);
    // 3. fields
    CsvOut O{};
    Buffer<DeferredFloat> deferred(al, kCsvMaxDeferred);
    Buffer<unsigned int> ndeferred(al, 1);
    LDF_CUDA(cudaMemsetAsync(ndeferred.get(), 0, sizeof(unsigned int), s));
    O.deferred  = deferred.get();
    O.ndeferred = ndeferred.get();
    std::vector<Buffer<int64_t>> str_bufs;
    for (int j = 0; j < ncols; ++j) {
      out[j]     = alloc_out_column(al, P.types[j], rows, n_nulls > 0);
      O.data[j]  = out[j].data;
      O.valid[j] = out[j].valid;
      if (P.types[j] == LDF_STRING) {
        str_bufs.emplace_back(al, std::max<int64_t>(rows, 1));
        O.str_src[j] = str_bufs.back().get();
        str_bufs.emplace_back(al, std::max<int64_t>(rows, 1));
        O.str_len[j] = str_bufs.back().get();
      }
    }
    if (rows > 0) {
      launch("csv_parse", csv_parse_kernel, csv_blocks(nrec, kParseRecords), kParseRecords, 0, s, P, O,
             static_cast<const int64_t*>(lstart.get()), static_cast<const int64_t*>(lend.get()),
             static_cast<const int64_t*>(rowidx.get()), nrec, static_cast<int64_t>(h_first), skip_first ? 1 : 0,
             h_nfields, first.get() + 1);
    }
    unsigned long long h_err = ~0ull;
    unsigned int h_deferred  = 0;
    LDF_CUDA(cudaMemcpyAsync(&h_err, first.get() + 1, sizeof(h_err), cudaMemcpyDeviceToHost, s));
    LDF_CUDA(cudaMemcpyAsync(&h_deferred, ndeferred.get(), sizeof(h_deferred), cudaMemcpyDeviceToHost, s));
    ctx.finish();
    if (h_err == ~0ull && h_deferred > 0) {  // floats the 19-digit conversion could not round
      const unsigned int count = std::min<unsigned int>(h_deferred, kCsvMaxDeferred);
      launch("csv_exact_float", csv_exact_float_kernel, csv_blocks(count, 64), 64, 0, s, P, O, count, first.get() + 1);
      LDF_CUDA(cudaMemcpyAsync(&h_err, first.get() + 1, sizeof(h_err), cudaMemcpyDeviceToHost, s));
      ctx.finish();
    }
    if (h_err != ~0ull) {
      for (int j = 0; j < ncols; ++j) free_out_column(al, out[j]);
      const int64_t line = static_cast<int64_t>(h_err >> 16);
      const int col      = static_cast<int>((h_err >> 8) & 0xff);
      const uint32_t code = static_cast<uint32_t>(h_err & 0xff);
      const std::string where = " in record " + std::to_string(line + 1);
      if (code == kErrFields) fail(LDF_ERR_INVALID_ARGUMENT, "CSV parse error: expected " + std::to_string(h_nfields) + " columns" + where);
      if (code == kErrUtf8) fail(LDF_ERR_INVALID_ARGUMENT, "CSV conversion error to string: invalid UTF8 data in column " + std::to_string(col) + where);
      if (code == kErrUnsupported)
        fail(LDF_ERR_UNSUPPORTED, "CSV value of column " + std::to_string(col) + where +
                                    ": a number needing more than 19 significant digits to round, or a quoted number of more than 96 bytes");
      fail(LDF_ERR_INVALID_ARGUMENT, "CSV conversion error: invalid value in column " + std::to_string(col) + where);
    }
    // strings: lengths -> offsets -> characters
    for (int j = 0; j < ncols; ++j) {
      if (P.types[j] != LDF_STRING) continue;
      Buffer<int64_t> offs(al, std::max<int64_t>(rows, 1));
      exclusive_scan_i64(O.str_len[j], offs.get(), rows, misc.get(), ctx);
      const int64_t nchars = ctx.read_i64(misc.get());
      out[j].chars         = static_cast<char*>(al.allocate(static_cast<size_t>(std::max<int64_t>(nchars, 1))));
      out[j].num_chars     = nchars;
      out[j].chars_base    = 0;
      if (rows > 0)
        launch("csv_strings", csv_copy_strings_kernel, csv_blocks(ceil_div(rows, kCsvStrRows), 256), 256, 0, s, text,
               n, static_cast<const int64_t*>(O.str_src[j]), static_cast<const int64_t*>(O.str_len[j]),
               static_cast<const int64_t*>(offs.get()), rows, nchars, reinterpret_cast<uint8_t*>(out[j].chars),
               static_cast<ldf_range*>(out[j].data));
    }
    ctx.finish();
  } else {
    for (int j = 0; j < ncols; ++j) {
      out[j] = alloc_out_column(al, types[j], 0, n_nulls > 0);
      if (types[j] == LDF_STRING) {
        out[j].chars     = static_cast<char*>(al.allocate(16));
        out[j].num_chars = 0;
      }
    }
  }
  *nrows = rows;
}

}  // namespace ldf
