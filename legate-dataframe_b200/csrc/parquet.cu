// Parquet pages -> columns in the legate layout, decoded on the device.
// Replaces cudf::io::read_parquet in ParquetRead::gpu_variant
// (parquet.cu:48-101); the results match the reference's CPU reader (Arrow).
//
// The caller walks the footer and the page headers (Thrift, a few bytes per
// page) and hands over one entry per page; the whole file is in device
// memory.  Then:
// 1. Snappy pages are decompressed, one warp per page, with the compressed
//    stream staged and the recent output kept in shared memory; every lane
//    parses the same element tags and the warp copies each element's bytes
//    together.
// 2. Dictionary pages of byte arrays get an entry table (offset, length),
//    one block per page walking the length prefixes from shared memory.
// 3. One block per data page decodes its rows in tiles of kPqTile: thread 0
//    cuts the next tile out of the RLE / bit-packed hybrid streams (the
//    definition levels, the dictionary indices) as a list of run segments,
//    and every thread decodes its values from the segment it falls in; a
//    block scan of the definition levels gives each valid row its value
//    index; PLAIN values are read at that index, dictionary values through
//    the decoded index, and byte arrays by a walk of their length prefixes.
// 4. String columns: lengths -> offsets (scan) -> characters copied.
#include <algorithm>

#include "scan.cuh"
#include "table_ops.cuh"

namespace ldf {
namespace {

constexpr int kLanes     = 32;    // threads of a warp
constexpr int kPqThreads = 128;
constexpr int kPqTile    = 1024;  // rows of a data page decoded per round

// Device view of one page.
struct PqPage {
  ldf_parquet_page h;
  const uint8_t* data;    // payload, decompressed (the file's bytes for an uncompressed page)
  int64_t data_bytes;
  int64_t dict_entry0;    // byte-array dictionary pages: first entry in the entry table
};

// Error record: (page << 8 | code), the smallest kept.
enum : uint32_t { kPqErrSnappy = 1, kPqErrStream = 2, kPqErrDictIndex = 3, kPqErrValues = 4 };
__device__ __forceinline__ void pq_error(unsigned long long* err, int64_t page, uint32_t code)
{
  atomicMin(err, (static_cast<unsigned long long>(page) << 8) | code);
}

__device__ __forceinline__ uint32_t le_bytes(const uint8_t* p, int n)
{
  uint32_t v = 0;
  for (int k = 0; k < n; ++k) v |= static_cast<uint32_t>(p[k]) << (8 * k);
  return v;
}

// ---- 1. Snappy ------------------------------------------------------------------
// One warp per page.  The compressed stream is staged kSnapIn bytes at a time
// in shared memory (16-byte granules loaded by all lanes), and the last
// kSnapWin output bytes are kept in a shared ring, so tag parsing and most
// back-references run at shared-memory latency; the output goes to global
// memory as it is produced.
// One warp per block: the 32 KB ring covers all but a few back-references
// (Snappy's offsets stay below 64 KB) and six such blocks fit an SM.
constexpr int kSnapIn    = 2048;   // staged compressed bytes per warp
constexpr int kSnapWin   = 32768;  // output ring per warp (a power of two, a multiple of 32)

constexpr int kSnapBatch      = 32;    // short elements decoded together
constexpr int kSnapBatchBytes = 1024;  // output bytes of a batch at most
constexpr int kSnapShort      = 64;    // longer literals are copied on their own
constexpr int kSnapPerLane    = 4;     // output bytes per lane per window of a batch

struct alignas(16) SnapShared {
  uint8_t in[kSnapIn];
  uint8_t win[kSnapWin];
  uint16_t size[kSnapIn];         // input bytes of an element whose tag is at in[x] (0xffff: unknown)
  uint8_t elem[kSnapBatchBytes];  // batch element of each output byte
  int64_t off[kSnapBatch];        // copy: offset
  int32_t epos[kSnapBatch];       // staged index of the element's tag
  int32_t rstart[kSnapBatch];     // first output byte in the batch
  int32_t len[kSnapBatch];        // output bytes (kSnapBatchBytes + 1 for longer literals)
  int32_t src[kSnapBatch];        // literal: staged index of its first byte; copy: -1
  int32_t flags[kSnapBatch];      // 1: malformed on its own, 2: short enough for a batch
  int32_t cut, bad;
};

struct SnapStage {
  const uint8_t* src;
  int64_t n;
  int64_t ib;  // stream index of in[0] (negative before a misaligned start)
  bool sized;  // size[] describes the staged bytes
};

__device__ __forceinline__ void copy16(uint8_t* dst, const uint8_t* src)
{
#ifdef __CUDA_ARCH__
  *reinterpret_cast<uint4*>(dst) = *reinterpret_cast<const uint4*>(src);
#else
  for (int k = 0; k < 16; ++k) dst[k] = src[k];
#endif
}

// One element's tag: t and the four bytes after it (x).
struct SnapElem {
  int hdr;      // tag bytes
  int64_t l;    // output bytes
  int64_t off;  // copy: offset
  bool literal;
};

__device__ __forceinline__ SnapElem snap_decode(uint32_t t, uint32_t x)
{
  SnapElem e{1, 0, 0, (t & 3) == 0};
  if (e.literal) {
    e.l = t >> 2;
    if (e.l >= 60) {
      const int nbytes = static_cast<int>(e.l) - 59;
      e.hdr += nbytes;
      e.l = nbytes == 4 ? x : (x & ((1u << (8 * nbytes)) - 1));
    }
    e.l += 1;
  } else if ((t & 3) == 1) {
    e.hdr = 2;
    e.l   = 4 + ((t >> 2) & 7);
    e.off = (static_cast<int64_t>(t >> 5) << 8) | (x & 0xff);
  } else {
    const bool two = (t & 3) == 2;
    e.hdr = two ? 3 : 5;
    e.l   = (t >> 2) + 1;
    e.off = two ? (x & 0xffff) : x;
  }
  return e;
}

// The tag at staged index r and the four bytes after it (r + 5 <= kSnapIn).
__device__ __forceinline__ SnapElem snap_at(const SnapShared& sh, int r)
{
  const uint8_t* q = sh.in + r;
  const uint32_t x = static_cast<uint32_t>(q[1]) | static_cast<uint32_t>(q[2]) << 8 |
                     static_cast<uint32_t>(q[3]) << 16 | static_cast<uint32_t>(q[4]) << 24;
  return snap_decode(q[0], x);
}

__device__ __forceinline__ void store_u32(uint8_t* p, uint32_t v)  // p 4-byte aligned
{
#ifdef __CUDA_ARCH__
  *reinterpret_cast<uint32_t*>(p) = v;
#else
  memcpy(p, &v, 4);
#endif
}

__device__ __forceinline__ uint32_t load_u32(const uint8_t* p)  // p 4-byte aligned
{
#ifdef __CUDA_ARCH__
  return *reinterpret_cast<const uint32_t*>(p);
#else
  uint32_t v;
  memcpy(&v, p, 4);
  return v;
#endif
}

// Input bytes of an element whose tag is t, followed by the bytes x (capped at 0xffff).
// Branch-free: every lane of the warp takes the same path.
__device__ __forceinline__ uint32_t snap_size(uint32_t t, uint32_t x)
{
  const uint32_t type = t & 3, L = t >> 2;
  const uint32_t copy = (0x05030200u >> (8 * type)) & 0xff;  // 2, 3, 5 bytes of tag
  const uint32_t nbytes = L >= 60 ? L - 59 : 1;               // extra length bytes (1..4)
  const uint32_t mask   = nbytes == 4 ? 0xffffffffu : (1u << (8 * nbytes)) - 1;
  const uint32_t big    = (x & mask) >= 0xfff0u ? 0xffffu : 2 + nbytes + (x & mask);  // 1 + nbytes + (len + 1)
  const uint32_t lit    = L < 60 ? L + 2 : big;
  return type != 0 ? copy : lit;
}

// size[] of the staged bytes: every position read as a tag, in parallel,
// four positions from two aligned words at a time.
__device__ void snap_sizes(SnapStage& st, SnapShared& sh)
{
  const int lane = threadIdx.x % kLanes;
#pragma unroll 2
  for (int w = lane; w < kSnapIn / 4; w += kLanes) {
    const uint32_t lo = load_u32(sh.in + 4 * w);
    const uint32_t hi = w + 1 < kSnapIn / 4 ? load_u32(sh.in + 4 * w + 4) : 0;
    const uint64_t v  = static_cast<uint64_t>(hi) << 32 | lo;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int r = 4 * w + k;
      const uint32_t t = static_cast<uint32_t>(v >> (8 * k)) & 0xff;
      const uint32_t x = static_cast<uint32_t>(v >> (8 * k + 8));
      sh.size[r] = static_cast<uint16_t>(r + 5 <= kSnapIn ? snap_size(t, x) : 0xffff);
    }
  }
  st.sized = true;
  __syncwarp();
}

constexpr int kSnapPer = kSnapIn / 16 / kLanes;  // staged 16-byte granules per lane
struct alignas(16) SnapGranule {
  uint8_t b[16];
};

// Loads the stage that starts at the 16-byte boundary at or below stream
// index i into registers (the bytes inside [0, n)); returns its first index.
__device__ int64_t snap_load(const SnapStage& st, int64_t i, SnapGranule (&reg)[kSnapPer])
{
  const int lane   = threadIdx.x % kLanes;
  const int64_t ib = i - static_cast<int64_t>(reinterpret_cast<uintptr_t>(st.src + i) & 15);
  for (int r = 0; r < kSnapPer; ++r) {
    const int64_t b = ib + 16 * (lane + r * kLanes);
    if (b >= 0 && b + 16 <= st.n) {
      copy16(reg[r].b, st.src + b);
    } else {
      for (int k = 0; k < 16; ++k) reg[r].b[k] = b + k >= 0 && b + k < st.n ? st.src[b + k] : 0;
    }
  }
  return ib;
}

// Makes the loaded stage the staged one: in[k] = src[ib + k].
__device__ void snap_commit(SnapStage& st, SnapShared& sh, int64_t ib, const SnapGranule (&reg)[kSnapPer])
{
  const int lane = threadIdx.x % kLanes;
  __syncwarp();  // every lane is done with the previous contents
  st.ib    = ib;
  st.sized = false;
  for (int r = 0; r < kSnapPer; ++r) copy16(sh.in + 16 * (lane + r * kLanes), reg[r].b);
  __syncwarp();
}

// Stages the stream from the 16-byte boundary at or below stream index i;
// with `sizes`, size[] too.
__device__ void snap_stage(SnapStage& st, SnapShared& sh, int64_t i, bool sizes)
{
  SnapGranule reg[kSnapPer];
  const int64_t ib = snap_load(st, i, reg);  // all loads first, then the stores
  snap_commit(st, sh, ib, reg);
  if (sizes) snap_sizes(st, sh);
}

// src[0, n) -> dst (at most cap bytes) by the calling warp; false when the
// stream is malformed.  The stream is a chain of elements (literals and
// back-references) whose boundaries are known only by parsing them in turn.
// Per batch of up to kSnapBatch short elements: the warp walks the chain
// through size[] (one shared load per element; the sizes of every staged
// position were tabulated in parallel), each lane decodes one element, and
// the batch's output bytes are produced all at once: byte r of the batch is
// a literal's input byte, or a back-reference's source byte -- at
// out[o - d + k % d] for byte k of a copy of offset d -- followed back
// through the batch until it reaches a literal or output written before the
// batch (ring or global).  Long literals are copied on their own.
__device__ bool snappy_warp(const uint8_t* src, int64_t n, uint8_t* dst, int64_t cap, int64_t& produced,
                            SnapShared& sh)
{
  const int lane = threadIdx.x % kLanes;
  SnapStage st{src, n, 0, false};
  snap_stage(st, sh, 0, false);
  int64_t i    = 0;
  uint64_t len = 0;
  for (int sh_ = 0;; sh_ += 7) {  // preamble: the uncompressed length as a varint
    if (i >= n || sh_ > 35) return false;
    const uint8_t b = sh.in[i++ - st.ib];
    len |= static_cast<uint64_t>(b & 0x7f) << sh_;
    if (!(b & 0x80)) break;
  }
  if (len > static_cast<uint64_t>(cap)) return false;
  const int64_t total = static_cast<int64_t>(len);
  constexpr int64_t kMask = kSnapWin - 1;
  int64_t o = 0;
  while (o < total) {
    if (i >= n) return false;
    if (i + 5 > st.ib + kSnapIn) snap_stage(st, sh, i, true);  // a tag and its extra bytes
    else if (!st.sized) snap_sizes(st, sh);
    // walk the chain (every lane the same)
    int nb = 0, r = static_cast<int>(i - st.ib);
    while (nb < kSnapBatch && st.ib + r < n && r + 5 <= kSnapIn) {
      if (lane == 0) sh.epos[nb] = r;
      ++nb;
      r += sh.size[r];
    }
    const int walk_end = r;
    if (lane == 0) {
      sh.cut = nb;
      sh.bad = kSnapBatch;
    }
    __syncwarp();
    // decode, one element per lane
    for (int j = lane; j < nb; j += kLanes) {
      const int er      = sh.epos[j];
      const SnapElem e  = snap_at(sh, er);
      const int64_t body = st.ib + er + e.hdr;  // stream index
      bool alone_bad = body > n;
      bool is_short  = true;
      if (e.literal) {
        alone_bad = alone_bad || body + e.l > n;
        is_short  = e.l <= kSnapShort && body + e.l <= st.ib + kSnapIn;
      } else {
        alone_bad = alone_bad || e.off == 0;
      }
      sh.len[j]   = static_cast<int32_t>(e.l > kSnapBatchBytes ? kSnapBatchBytes + 1 : e.l);
      sh.src[j]   = e.literal ? er + e.hdr : -1;
      sh.off[j]   = e.off;
      sh.flags[j] = (alone_bad ? 1 : 0) | (is_short ? 2 : 0);
    }
    __syncwarp();
    // output positions; the batch ends before the first element that is past
    // the end, long, or does not fit
    int cut, first_bad;
    if (kLanes == 32) {  // one element per lane: a shuffle scan and ballots
      const int lj = lane < nb ? sh.len[lane] : 0;
      int incl     = lj;
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= d) incl += u;
      }
      const int rs     = incl - lj;
      const int64_t at = o + rs;
      bool stop = false, bad = false;
      if (lane < nb) {
        sh.rstart[lane] = rs;
        const int fl    = sh.flags[lane];
        const bool end  = at >= total;
        stop            = end || !(fl & 2) || rs + lj > kSnapBatchBytes;
        bad             = !end && ((fl & 1) || at + lj > total || (sh.src[lane] < 0 && sh.off[lane] > at));
      }
      const unsigned sm = __ballot_sync(0xffffffffu, stop), bm = __ballot_sync(0xffffffffu, bad);
      cut       = sm ? __ffs(sm) - 1 : nb;
      first_bad = bm ? __ffs(bm) - 1 : kSnapBatch;
    } else {
      for (int j = lane; j < nb; j += kLanes) {
        int rs = 0;
        for (int k = 0; k < j; ++k) rs += sh.len[k];
        sh.rstart[j]     = rs;
        const int64_t at = o + rs;
        const int lj     = sh.len[j];
        const int fl     = sh.flags[j];
        const bool end   = at >= total;
        const bool stop  = end || !(fl & 2) || rs + lj > kSnapBatchBytes;
        const bool bad   = !end && ((fl & 1) || at + lj > total || (sh.src[j] < 0 && sh.off[j] > at));
        if (stop) atomicMin(&sh.cut, j);
        if (bad) atomicMin(&sh.bad, j);
      }
      __syncwarp();
      cut       = sh.cut;
      first_bad = sh.bad;
    }
    __syncwarp();
    if (first_bad < cut) return false;
    if (cut == 0) {  // a long literal (or one past the staged bytes), straight from the input
      const SnapElem e   = snap_at(sh, static_cast<int>(i - st.ib));
      const int64_t body = i + e.hdr;
      if (body > n || body + e.l > n || o + e.l > total) return false;
      // Copied a stage at a time with four-byte stores, the next stage's
      // loads in flight meanwhile; the ring keeps only the literal's last
      // kSnapWin bytes.
      const int64_t l         = e.l;
      const int64_t ring_from = l > kSnapWin ? l - kSnapWin : 0;
      int64_t from_i          = body;
      if (from_i >= st.ib + kSnapIn) snap_stage(st, sh, from_i, false);
      for (int64_t done = 0; done < l;) {
        const int64_t avail = st.ib + kSnapIn - from_i;
        const int64_t piece = l - done < avail ? l - done : avail;
        const bool more     = done + piece < l;
        SnapGranule reg[kSnapPer];
        int64_t next_ib = 0;
        if (more) next_ib = snap_load(st, from_i + piece, reg);
        const uint8_t* f = sh.in + (from_i - st.ib);
        uint8_t* to      = dst + o + done;
        int64_t head     = (4 - static_cast<int64_t>(reinterpret_cast<uintptr_t>(to) & 3)) & 3;
        if (head > piece) head = piece;
        for (int64_t k = lane; k < head; k += kLanes) to[k] = f[k];
        const int64_t words = (piece - head) >> 2;
#pragma unroll 4
        for (int64_t w = lane; w < words; w += kLanes) {
          const uint8_t* q = f + head + 4 * w;
          store_u32(to + head + 4 * w, static_cast<uint32_t>(q[0]) | static_cast<uint32_t>(q[1]) << 8 |
                                         static_cast<uint32_t>(q[2]) << 16 | static_cast<uint32_t>(q[3]) << 24);
        }
        for (int64_t k = head + 4 * words + lane; k < piece; k += kLanes) to[k] = f[k];
        for (int64_t k = (ring_from > done ? ring_from - done : 0) + lane; k < piece; k += kLanes)
          sh.win[(o + done + k) & kMask] = f[k];
        done += piece;
        from_i += piece;
        if (more) snap_commit(st, sh, next_ib, reg);
      }
      o += l;
      i = from_i;
      __syncwarp();
      continue;
    }
    const int B = sh.rstart[cut - 1] + sh.len[cut - 1];
    for (int j = lane; j < cut; j += kLanes) {
      const int r0 = sh.rstart[j], lj = sh.len[j];
      for (int k = 0; k < lj; ++k) sh.elem[r0 + k] = static_cast<uint8_t>(j);
    }
    __syncwarp();
    // The batch is written a window of kSnapPerLane * kLanes bytes at a time,
    // ring included, so a source inside the batch but before the window is
    // read from the ring and only sources inside the window are followed
    // back.  A batch writes ring slots of [o, o + B), B <= kSnapBatchBytes;
    // the slots of positions from o + kSnapBatchBytes - kSnapWin on are not
    // among them, so those are read from the ring and older ones from dst.
    for (int base = 0; base < B; base += kSnapPerLane * kLanes) {
      uint8_t bv[kSnapPerLane];
      int64_t nrq[kSnapPerLane];
      bool chase[kSnapPerLane];
#pragma unroll
      for (int q = 0; q < kSnapPerLane; ++q) {  // first hop of every byte, side by side
        const int rb = base + q * kLanes + lane;
        const int rr = rb < B ? rb : 0;
        const int e  = sh.elem[rr];
        const int r0 = sh.rstart[e];
        const int si = sh.src[e];
        const int64_t d = sh.off[e];
        int k = rr - r0;
        if (si < 0 && d < sh.len[e]) k %= static_cast<int>(d);  // an overlapping copy: d < len <= 64
        const int64_t nr = si >= 0 ? 0 : r0 - d + k;
        const bool far   = si < 0 && nr < base;
        const int64_t at = o + nr;
        bv[q]    = si >= 0 ? sh.in[si + k] : (far ? (nr >= kSnapBatchBytes - kSnapWin ? sh.win[at & kMask] : dst[at]) : 0);
        chase[q] = rb < B && si < 0 && !far;
        nrq[q]   = nr;
      }
#pragma unroll
      for (int q = 0; q < kSnapPerLane; ++q) {
        if (!chase[q]) continue;
        int64_t rr = nrq[q];  // a source inside this window: follow it back
        while (true) {
          const int e  = sh.elem[rr];
          const int r0 = sh.rstart[e];
          const int si = sh.src[e];
          if (si >= 0) {
            bv[q] = sh.in[si + (rr - r0)];
            break;
          }
          const int64_t d = sh.off[e];
          int64_t nr;
          if (d >= sh.len[e]) nr = rr - d;  // no overlap
          else nr = r0 - d + static_cast<int>(rr - r0) % static_cast<int>(d);  // d < len <= 64
          if (nr < base) {
            const int64_t at = o + nr;
            bv[q] = nr >= kSnapBatchBytes - kSnapWin ? sh.win[at & kMask] : dst[at];
            break;
          }
          rr = nr;
        }
      }
#pragma unroll
      for (int q = 0; q < kSnapPerLane; ++q) {
        const int rb = base + q * kLanes + lane;
        if (rb < B) {
          dst[o + rb]              = bv[q];
          sh.win[(o + rb) & kMask] = bv[q];
        }
      }
      __syncwarp();  // the next window may read these bytes from the ring
    }
    o += B;
    i = st.ib + (cut < nb ? sh.epos[cut] : walk_end);
    __syncwarp();  // the next batch reads these bytes and rewrites the descriptors
  }
  produced = o;
  return true;
}

// ---- 2. byte-array dictionary pages ---------------------------------------------------
constexpr int kDictStage = 8192;  // staged page bytes per round
struct alignas(16) DictStage {
  uint8_t b[kDictStage];
};

// ---- 3. RLE / bit-packed hybrid streams ----------------------------------------------
// Streaming state of one hybrid stream of `bw`-bit values in [pos, end).
struct RleStream {
  const uint8_t* p;
  int64_t pos, end;
  int bw;
  uint32_t left;    // values left in the current run
  bool packed;
  uint32_t value;   // RLE run value
  int64_t bitpos;   // bit-packed run: bit offset (from p) of its next value
  bool bad;
};

// One run segment of a tile: values [start, start + count) of the tile.
struct RleSeg {
  uint32_t start, count;
  uint32_t value;   // RLE
  uint32_t packed;
  int64_t bitpos;   // bit-packed: bit offset of the segment's first value
};

__device__ __forceinline__ uint32_t read_bits(const uint8_t* p, int64_t end, int64_t bitpos, int bw)
{
  const int64_t b0 = bitpos >> 3;
  uint64_t w       = 0;
#pragma unroll
  for (int k = 0; k < 5; ++k)
    if (b0 + k < end) w |= static_cast<uint64_t>(p[b0 + k]) << (8 * k);
  w >>= bitpos & 7;
  return static_cast<uint32_t>(bw == 32 ? w : (w & ((1ull << bw) - 1)));
}

// Thread 0: cut the next n values of the stream into segments (at most n).
// Values past a stream's end read as 0 and mark it bad.
__device__ int rle_cut(RleStream& s, uint32_t n, RleSeg* seg)
{
  uint32_t got = 0;
  int ns       = 0;
  while (got < n) {
    if (s.left == 0) {
      uint64_t h = 0;
      int sh     = 0;
      while (true) {
        if (s.pos >= s.end || sh > 35) {
          s.bad = true;
          break;
        }
        const uint8_t b = s.p[s.pos++];
        h |= static_cast<uint64_t>(b & 0x7f) << sh;
        if (!(b & 0x80)) break;
        sh += 7;
      }
      if (s.bad) {  // fill the rest with zeros
        seg[ns++] = RleSeg{got, n - got, 0, 0, 0};
        return ns;
      }
      if (h & 1) {
        const uint64_t groups = h >> 1;
        s.packed              = true;
        s.left                = static_cast<uint32_t>(groups * 8 < (1ull << 31) ? groups * 8 : (1ull << 31));
        s.bitpos              = s.pos * 8;
        s.pos += static_cast<int64_t>(groups) * s.bw;
        if (s.pos > s.end) s.bad = true;  // values past the end read as 0
      } else {
        const int nb = (s.bw + 7) / 8;
        s.packed     = false;
        s.left       = static_cast<uint32_t>(h >> 1 < (1ull << 31) ? h >> 1 : (1ull << 31));
        s.value      = s.pos + nb <= s.end ? le_bytes(s.p + s.pos, nb) : 0;
        if (s.pos + nb > s.end) s.bad = true;
        s.pos += nb;
      }
      continue;
    }
    const uint32_t take = s.left < n - got ? s.left : n - got;
    seg[ns++]           = RleSeg{got, take, s.value, s.packed ? 1u : 0u, s.bitpos};
    got += take;
    s.left -= take;
    if (s.packed) s.bitpos += static_cast<int64_t>(take) * s.bw;
  }
  return ns;
}

// Value i of a tile cut into segs[0, ns).
__device__ __forceinline__ uint32_t rle_value(const RleStream& s, const RleSeg* seg, int ns, uint32_t i)
{
  int lo = 0, hi = ns - 1;
  while (lo < hi) {  // last segment with start <= i
    const int mid = (lo + hi + 1) >> 1;
    if (seg[mid].start <= i) lo = mid;
    else hi = mid - 1;
  }
  const RleSeg& g = seg[lo];
  if (!g.packed) return g.value;
  return read_bits(s.p, s.end, g.bitpos + static_cast<int64_t>(i - g.start) * s.bw, s.bw);
}

// ---- kernels ------------------------------------------------------------------------
// Compressed pages, one warp each: payload -> scratch (a v2 page's levels are
// stored uncompressed in front of its values and copied as they are).
__global__ void __launch_bounds__(kLanes) pq_snappy_kernel(const uint8_t* file, PqPage* pages, const int* list,
                                                          int nlist, uint8_t* scratch, const int64_t* soff,
                                                          unsigned long long* err)
{
  __shared__ SnapShared sm;
  const int w = blockIdx.x;
  if (w >= nlist) return;
  const int p           = list[w];
  const PqPage& pg      = pages[p];
  const int64_t lv      = pg.h.kind == LDF_PQ_DATA_V2 ? pg.h.levels_bytes : 0;
  const uint8_t* src    = file + pg.h.offset;
  uint8_t* dst          = scratch + soff[w];
  const int lane        = threadIdx.x % kLanes;
  for (int64_t k = lane; k < lv; k += kLanes) dst[k] = src[k];
  int64_t got = 0;
  const bool ok = snappy_warp(src + lv, pg.h.compressed - lv, dst + lv, pg.h.uncompressed - lv, got, sm);
  if (lane == 0 && (!ok || got != pg.h.uncompressed - lv)) pq_error(err, p, kPqErrSnappy);
}

// Byte-array dictionary pages, one block each: the entry table (offset in
// the page's data, length) of every value.  The page is staged kDictStage
// bytes at a time by the block and thread 0 walks the length prefixes.
__global__ void __launch_bounds__(kPqThreads) pq_dict_strings_kernel(const PqPage* pages, const int* list,
                                                                     int nlist, int64_t* entry_off,
                                                                     int32_t* entry_len, unsigned long long* err)
{
  __shared__ DictStage stage;
  __shared__ int64_t s_pos;
  __shared__ int s_v;
  for (int q = blockIdx.x; q < nlist; q += gridDim.x) {
    const int p         = list[q];
    const PqPage& pg    = pages[p];
    const uint8_t* data = pg.data;
    const int64_t bytes = pg.data_bytes;
    const int nv        = pg.h.num_values;
    int64_t pos         = 0;
    int v               = 0;
    uint8_t* buf        = stage.b;
    while (v < nv) {
      const int64_t base = pos - static_cast<int64_t>(reinterpret_cast<uintptr_t>(data + pos) & 15);
      for (int g = threadIdx.x; g < kDictStage / 16; g += blockDim.x) {
        const int64_t b = base + 16 * g;
        if (b >= 0 && b + 16 <= bytes) {
          copy16(buf + 16 * g, data + b);
        } else {
          for (int k = 0; k < 16; ++k)
            if (b + k >= 0 && b + k < bytes) buf[16 * g + k] = data[b + k];
        }
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        while (v < nv) {
          int64_t len = -1;
          if (pos + 4 <= bytes) {
            if (pos + 4 > base + kDictStage) break;  // the next prefix is past the staged bytes
            len = le_bytes(buf + (pos - base), 4);
          }
          if (len < 0 || pos + 4 + len > bytes) {
            pq_error(err, p, kPqErrValues);
            len = 0;
            pos = bytes;
          } else {
            pos += 4;
          }
          entry_off[pg.dict_entry0 + v] = pos;
          entry_len[pg.dict_entry0 + v] = static_cast<int32_t>(len);
          pos += len;
          ++v;
        }
        s_pos = pos;
        s_v   = v;
      }
      __syncthreads();
      pos = s_pos;
      v   = s_v;
      __syncthreads();  // s_pos / s_v and buf are rewritten next round
    }
  }
}

// ---- large byte-array Snappy pages: the element chain ranked in parallel ----------
// A Snappy page of a byte-array column can hold hundreds of thousands of short
// elements (a 1 MB dictionary page of short strings about 60,000), which one
// warp parses in turn.  Such pages are decoded by the whole GPU instead:
//  1. every position of the stream gets the position of the element that would
//     follow a tag there (nxt), and doubling gives the position kChainStep
//     elements on;
//  2. one thread per page lays checkpoints kChainStep elements apart through the
//     doubled table, one thread per checkpoint walks its kChainStep elements;
//  3. every element is decoded on its own; a scan of the output lengths gives
//     its output position;
//  4. every output byte points at its source: a literal's input byte, or for
//     byte k of a copy of offset d the output byte o - d + k % d; pointer
//     jumping (log2 of the page size rounds) takes every byte to a literal
//     input byte, which is then copied.
constexpr int64_t kChainMinBytes = 131072;  // Snappy pages from this many output bytes
constexpr int64_t kDictChainMinBytes = 16384;  // dictionary pages from this many data bytes
constexpr int kChainLog          = 8;
constexpr int kChainStep         = 1 << kChainLog;  // elements between checkpoints
constexpr int64_t kChainMaxInput = int64_t(32) << 20;  // bytes per call and kind (pages beyond: the per-page kernels)

struct ChainPage {
  int page;           // index in the page table
  int64_t file_off;   // file offset of the Snappy stream (behind a v2 page's levels)
  int64_t n;          // compressed stream bytes
  int64_t lv;         // v2 levels in front of the stream (copied as they are)
  int64_t u;          // stream output bytes
  int64_t elem_cap;   // element slots (every element takes 2 input bytes or more)
  int64_t ck_cap;     // checkpoint slots
};
struct ChainState {
  int64_t start;  // first tag (behind the length preamble); -1 when the preamble is bad
  int64_t nck;    // checkpoints laid
  int64_t nelem;  // elements (set by the walk that reaches the stream's end)
};
struct ChainBases {  // the flattened index spaces: first index of each page
  const int64_t* in;    // stream positions
  const int64_t* out;   // output bytes (the page's scratch offset; levels included)
  const int64_t* elem;  // element slots
  const int64_t* ck;    // checkpoint slots
  int n;                // chain pages
};

// Last page q with bases[q] <= g.
__device__ __forceinline__ int chain_page_of(const int64_t* bases, int n, int64_t g)
{
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (bases[mid] <= g) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Input bytes of the element whose tag is at b[x] (x < n), or -1 when its
// extra length bytes run past n.
__device__ __forceinline__ int64_t chain_elem_size(const uint8_t* b, int64_t x, int64_t n)
{
  const uint32_t t = b[x];
  if ((t & 3) != 0) return (t & 3) == 1 ? 2 : ((t & 3) == 2 ? 3 : 5);
  const uint32_t L = t >> 2;
  if (L < 60) return L + 2;
  const int nb = static_cast<int>(L) - 59;
  if (x + 1 + nb > n) return -1;
  uint64_t len = 0;
  for (int k = 0; k < nb; ++k) len |= static_cast<uint64_t>(b[x + 1 + k]) << (8 * k);
  return 1 + nb + static_cast<int64_t>(len) + 1;
}

__global__ void chain_start_kernel(const uint8_t* file, const ChainPage* cp, ChainState* st, int npages,
                                   unsigned long long* err)
{
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < npages; q += gridDim.x * blockDim.x) {
    const ChainPage& c = cp[q];
    const uint8_t* b   = file + c.file_off;
    int64_t i = 0, start = -1;
    uint64_t len = 0;
    for (int sh = 0; sh <= 35; sh += 7) {
      if (i >= c.n) break;
      const uint8_t v = b[i++];
      len |= static_cast<uint64_t>(v & 0x7f) << sh;
      if (!(v & 0x80)) {
        start = i;
        break;
      }
    }
    if (start < 0 || len != static_cast<uint64_t>(c.u)) {
      start = -1;
      pq_error(err, c.page, kPqErrSnappy);
    }
    st[q] = ChainState{start, 0, 0};
  }
}

__global__ void chain_next_kernel(const uint8_t* file, const ChainPage* cp, const ChainState* st, ChainBases B,
                                  int64_t total, int64_t* nxt)
{
  for (int64_t g = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; g < total;
       g += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int q        = chain_page_of(B.in, B.n, g);
    const ChainPage& c = cp[q];
    const int64_t x    = g - B.in[q];
    int64_t v          = -1;
    if (st[q].start >= 0 && x >= st[q].start && x < c.n) {
      const int64_t sz = chain_elem_size(file + c.file_off, x, c.n);
      if (sz > 0 && x + sz < c.n) v = B.in[q] + x + sz;
    }
    nxt[g] = v;
  }
}

__global__ void chain_double_kernel(const int64_t* in, int64_t* out, int64_t total)
{
  for (int64_t g = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; g < total;
       g += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t v = in[g];
    out[g]          = v < 0 ? -1 : in[v];
  }
}

// One thread per page: checkpoints kChainStep elements apart.
__global__ void chain_checkpoints_kernel(const ChainPage* cp, ChainState* st, ChainBases B, const int64_t* jump,
                                         int64_t* ck)
{
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < B.n; q += gridDim.x * blockDim.x) {
    int64_t c = st[q].start >= 0 ? B.in[q] + st[q].start : -1;
    int64_t j = 0;
    while (c >= 0 && j < cp[q].ck_cap) {
      ck[B.ck[q] + j++] = c;
      c = jump[c];
    }
    st[q].nck = j;
  }
}

// One thread per checkpoint: the element positions of its kChainStep elements.
__global__ void chain_walk_kernel(const uint8_t* file, const ChainPage* cp, ChainState* st, ChainBases B,
                                  int64_t total_ck, const int64_t* ck, int64_t* epos, unsigned long long* err)
{
  for (int64_t g = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; g < total_ck;
       g += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int q        = chain_page_of(B.ck, B.n, g);
    const int64_t j    = g - B.ck[q];
    if (j >= st[q].nck) continue;
    const ChainPage& c = cp[q];
    const uint8_t* b   = file + c.file_off;
    int64_t x          = ck[g] - B.in[q];
    for (int t = 0; t < kChainStep; ++t) {
      const int64_t k = j * kChainStep + t;
      if (k >= c.elem_cap) {
        pq_error(err, c.page, kPqErrSnappy);
        break;
      }
      epos[B.elem[q] + k] = x;
      const int64_t sz    = chain_elem_size(b, x, c.n);
      if (sz < 0 || x + sz > c.n) {
        pq_error(err, c.page, kPqErrSnappy);
        break;
      }
      x += sz;
      if (x == c.n) {
        st[q].nelem = k + 1;
        break;
      }
    }
  }
}

// Every element slot: output length and (copy) offset or (literal) -(body + 1).
__global__ void chain_decode_kernel(const uint8_t* file, const ChainPage* cp, const ChainState* st, ChainBases B,
                                    int64_t total_elem, const int64_t* epos, int64_t* elen, int64_t* emeta)
{
  for (int64_t g = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; g < total_elem;
       g += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int q     = chain_page_of(B.elem, B.n, g);
    const int64_t k = g - B.elem[q];
    if (k >= st[q].nelem) {
      elen[g]  = 0;
      emeta[g] = 0;
      continue;
    }
    const ChainPage& c = cp[q];
    const uint8_t* b   = file + c.file_off;
    const int64_t x    = epos[g];
    const uint32_t t   = b[x];
    int64_t l, meta;
    if ((t & 3) == 0) {
      l       = t >> 2;
      int hdr = 1;
      if (l >= 60) {
        const int nb = static_cast<int>(l) - 59;
        l            = 0;
        for (int i = 0; i < nb; ++i) l |= static_cast<int64_t>(b[x + 1 + i]) << (8 * i);
        hdr += nb;
      }
      l += 1;
      meta = -(x + hdr) - 1;
    } else if ((t & 3) == 1) {
      l    = 4 + ((t >> 2) & 7);
      meta = (static_cast<int64_t>(t >> 5) << 8) | b[x + 1];
    } else {
      l    = (t >> 2) + 1;
      meta = (t & 3) == 2 ? (b[x + 1] | b[x + 2] << 8)
                          : static_cast<int64_t>(static_cast<uint32_t>(b[x + 1]) | static_cast<uint32_t>(b[x + 2]) << 8 |
                                                 static_cast<uint32_t>(b[x + 3]) << 16 |
                                                 static_cast<uint32_t>(b[x + 4]) << 24);
    }
    elen[g]  = l;
    emeta[g] = meta;
  }
}

// Every output byte: its source, another output byte (>= 0, scratch index) or
// a file byte (-(offset + 1)).
__global__ void chain_ptr_kernel(const ChainPage* cp, const ChainState* st, ChainBases B, int64_t total_out,
                                 const int64_t* eoff, const int64_t* elen, const int64_t* emeta, int64_t* ptr,
                                 unsigned long long* err)
{
  for (int64_t g = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; g < total_out;
       g += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int q        = chain_page_of(B.out, B.n, g);
    const ChainPage& c = cp[q];
    const int64_t r    = g - B.out[q];
    if (r >= c.lv + c.u) {  // alignment padding behind the page
      ptr[g] = -1;
      continue;
    }
    if (r < c.lv) {  // a v2 page's levels, stored uncompressed
      ptr[g] = -(c.file_off - c.lv + r) - 1;
      continue;
    }
    const int64_t s  = r - c.lv;
    const int64_t e0 = B.elem[q], ne = st[q].nelem;
    if (ne <= 0) {
      ptr[g] = -1;
      pq_error(err, c.page, kPqErrSnappy);
      continue;
    }
    const int64_t base = eoff[e0];
    int64_t lo = 0, hi = ne - 1;  // last element starting at or before s
    while (lo < hi) {
      const int64_t mid = (lo + hi + 1) >> 1;
      if (eoff[e0 + mid] - base <= s) lo = mid;
      else hi = mid - 1;
    }
    const int64_t o = eoff[e0 + lo] - base, l = elen[e0 + lo], m = emeta[e0 + lo];
    if (s >= o + l || (s == o && o + l > c.u) || (m >= 0 && (m == 0 || m > o))) {
      ptr[g] = -1;
      pq_error(err, c.page, kPqErrSnappy);
      continue;
    }
    if (m < 0) {
      ptr[g] = -(c.file_off + (-m - 1) + (s - o)) - 1;
    } else {
      const int64_t src = m >= l ? s - m : o - m + (s - o) % m;
      ptr[g]            = B.out[q] + c.lv + src;
    }
  }
}

__global__ void chain_jump_kernel(const int64_t* in, int64_t* out, int64_t total)
{
  for (int64_t g = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; g < total;
       g += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t p = in[g];
    out[g]          = p >= 0 ? in[p] : p;
  }
}

__global__ void chain_final_kernel(const uint8_t* file, const ChainPage* cp, ChainBases B, const int64_t* ptr,
                                   int64_t total, uint8_t* scratch, unsigned long long* err)
{
  for (int64_t g = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; g < total;
       g += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t p = ptr[g];
    if (p < 0) {
      scratch[g] = file[-p - 1];
    } else {
      scratch[g] = 0;
      pq_error(err, cp[chain_page_of(B.out, B.n, g)].page, kPqErrSnappy);
    }
  }
}

// Byte-array dictionary pages from kDictChainMinBytes: the chain of length
// prefixes ranked the same way (next entry at x + 4 + length), each
// checkpoint's thread writing its entries.
struct DictChain {
  int page;
  const uint8_t* data;  // the page's data (decompressed)
  int64_t n;            // data bytes
  int64_t nv;           // entries
  int64_t entry0;       // first entry in the entry table
  int64_t ck_cap;
};

__device__ __forceinline__ int64_t dict_len_at(const uint8_t* d, int64_t x)
{
  return static_cast<int64_t>(static_cast<uint32_t>(d[x]) | static_cast<uint32_t>(d[x + 1]) << 8 |
                              static_cast<uint32_t>(d[x + 2]) << 16 | static_cast<uint32_t>(d[x + 3]) << 24);
}

__global__ void dict_next_kernel(const DictChain* dc, ChainBases B, int64_t total, int64_t* nxt)
{
  for (int64_t g = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; g < total;
       g += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int q        = chain_page_of(B.in, B.n, g);
    const DictChain& c = dc[q];
    const int64_t x    = g - B.in[q];
    int64_t v          = -1;
    if (x + 4 <= c.n) {
      const int64_t e = x + 4 + dict_len_at(c.data, x);
      if (e < c.n) v = B.in[q] + e;
    }
    nxt[g] = v;
  }
}

__global__ void dict_checkpoints_kernel(const DictChain* dc, ChainBases B, const int64_t* jump, int64_t* ck,
                                        int64_t* nck)
{
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < B.n; q += gridDim.x * blockDim.x) {
    const DictChain& c = dc[q];
    int64_t x          = c.n > 0 ? B.in[q] : -1;
    int64_t j          = 0;
    while (x >= 0 && j < c.ck_cap && j * kChainStep < c.nv) {
      ck[B.ck[q] + j++] = x;
      x = jump[x];
    }
    nck[q] = j;
  }
}

__global__ void dict_walk_kernel(const DictChain* dc, ChainBases B, int64_t total_ck, const int64_t* ck,
                                 const int64_t* nck, int64_t* entry_off, int32_t* entry_len, unsigned long long* err)
{
  for (int64_t g = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; g < total_ck;
       g += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int q     = chain_page_of(B.ck, B.n, g);
    const int64_t j = g - B.ck[q];
    const DictChain& c = dc[q];
    if (j == 0 && nck[q] == 0 && c.nv > 0) pq_error(err, c.page, kPqErrValues);
    if (j >= nck[q]) continue;
    int64_t x = ck[g] - B.in[q];
    for (int t = 0; t < kChainStep; ++t) {
      const int64_t k = j * kChainStep + t;
      if (k >= c.nv) break;
      const int64_t len = x + 4 <= c.n ? dict_len_at(c.data, x) : -1;
      if (len < 0 || x + 4 + len > c.n) {
        pq_error(err, c.page, kPqErrValues);
        break;
      }
      entry_off[c.entry0 + k] = x + 4;
      entry_len[c.entry0 + k] = static_cast<int32_t>(len);
      x += 4 + len;
    }
  }
}

struct PqColumns {
  int ncols;
  int32_t physical[64];
  int32_t width[64];                // output bytes per value (strings: 16)
  int32_t nullable[64];
  void* data[64];
  uint8_t* valid[64];
  const uint8_t** str_src[64];      // strings: source of each row's bytes
  int64_t* str_len[64];             // strings: length (0 for null)
};

__device__ __forceinline__ void store_value(void* dst, int width, int64_t row, uint64_t v)
{
  switch (width) {
    case 1: static_cast<uint8_t*>(dst)[row] = static_cast<uint8_t>(v); break;
    case 2: static_cast<uint16_t*>(dst)[row] = static_cast<uint16_t>(v); break;
    case 4: static_cast<uint32_t*>(dst)[row] = static_cast<uint32_t>(v); break;
    default: static_cast<unsigned long long*>(dst)[row] = v; break;
  }
}

// PLAIN value v of a fixed-width physical type (bit v for booleans).
__device__ __forceinline__ uint64_t plain_value(const uint8_t* vals, int physical, int64_t v)
{
  switch (physical) {
    case LDF_PQ_BOOLEAN: return (vals[v >> 3] >> (v & 7)) & 1u;
    case LDF_PQ_INT32:
    case LDF_PQ_FLOAT: return le_bytes(vals + 4 * v, 4);
    default: return static_cast<uint64_t>(le_bytes(vals + 8 * v, 4)) | (static_cast<uint64_t>(le_bytes(vals + 8 * v + 4, 4)) << 32);
  }
}

__device__ __forceinline__ int plain_bits(int physical)
{
  return physical == LDF_PQ_BOOLEAN ? 1 : (physical == LDF_PQ_INT32 || physical == LDF_PQ_FLOAT ? 32 : 64);
}

// One block per data page, kPqTile rows per round (kPqRows per thread).
constexpr int kPqRows = kPqTile / kPqThreads;
__global__ void __launch_bounds__(kPqThreads) pq_data_kernel(const PqPage* pages, const int* list, PqColumns C,
                                                             const int64_t* entry_off, const int32_t* entry_len,
                                                             unsigned long long* err)
{
  __shared__ RleSeg seg[kPqTile];
  __shared__ uint8_t lev[kPqTile];
  __shared__ uint32_t idx[kPqTile];
  __shared__ int64_t str_off[kPqTile];
  __shared__ int32_t str_len[kPqTile];
  __shared__ RleStream def, ids;
  __shared__ int nseg;
  __shared__ int64_t walk;  // byte-array values: next value's offset in the value bytes
  __shared__ int bad;
  __shared__ int64_t s_scan[kPqThreads / kLanes + 1];

  const int p       = list[blockIdx.x];
  const PqPage& pg  = pages[p];
  const int col     = pg.h.column;
  const int phys    = C.physical[col];
  const bool nulls  = C.nullable[col] != 0;
  const bool dict   = pg.h.encoding == 2 || pg.h.encoding == 8;
  const bool rle    = pg.h.encoding == 3;  // RLE booleans (v2 pages): 4-byte length, then a 1-bit hybrid stream
  const bool strs   = phys == LDF_PQ_BYTE_ARRAY;
  const uint8_t* d  = pg.data;
  const int64_t nb  = pg.data_bytes;
  // the value stream, after the definition levels
  int64_t lv_off = 0, lv_len = 0, v_off = 0;
  if (pg.h.kind == LDF_PQ_DATA_V2) {
    lv_len = pg.h.levels_bytes;
    v_off  = lv_len;
  } else if (nulls) {
    lv_off = 4;
    lv_len = nb >= 4 ? le_bytes(d, 4) : 0;
    v_off  = 4 + lv_len;
  }
  const uint8_t* vals  = d + v_off;
  const int64_t vbytes = nb - v_off;
  if (threadIdx.x == 0) {
    bad  = (v_off > nb || lv_off + lv_len > nb) ? 1 : 0;
    def  = RleStream{d + lv_off, 0, bad ? 0 : lv_len, 1, 0, false, 0, 0, false};
    if (rle) {
      const int64_t len = vbytes >= 4 ? le_bytes(vals, 4) : -1;
      if (len < 0 || 4 + len > vbytes) bad = 1;
      ids = RleStream{vals + 4, 0, bad ? 0 : len, 1, 0, false, 0, 0, false};
    } else {
      const int bw = dict && vbytes >= 1 ? vals[0] : 0;
      if (dict && (vbytes < 1 || bw > 32)) bad = 1;
      ids = RleStream{vals + 1, 0, dict && vbytes >= 1 ? vbytes - 1 : 0, bw, 0, false, 0, 0, false};
    }
    walk = 0;
  }
  __syncthreads();
  if (bad) {
    if (threadIdx.x == 0) pq_error(err, p, kPqErrStream);
    return;
  }
  const PqPage* dp       = dict && pg.h.dict >= 0 ? &pages[pg.h.dict] : nullptr;
  const int64_t ndict    = dp ? dp->h.num_values : 0;
  const int width        = C.width[col];
  const int pbits        = plain_bits(phys);
  int64_t vbase          = 0;  // values (non-null rows) before the tile
  for (int64_t t0 = 0; t0 < pg.h.num_values; t0 += kPqTile) {
    const uint32_t n = static_cast<uint32_t>(pg.h.num_values - t0 < kPqTile ? pg.h.num_values - t0 : kPqTile);
    // definition levels
    if (nulls) {
      if (threadIdx.x == 0) nseg = rle_cut(def, n, seg);
      __syncthreads();
      for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) lev[i] = rle_value(def, seg, nseg, i) != 0 ? 1 : 0;
    } else {
      for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) lev[i] = 1;
    }
    __syncthreads();
    // value index of each row: kPqRows consecutive rows per thread
    const uint32_t r0 = threadIdx.x * kPqRows;
    int64_t mine = 0;
#pragma unroll
    for (int k = 0; k < kPqRows; ++k) mine += (r0 + k < n) ? lev[r0 + k] : 0;
    int64_t tile_valid;
    const int64_t before = block_exclusive_scan<int64_t, kPqThreads>(mine, s_scan, &tile_valid);
    // dictionary indices / byte-array offsets of the tile's values
    if (dict || rle) {
      if (threadIdx.x == 0) nseg = rle_cut(ids, static_cast<uint32_t>(tile_valid), seg);
      __syncthreads();
      for (uint32_t k = threadIdx.x; k < tile_valid; k += blockDim.x) idx[k] = rle_value(ids, seg, nseg, k);
    } else if (strs && threadIdx.x == 0) {
      int64_t pos = walk;
      for (int64_t k = 0; k < tile_valid; ++k) {
        int64_t len = -1;
        if (pos + 4 <= vbytes) len = le_bytes(vals + pos, 4);
        if (len < 0 || pos + 4 + len > vbytes) {
          pq_error(err, p, kPqErrValues);
          str_off[k] = 0;
          str_len[k] = 0;
          pos        = vbytes;
          continue;
        }
        str_off[k] = pos + 4;
        str_len[k] = static_cast<int32_t>(len);
        pos += 4 + len;
      }
      walk = pos;
    }
    __syncthreads();
    if (threadIdx.x == 0 && (def.bad || ids.bad)) pq_error(err, p, kPqErrStream);
    // outputs
    int64_t k = before;  // value index (in the tile) of the thread's next valid row
#pragma unroll 1
    for (int q = 0; q < kPqRows; ++q) {
      const uint32_t i = r0 + q;
      if (i >= n) break;
      const int64_t row = pg.h.row0 + t0 + i;
      if (C.valid[col]) C.valid[col][row] = lev[i];
      if (!lev[i]) {
        if (strs) {
          C.str_src[col][row] = nullptr;
          C.str_len[col][row] = 0;
        } else {
          store_value(C.data[col], width, row, 0);
        }
        continue;
      }
      if (strs) {
        const uint8_t* src = nullptr;
        int64_t len        = 0;
        if (dict) {
          const uint32_t e = idx[k];
          if (e < ndict) {
            src = dp->data + entry_off[dp->dict_entry0 + e];
            len = entry_len[dp->dict_entry0 + e];
          } else {
            pq_error(err, p, kPqErrDictIndex);
          }
        } else {
          src = vals + str_off[k];
          len = str_len[k];
        }
        C.str_src[col][row] = src;
        C.str_len[col][row] = len;
      } else {
        uint64_t v = 0;
        if (rle) {
          v = idx[k];
        } else if (dict) {
          const uint32_t e = idx[k];
          if (e < ndict && (static_cast<int64_t>(e) + 1) * pbits <= dp->data_bytes * 8) v = plain_value(dp->data, phys, e);
          else pq_error(err, p, kPqErrDictIndex);
        } else {
          const int64_t v_ix = vbase + k;
          if ((v_ix + 1) * pbits <= vbytes * 8) v = plain_value(vals, phys, v_ix);
          else pq_error(err, p, kPqErrValues);
        }
        store_value(C.data[col], width, row, v);
      }
      ++k;
    }
    vbase += tile_valid;
    __syncthreads();
  }
}

// Characters of one string column: row i's bytes at offs[i], local ranges.
// A block takes kPqStrRows rows a thread; every thread reads its strings
// eight bytes at a time with the loads in flight together into a shared
// stage laid out at the output's 16-byte phase, and the block writes the
// stage with 16-byte stores (the range's two end chunks, shared with the
// neighbouring tiles, byte by byte).  A tile whose characters exceed the
// stage writes them directly.
constexpr int kPqStrRows  = 2;
constexpr int kPqStrStage = 16 * 1024;
struct alignas(16) PqStrStage {
  uint8_t b[kPqStrStage];
};

__global__ void __launch_bounds__(256) pq_copy_strings_kernel(const uint8_t* const* src, const int64_t* len,
                                                              const int64_t* offs, int64_t rows, int64_t nchars,
                                                              uint8_t* chars, ldf_range* ranges)
{
  __shared__ PqStrStage stage;
  const int64_t per_tile = static_cast<int64_t>(blockDim.x) * kPqStrRows;
  for (int64_t tile = blockIdx.x; tile * per_tile < rows; tile += gridDim.x) {
    const int64_t i0 = tile * per_tile;
    const int64_t lo = offs[i0];
    const int64_t hi = i0 + per_tile < rows ? offs[i0 + per_tile] : nchars;
    // stage.b[k] <-> chars[abase + k], with chars + abase 16-byte aligned
    const int64_t abase = lo - static_cast<int64_t>(reinterpret_cast<uintptr_t>(chars + lo) & 15);
    const bool staged   = hi - abase <= kPqStrStage;
    for (int j = 0; j < kPqStrRows; ++j) {
      const int64_t i = i0 + j * blockDim.x + threadIdx.x;
      if (i >= rows) continue;
      const int64_t o = offs[i], n = len[i];
      ranges[i]        = ldf_range{o, o + n - 1};
      const uint8_t* s = src[i];
      uint8_t* q       = staged ? stage.b + (o - abase) : chars + o;
      for (int64_t k = 0; k < n; k += 8) {
        uint8_t b[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) b[u] = k + u < n ? s[k + u] : 0;
#pragma unroll
        for (int u = 0; u < 8; ++u)
          if (k + u < n) q[k + u] = b[u];
      }
    }
    if (staged) {
      __syncthreads();
      const int64_t nchunks = (hi - abase + 15) >> 4;  // chunk c: chars [abase + 16c, abase + 16c + 16)
      for (int64_t c = threadIdx.x; c < nchunks; c += blockDim.x) {
        const int64_t a0 = abase + 16 * c;
        if (a0 >= lo && a0 + 16 <= hi) {
          copy16(chars + a0, stage.b + 16 * c);
        } else {
          for (int k = 0; k < 16; ++k)
            if (a0 + k >= lo && a0 + k < hi) chars[a0 + k] = stage.b[16 * c + k];
        }
      }
      __syncthreads();
    }
  }
}

unsigned pq_blocks(int64_t work, int threads)
{
  const int64_t b   = ceil_div(work, threads);
  const int64_t cap = static_cast<int64_t>(num_sms()) * 16;
  return static_cast<unsigned>(b < 1 ? 1 : (b > cap ? cap : b));
}

}  // namespace

void parquet_decode(const uint8_t* file, int64_t file_bytes, const ldf_parquet_page* pages, int npages,
                    const int32_t* physical, const int32_t* types, const int32_t* nullable, int ncols, int64_t nrows,
                    ldf_column* out, const OpContext& ctx)
{
  LDF_REQUIRE(ncols >= 1 && ncols <= 64, "parquet_decode: between 1 and 64 columns");
  LDF_REQUIRE(npages >= 0 && (npages == 0 || pages != nullptr), "parquet_decode: no pages");
  LDF_REQUIRE(nrows >= 0 && file_bytes >= 0 && (file_bytes == 0 || file != nullptr), "parquet_decode: no file");
  PqColumns C{};
  C.ncols = ncols;
  for (int j = 0; j < ncols; ++j) {
    const int ph = physical[j], t = types[j];
    LDF_REQUIRE(ph == LDF_PQ_BOOLEAN || ph == LDF_PQ_INT32 || ph == LDF_PQ_INT64 || ph == LDF_PQ_FLOAT ||
                  ph == LDF_PQ_DOUBLE || ph == LDF_PQ_BYTE_ARRAY,
                "parquet_decode: unsupported physical type");
    const bool ok = (ph == LDF_PQ_BOOLEAN && t == LDF_BOOL8) || (ph == LDF_PQ_BYTE_ARRAY && t == LDF_STRING) ||
                    (ph == LDF_PQ_FLOAT && t == LDF_FLOAT32) || (ph == LDF_PQ_DOUBLE && t == LDF_FLOAT64) ||
                    (ph == LDF_PQ_INT32 && (t == LDF_INT8 || t == LDF_INT16 || t == LDF_INT32 || t == LDF_UINT8 ||
                                            t == LDF_UINT16 || t == LDF_UINT32)) ||
                    (ph == LDF_PQ_INT64 && (t == LDF_INT64 || t == LDF_UINT64 || t == LDF_TIMESTAMP_US));
    LDF_REQUIRE(ok, "parquet_decode: output type does not match the physical type");
    C.physical[j] = ph;
    C.width[j]    = type_width(t);
    C.nullable[j] = nullable[j] ? 1 : 0;
  }
  // check the page table, lay out the decompression scratch
  std::vector<int64_t> covered(ncols, 0);
  std::vector<int> snappy, chain, dict_strings, dict_chain, data_pages;
  std::vector<int64_t> soff;
  int64_t scratch_bytes = 0, nentries = 0, chain_in = 0, dict_in = 0;
  std::vector<PqPage> dev_pages(npages);
  for (int p = 0; p < npages; ++p) {
    const ldf_parquet_page& h = pages[p];
    LDF_REQUIRE(h.column >= 0 && h.column < ncols, "parquet_decode: page column out of range");
    LDF_REQUIRE(h.offset >= 0 && h.compressed >= 0 && h.offset + h.compressed <= file_bytes,
                "parquet_decode: page outside the file");
    LDF_REQUIRE(h.uncompressed >= 0 && h.num_values >= 0, "parquet_decode: negative page sizes");
    LDF_REQUIRE(h.kind == LDF_PQ_DICT_PAGE || h.kind == LDF_PQ_DATA_V1 || h.kind == LDF_PQ_DATA_V2,
                "parquet_decode: unsupported page kind");
    LDF_REQUIRE(h.codec == LDF_PQ_UNCOMPRESSED || h.codec == LDF_PQ_SNAPPY, "parquet_decode: unsupported codec");
    LDF_REQUIRE(h.kind != LDF_PQ_DATA_V2 || (h.levels_bytes >= 0 && h.levels_bytes <= h.compressed &&
                                             h.levels_bytes <= h.uncompressed),
                "parquet_decode: bad level bytes");
    dev_pages[p].h          = h;
    dev_pages[p].data_bytes = h.codec == LDF_PQ_SNAPPY ? h.uncompressed : h.compressed;
    if (h.codec == LDF_PQ_SNAPPY) {
      const int64_t lv = h.kind == LDF_PQ_DATA_V2 ? h.levels_bytes : 0;
      if (C.physical[h.column] == LDF_PQ_BYTE_ARRAY && h.uncompressed - lv >= kChainMinBytes &&
          chain_in + h.compressed <= kChainMaxInput) {
        chain.push_back(p);  // decoded by the whole GPU (scratch laid out below)
        chain_in += h.compressed - lv;
      } else {
        snappy.push_back(p);
      }
    }
    if (h.kind == LDF_PQ_DICT_PAGE) {
      LDF_REQUIRE(h.encoding == 0 || h.encoding == 2, "parquet_decode: dictionary pages must be PLAIN");
      if (C.physical[h.column] == LDF_PQ_BYTE_ARRAY) {
        dev_pages[p].dict_entry0 = nentries;
        nentries += h.num_values;
        const int64_t bytes = dev_pages[p].data_bytes;
        if (bytes >= kDictChainMinBytes && dict_in + bytes <= kChainMaxInput) {
          dict_chain.push_back(p);  // ranked by the whole GPU
          dict_in += bytes;
        } else {
          dict_strings.push_back(p);
        }
      }
    } else {
      LDF_REQUIRE(h.encoding == 0 || h.encoding == 2 || h.encoding == 8 ||
                    (h.encoding == 3 && C.physical[h.column] == LDF_PQ_BOOLEAN),
                  "parquet_decode: unsupported encoding");
      if (h.encoding == 2 || h.encoding == 8)
        LDF_REQUIRE(h.dict >= 0 && h.dict < npages && pages[h.dict].kind == LDF_PQ_DICT_PAGE &&
                      pages[h.dict].column == h.column,
                    "parquet_decode: a dictionary-encoded page without its dictionary");
      LDF_REQUIRE(h.row0 >= 0 && h.row0 + h.num_values <= nrows, "parquet_decode: page rows out of range");
      covered[h.column] += h.num_values;
      data_pages.push_back(p);
    }
  }
  for (int j = 0; j < ncols; ++j)
    LDF_REQUIRE(covered[j] == nrows, "parquet_decode: the data pages do not cover every row of a column");
  // scratch: the chain pages' outputs first (one index space), then the others
  std::vector<ChainPage> cpages;
  std::vector<int64_t> cbases;  // in | out | elem | ck, one entry per chain page each
  int64_t chain_elems = 0, chain_cks = 0, chain_out = 0, chain_maxu = 1;
  {
    std::vector<int64_t> in_b, out_b, el_b, ck_b;
    int64_t in_run = 0;
    for (int p : chain) {
      const ldf_parquet_page& h = pages[p];
      const int64_t lv          = h.kind == LDF_PQ_DATA_V2 ? h.levels_bytes : 0;
      ChainPage c{};
      c.page     = p;
      c.file_off = h.offset + lv;
      c.n        = h.compressed - lv;
      c.lv       = lv;
      c.u        = h.uncompressed - lv;
      c.elem_cap = c.n / 2 + 1;
      c.ck_cap   = c.elem_cap / kChainStep + 2;
      in_b.push_back(in_run);
      out_b.push_back(scratch_bytes);
      el_b.push_back(chain_elems);
      ck_b.push_back(chain_cks);
      in_run += c.n;
      chain_elems += c.elem_cap;
      chain_cks += c.ck_cap;
      chain_maxu = std::max(chain_maxu, h.uncompressed);
      scratch_bytes += (h.uncompressed + 15) & ~int64_t(15);
      cpages.push_back(c);
    }
    chain_out = scratch_bytes;
    for (auto* v : {&in_b, &out_b, &el_b, &ck_b}) cbases.insert(cbases.end(), v->begin(), v->end());
    for (int p : snappy) {
      soff.push_back(scratch_bytes);
      scratch_bytes += (pages[p].uncompressed + 15) & ~int64_t(15);
    }
  }
  {  // decompress the largest pages first: a page is one warp's sequential work
    std::vector<int> order(snappy.size());
    for (size_t q = 0; q < order.size(); ++q) order[q] = static_cast<int>(q);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
      return pages[snappy[a]].uncompressed > pages[snappy[b]].uncompressed;
    });
    std::vector<int> sp(order.size());
    std::vector<int64_t> so(order.size());
    for (size_t q = 0; q < order.size(); ++q) {
      sp[q] = snappy[order[q]];
      so[q] = soff[order[q]];
    }
    snappy.swap(sp);
    soff.swap(so);
  }
  const Allocator& al = ctx.alloc();
  cudaStream_t s      = ctx.stream();
  Buffer<uint8_t> scratch(al, std::max<int64_t>(scratch_bytes, 16));
  for (size_t q = 0; q < snappy.size(); ++q) dev_pages[snappy[q]].data = scratch.get() + soff[q];
  for (size_t q = 0; q < chain.size(); ++q) dev_pages[chain[q]].data = scratch.get() + cbases[chain.size() + q];
  for (int p = 0; p < npages; ++p)
    if (pages[p].codec != LDF_PQ_SNAPPY) dev_pages[p].data = file + pages[p].offset;
  Buffer<PqPage> d_pages(al, std::max(npages, 1));
  std::vector<int> lists;  // snappy | dict strings | data pages
  lists.insert(lists.end(), snappy.begin(), snappy.end());
  lists.insert(lists.end(), dict_strings.begin(), dict_strings.end());
  lists.insert(lists.end(), data_pages.begin(), data_pages.end());
  Buffer<int> d_lists(al, std::max<size_t>(lists.size(), 1));
  Buffer<int64_t> d_soff(al, std::max<size_t>(soff.size(), 1));
  Buffer<unsigned long long> d_err(al, 1);
  LDF_CUDA(cudaMemcpyAsync(d_pages.get(), dev_pages.data(), npages * sizeof(PqPage), cudaMemcpyHostToDevice, s));
  LDF_CUDA(cudaMemcpyAsync(d_lists.get(), lists.data(), lists.size() * sizeof(int), cudaMemcpyHostToDevice, s));
  LDF_CUDA(cudaMemcpyAsync(d_soff.get(), soff.data(), soff.size() * sizeof(int64_t), cudaMemcpyHostToDevice, s));
  LDF_CUDA(cudaMemsetAsync(d_err.get(), 0xff, sizeof(unsigned long long), s));
  // outputs
  std::vector<Buffer<const uint8_t*>> src_bufs;
  std::vector<Buffer<int64_t>> len_bufs;
  for (int j = 0; j < ncols; ++j) {
    out[j]     = alloc_out_column(al, types[j], nrows, nullable[j] != 0);
    C.data[j]  = out[j].data;
    C.valid[j] = out[j].valid;
    if (C.physical[j] == LDF_PQ_BYTE_ARRAY) {
      src_bufs.emplace_back(al, std::max<int64_t>(nrows, 1));
      len_bufs.emplace_back(al, std::max<int64_t>(nrows, 1));
      C.str_src[j] = src_bufs.back().get();
      C.str_len[j] = len_bufs.back().get();
    }
  }
  Buffer<int64_t> entry_off(al, std::max<int64_t>(nentries, 1));
  Buffer<int32_t> entry_len(al, std::max<int64_t>(nentries, 1));
  const int nsn = static_cast<int>(snappy.size()), nds = static_cast<int>(dict_strings.size()),
            ndp = static_cast<int>(data_pages.size());
  if (!chain.empty()) {  // large byte-array pages: the element chains ranked by the whole GPU
    const int nc          = static_cast<int>(chain.size());
    const int64_t cin     = chain_in;
    Buffer<ChainPage> d_cp(al, nc);
    Buffer<ChainState> d_st(al, nc);
    Buffer<int64_t> d_cb(al, cbases.size());
    LDF_CUDA(cudaMemcpyAsync(d_cp.get(), cpages.data(), nc * sizeof(ChainPage), cudaMemcpyHostToDevice, s));
    LDF_CUDA(cudaMemcpyAsync(d_cb.get(), cbases.data(), cbases.size() * sizeof(int64_t), cudaMemcpyHostToDevice, s));
    const ChainBases B{d_cb.get(), d_cb.get() + nc, d_cb.get() + 2 * nc, d_cb.get() + 3 * nc, nc};
    Buffer<int64_t> j0(al, cin), j1(al, cin), j2(al, cin);
    launch("chain_start", chain_start_kernel, pq_blocks(nc, 128), 128, 0, s, file,
           static_cast<const ChainPage*>(d_cp.get()), d_st.get(), nc, d_err.get());
    launch("chain_next", chain_next_kernel, pq_blocks(cin, 256), 256, 0, s, file,
           static_cast<const ChainPage*>(d_cp.get()), static_cast<const ChainState*>(d_st.get()), B, cin, j0.get());
    const int64_t* jump = j0.get();
    for (int r = 0; r < kChainLog; ++r) {
      int64_t* out = (r % 2 == 0) ? j1.get() : j2.get();
      launch("chain_double", chain_double_kernel, pq_blocks(cin, 256), 256, 0, s, jump, out, cin);
      jump = out;
    }
    Buffer<int64_t> ck(al, chain_cks);
    launch("chain_checkpoints", chain_checkpoints_kernel, pq_blocks(nc, 128), 128, 0, s,
           static_cast<const ChainPage*>(d_cp.get()), d_st.get(), B, jump, ck.get());
    Buffer<int64_t> epos(al, chain_elems), elen(al, chain_elems), emeta(al, chain_elems), eoff(al, chain_elems);
    launch("chain_walk", chain_walk_kernel, pq_blocks(chain_cks, 128), 128, 0, s, file,
           static_cast<const ChainPage*>(d_cp.get()), d_st.get(), B, chain_cks, static_cast<const int64_t*>(ck.get()),
           epos.get(), d_err.get());
    launch("chain_decode", chain_decode_kernel, pq_blocks(chain_elems, 256), 256, 0, s, file,
           static_cast<const ChainPage*>(d_cp.get()), static_cast<const ChainState*>(d_st.get()), B, chain_elems,
           static_cast<const int64_t*>(epos.get()), elen.get(), emeta.get());
    Buffer<int64_t> etotal(al, 1);
    exclusive_scan_i64(elen.get(), eoff.get(), chain_elems, etotal.get(), ctx);
    Buffer<int64_t> p0(al, chain_out), p1(al, chain_out);
    launch("chain_ptr", chain_ptr_kernel, pq_blocks(chain_out, 256), 256, 0, s,
           static_cast<const ChainPage*>(d_cp.get()), static_cast<const ChainState*>(d_st.get()), B, chain_out,
           static_cast<const int64_t*>(eoff.get()), static_cast<const int64_t*>(elen.get()),
           static_cast<const int64_t*>(emeta.get()), p0.get(), d_err.get());
    int rounds = 1;  // every pointer moves back one byte or more: log2 of the page size rounds reach a literal
    while ((int64_t(1) << rounds) <= chain_maxu) ++rounds;
    int64_t* pin = p0.get();
    int64_t* pout = p1.get();
    for (int r = 0; r < rounds; ++r) {
      launch("chain_jump", chain_jump_kernel, pq_blocks(chain_out, 256), 256, 0, s,
             static_cast<const int64_t*>(pin), pout, chain_out);
      std::swap(pin, pout);
    }
    launch("chain_final", chain_final_kernel, pq_blocks(chain_out, 256), 256, 0, s, file,
           static_cast<const ChainPage*>(d_cp.get()), B, static_cast<const int64_t*>(pin), chain_out, scratch.get(),
           d_err.get());
  }
  if (nsn > 0)
    launch("pq_snappy", pq_snappy_kernel, static_cast<unsigned>(nsn), kLanes, 0, s,
           file, d_pages.get(), static_cast<const int*>(d_lists.get()), nsn, scratch.get(),
           static_cast<const int64_t*>(d_soff.get()), d_err.get());
  if (nds > 0)
    launch("pq_dict_strings", pq_dict_strings_kernel, static_cast<unsigned>(nds), kPqThreads, 0, s,
           static_cast<const PqPage*>(d_pages.get()), static_cast<const int*>(d_lists.get()) + nsn, nds,
           entry_off.get(), entry_len.get(), d_err.get());
  if (!dict_chain.empty()) {  // large dictionary pages: the length-prefix chains ranked by the whole GPU
    const int nc = static_cast<int>(dict_chain.size());
    std::vector<DictChain> dc;
    std::vector<int64_t> in_b, ck_b;
    int64_t in_run = 0, ck_run = 0;
    for (int p : dict_chain) {
      DictChain c{};
      c.page   = p;
      c.data   = dev_pages[p].data;
      c.n      = dev_pages[p].data_bytes;
      c.nv     = pages[p].num_values;
      c.entry0 = dev_pages[p].dict_entry0;
      c.ck_cap = c.nv / kChainStep + 2;
      in_b.push_back(in_run);
      ck_b.push_back(ck_run);
      in_run += c.n;
      ck_run += c.ck_cap;
      dc.push_back(c);
    }
    std::vector<int64_t> bases(in_b);
    bases.insert(bases.end(), ck_b.begin(), ck_b.end());
    Buffer<DictChain> d_dc(al, nc);
    Buffer<int64_t> d_b(al, bases.size()), d_nck(al, nc), ck(al, ck_run);
    LDF_CUDA(cudaMemcpyAsync(d_dc.get(), dc.data(), nc * sizeof(DictChain), cudaMemcpyHostToDevice, s));
    LDF_CUDA(cudaMemcpyAsync(d_b.get(), bases.data(), bases.size() * sizeof(int64_t), cudaMemcpyHostToDevice, s));
    const ChainBases B{d_b.get(), nullptr, nullptr, d_b.get() + nc, nc};
    Buffer<int64_t> j0(al, in_run), j1(al, in_run), j2(al, in_run);
    launch("dict_next", dict_next_kernel, pq_blocks(in_run, 256), 256, 0, s,
           static_cast<const DictChain*>(d_dc.get()), B, in_run, j0.get());
    const int64_t* jump = j0.get();
    for (int r = 0; r < kChainLog; ++r) {
      int64_t* out = (r % 2 == 0) ? j1.get() : j2.get();
      launch("chain_double", chain_double_kernel, pq_blocks(in_run, 256), 256, 0, s, jump, out, in_run);
      jump = out;
    }
    launch("dict_checkpoints", dict_checkpoints_kernel, pq_blocks(nc, 128), 128, 0, s,
           static_cast<const DictChain*>(d_dc.get()), B, jump, ck.get(), d_nck.get());
    launch("dict_walk", dict_walk_kernel, pq_blocks(ck_run, 128), 128, 0, s,
           static_cast<const DictChain*>(d_dc.get()), B, ck_run, static_cast<const int64_t*>(ck.get()),
           static_cast<const int64_t*>(d_nck.get()), entry_off.get(), entry_len.get(), d_err.get());
  }
  if (ndp > 0)
    launch("pq_data", pq_data_kernel, static_cast<unsigned>(ndp), kPqThreads, 0, s,
           static_cast<const PqPage*>(d_pages.get()), static_cast<const int*>(d_lists.get()) + nsn + nds, C,
           static_cast<const int64_t*>(entry_off.get()), static_cast<const int32_t*>(entry_len.get()), d_err.get());
  unsigned long long h_err = ~0ull;
  LDF_CUDA(cudaMemcpyAsync(&h_err, d_err.get(), sizeof(h_err), cudaMemcpyDeviceToHost, s));
  ctx.finish();
  if (h_err != ~0ull) {
    for (int j = 0; j < ncols; ++j) free_out_column(al, out[j]);
    static const char* what[] = {"", "a Snappy stream is malformed", "a level or index stream is malformed",
                                 "a dictionary index is out of range", "the page's values are truncated"};
    const uint32_t code = static_cast<uint32_t>(h_err & 0xff);
    fail(LDF_ERR_INVALID_ARGUMENT, std::string("Parquet page ") + std::to_string(h_err >> 8) + ": " +
                                     (code < 5 ? what[code] : "decode error"));
  }
  // strings: lengths -> offsets -> characters
  Buffer<int64_t> misc(al, 1);
  for (int j = 0; j < ncols; ++j) {
    if (C.physical[j] != LDF_PQ_BYTE_ARRAY) continue;
    Buffer<int64_t> offs(al, std::max<int64_t>(nrows, 1));
    exclusive_scan_i64(C.str_len[j], offs.get(), nrows, misc.get(), ctx);
    const int64_t nchars = ctx.read_i64(misc.get());
    out[j].chars         = static_cast<char*>(al.allocate(static_cast<size_t>(std::max<int64_t>(nchars, 1))));
    out[j].num_chars     = nchars;
    out[j].chars_base    = 0;
    if (nrows > 0)
      launch("pq_strings", pq_copy_strings_kernel, pq_blocks(ceil_div(nrows, kPqStrRows), 256), 256, 0, s,
             static_cast<const uint8_t* const*>(C.str_src[j]), static_cast<const int64_t*>(C.str_len[j]),
             static_cast<const int64_t*>(offs.get()), nrows, nchars, reinterpret_cast<uint8_t*>(out[j].chars),
             static_cast<ldf_range*>(out[j].data));
  }
  ctx.finish();
}

}  // namespace ldf

// ---- page headers on the host (Thrift compact protocol) -----------------------------
namespace ldf {
namespace {

struct ThriftReader {
  const uint8_t* b;
  int64_t pos, end;
  uint8_t byte()
  {
    if (pos >= end) fail(LDF_ERR_INVALID_ARGUMENT, "truncated Parquet page header");
    return b[pos++];
  }
  uint64_t varint()
  {
    uint64_t v = 0;
    for (int sh = 0;; sh += 7) {
      if (sh > 63) fail(LDF_ERR_INVALID_ARGUMENT, "bad varint in a Parquet page header");
      const uint8_t c = byte();
      v |= static_cast<uint64_t>(c & 0x7f) << sh;
      if (!(c & 0x80)) return v;
    }
  }
  int64_t zigzag()
  {
    const uint64_t v = varint();
    return static_cast<int64_t>(v >> 1) ^ -static_cast<int64_t>(v & 1);
  }
  // Skips a value of Thrift compact type t.
  void skip(int t)
  {
    switch (t) {
      case 1:
      case 2: return;
      case 3: byte(); return;
      case 4:
      case 5:
      case 6: varint(); return;
      case 7: pos += 8; return;
      case 8: pos += static_cast<int64_t>(varint()); return;
      case 9:
      case 10: {
        const uint8_t h = byte();
        uint64_t n      = h >> 4;
        if (n == 15) n = varint();
        for (uint64_t k = 0; k < n; ++k) skip((h & 15) == 1 || (h & 15) == 2 ? 3 : (h & 15));
        return;
      }
      case 11: {
        const uint64_t n = varint();
        if (n) {
          const uint8_t kv = byte();
          for (uint64_t k = 0; k < n; ++k) {
            skip(kv >> 4);
            skip(kv & 15);
          }
        }
        return;
      }
      case 12: struct_fields([](int, int, ThriftReader&) { return false; }); return;
      default: fail(LDF_ERR_INVALID_ARGUMENT, "unknown Thrift type in a Parquet page header");
    }
  }
  // Calls f(field id, type, *this) for each field; f reads the value and
  // returns true, or returns false to have it skipped.
  template <typename F>
  void struct_fields(F&& f)
  {
    int last = 0;
    while (true) {
      const uint8_t h = byte();
      if (h == 0) return;
      const int t   = h & 15;
      const int fid = (h >> 4) ? last + (h >> 4) : static_cast<int>(zigzag());
      if (!f(fid, t, *this)) skip(t);
      last = fid;
    }
  }
  int64_t int_value(int t) { return t == 1 ? 1 : (t == 2 ? 0 : zigzag()); }
};

}  // namespace

void parquet_pages(const uint8_t* file, int64_t file_bytes, const int64_t* chunk_start, const int64_t* chunk_bytes,
                   const int64_t* chunk_row0, const int32_t* chunk_column, const int32_t* chunk_codec,
                   const int32_t* chunk_physical, int nchunks, ldf_parquet_page* pages, int max_pages, int* npages)
{
  LDF_REQUIRE(nchunks >= 0 && file != nullptr && npages != nullptr, "parquet_pages: null argument");
  int count = 0;
  for (int k = 0; k < nchunks; ++k) {
    LDF_REQUIRE(chunk_start[k] >= 0 && chunk_bytes[k] >= 0 && chunk_start[k] + chunk_bytes[k] <= file_bytes,
                "parquet_pages: column chunk outside the file");
    const int64_t end = chunk_start[k] + chunk_bytes[k];
    int64_t pos = chunk_start[k], row = chunk_row0[k];
    int dict    = -1;
    while (pos < end) {
      ThriftReader rd{file, pos, end};
      int64_t type = -1, usize = 0, csize = 0;
      int64_t nvals = 0, enc = 0, lv = 0, rep = 0, compressed = 1;
      rd.struct_fields([&](int fid, int t, ThriftReader& r) {
        switch (fid) {
          case 1: type = r.int_value(t); return true;
          case 2: usize = r.int_value(t); return true;
          case 3: csize = r.int_value(t); return true;
          case 5:  // DataPageHeader
          case 7:  // DictionaryPageHeader
          case 8:  // DataPageHeaderV2
            if (t != 12) return false;
            r.struct_fields([&](int g, int tt, ThriftReader& q) {
              if (fid == 8) {
                switch (g) {
                  case 1: nvals = q.int_value(tt); return true;
                  case 4: enc = q.int_value(tt); return true;
                  case 5: lv = q.int_value(tt); return true;
                  case 6: rep = q.int_value(tt); return true;
                  case 7: compressed = q.int_value(tt); return true;
                  default: return false;
                }
              }
              if (g == 1) nvals = q.int_value(tt);
              else if (g == 2) enc = q.int_value(tt);
              else return false;
              return true;
            });
            return true;
          default: return false;
        }
      });
      const int64_t payload = rd.pos;
      LDF_REQUIRE(csize >= 0 && payload + csize <= end, "parquet_pages: page outside its column chunk");
      if (type == 0 || type == 2 || type == 3) {
        if (type != 2) {
          const bool rle_bool = enc == 3 && chunk_physical[k] == LDF_PQ_BOOLEAN;
          if (!(enc == 0 || enc == 2 || enc == 8 || rle_bool))
            fail(LDF_ERR_UNSUPPORTED, "parquet_pages: page encoding " + std::to_string(enc));
          if (rep != 0) fail(LDF_ERR_UNSUPPORTED, "parquet_pages: repetition levels");
        }
        if (pages != nullptr) {
          LDF_REQUIRE(count < max_pages, "parquet_pages: more pages than max_pages");
          ldf_parquet_page& e = pages[count];
          e                   = ldf_parquet_page{};
          e.offset            = payload;
          e.compressed        = csize;
          e.uncompressed      = usize;
          e.num_values        = static_cast<int32_t>(nvals);
          e.encoding          = static_cast<int32_t>(enc);
          e.codec             = chunk_codec[k];
          e.column            = chunk_column[k];
          e.dict              = -1;
          if (type == 2) {
            e.kind = LDF_PQ_DICT_PAGE;
          } else {
            e.kind = type == 0 ? LDF_PQ_DATA_V1 : LDF_PQ_DATA_V2;
            e.row0 = row;
            e.dict = (enc == 2 || enc == 8) ? dict : -1;
            if (type == 3) {
              e.levels_bytes = static_cast<int32_t>(lv);
              if (!compressed) e.codec = LDF_PQ_UNCOMPRESSED;
            }
          }
        }
        if (type == 2) dict = count;
        else row += nvals;
        ++count;
      }
      pos = payload + csize;
    }
  }
  *npages = count;
}

}  // namespace ldf
