// Parquet pages -> columns in the legate layout, decoded on the device.
// Replaces cudf::io::read_parquet in ParquetRead::gpu_variant
// (parquet.cu:48-101); the results match the reference's CPU reader (Arrow).
//
// The caller walks the footer and the page headers (Thrift, a few bytes per
// page) and hands over one entry per page; the whole file is in device
// memory.  Then:
// 1. Snappy pages are decompressed, one warp per page: every lane parses the
//    same element tags (broadcast loads), the warp copies the element's bytes
//    together (a back-reference of offset d repeats its last d bytes, so
//    byte k of it is dst[o - d + k % d] and all of it copies at once).
// 2. Dictionary pages of byte arrays get an entry table (offset, length).
// 3. One block per data page decodes its rows in tiles of kPqTile: thread 0
//    cuts the next tile out of the RLE / bit-packed hybrid streams (the
//    definition levels, the dictionary indices) as a list of run segments,
//    and every thread decodes its values from the segment it falls in; a
//    block scan of the definition levels gives each valid row its value
//    index; PLAIN values are read at that index, dictionary values through
//    the decoded index, and byte arrays by a walk of their length prefixes.
// 4. String columns: lengths -> offsets (scan) -> characters copied.
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
// src[0, n) -> dst (at most cap bytes) by the calling warp; false when the
// stream is malformed.  Every lane parses the same tags.
__device__ bool snappy_warp(const uint8_t* src, int64_t n, uint8_t* dst, int64_t cap, int64_t& produced)
{
  const int lane = threadIdx.x % kLanes;
  int64_t i      = 0;
  uint64_t len   = 0;
  for (int sh = 0;; sh += 7) {  // preamble: the uncompressed length as a varint
    if (i >= n || sh > 35) return false;
    const uint8_t b = src[i++];
    len |= static_cast<uint64_t>(b & 0x7f) << sh;
    if (!(b & 0x80)) break;
  }
  if (len > static_cast<uint64_t>(cap)) return false;
  int64_t o = 0;
  while (o < static_cast<int64_t>(len)) {
    if (i >= n) return false;
    const uint32_t t = src[i++];
    int64_t l;
    if ((t & 3) == 0) {  // literal
      l = t >> 2;
      if (l >= 60) {
        const int nb = static_cast<int>(l) - 59;
        if (i + nb > n) return false;
        l = le_bytes(src + i, nb);
        i += nb;
      }
      l += 1;
      if (i + l > n || o + l > static_cast<int64_t>(len)) return false;
      for (int64_t k = lane; k < l; k += kLanes) dst[o + k] = src[i + k];
      i += l;
    } else {  // back-reference
      int64_t off;
      if ((t & 3) == 1) {
        if (i >= n) return false;
        l   = 4 + ((t >> 2) & 7);
        off = (static_cast<int64_t>(t >> 5) << 8) | src[i++];
      } else {
        const int nb = (t & 3) == 2 ? 2 : 4;
        if (i + nb > n) return false;
        l   = (t >> 2) + 1;
        off = le_bytes(src + i, nb);
        i += nb;
      }
      if (off == 0 || off > o || o + l > static_cast<int64_t>(len)) return false;
      for (int64_t k = lane; k < l; k += kLanes) dst[o + k] = dst[o - off + k % off];
    }
    o += l;
    __syncwarp();  // the next element may read these bytes
  }
  produced = o;
  return true;
}

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
__global__ void __launch_bounds__(kPqThreads) pq_snappy_kernel(const uint8_t* file, PqPage* pages,
                                                               const int* list, int nlist, uint8_t* scratch,
                                                               const int64_t* soff, unsigned long long* err)
{
  const int w = blockIdx.x * (kPqThreads / kLanes) + threadIdx.x / kLanes;
  if (w >= nlist) return;
  const int p           = list[w];
  const PqPage& pg      = pages[p];
  const int64_t lv      = pg.h.kind == LDF_PQ_DATA_V2 ? pg.h.levels_bytes : 0;
  const uint8_t* src    = file + pg.h.offset;
  uint8_t* dst          = scratch + soff[w];
  const int lane        = threadIdx.x % kLanes;
  for (int64_t k = lane; k < lv; k += kLanes) dst[k] = src[k];
  int64_t got = 0;
  const bool ok = snappy_warp(src + lv, pg.h.compressed - lv, dst + lv, pg.h.uncompressed - lv, got);
  if (lane == 0 && (!ok || got != pg.h.uncompressed - lv)) pq_error(err, p, kPqErrSnappy);
}

// Byte-array dictionary pages, one thread each: entry (offset in the page's
// data, length) of every value.
__global__ void pq_dict_strings_kernel(const PqPage* pages, const int* list, int nlist, int64_t* entry_off,
                                       int32_t* entry_len, unsigned long long* err)
{
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nlist; q += gridDim.x * blockDim.x) {
    const int p      = list[q];
    const PqPage& pg = pages[p];
    int64_t pos      = 0;
    for (int v = 0; v < pg.h.num_values; ++v) {
      int64_t len = -1;
      if (pos + 4 <= pg.data_bytes) len = le_bytes(pg.data + pos, 4);
      if (len < 0 || pos + 4 + len > pg.data_bytes) {
        pq_error(err, p, kPqErrValues);
        len = 0;
        pos = pg.data_bytes;
      } else {
        pos += 4;
      }
      entry_off[pg.dict_entry0 + v] = pos;
      entry_len[pg.dict_entry0 + v] = static_cast<int32_t>(len);
      pos += len;
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
__global__ void pq_copy_strings_kernel(const uint8_t* const* src, const int64_t* len, const int64_t* offs, int64_t rows,
                                       uint8_t* chars, ldf_range* ranges)
{
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < rows; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t o = offs[i], n = len[i];
    ranges[i]       = ldf_range{o, o + n - 1};
    const uint8_t* s = src[i];
    for (int64_t k = 0; k < n; ++k) chars[o + k] = s[k];
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
  std::vector<int> snappy, dict_strings, data_pages;
  std::vector<int64_t> soff;
  int64_t scratch_bytes = 0, nentries = 0;
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
      snappy.push_back(p);
      soff.push_back(scratch_bytes);
      scratch_bytes += (h.uncompressed + 15) & ~int64_t(15);
    }
    if (h.kind == LDF_PQ_DICT_PAGE) {
      LDF_REQUIRE(h.encoding == 0 || h.encoding == 2, "parquet_decode: dictionary pages must be PLAIN");
      if (C.physical[h.column] == LDF_PQ_BYTE_ARRAY) {
        dev_pages[p].dict_entry0 = nentries;
        nentries += h.num_values;
        dict_strings.push_back(p);
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
  const Allocator& al = ctx.alloc();
  cudaStream_t s      = ctx.stream();
  Buffer<uint8_t> scratch(al, std::max<int64_t>(scratch_bytes, 16));
  for (size_t q = 0; q < snappy.size(); ++q) dev_pages[snappy[q]].data = scratch.get() + soff[q];
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
  if (nsn > 0)
    launch("pq_snappy", pq_snappy_kernel, static_cast<unsigned>(ceil_div(nsn, kPqThreads / kLanes)), kPqThreads, 0, s,
           file, d_pages.get(), static_cast<const int*>(d_lists.get()), nsn, scratch.get(),
           static_cast<const int64_t*>(d_soff.get()), d_err.get());
  if (nds > 0)
    launch("pq_dict_strings", pq_dict_strings_kernel, pq_blocks(nds, 128), 128, 0, s,
           static_cast<const PqPage*>(d_pages.get()), static_cast<const int*>(d_lists.get()) + nsn, nds,
           entry_off.get(), entry_len.get(), d_err.get());
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
      launch("pq_strings", pq_copy_strings_kernel, pq_blocks(nrows, 256), 256, 0, s,
             static_cast<const uint8_t* const*>(C.str_src[j]), static_cast<const int64_t*>(C.str_len[j]),
             static_cast<const int64_t*>(offs.get()), nrows, reinterpret_cast<uint8_t*>(out[j].chars),
             static_cast<ldf_range*>(out[j].data));
  }
  ctx.finish();
}

}  // namespace ldf
