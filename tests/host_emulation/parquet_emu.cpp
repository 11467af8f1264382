// Host emulation of the Parquet decoder's device code
// (legate-dataframe_b200/csrc/parquet.cu): Snappy, the RLE / bit-packed
// hybrid cutter, dictionary entries and the data-page kernel compiled as host
// C++ with one thread per block (a warp of one lane, tiles of 8 rows), the
// kernels run block after block over host memory.  The test that builds it
// (tests/test_parquet_emulated.py) extracts the kernels' section from the
// CUDA source and substitutes the thread counts; this file supplies the CUDA
// built-ins and a driver laid out like parquet_decode.
//
// Input file (argv[1]): int64 file_bytes, npages, ncols, nrows; the file's
// bytes; npages ldf_parquet_page records; ncols x (physical, type,
// nullable) int32.  Output: "rows R" and per column one line per row ("N",
// "I <int64>", "U <uint64>", "F <hex bits>", "S <hex bytes>"), or
// "error <code> <page>".
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <algorithm>
#include <vector>

#include "ldf_b200.h"

#define __global__
#define __device__
#define __host__
#define __shared__ static
#define __forceinline__ inline
#define __launch_bounds__(...)
struct dim3 { unsigned x; };
static dim3 threadIdx{0}, blockIdx{0}, blockDim{1}, gridDim{1};
static inline void __syncthreads() {}
static inline void __syncwarp() {}
template <typename T> static inline T atomicMin(T* p, T v) { T o = *p; if (v < o) *p = v; return o; }
template <typename T, int NT> static inline T block_exclusive_scan(T v, T*, T* total) { *total = v; return 0; }
// warp intrinsics of the 32-lane paths, which a one-lane build never takes
static inline int __shfl_up_sync(unsigned, int v, int) { abort(); return v; }
static inline unsigned __ballot_sync(unsigned, bool) { abort(); return 0; }
static inline int __ffs(unsigned) { abort(); return 0; }

namespace ldf {
inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }
inline int num_sms() { return 1; }
#include "parquet_sections.inc"
}  // namespace ldf

using namespace ldf;

int main(int argc, char** argv)
{
  FILE* f = fopen(argv[1], "rb");
  int64_t hdr[4];
  if (fread(hdr, 8, 4, f) != 4) return 2;
  const int64_t file_bytes = hdr[0], nrows = hdr[3];
  const int npages = (int)hdr[1], ncols = (int)hdr[2];
  std::vector<uint8_t> file(std::max<int64_t>(file_bytes, 1));
  if ((int64_t)fread(file.data(), 1, file_bytes, f) != file_bytes) return 2;
  std::vector<ldf_parquet_page> pages(std::max(npages, 1));
  if ((int)fread(pages.data(), sizeof(ldf_parquet_page), npages, f) != npages) return 2;
  std::vector<int32_t> spec(3 * ncols);
  if ((int)fread(spec.data(), 4, 3 * ncols, f) != 3 * ncols) return 2;
  fclose(f);
  static const int widths[] = {0, 1, 1, 2, 4, 8, 1, 2, 4, 8, 4, 8, 16, 8};
  PqColumns C;
  memset(&C, 0, sizeof(C));
  C.ncols = ncols;
  std::vector<std::vector<uint8_t>> data(ncols), valid(ncols);
  std::vector<std::vector<const uint8_t*>> ssrc(ncols);
  std::vector<std::vector<int64_t>> slen(ncols);
  for (int j = 0; j < ncols; ++j) {
    C.physical[j] = spec[3 * j];
    C.width[j]    = widths[spec[3 * j + 1]];
    C.nullable[j] = spec[3 * j + 2];
    data[j].assign(std::max<int64_t>(nrows, 1) * C.width[j], 0xAB);
    C.data[j] = data[j].data();
    if (C.nullable[j]) {
      valid[j].assign(std::max<int64_t>(nrows, 1), 0xAB);
      C.valid[j] = valid[j].data();
    }
    if (C.physical[j] == LDF_PQ_BYTE_ARRAY) {
      ssrc[j].assign(std::max<int64_t>(nrows, 1), nullptr);
      slen[j].assign(std::max<int64_t>(nrows, 1), -1);
      C.str_src[j] = ssrc[j].data();
      C.str_len[j] = slen[j].data();
    }
  }
  // page table and lists, as parquet_decode lays them out
  std::vector<PqPage> dp(std::max(npages, 1));
  std::vector<int> snappy, dict_strings, data_pages;
  std::vector<int64_t> soff;
  int64_t scratch_bytes = 0, nentries = 0;
  for (int p = 0; p < npages; ++p) {
    const ldf_parquet_page& h = pages[p];
    dp[p].h          = h;
    dp[p].data_bytes = h.codec == LDF_PQ_SNAPPY ? h.uncompressed : h.compressed;
    if (h.codec == LDF_PQ_SNAPPY) {
      snappy.push_back(p);
      soff.push_back(scratch_bytes);
      scratch_bytes += (h.uncompressed + 15) & ~int64_t(15);
    }
    if (h.kind == LDF_PQ_DICT_PAGE) {
      if (C.physical[h.column] == LDF_PQ_BYTE_ARRAY) {
        dp[p].dict_entry0 = nentries;
        nentries += h.num_values;
        dict_strings.push_back(p);
      }
    } else {
      data_pages.push_back(p);
    }
  }
  std::vector<uint8_t> scratch(std::max<int64_t>(scratch_bytes, 16));
  for (size_t q = 0; q < snappy.size(); ++q) dp[snappy[q]].data = scratch.data() + soff[q];
  for (int p = 0; p < npages; ++p)
    if (pages[p].codec != LDF_PQ_SNAPPY) dp[p].data = file.data() + pages[p].offset;
  std::vector<int> lists;
  lists.insert(lists.end(), snappy.begin(), snappy.end());
  lists.insert(lists.end(), dict_strings.begin(), dict_strings.end());
  lists.insert(lists.end(), data_pages.begin(), data_pages.end());
  std::vector<int64_t> entry_off(std::max<int64_t>(nentries, 1));
  std::vector<int32_t> entry_len(std::max<int64_t>(nentries, 1));
  unsigned long long err = ~0ull;
  for (unsigned b = 0; b < snappy.size(); ++b) {
    blockIdx.x = b;
    pq_snappy_kernel(file.data(), dp.data(), lists.data(), (int)snappy.size(), scratch.data(), soff.data(), &err);
  }
  blockIdx.x = 0;
  if (!dict_strings.empty())
    pq_dict_strings_kernel(dp.data(), lists.data() + snappy.size(), (int)dict_strings.size(), entry_off.data(),
                           entry_len.data(), &err);
  for (unsigned b = 0; b < data_pages.size(); ++b) {
    blockIdx.x = b;
    pq_data_kernel(dp.data(), lists.data() + snappy.size() + dict_strings.size(), C, entry_off.data(),
                   entry_len.data(), &err);
  }
  if (err != ~0ull) {
    printf("error %llu %llu\n", err & 0xff, err >> 8);
    return 0;
  }
  printf("rows %lld\n", (long long)nrows);
  for (int j = 0; j < ncols; ++j) {
    const int t = spec[3 * j + 1];
    std::vector<uint8_t> chars;
    std::vector<ldf_range> ranges(std::max<int64_t>(nrows, 1));
    std::vector<int64_t> offs(std::max<int64_t>(nrows, 1));
    if (C.physical[j] == LDF_PQ_BYTE_ARRAY) {
      int64_t o = 0;
      for (int64_t r = 0; r < nrows; ++r) {
        offs[r] = o;
        o += slen[j][r];
      }
      chars.assign(std::max<int64_t>(o, 1), 0);
      blockIdx.x = 0;
      pq_copy_strings_kernel(ssrc[j].data(), slen[j].data(), offs.data(), nrows, chars.data(), ranges.data());
    }
    for (int64_t r = 0; r < nrows; ++r) {
      if (C.nullable[j] && !valid[j][r]) {
        printf("N\n");
        continue;
      }
      if (C.nullable[j] && valid[j][r] != 1) {
        printf("BADMASK\n");
        continue;
      }
      if (t == LDF_STRING) {
        printf("S ");
        for (int64_t k = ranges[r].lo; k <= ranges[r].hi; ++k) printf("%02x", chars[k]);
        printf("\n");
        continue;
      }
      uint64_t v = 0;
      memcpy(&v, data[j].data() + r * C.width[j], C.width[j]);
      if (t == LDF_FLOAT32 || t == LDF_FLOAT64) printf("F %llx\n", (unsigned long long)v);
      else if (t == LDF_INT8 || t == LDF_INT16 || t == LDF_INT32 || t == LDF_INT64 || t == LDF_TIMESTAMP_US) {
        const int w = C.width[j] * 8;
        const int64_t sv = w == 64 ? (int64_t)v : ((int64_t)(v << (64 - w)) >> (64 - w));
        printf("I %lld\n", (long long)sv);
      } else {
        printf("U %llu\n", (unsigned long long)v);
      }
    }
  }
  return 0;
}
