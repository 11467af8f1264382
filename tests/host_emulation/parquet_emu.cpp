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
  // page table and lists, as parquet_decode lays them out (chain pages first in scratch)
  std::vector<PqPage> dp(std::max(npages, 1));
  std::vector<int> snappy, chain, dict_strings, dict_chain, data_pages;
  std::vector<int64_t> soff;
  int64_t scratch_bytes = 0, nentries = 0, chain_in = 0, dict_in = 0;
  for (int p = 0; p < npages; ++p) {
    const ldf_parquet_page& h = pages[p];
    dp[p].h          = h;
    dp[p].data_bytes = h.codec == LDF_PQ_SNAPPY ? h.uncompressed : h.compressed;
    if (h.codec == LDF_PQ_SNAPPY) {
      const int64_t lv = h.kind == LDF_PQ_DATA_V2 ? h.levels_bytes : 0;
      if (C.physical[h.column] == LDF_PQ_BYTE_ARRAY && h.uncompressed - lv >= kChainMinBytes &&
          chain_in + h.compressed <= kChainMaxInput) {
        chain.push_back(p);
        chain_in += h.compressed - lv;
      } else {
        snappy.push_back(p);
      }
    }
    if (h.kind == LDF_PQ_DICT_PAGE) {
      if (C.physical[h.column] == LDF_PQ_BYTE_ARRAY) {
        dp[p].dict_entry0 = nentries;
        nentries += h.num_values;
        const int64_t bytes = dp[p].data_bytes;
        if (bytes >= kDictChainMinBytes && dict_in + bytes <= kChainMaxInput) {
          dict_chain.push_back(p);
          dict_in += bytes;
        } else {
          dict_strings.push_back(p);
        }
      }
    } else {
      data_pages.push_back(p);
    }
  }
  std::vector<ChainPage> cpages;
  std::vector<int64_t> in_b, out_b, el_b, ck_b;
  int64_t chain_elems = 0, chain_cks = 0, chain_maxu = 1, in_run = 0;
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
    chain_maxu = std::max<int64_t>(chain_maxu, h.uncompressed);
    scratch_bytes += (h.uncompressed + 15) & ~int64_t(15);
    cpages.push_back(c);
  }
  const int64_t chain_out = scratch_bytes;
  for (int p : snappy) {
    soff.push_back(scratch_bytes);
    scratch_bytes += (pages[p].uncompressed + 15) & ~int64_t(15);
  }
  std::vector<uint8_t> scratch(std::max<int64_t>(scratch_bytes, 16));
  for (size_t q = 0; q < snappy.size(); ++q) dp[snappy[q]].data = scratch.data() + soff[q];
  for (size_t q = 0; q < chain.size(); ++q) dp[chain[q]].data = scratch.data() + out_b[q];
  for (int p = 0; p < npages; ++p)
    if (pages[p].codec != LDF_PQ_SNAPPY) dp[p].data = file.data() + pages[p].offset;
  unsigned long long err = ~0ull;
  if (!chain.empty()) {  // the chain kernels: one thread runs each grid-stride loop
    blockIdx.x = 0;
    const int nc = (int)chain.size();
    const ChainBases B{in_b.data(), out_b.data(), el_b.data(), ck_b.data(), nc};
    std::vector<ChainState> st(nc);
    const int64_t cin = in_run;
    std::vector<int64_t> j0(std::max<int64_t>(cin, 1)), j1(j0.size()), j2(j0.size());
    chain_start_kernel(file.data(), cpages.data(), st.data(), nc, &err);
    chain_next_kernel(file.data(), cpages.data(), st.data(), B, cin, j0.data());
    const int64_t* jump = j0.data();
    for (int r = 0; r < kChainLog; ++r) {
      int64_t* out = (r % 2 == 0) ? j1.data() : j2.data();
      chain_double_kernel(jump, out, cin);
      jump = out;
    }
    std::vector<int64_t> ck(std::max<int64_t>(chain_cks, 1));
    chain_checkpoints_kernel(cpages.data(), st.data(), B, jump, ck.data());
    std::vector<int64_t> epos(std::max<int64_t>(chain_elems, 1)), elen(epos.size()), emeta(epos.size()),
      eoff(epos.size());
    chain_walk_kernel(file.data(), cpages.data(), st.data(), B, chain_cks, ck.data(), epos.data(), &err);
    chain_decode_kernel(file.data(), cpages.data(), st.data(), B, chain_elems, epos.data(), elen.data(),
                        emeta.data());
    int64_t run = 0;
    for (int64_t k = 0; k < chain_elems; ++k) {
      eoff[k] = run;
      run += elen[k];
    }
    std::vector<int64_t> p0(std::max<int64_t>(chain_out, 1)), p1(p0.size());
    chain_ptr_kernel(cpages.data(), st.data(), B, chain_out, eoff.data(), elen.data(), emeta.data(), p0.data(),
                     &err);
    int rounds = 1;
    while ((int64_t(1) << rounds) <= chain_maxu) ++rounds;
    int64_t* pin  = p0.data();
    int64_t* pout = p1.data();
    for (int r = 0; r < rounds; ++r) {
      chain_jump_kernel(pin, pout, chain_out);
      std::swap(pin, pout);
    }
    chain_final_kernel(file.data(), cpages.data(), B, pin, chain_out, scratch.data(), &err);
  }
  std::vector<int> lists;
  lists.insert(lists.end(), snappy.begin(), snappy.end());
  lists.insert(lists.end(), dict_strings.begin(), dict_strings.end());
  lists.insert(lists.end(), data_pages.begin(), data_pages.end());
  std::vector<int64_t> entry_off(std::max<int64_t>(nentries, 1));
  std::vector<int32_t> entry_len(std::max<int64_t>(nentries, 1));
  for (unsigned b = 0; b < snappy.size(); ++b) {
    blockIdx.x = b;
    pq_snappy_kernel(file.data(), dp.data(), lists.data(), (int)snappy.size(), scratch.data(), soff.data(), &err);
  }
  blockIdx.x = 0;
  if (!dict_strings.empty())
    pq_dict_strings_kernel(dp.data(), lists.data() + snappy.size(), (int)dict_strings.size(), entry_off.data(),
                           entry_len.data(), &err);
  if (!dict_chain.empty()) {  // the dictionary chain kernels, one thread each loop
    blockIdx.x   = 0;
    const int nc = (int)dict_chain.size();
    std::vector<DictChain> dc;
    std::vector<int64_t> in_b, ck_b;
    int64_t in_run = 0, ck_run = 0;
    for (int p : dict_chain) {
      DictChain c{};
      c.page   = p;
      c.data   = dp[p].data;
      c.n      = dp[p].data_bytes;
      c.nv     = pages[p].num_values;
      c.entry0 = dp[p].dict_entry0;
      c.ck_cap = c.nv / kChainStep + 2;
      in_b.push_back(in_run);
      ck_b.push_back(ck_run);
      in_run += c.n;
      ck_run += c.ck_cap;
      dc.push_back(c);
    }
    const ChainBases B{in_b.data(), nullptr, nullptr, ck_b.data(), nc};
    std::vector<int64_t> j0(std::max<int64_t>(in_run, 1)), j1(j0.size()), j2(j0.size()), ck(ck_run), nck(nc);
    dict_next_kernel(dc.data(), B, in_run, j0.data());
    const int64_t* jump = j0.data();
    for (int r = 0; r < kChainLog; ++r) {
      int64_t* out = (r % 2 == 0) ? j1.data() : j2.data();
      chain_double_kernel(jump, out, in_run);
      jump = out;
    }
    dict_checkpoints_kernel(dc.data(), B, jump, ck.data(), nck.data());
    dict_walk_kernel(dc.data(), B, ck_run, ck.data(), nck.data(), entry_off.data(), entry_len.data(), &err);
  }
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
      pq_copy_strings_kernel(ssrc[j].data(), slen[j].data(), offs.data(), nrows, o, chars.data(), ranges.data());
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
