// sort (stable, multi-key) and the local hash_partition.
//
// sort: reference SortTask::gpu_variant (cpp/src/sort.cu:295-379): keys in
// order, per-key ascending/descending, `nulls_at_end` for every key regardless
// of direction (the null-precedence flip of sort.cu:309-323, which makes the
// GPU agree with Arrow SortIndices, sort.cpp:324-342), head/tail `limit`
// (apply_limit, sort.cu:275-291).  The radix sort is stable, so `stable=false`
// returns the stable order too.
//
// String keys are replaced by their dense rank among the distinct strings
// (bytewise order, shorter prefix first): distinct strings come from a hash
// table, are ranked by repeated stable radix passes over 8-byte big-endian
// chunks (rank of the previous chunks as the major key), and every row then
// sorts on the uint32 rank.
//
// Output: a sort that returns the whole table lets its last radix pass move
// the first four columns into sorted order (the non-nullable fixed-width ones
// packed into one 16-byte record per row, a string key as the row id of a
// representative of its string, other strings as their ranges); the other
// columns, and the rows of a `limit`, are gathered through the permutation.
//
// hash_partition: reference task::repartition_by_hash local step
// (cpp/src/core/repartition_by_hash.cu:296-310): bucket = hash(keys) % nparts,
// rows grouped by bucket, start offsets returned; here one pass hashes the
// keys into a bucket id per row (and counts the buckets), then one stable
// radix pass on the bucket ids (two for more than 256 buckets) that also
// moves up to four columns into bucket order itself.
#include <algorithm>

#include "radix.cuh"

namespace ldf {
namespace {

constexpr uint64_t kEmpty = ~0ull;

// ---- string ranking --------------------------------------------------------
// A row's string held for the dedupe: its bytes, length and (when it fits)
// its 8-byte words, loaded once for the hash and the comparisons.
struct StrRow {
  const uint8_t* p;
  int64_t n;
  uint64_t w[4];
  bool words;
  bool valid;
};

__device__ __forceinline__ void load_str_row(const DCol& col, int64_t r, StrRow& s)
{
  s.valid = dvalid(col, r);
  s.words = false;
  if (!s.valid) return;
  s.p     = dstr_ptr(col, r);
  s.n     = dstr_len(col, r);
  s.words = str_words(col, s.p, s.n, s.w);
}

// The string of row `rb` equals `s`.
__device__ __forceinline__ bool str_row_equals(const DCol& col, const StrRow& s, int64_t rb)
{
  if (!dvalid(col, rb) || dstr_len(col, rb) != s.n) return false;
  const uint8_t* pb = dstr_ptr(col, rb);
  uint64_t wb[4];
  if (s.words && str_words(col, pb, s.n, wb))
    return wb[0] == s.w[0] && wb[1] == s.w[1] && wb[2] == s.w[2] && wb[3] == s.w[3];
  return bytes_equal(s.p, pb, s.n);
}

// Slot of each string (rows r = i * stride, i < n) in the dedupe table;
// row_slot[i] = -1 for a null row.  One row per thread per step (two in
// flight measured slower: 4.9 against 4.3 ms for 100M rows).
constexpr int kDedupeRows = 1;
__global__ void __launch_bounds__(256) str_find_insert_kernel(DCol col, int64_t n, int64_t stride,
                                                              unsigned long long* slots, uint64_t cap,
                                                              int32_t* row_slot, int* overflow)
{
  const int64_t per_iter = static_cast<int64_t>(blockDim.x) * kDedupeRows;
  for (int64_t base = blockIdx.x * per_iter; base < n; base += static_cast<int64_t>(gridDim.x) * per_iter) {
    StrRow sr[kDedupeRows];
    uint64_t h[kDedupeRows], idx[kDedupeRows], first[kDedupeRows];
#pragma unroll
    for (int j = 0; j < kDedupeRows; ++j) {
      const int64_t i = base + j * blockDim.x + threadIdx.x;
      sr[j].valid     = false;
      if (i < n) load_str_row(col, i * stride, sr[j]);
    }
#pragma unroll
    for (int j = 0; j < kDedupeRows; ++j) {
      h[j]     = sr[j].valid ? (sr[j].words ? hash_words(sr[j].w, sr[j].n) : hash_bytes(sr[j].p, sr[j].n)) : 0;
      idx[j]   = fastrange(h[j], cap);
      first[j] = sr[j].valid ? slots[idx[j]] : kEmpty;
    }
#pragma unroll
    for (int j = 0; j < kDedupeRows; ++j) {
      const int64_t i = base + j * blockDim.x + threadIdx.x;
      if (i >= n) continue;
      if (!sr[j].valid) {
        row_slot[i] = -1;
        continue;
      }
      const int64_t r      = i * stride;
      const uint64_t entry = (static_cast<uint64_t>(r) << 32) | static_cast<uint32_t>(h[j]);
      uint64_t at          = idx[j];
      int64_t found        = -1;
      for (int probe = 0; probe < 4096; ++probe) {
        // a long probe sequence means a full table: stop once any row has
        // reported the overflow (the pass is redone with a larger table)
        if ((probe & 31) == 31 && *static_cast<volatile int*>(overflow)) break;
        uint64_t v = probe == 0 ? first[j] : slots[at];
        if (v == kEmpty) {
          v = atomicCAS(&slots[at], kEmpty, entry);
          if (v == kEmpty) {
            found = static_cast<int64_t>(at);
            break;
          }
        }
        if (static_cast<uint32_t>(v) == static_cast<uint32_t>(h[j]) &&
            str_row_equals(col, sr[j], static_cast<int64_t>(v >> 32))) {
          found = static_cast<int64_t>(at);
          break;
        }
        at = at + 1 == cap ? 0 : at + 1;
      }
      if (found < 0) atomicExch(overflow, 1);
      row_slot[i] = static_cast<int32_t>(found);
    }
  }
}

// Occurrences per slot of a sample (lanes of a warp on the same slot add once:
// frequent strings would serialize on one counter).
__global__ void slot_count_kernel(const int32_t* row_slot, int64_t n, unsigned int* count)
{
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t sl = row_slot[i];
    if (sl < 0) continue;
    const uint32_t peers = __match_any_sync(__activemask(), sl);
    if ((threadIdx.x & 31) == static_cast<unsigned>(__ffs(peers) - 1))
      atomicAdd(count + sl, static_cast<unsigned>(__popc(peers)));
  }
}

// out[0] += slots seen, out[1] += slots seen once.
__global__ void distinct_stats_kernel(const unsigned int* count, int64_t cap, unsigned long long* out)
{
  unsigned long long d = 0, f1 = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < cap; i += (int64_t)gridDim.x * blockDim.x) {
    d += count[i] != 0;
    f1 += count[i] == 1;
  }
  for (int o = 16; o > 0; o >>= 1) {
    d += __shfl_xor_sync(0xffffffffu, d, o);
    f1 += __shfl_xor_sync(0xffffffffu, f1, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(out, d);
    atomicAdd(out + 1, f1);
  }
}

// slot -> dense distinct id; distinct id -> representative row.  The
// occupied slots of a warp take their ids with one atomic (order is
// irrelevant: the ids get sorted).
__global__ void str_compact_kernel(const unsigned long long* slots, uint64_t cap, int32_t* slot_id,
                                   int32_t* repr, unsigned long long* count)
{
  const int lane = threadIdx.x & 31;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  // every lane of a warp runs the same number of iterations (ballots below)
  for (int64_t base = blockIdx.x * (int64_t)blockDim.x + (threadIdx.x & ~31); base < static_cast<int64_t>(cap);
       base += stride) {
    const int64_t i       = base + lane;
    const uint64_t v      = i < static_cast<int64_t>(cap) ? slots[i] : kEmpty;
    const bool used       = v != kEmpty;
    const uint32_t ballot = __ballot_sync(0xffffffffu, used);
    if (ballot == 0) continue;
    unsigned long long first = 0;
    if (lane == 0) first = atomicAdd(count, static_cast<unsigned long long>(__popc(ballot)));
    first = __shfl_sync(0xffffffffu, first, 0);
    if (!used) continue;
    const unsigned long long d = first + __popc(ballot & ((1u << lane) - 1u));
    slot_id[i]                 = static_cast<int32_t>(d);
    repr[d]                    = static_cast<int32_t>(v >> 32);
  }
}

// chunk c (8 bytes, big-endian, zero padded) of each distinct string
__global__ void str_chunk_kernel(DCol col, const int32_t* repr, int64_t D, int chunk, uint64_t* out,
                                 uint32_t* lens)
{
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < D; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r   = repr[i];
    const int64_t len = dstr_len(col, r);
    const uint8_t* p  = dstr_ptr(col, r);
    uint64_t w        = 0;
    for (int b = 0; b < 8; ++b) {
      int64_t o = static_cast<int64_t>(chunk) * 8 + b;
      w         = (w << 8) | (o < len ? p[o] : 0);
    }
    out[i] = w;
    if (lens) lens[i] = static_cast<uint32_t>(len);
  }
}

// new rank = number of (prev rank, word) changes along the sorted order
__global__ void rank_flags_kernel(const int32_t* perm, int64_t D, const uint32_t* prev, const uint64_t* word,
                                  uint32_t* flags)
{
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < D; i += (int64_t)gridDim.x * blockDim.x) {
    if (i == 0) {
      flags[0] = 0;
      continue;
    }
    const int32_t a = perm[i - 1], b = perm[i];
    flags[i] = (prev[a] != prev[b] || word[a] != word[b]) ? 1u : 0u;
  }
}
__global__ void rank_scatter_kernel(const int32_t* perm, int64_t D, const int64_t* scanned, const uint32_t* flags,
                                    uint32_t* rank)
{
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < D; i += (int64_t)gridDim.x * blockDim.x)
    rank[perm[i]] = static_cast<uint32_t>(scanned[i] + flags[i]);
}
// rank of every row's string (0 for null rows); with rep_out, also the
// representative row of its string (-1 for null rows)
__global__ void row_rank_kernel(const int32_t* row_slot, const int32_t* slot_id, const uint32_t* rank, int64_t n,
                                uint32_t* out, const int32_t* repr, int32_t* rep_out)
{
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
    const int32_t s = row_slot[r];
    const int32_t d = s >= 0 ? slot_id[s] : -1;
    out[r]          = d >= 0 ? rank[d] : 0u;
    if (rep_out) rep_out[r] = d >= 0 ? repr[d] : -1;
  }
}
__global__ void max_len_kernel(DCol col, const int32_t* repr, int64_t D, unsigned long long* out)
{
  unsigned long long m = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < D; i += (int64_t)gridDim.x * blockDim.x)
    m = max(m, static_cast<unsigned long long>(dstr_len(col, repr[i])));
  for (int d = 16; d > 0; d >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, d));
  if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

unsigned blocks_for(int64_t n)
{
  int64_t b   = ceil_div(n, 256);
  int64_t cap = static_cast<int64_t>(num_sms()) * 8;
  return static_cast<unsigned>(b < 1 ? 1 : (b > cap ? cap : b));
}

DCol u32_col(const uint32_t* p)
{
  DCol d{};
  d.data  = p;
  d.type  = LDF_UINT32;
  d.width = 4;
  return d;
}
DCol i32_col(const int32_t* p)
{
  DCol d{};
  d.data  = p;
  d.type  = LDF_INT32;
  d.width = 4;
  return d;
}
DCol u64_col(const uint64_t* p)
{
  DCol d{};
  d.data  = p;
  d.type  = LDF_UINT64;
  d.width = 8;
  return d;
}

void add_word_passes(std::vector<RadixPass>& v, const SortKeyDesc& k)
{
  for (int b = 0; b < k.key_bytes; ++b) {
    RadixPass p{};
    p.src   = DigitSrc::COLUMN;
    p.shift = 8 * b;
    p.key   = k;
    v.push_back(p);
  }
}

}  // namespace

// Dense bytewise rank of every row's string (nulls get 0; they are ordered
// by the CLASS pass).  `out` has n entries.
// Rank of every row's string among the column's distinct strings (bytewise
// order, shorter prefix first); rep_out (optional): a row holding the same
// string for every row, -1 for null rows.
// Returns the number of distinct non-null strings D (ranks lie in [0, D)).
int64_t string_ranks(const OpContext& ctx, const DCol& col, int64_t n, uint32_t* out, int32_t* rep_out = nullptr)
{
  const Allocator& al = ctx.alloc();
  cudaStream_t s      = ctx.stream();
  if (n == 0) return 0;
  // Dedupe table size from a strided sample of 2^20 rows: distinct strings
  // estimated by GEE (Charikar et al. 2000), room for twice the estimate at
  // a load of one half (a table that stays in L2 for a dictionary of a few
  // million strings).  GEE can underestimate heavy tails; a table too small
  // for the real count overflows (inserts stop at the first full probe
  // window) and the pass is redone with room for every row.
  uint64_t cap          = static_cast<uint64_t>(2 * n + 64);
  const int64_t kSample = int64_t(1) << 20;
  if (n > 4 * kSample) {
    const int64_t stride = n / kSample;
    const uint64_t scap  = static_cast<uint64_t>(2 * kSample + 64);
    Buffer<unsigned long long> sslots(al, scap);
    Buffer<int32_t> sslot(al, kSample);
    Buffer<unsigned int> scount(al, scap);
    Buffer<unsigned long long> sm(al, 4);
    LDF_CUDA(cudaMemsetAsync(sslots.get(), 0xff, scap * 8, s));
    LDF_CUDA(cudaMemsetAsync(scount.get(), 0, scap * 4, s));
    LDF_CUDA(cudaMemsetAsync(sm.get(), 0, 32, s));
    launch("str_find_insert", str_find_insert_kernel, blocks_for(kSample), 256, 0, s, col, kSample, stride,
           sslots.get(), scap, sslot.get(), reinterpret_cast<int*>(sm.get() + 2));
    launch("slot_count", slot_count_kernel, blocks_for(kSample), 256, 0, s, static_cast<const int32_t*>(sslot.get()),
           kSample, scount.get());
    launch("distinct_stats", distinct_stats_kernel, blocks_for(static_cast<int64_t>(scap)), 256, 0, s,
           static_cast<const unsigned int*>(scount.get()), static_cast<int64_t>(scap), sm.get());
    unsigned long long h[3];
    LDF_CUDA(cudaMemcpyAsync(h, sm.get(), sizeof(h), cudaMemcpyDeviceToHost, s));
    ctx.finish();
    if (h[2] == 0) {
      const double est = std::sqrt(static_cast<double>(n) / kSample) * static_cast<double>(h[1]) +
                         static_cast<double>(h[0] - h[1]);
      const int64_t groups = std::min<int64_t>(n, static_cast<int64_t>(2 * est) + 1024);
      cap                  = static_cast<uint64_t>(2 * groups + 64);
    }
  }
  Buffer<int32_t> row_slot(al, n);
  Buffer<int64_t> misc(al, 4);
  Buffer<unsigned long long> slots;
  int* overflow              = reinterpret_cast<int*>(misc.get());
  unsigned long long* dcount = reinterpret_cast<unsigned long long*>(misc.get() + 1);
  unsigned long long* maxlen = reinterpret_cast<unsigned long long*>(misc.get() + 2);
  for (int attempt = 0;; ++attempt) {
    slots = Buffer<unsigned long long>(al, cap);
    LDF_CUDA(cudaMemsetAsync(slots.get(), 0xff, cap * 8, s));
    LDF_CUDA(cudaMemsetAsync(misc.get(), 0, 32, s));
    launch("str_find_insert", str_find_insert_kernel, blocks_for(n), 256, 0, s, col, n, int64_t(1), slots.get(), cap,
           row_slot.get(), overflow);
    int ov = 0;
    LDF_CUDA(cudaMemcpyAsync(&ov, overflow, sizeof(int), cudaMemcpyDeviceToHost, s));
    ctx.finish();
    if (ov == 0) break;
    const uint64_t full = static_cast<uint64_t>(2 * n + 64);
    if (attempt > 0 || cap >= full) fail(LDF_ERR_INTERNAL, "string dictionary overflow");
    cap = full;  // the estimate was too low: room for every row
  }
  Buffer<int32_t> slot_id(al, cap);
  Buffer<int32_t> repr(al, n);
  launch("str_compact", str_compact_kernel, blocks_for(cap), 256, 0, s, slots.get(), cap, slot_id.get(), repr.get(), dcount);
  LDF_CHECK_LAUNCH();
  const int64_t D = ctx.read_i64(misc.get() + 1);
  Buffer<uint32_t> rank(al, std::max<int64_t>(D, 1));
  if (D > 0) {
    launch("max_len", max_len_kernel, blocks_for(D), 256, 0, s, col, repr.get(), D, maxlen);
    LDF_CHECK_LAUNCH();
    const int64_t L = ctx.read_i64(misc.get() + 2);
    LDF_CUDA(cudaMemsetAsync(rank.get(), 0, D * 4, s));
    Buffer<uint64_t> word(al, D);
    Buffer<uint32_t> lens(al, D);
    Buffer<int32_t> perm(al, D);
    Buffer<uint32_t> flags(al, D);
    Buffer<int64_t> scanned(al, D);
    Buffer<int64_t> total(al, 1);
    const int nchunks = static_cast<int>((L + 7) / 8);
    // chunks, then the length as the final tie-break (shorter prefix first)
    for (int c = 0; c <= nchunks; ++c) {
      if (c < nchunks) {
        launch("str_chunk", str_chunk_kernel, blocks_for(D), 256, 0, s, col, repr.get(), D, c, word.get(), nullptr);
      } else {
        launch("str_chunk", str_chunk_kernel, blocks_for(D), 256, 0, s, col, repr.get(), D, 0, word.get(), lens.get());
        // word := length (zero-extended)
        LDF_CUDA(cudaMemsetAsync(word.get(), 0, D * 8, s));
        LDF_CUDA(cudaMemcpy2DAsync(word.get(), 8, lens.get(), 4, 4, D, cudaMemcpyDeviceToDevice, s));
      }
      LDF_CHECK_LAUNCH();
      std::vector<RadixPass> passes;
      SortKeyDesc wk{u64_col(word.get()), 0, 1, 8};
      SortKeyDesc rk{u32_col(rank.get()), 0, 1, 4};
      add_word_passes(passes, wk);
      add_word_passes(passes, rk);
      radix_sort_rows(ctx, passes, D, perm.get());
      launch("rank_flags", rank_flags_kernel, blocks_for(D), 256, 0, s, perm.get(), D, rank.get(), word.get(), flags.get());
      LDF_CHECK_LAUNCH();
      exclusive_scan_u32(flags.get(), scanned.get(), D, total.get(), ctx);
      launch("rank_scatter", rank_scatter_kernel, blocks_for(D), 256, 0, s, perm.get(), D, scanned.get(), flags.get(), rank.get());
      LDF_CHECK_LAUNCH();
      const int64_t ndistinct_ranks = ctx.read_i64(total.get()) + 1;
      if (ndistinct_ranks == D) break;
    }
  }
  launch("row_rank", row_rank_kernel, blocks_for(n), 256, 0, s, row_slot.get(), slot_id.get(), rank.get(), n, out,
         static_cast<const int32_t*>(repr.get()), rep_out);
  LDF_CHECK_LAUNCH();
  return D;
}

void gather_table(const OpContext& ctx, const ldf_column* table, int ncols, const int32_t* map, int64_t rows,
                  ldf_column* out)
{
  std::vector<DCol> fsrc;
  std::vector<ldf_column*> fdst;
  for (int j = 0; j < ncols; ++j) {
    const ldf_column& c = table[j];
    out[j]              = alloc_out_column(ctx.alloc(), c.type, rows, c.valid != nullptr);
    if (c.type == LDF_STRING) {
      gather_strings(ctx, make_dcol(c), map, rows, out[j]);
    } else {
      fsrc.push_back(make_dcol(c));
      fdst.push_back(&out[j]);
    }
  }
  gather_fixed_columns(ctx, fsrc.data(), map, rows, fdst.data(), static_cast<int>(fsrc.size()));
}

namespace {
// Columns that the last radix pass moves itself, up to kPassPayload of them in
// table order (written with the pass's runs while the tile's rows are in
// cache, instead of gathered through the permutation afterwards): fixed
// widths straight into the allocated outputs, a string column's ranges (and
// mask) into scratch in output order, from which move_strings_in_order then
// copies its characters.  A string column with representative rows (rep[j]:
// for every row, a row holding the same string, -1 for null) moves those
// 4-byte row ids instead, and its strings are then copied from the
// representatives: as many source strings as distinct values, which stay in
// L2 when there are few.
struct PassMove {
  RadixPayload pay{};
  int col[kPassPayload];              // table column of each payload entry
  bool by_rep[kPassPayload];          // the entry moves representative rows
  std::vector<char> moved;            // per table column
  std::vector<Buffer<uint8_t>> scratch;
};

void plan_pass_move(const Allocator& al, const ldf_column* table, int ncols, int64_t n, ldf_column* out,
                    PassMove& m, const std::vector<const int32_t*>* rep = nullptr)
{
  m.moved.assign(ncols, 0);
  for (int j = 0; j < ncols && m.pay.n < kPassPayload; ++j) {
    const ldf_column& c = table[j];
    const int q         = m.pay.n++;
    m.col[q]            = j;
    m.by_rep[q]         = false;
    m.moved[j]          = 1;
    m.pay.src[q]        = make_dcol(c);
    if (c.type == LDF_STRING && rep && (*rep)[j]) {
      m.by_rep[q]        = true;
      m.pay.src[q]       = i32_col((*rep)[j]);
      m.scratch.emplace_back(al, std::max<int64_t>(n, 1) * sizeof(int32_t));
      m.pay.dst[q]       = m.scratch.back().get();
      m.pay.dst_valid[q] = nullptr;
    } else if (c.type == LDF_STRING) {
      m.scratch.emplace_back(al, std::max<int64_t>(n, 1) * sizeof(ldf_range));
      m.pay.dst[q]       = m.scratch.back().get();
      m.pay.dst_valid[q] = nullptr;
      if (c.valid) {
        m.scratch.emplace_back(al, std::max<int64_t>(n, 1));
        m.pay.dst_valid[q] = m.scratch.back().get();
      }
    } else {
      m.pay.dst[q]       = out[j].data;
      m.pay.dst_valid[q] = out[j].valid;
    }
  }
}

struct PackArgs {
  const void* src[kPassPayload];
  int width[kPassPayload];
  int off[kPassPayload];
  int nparts;
};

constexpr int kPackRows = 4;  // rows per thread, their loads in flight together

__device__ __forceinline__ unsigned long long load_part(const void* p, int width, int64_t r)
{
  switch (width) {
    case 1: return static_cast<const uint8_t*>(p)[r];
    case 2: return static_cast<const uint16_t*>(p)[r];
    case 4: return static_cast<const uint32_t*>(p)[r];
    default: return static_cast<const unsigned long long*>(p)[r];
  }
}

// rec[r] = the parts of row r at their byte offsets (in order over the rows)
__global__ void __launch_bounds__(256) pack_records_kernel(PackArgs a, int64_t n, ulonglong2* rec)
{
  const int64_t per = static_cast<int64_t>(blockDim.x) * kPackRows;
  for (int64_t base = blockIdx.x * per; base < n; base += static_cast<int64_t>(gridDim.x) * per) {
    unsigned long long v[kPassPayload][kPackRows];
#pragma unroll
    for (int q = 0; q < kPassPayload; ++q)
#pragma unroll
      for (int k = 0; k < kPackRows; ++k) {
        const int64_t r = base + k * blockDim.x + threadIdx.x;
        v[q][k]         = q < a.nparts && r < n ? load_part(a.src[q], a.width[q], r) : 0;
      }
#pragma unroll
    for (int k = 0; k < kPackRows; ++k) {
      const int64_t r = base + k * blockDim.x + threadIdx.x;
      if (r >= n) continue;
      unsigned long long w[2] = {0, 0};
#pragma unroll
      for (int q = 0; q < kPassPayload; ++q)
        if (q < a.nparts) w[a.off[q] >> 3] |= v[q][k] << ((a.off[q] & 7) * 8);
      rec[r] = make_ulonglong2(w[0], w[1]);
    }
  }
}

// The payload a pass over rows in random order runs with: the non-nullable
// fixed-width entries of `pay` (representative rows included) packed into
// one 16-byte record per row while they fit, widest first so that every part
// sits at an offset that is a multiple of its width, and the other entries
// as they are.  The pass then loads one record per row instead of one value
// per column; packing costs one read and write of the records in order.
RadixPayload pack_payload(const OpContext& ctx, const RadixPayload& pay, int64_t n, Buffer<ulonglong2>& rec)
{
  int order[kPassPayload];
  int m = 0;
  for (int q = 0; q < pay.n; ++q) {
    const DCol& c = pay.src[q];
    if (c.type != LDF_STRING && c.width <= 8 && c.valid == nullptr && pay.dst_valid[q] == nullptr) order[m++] = q;
  }
  std::stable_sort(order, order + m, [&](int x, int y) { return pay.src[x].width > pay.src[y].width; });
  RadixPayload out{};
  PackArgs pa{};
  bool in_rec[kPassPayload] = {};
  int used                  = 0;
  for (int i = 0; i < m; ++i) {
    const int q = order[i];
    const int w = pay.src[q].width;
    if (used + w > 16) continue;
    in_rec[q]              = true;
    pa.src[pa.nparts]      = pay.src[q].data;
    pa.width[pa.nparts]    = w;
    pa.off[pa.nparts]      = used;
    out.pdst[pa.nparts]    = pay.dst[q];
    out.pwidth[pa.nparts]  = w;
    out.poff[pa.nparts]    = used;
    used += w;
    ++pa.nparts;
  }
  if (pa.nparts < 2 || n == 0) return pay;
  out.nparts = pa.nparts;
  for (int q = 0; q < pay.n; ++q) {
    if (in_rec[q]) continue;
    out.src[out.n]       = pay.src[q];
    out.dst[out.n]       = pay.dst[q];
    out.dst_valid[out.n] = pay.dst_valid[q];
    ++out.n;
  }
  rec = Buffer<ulonglong2>(ctx.alloc(), static_cast<size_t>(n));
  launch("pack_records", pack_records_kernel, blocks_for(ceil_div(n, int64_t(kPackRows))), 256, 0, ctx.stream(), pa, n,
         rec.get());
  LDF_CHECK_LAUNCH();
  out.packed = rec.get();
  return out;
}

void move_strings_in_order(const OpContext& ctx, const ldf_column* table, const PassMove& m, int64_t n,
                           ldf_column* out)
{
  for (int q = 0; q < m.pay.n; ++q) {
    if (m.by_rep[q]) {
      gather_strings(ctx, make_dcol(table[m.col[q]]), static_cast<const int32_t*>(m.pay.dst[q]), n, out[m.col[q]]);
      continue;
    }
    const DCol& src = m.pay.src[q];
    if (src.type != LDF_STRING) continue;
    DCol ordered  = src;  // same characters; ranges and mask already in output order
    ordered.data  = m.pay.dst[q];
    ordered.valid = m.pay.dst_valid[q];
    gather_strings(ctx, ordered, nullptr, n, out[m.col[q]]);
  }
}
}  // namespace

void sort_table(const ldf_column* table, int ncols, const int32_t* keys, const uint8_t* ascending, int nkeys,
                bool nulls_at_end, int64_t limit, ldf_column* out, const OpContext& ctx)
{
  if (nkeys < 1) fail(LDF_ERR_INVALID_ARGUMENT, "must sort along at least one column");
  for (int j = 0; j < nkeys; ++j) {
    LDF_REQUIRE(keys[j] >= 0 && keys[j] < ncols, "sort key column out of range");
    for (int q = 0; q < j; ++q) LDF_REQUIRE(keys[q] != keys[j], "duplicate sort keys");
  }
  const Allocator& al = ctx.alloc();
  const int64_t n     = ncols > 0 ? table[0].size : 0;
  LDF_REQUIRE(n < (int64_t(1) << 31), "tables of 2^31 rows or more per task are not supported");
  int64_t first = 0, rows = n;
  if (limit != INT64_MIN && (limit < 0 ? -limit : limit) < n) {
    if (limit < 0) {
      first = n + limit;
      rows  = -limit;
    } else {
      rows = limit;
    }
  }
  const bool whole = rows == n;
  std::vector<Buffer<uint32_t>> ranks;
  std::vector<Buffer<int32_t>> reps;                   // representative rows of string keys
  std::vector<const int32_t*> rep_of(ncols, nullptr);  // per table column
  std::vector<RadixPass> passes;
  std::vector<SortKeyDesc> kd;  // least significant key first
  std::vector<int64_t> ndistinct;  // string keys: distinct strings (their ranks' range); -1 otherwise
  bool fusable = nkeys >= 2 && nkeys <= kFuseMax;
  for (int j = nkeys - 1; j >= 0; --j) {
    const ldf_column& c = table[keys[j]];
    SortKeyDesc k{};
    k.col          = make_dcol(c);
    k.descending   = ascending[j] ? 0 : 1;
    k.nulls_at_end = nulls_at_end ? 1 : 0;
    if (c.type == LDF_STRING) {
      ranks.emplace_back(al, std::max<int64_t>(n, 1));
      int32_t* rep = nullptr;
      if (whole && keys[j] < kPassPayload) {  // a column the last pass moves
        reps.emplace_back(al, std::max<int64_t>(n, 1));
        rep            = reps.back().get();
        rep_of[keys[j]] = rep;
      }
      ndistinct.push_back(string_ranks(ctx, k.col, n, ranks.back().get(), rep));
      DCol rc  = u32_col(ranks.back().get());
      rc.valid = c.valid;
      k.col    = rc;
    } else {
      ndistinct.push_back(-1);
    }
    k.key_bytes = k.col.width;
    if (c.valid != nullptr || is_float(c.type)) fusable = false;  // those need CLASS passes
    kd.push_back(k);
  }
  // Keys without nulls or floats whose value ranges fit one word of at most
  // kFusedMaxBits bits are sorted on that word: its first pass loads every key
  // in input order, and no pass gathers a key through the permutation.
  FusedKey fk{};
  bool fused = false;
  if (fusable && n > 0) {
    // ranges: string ranks lie in [0, D) (inverted when descending); the other
    // keys' ranges come from one read of their columns
    uint64_t mn[kFuseMax], mx[kFuseMax];
    std::vector<SortKeyDesc> scan;
    std::vector<int> scan_of;
    for (size_t k = 0; k < kd.size(); ++k) {
      if (ndistinct[k] >= 0) {
        const uint64_t top = std::max<int64_t>(ndistinct[k], 1) - 1;
        mn[k]              = kd[k].descending ? 0xffffffffull - top : 0;
        mx[k]              = kd[k].descending ? 0xffffffffull : top;
      } else {
        scan.push_back(kd[k]);
        scan_of.push_back(static_cast<int>(k));
      }
    }
    if (!scan.empty()) {
      uint64_t smn[kFuseMax], smx[kFuseMax];
      sort_word_ranges(ctx, scan.data(), static_cast<int>(scan.size()), n, smn, smx);
      for (size_t q = 0; q < scan.size(); ++q) {
        mn[scan_of[q]] = smn[q];
        mx[scan_of[q]] = smx[q];
      }
    }
    int bits = 0;
    fk.n     = static_cast<int>(kd.size());
    for (int k = 0; k < fk.n; ++k) {
      const uint64_t span = mx[k] - mn[k];
      int b               = 0;
      while (b < 64 && (span >> b) != 0) ++b;
      fk.key[k] = kd[k];
      fk.min[k] = mn[k];
      fk.off[k] = bits;
      bits += b;
    }
    if (bits <= kFusedMaxBits) {
      fused = true;
      for (int q = 0; 8 * q < bits; ++q) {
        RadixPass p{};
        p.src       = DigitSrc::FUSED;
        p.fused_low = q == 0 ? 1 : 0;
        p.shift     = q == 0 ? 0 : 8 * (q - 1);  // byte q of W is byte q - 1 of C = W >> 8
        passes.push_back(p);
      }
    }
  }
  if (!fused) {
    for (size_t q = 0; q < kd.size(); ++q) {
      const ldf_column& c = table[keys[nkeys - 1 - static_cast<int>(q)]];
      add_word_passes(passes, kd[q]);
      if (c.valid != nullptr || is_float(c.type)) {
        RadixPass p{};
        p.src = DigitSrc::CLASS;
        p.key = kd[q];
        passes.push_back(p);
      }
    }
  }
  const FusedKey* fkp = fused ? &fk : nullptr;
  Buffer<int32_t> perm(al, std::max<int64_t>(n, 1));
  if (!whole) {
    radix_sort_rows(ctx, passes, n, perm.get(), nullptr, nullptr, nullptr, fkp);
    gather_table(ctx, table, ncols, perm.get() + first, rows, out);
    ctx.finish();
    return;
  }
  // the whole table: the last pass moves the first kPassPayload columns
  // (string keys as their representative rows), the rest are gathered
  // through the permutation
  for (int j = 0; j < ncols; ++j) out[j] = alloc_out_column(al, table[j].type, n, table[j].valid != nullptr);
  PassMove mv;
  plan_pass_move(al, table, ncols, n, out, mv, &rep_of);
  Buffer<ulonglong2> rec;
  const RadixPayload pay = pack_payload(ctx, mv.pay, n, rec);
  radix_sort_rows(ctx, passes, n, perm.get(), nullptr, nullptr, &pay, fkp);
  move_strings_in_order(ctx, table, mv, n, out);
  std::vector<DCol> fsrc;
  std::vector<ldf_column*> fdst;
  for (int j = 0; j < ncols; ++j) {
    if (mv.moved[j]) continue;
    if (table[j].type == LDF_STRING) {
      gather_strings(ctx, make_dcol(table[j]), perm.get(), n, out[j]);
    } else {
      fsrc.push_back(make_dcol(table[j]));
      fdst.push_back(&out[j]);
    }
  }
  gather_fixed_columns(ctx, fsrc.data(), perm.get(), n, fdst.data(), static_cast<int>(fsrc.size()));
  ctx.finish();
}

namespace {
// Bucket id of every row (hash of the key columns % nparts), written once so
// that the radix passes read 4 bytes per row instead of hashing the keys
// again, and the bucket sizes.
__global__ void bucket_ids_kernel(KeyCols k, int64_t n, uint32_t nparts, uint32_t* ids, unsigned long long* counts)
{
  extern __shared__ unsigned int sc[];
  const bool use_smem = nparts <= 8192;
  if (use_smem)
    for (uint32_t i = threadIdx.x; i < nparts; i += blockDim.x) sc[i] = 0;
  __syncthreads();
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t b = static_cast<uint32_t>(key_bits<KeyMode::GEN>(k, r) % nparts);
    ids[r]           = b;
    if (use_smem) atomicAdd(&sc[b], 1u);
    else atomicAdd(&counts[b], 1ull);
  }
  __syncthreads();
  if (use_smem)
    for (uint32_t i = threadIdx.x; i < nparts; i += blockDim.x)
      if (sc[i]) atomicAdd(&counts[i], static_cast<unsigned long long>(sc[i]));
}
}  // namespace

void hash_partition(const ldf_column* table, int ncols, const int32_t* keys, int nkeys, int nparts,
                    ldf_column* out, int64_t* offsets, const OpContext& ctx)
{
  LDF_REQUIRE(nparts >= 1, "nparts must be positive");
  KeyCols k       = make_keys(table, ncols, keys, nkeys);
  const int64_t n = ncols > 0 ? table[0].size : 0;
  LDF_REQUIRE(n < (int64_t(1) << 31), "tables of 2^31 rows or more per task are not supported");
  const Allocator& al = ctx.alloc();
  cudaStream_t s      = ctx.stream();
  // bucket id of every row, and the bucket sizes
  Buffer<uint32_t> ids(al, std::max<int64_t>(n, 1));
  Buffer<unsigned long long> counts(al, nparts);
  LDF_CUDA(cudaMemsetAsync(counts.get(), 0, static_cast<size_t>(nparts) * 8, s));
  if (n > 0) {
    size_t smem = nparts <= 8192 ? static_cast<size_t>(nparts) * 4 : 0;
    launch("bucket_ids", bucket_ids_kernel, blocks_for(n), 256, smem, s, k, n, static_cast<uint32_t>(nparts), ids.get(),
           counts.get());
    LDF_CHECK_LAUNCH();
  }
  // stable radix passes over the bucket ids (a uint32 column, no nulls)
  ldf_column idc{};
  idc.type = LDF_UINT32;
  idc.size = n;
  idc.data = ids.get();
  std::vector<RadixPass> passes;
  for (uint64_t span = 1, shift = 0; span < static_cast<uint64_t>(nparts); span <<= 8, shift += 8) {
    RadixPass p{};
    p.src              = DigitSrc::COLUMN;
    p.shift            = static_cast<int>(shift);
    p.key.col          = make_dcol(idc);
    p.key.descending   = 0;
    p.key.nulls_at_end = 1;
    p.key.key_bytes    = 4;
    passes.push_back(p);
  }
  // The radix pass itself moves up to kPassPayload columns into bucket order
  // (one pass over the rows in input order, so its reads are sequential).
  // Any further fixed-width columns are scattered through the inverse
  // permutation, further string columns gathered.
  for (int j = 0; j < ncols; ++j) out[j] = alloc_out_column(al, table[j].type, n, table[j].valid != nullptr);
  PassMove mv;
  plan_pass_move(al, table, ncols, n, out, mv);
  std::vector<DCol> fsrc;
  std::vector<ldf_column*> fdst;
  for (int j = 0; j < ncols; ++j)
    if (!mv.moved[j] && table[j].type != LDF_STRING) {
      fsrc.push_back(make_dcol(table[j]));
      fdst.push_back(&out[j]);
    }
  Buffer<int32_t> perm(al, std::max<int64_t>(n, 1));
  Buffer<int32_t> inv;
  if (!fsrc.empty()) inv = Buffer<int32_t>(al, std::max<int64_t>(n, 1));
  radix_sort_rows(ctx, passes, n, perm.get(), nullptr, fsrc.empty() ? nullptr : inv.get(), &mv.pay);
  std::vector<unsigned long long> h(nparts);
  LDF_CUDA(cudaMemcpyAsync(h.data(), counts.get(), static_cast<size_t>(nparts) * 8, cudaMemcpyDeviceToHost, s));
  scatter_fixed_columns(ctx, fsrc.data(), inv.get(), n, fdst.data(), static_cast<int>(fsrc.size()));
  move_strings_in_order(ctx, table, mv, n, out);
  for (int j = 0; j < ncols; ++j)
    if (table[j].type == LDF_STRING && !mv.moved[j]) gather_strings(ctx, make_dcol(table[j]), perm.get(), n, out[j]);
  ctx.finish();
  int64_t acc = 0;
  for (int b = 0; b < nparts; ++b) {
    offsets[b] = acc;
    acc += static_cast<int64_t>(h[b]);
  }
  offsets[nparts] = acc;
}

}  // namespace ldf
