// Onesweep-style LSD radix sort of (key, row) pairs with 8-bit digits, used by
// `sort` (multi-key, stable) and by `hash_partition` (stable bucket order).
#pragma once

#include "table_ops.cuh"

namespace ldf {

// Rows per onesweep tile (threads x items per thread).
constexpr int kRadixThreads = 256;
constexpr int kRadixItems   = 12;
constexpr int kRadixTile    = kRadixThreads * kRadixItems;
// Resident onesweep CTAs per SM the register budget is sized for.
constexpr int kRadixMinBlocks = 4;

// How a pass obtains the digit of a row.
enum class DigitSrc : int {
  CARRIED = 0,  // byte `shift/8` of the carried key word
  COLUMN  = 1,  // load the key column at the row, transform, then byte
  CLASS   = 2,  // 0/1/2 class of the row: value / NaN / null, ordered by nulls_at_end
  BUCKET  = 3,  // hash of the key columns % nparts (then byte)
  FUSED   = 4   // byte of the fused word of several keys (FusedKey)
};

// Value transform of one sort key column into an order-preserving unsigned
// word (ascending), inverted for descending; null and NaN rows give 0 (their
// order comes from the CLASS pass).
struct SortKeyDesc {
  DCol col;
  int descending;
  int nulls_at_end;
  int key_bytes;  // bytes of the transformed word (1..8)
};

struct RadixPass {
  DigitSrc src;
  int shift;      // bit offset of the digit in the key word (FUSED: in C)
  int fused_low;  // FUSED: the pass of the fused word's low byte
  SortKeyDesc key;
  KeyCols hash_keys;  // BUCKET
  uint32_t nparts;    // BUCKET
};

// Several sort keys without nulls or floating-point values packed into one
// word, least significant key first: W = sum_k (word_k - min_k) << off_k,
// word_k the key's order-preserving word (inverted when descending) and
// min_k its minimum over the rows, at most kFusedMaxBits bits in all.  The
// pass of W's low byte loads every key at the row and carries C = W >> 8
// (64 bits); the later passes take byte shift / 8 of C.  One word for all
// the keys means that no pass gathers a key column through the permutation.
constexpr int kFuseMax      = 4;
constexpr int kFusedMaxBits = 72;
struct FusedKey {
  int n;
  SortKeyDesc key[kFuseMax];
  uint64_t min[kFuseMax];
  int off[kFuseMax];
};

// Minimum and maximum of the order-preserving words of `keys` (no nulls)
// over n rows, one read of each column.
void sort_word_ranges(const OpContext& ctx, const SortKeyDesc* keys, int nkeys, int64_t n, uint64_t* mn,
                      uint64_t* mx);

// Stable sort of rows by a list of passes (least significant first).
// Returns the permutation (row ids) in `perm` (n entries, caller allocated).
// `hist_only` variants are used by the planner.
struct RadixPlan {
  std::vector<RadixPass> passes;  // in execution order (LS first)
};

// Upfront digit histograms of every candidate pass: hist[p * 256 + d].
void radix_histograms(const OpContext& ctx, const std::vector<RadixPass>& passes, int64_t n,
                      uint32_t* d_hist, const FusedKey* fused = nullptr);

// Run the passes; `perm` receives the row order.  Passes whose histogram has a
// single bucket holding every row are skipped.
// Columns the last radix pass moves into sorted order itself: dst[j][pos] =
// src[j][row] (and the null masks), written as the pass's coalesced runs
// while the tile's source rows are still in cache.  Widths 1, 2, 4, 8, and 16
// (the ranges of a string column; its characters stay where they are).
// A payload may also carry one 16-byte record per row (`packed`, 16-byte
// aligned) holding up to kPassPayload non-nullable fixed-width values: part k
// is pwidth[k] bytes at byte offset poff[k] (a multiple of its width) and goes
// to pdst[k].  One random load per row then serves all of them.
constexpr int kPassPayload = 4;
struct RadixPayload {
  int n;
  DCol src[kPassPayload];
  void* dst[kPassPayload];
  uint8_t* dst_valid[kPassPayload];
  const ulonglong2* packed;
  int nparts;
  int pwidth[kPassPayload];
  int poff[kPassPayload];
  void* pdst[kPassPayload];
};

inline bool payload_empty(const RadixPayload& p) { return p.n == 0 && p.nparts == 0; }

// `inv` (optional, n entries): inv[row] = the row's position in the sorted
// order, written by the last pass.  `payload` (optional): columns the last
// pass writes in sorted order.  `fused`: the FusedKey of FUSED passes.
void radix_sort_rows(const OpContext& ctx, const std::vector<RadixPass>& passes, int64_t n,
                     int32_t* perm, std::vector<uint32_t>* hist_out = nullptr, int32_t* inv = nullptr,
                     const RadixPayload* payload = nullptr, const FusedKey* fused = nullptr);

}  // namespace ldf
