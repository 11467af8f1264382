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
//  1. build   open-addressing table over the rhs keys, linear probing, load
//             factor 0.5, 8-byte slots {row, key32 | hash tag} (16-byte
//             {key64, row} for 8-byte keys).  Nullable single keys with
//             nulls_equal keep their null rows in a separate "null list".
//  2. unique? one self-probe over the build keys.  Unique build keys bound
//             the output by the probe size, so the probe runs ONCE with a
//             decoupled look-back for output offsets; otherwise a count pass
//             sizes the output exactly first.
//  3. probe   tiles of 256 threads x 4 rows: probe, block scan of match counts,
//             look-back, then the fixed-width output columns are written
//             directly from the probe kernel (the gather is fused: no gather
//             maps for fixed-width columns).  String output columns go
//             through int32 gather maps and a string gather.
//  4. FULL    unmatched rhs rows (never touched by a probe) are compacted and
//             appended after the probe output.
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

// Device-side view of the build table.
struct BuildTable {
  KeyCols bk;             // build keys (rhs)
  void* slots;            // uint64_t[cap] (K32, GEN) or Slot16[cap] (K64)
  uint64_t cap;
  const int32_t* null_list;  // rows with a null single key (nulls_equal, K32/K64)
  const int64_t* null_count;
  int nulls_equal;
};

__device__ __forceinline__ uint64_t next_slot(uint64_t i, uint64_t cap) { return i + 1 == cap ? 0 : i + 1; }

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
    uint64_t idx = fastrange(h, t.cap);
    if (M == KeyMode::K64) {
      Slot16* s = static_cast<Slot16*>(t.slots);
      while (true) {
        unsigned long long old = atomicCAS(reinterpret_cast<unsigned long long*>(&s[idx].row),
                                           kEmpty64, static_cast<unsigned long long>(r));
        if (old == kEmpty64) {
          s[idx].key = kb;
          break;
        }
        idx = next_slot(idx, t.cap);
      }
    } else {
      uint32_t tag   = M == KeyMode::GEN ? static_cast<uint32_t>(h) : static_cast<uint32_t>(kb);
      uint64_t entry = (static_cast<uint64_t>(r) << 32) | tag;
      uint64_t* s    = static_cast<uint64_t*>(t.slots);
      while (atomicCAS(reinterpret_cast<unsigned long long*>(&s[idx]), kEmpty64,
                       static_cast<unsigned long long>(entry)) != kEmpty64)
        idx = next_slot(idx, t.cap);
    }
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
  uint64_t kb  = key_bits<M>(pk, r);
  uint64_t h   = M == KeyMode::GEN ? kb : mix64(kb);
  uint64_t idx = fastrange(h, t.cap);
  if (M == KeyMode::K64) {
    const Slot16* s = static_cast<const Slot16*>(t.slots);
    while (true) {
      Slot16 v = s[idx];
      if (v.row == kEmpty64) return;
      if (v.key == kb && !f(static_cast<int64_t>(v.row))) return;
      idx = next_slot(idx, t.cap);
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
      idx = next_slot(idx, t.cap);
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
  const int64_t* tile_offsets;  // write pass with known offsets (null -> look-back)
  uint64_t* status;
  unsigned long long* counter;
  int64_t* total;  // device: number of rows written by the probe
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

// COUNT: per-tile output counts.  WRITE: probe again (or use the single match
// of a unique build side) and write output rows at the tile's offset.
template <KeyMode M, bool WRITE, bool UNIQUE>
__global__ void __launch_bounds__(kProbeThreads) probe_kernel(ProbeArgs a)
{
  __shared__ int64_t s_scan[kProbeThreads / 32 + 1];
  __shared__ int64_t s_tile;
  __shared__ uint64_t s_prefix;
  const bool lookback = WRITE && a.tile_offsets == nullptr;
  const int64_t tile  = lookback ? next_tile_id(a.counter, &s_tile) : static_cast<int64_t>(blockIdx.x);
  const int64_t base  = tile * kProbeTile;

  int m[kProbeItems];
  int64_t first[kProbeItems];
  int64_t cnt = 0;
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
    if (lookback) {
      s_prefix = lookback_exclusive(a.status, tile, static_cast<uint64_t>(tile_total), a.err);
      if (tile == static_cast<int64_t>(gridDim.x) - 1) *a.total = static_cast<int64_t>(s_prefix) + tile_total;
    } else {
      s_prefix = static_cast<uint64_t>(a.tile_offsets[tile]);
    }
  }
  __syncthreads();
  int64_t pos = static_cast<int64_t>(s_prefix) + excl;
  const int jt = a.join_type;
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
      if (a.matched) a.matched[first[i]] = 1;
    } else {
      for_each_match<M>(a.t, a.pk, r, [&](int64_t b) {
        emit(a, pos++, r, b);
        if (a.matched) a.matched[b] = 1;
        return true;
      });
    }
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
  uint64_t* status;
  unsigned long long* counter;
  int64_t* total;
  int* err;
};

__global__ void __launch_bounds__(kProbeThreads) full_tail_kernel(TailArgs a)
{
  __shared__ int64_t s_scan[kProbeThreads / 32 + 1];
  __shared__ int64_t s_tile;
  __shared__ uint64_t s_prefix;
  const int64_t tile = next_tile_id(a.counter, &s_tile);
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
  if (threadIdx.x == 0) {
    s_prefix = lookback_exclusive(a.status, tile, static_cast<uint64_t>(tot), a.err);
    if (tile == static_cast<int64_t>(gridDim.x) - 1) *a.total = static_cast<int64_t>(s_prefix) + tot;
  }
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

template <KeyMode M>
void run_join(const OpContext& ctx, const KeyCols& pk, int64_t n_probe, const KeyCols& bk,
              int64_t n_build, int join_type, bool nulls_equal, OutSpec lo, OutSpec ro,
              const std::vector<ldf_column*>& out_cols, const std::vector<int>& out_is_lhs,
              const std::vector<DCol>& out_src, const std::vector<int>& out_types,
              const std::vector<int>& out_nullable)
{
  const Allocator& al = ctx.alloc();
  cudaStream_t s      = ctx.stream();

  // ---- build ---------------------------------------------------------------
  BuildTable t{};
  t.bk          = bk;
  t.nulls_equal = nulls_equal ? 1 : 0;
  t.cap         = static_cast<uint64_t>(std::max<int64_t>(2 * n_build, 64));
  const size_t slot_bytes = M == KeyMode::K64 ? sizeof(Slot16) : sizeof(uint64_t);
  Buffer<uint8_t> slots(al, t.cap * slot_bytes);
  LDF_CUDA(cudaMemsetAsync(slots.get(), 0xff, t.cap * slot_bytes, s));
  t.slots = slots.get();

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
  if (n_build > 0) {
    launch("build", build_kernel<M>, grid_stride_blocks(n_build, 256), 256, 0, s, t, n_build);
    LDF_CHECK_LAUNCH();
  }

  // ---- uniqueness ----------------------------------------------------------
  bool unique = true;
  if (n_build > 1) {
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

  if (tiles > 0) {
    if (unique) {
      StatusBuf sb(ctx, tiles);
      a.status  = sb.status;
      a.counter = sb.counter;
      a.total   = d_total.get();
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
    StatusBuf sb(ctx, btiles);
    TailArgs ta{};
    ta.matched  = matched.get();
    ta.n_build  = n_build;
    ta.base_pos = d_total.get();
    ta.lo       = a.lo;
    ta.ro       = a.ro;
    ta.lmap     = a.lmap;
    ta.rmap     = a.rmap;
    ta.status   = sb.status;
    ta.counter  = sb.counter;
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

  switch (key_mode(bk)) {
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
