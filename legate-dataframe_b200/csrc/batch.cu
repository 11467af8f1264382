// Batched execution of many small joins and groupbys in one CUDA-graph replay.
//
// A batch is a list of requests (int64-key groupby SUM + COUNT(*), or int64-key
// inner join with one int64 payload per side) whose inputs are already on the
// device.  The engine turns the batch into a work list of row tiles and runs
// three persistent kernels over it, each a grid of (#SMs x k) CTAs that loop
// over items:
//   1. init     fill every request's hash table with the empty marker;
//   2. build    groupby rows aggregate into their request's table; join rhs
//               rows insert into their request's multimap;
//   3. emit     join lhs rows probe and write matches; groupby table slots are
//               compacted into the request's output.
// Outputs go through per-request cursors (per-warp aggregated atomics), so row
// order is unspecified; float sums use the exact fixed-point chunks of the
// groupby path, so values do not depend on which requests share a batch.
// The kernels read the item count and descriptors from device memory, so the
// whole sequence (descriptor upload, 3 kernels, status download) is captured
// once into a CUDA graph and replayed for every batch.  Every wait is bounded;
// a request whose table or output overflows its reservation is flagged and its
// caller re-runs it on the per-op path.
#include <cstring>

#include "scan.cuh"

namespace ldf {
namespace {

constexpr uint64_t kEmptyKey = 0x7ff4dead7ff4beefull;  // empty table key word
constexpr uint64_t kEmptyRow = ~0ull;
constexpr int kBThreads      = 256;
constexpr int kMaxProbeB     = 2048;
constexpr int64_t kMinTile   = 1024;  // smallest row tile of a work item

// flags
enum : int32_t { RQ_GROUPBY = 0, RQ_JOIN = 1 };
enum : int32_t { V_INT64 = 0, V_FLOAT64 = 1 };

struct ItemD {
  int32_t req;
  int32_t kind;  // 0 = table init, 1 = build/aggregate rows, 2 = emit (probe rows / table slots)
  int64_t begin, end;
};

// groupby slot record (words): key, count, sum (1 word int64, 6 words float64)
__device__ __forceinline__ int gb_stride(int vtype) { return vtype == V_FLOAT64 ? 8 : 3; }

__device__ __forceinline__ uint64_t bmix(uint64_t x)
{
  x ^= x >> 33;
  x *= 0xff51afd7ed558ccdull;
  x ^= x >> 33;
  x *= 0xc4ceb9fe1a85ec53ull;
  x ^= x >> 33;
  return x;
}

__device__ __forceinline__ void bred_add(unsigned long long* p, uint64_t v)
{
  asm volatile("red.relaxed.gpu.global.add.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// exact float64 -> fixed-point chunks (2^-96 LSB, 32-bit chunks), as in groupby
__device__ __forceinline__ bool bfixed(double x, uint64_t& m, int& s, bool& neg)
{
  const uint64_t b = __double_as_longlong(x);
  const int e      = static_cast<int>((b >> 52) & 0x7ff);
  neg              = (b >> 63) != 0;
  if (e == 0 && (b << 1) == 0) {
    m = 0;
    s = 0;
    return true;
  }
  const int E = e - 1023;
  if (e == 0 || E < -44 || E >= 95) return false;
  m = (b & ((1ull << 52) - 1)) | (1ull << 52);
  s = E + 44;
  return true;
}

// Warp-aggregated cursor: each lane with `want` gets a distinct slot.
__device__ __forceinline__ unsigned long long warp_claim(unsigned long long* cursor, bool want)
{
  const unsigned mask = __activemask();
  const unsigned w    = __ballot_sync(mask, want);
  if (w == 0) return 0;
  const int lane   = threadIdx.x & 31;
  const int leader = __ffs(w) - 1;
  unsigned long long base = 0;
  if (lane == leader) base = atomicAdd(cursor, static_cast<unsigned long long>(__popc(w)));
  base = __shfl_sync(mask, base, leader);
  return base + __popc(w & ((1u << lane) - 1u));
}

}  // namespace

// ---- public device-side request (mirrors ldf_batch_request) ----------------
struct BReq {
  int32_t kind, vtype;
  int64_t n, m;  // groupby: n rows; join: n lhs (probe) rows, m rhs (build) rows
  const long long* k1;
  const void* v1;
  const long long* k2;
  const long long* v2;
  const uint8_t* vvalid;
  unsigned long long* table;
  uint64_t cap;
  long long* o0;
  void* o1;
  long long* o2;
  long long* o3;
  int64_t out_cap;
  unsigned long long* status;  // [0] output rows, [1] overflow
};
static_assert(sizeof(BReq) % 8 == 0, "BReq is staged as 8-byte words");

namespace {

struct BatchArgs {
  const BReq* reqs;
  const ItemD* items;
  const int* nitems;  // device: number of items of this kind list
  int* err;
};

// Copy the batch descriptors (requests, the three item lists and their
// counts) from mapped pinned host memory to the device; only used entries.
struct StageArgs {
  const BReq* h_reqs;
  const ItemD* h_items;
  const int* h_counts;  // [0..2] item counts, [3] requests
  BReq* d_reqs;
  ItemD* d_items;
  int* d_counts;
  int max_items;
};
__global__ void batch_stage_kernel(StageArgs a)
{
  const int nreq = a.h_counts[3];
  const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x, nth = (int64_t)gridDim.x * blockDim.x;
  const int words = static_cast<int>(sizeof(BReq) / 8);
  for (int64_t i = tid; i < static_cast<int64_t>(nreq) * words; i += nth)
    reinterpret_cast<unsigned long long*>(a.d_reqs)[i] = reinterpret_cast<const unsigned long long*>(a.h_reqs)[i];
  for (int l = 0; l < 3; ++l) {
    const int cnt = a.h_counts[l];
    for (int64_t i = tid; i < cnt; i += nth) a.d_items[l * a.max_items + i] = a.h_items[l * a.max_items + i];
    if (tid == 0) a.d_counts[l] = cnt;
  }
}

__global__ void __launch_bounds__(kBThreads) batch_init_kernel(BatchArgs a)
{
  const int nit = *a.nitems;
  for (int it = blockIdx.x; it < nit; it += gridDim.x) {
    const ItemD w = a.items[it];
    const BReq& q = a.reqs[w.req];
    if (q.kind == RQ_GROUPBY) {
      const int st = gb_stride(q.vtype);
      for (int64_t i = w.begin + threadIdx.x; i < w.end; i += blockDim.x) {
        unsigned long long* s = q.table + i * st;
        s[0] = kEmptyKey;
        for (int j = 1; j < st; ++j) s[j] = 0;
      }
    } else {
      for (int64_t i = w.begin + threadIdx.x; i < w.end; i += blockDim.x) {
        q.table[2 * i]     = 0;
        q.table[2 * i + 1] = kEmptyRow;
      }
    }
    if (w.begin == 0 && threadIdx.x == 0) {
      q.status[0] = 0;
      q.status[1] = 0;
    }
  }
}

__global__ void __launch_bounds__(kBThreads) batch_build_kernel(BatchArgs a)
{
  const int nit = *a.nitems;
  for (int it = blockIdx.x; it < nit; it += gridDim.x) {
    const ItemD w = a.items[it];
    const BReq& q = a.reqs[w.req];
    if (q.kind == RQ_GROUPBY) {
      const int st = gb_stride(q.vtype);
      for (int64_t r = w.begin + threadIdx.x; r < w.end; r += blockDim.x) {
        const uint64_t key = static_cast<uint64_t>(__ldg(q.k1 + r));
        // the empty-marker key value lives in the extra slot `cap`
        uint64_t idx = key == kEmptyKey ? q.cap : __umul64hi(bmix(key), q.cap);
        bool ok      = key == kEmptyKey;
        for (int probe = 0; !ok && probe < kMaxProbeB; ++probe) {
          unsigned long long* s = q.table + idx * st;
          unsigned long long v  = s[0];
          if (v == kEmptyKey) v = atomicCAS(s, kEmptyKey, key);
          if (v == kEmptyKey || v == key) {
            ok = true;
            break;
          }
          idx = idx + 1 == q.cap ? 0 : idx + 1;
        }
        if (!ok) {
          atomicExch(reinterpret_cast<unsigned long long*>(q.status + 1), 1ull);
          continue;
        }
        unsigned long long* s = q.table + idx * st;
        if (key == kEmptyKey) s[0] = kEmptyKey ^ 1ull;  // mark the extra slot used (key restored at emit)
        if (q.vvalid != nullptr && __ldg(q.vvalid + r) == 0) continue;  // null value: group only
        bred_add(s + 1, 1);
        if (q.vtype == V_INT64) {
          bred_add(s + 2, static_cast<uint64_t>(__ldg(static_cast<const long long*>(q.v1) + r)));
        } else {
          const double x = __ldg(static_cast<const double*>(q.v1) + r);
          uint64_t m;
          int sh;
          bool neg;
          if (bfixed(x, m, sh, neg)) {
            if (m) {
              const int j0 = sh >> 5, j1 = (sh + 52) >> 5;
              for (int j = j0; j <= j1; ++j) {
                const int off  = 32 * j - sh;
                uint64_t chunk = (off >= 0 ? (m >> off) : (m << (-off))) & 0xffffffffull;
                if (chunk) bred_add(s + 2 + j, neg ? (0ull - chunk) : chunk);
              }
            }
          } else {
            atomicExch(reinterpret_cast<unsigned long long*>(q.status + 1), 2ull);  // not exact here: per-op path
          }
        }
      }
    } else {
      // join build: rhs rows into the multimap {key, row}
      for (int64_t r = w.begin + threadIdx.x; r < w.end; r += blockDim.x) {
        const uint64_t key = static_cast<uint64_t>(__ldg(q.k2 + r));
        uint64_t idx       = __umul64hi(bmix(key), q.cap);
        bool ok            = false;
        for (int probe = 0; probe < kMaxProbeB; ++probe) {
          unsigned long long* s = q.table + 2 * idx;
          if (atomicCAS(s + 1, kEmptyRow, static_cast<unsigned long long>(r)) == kEmptyRow) {
            s[0] = key;
            ok   = true;
            break;
          }
          idx = idx + 1 == q.cap ? 0 : idx + 1;
        }
        if (!ok) atomicExch(reinterpret_cast<unsigned long long*>(q.status + 1), 1ull);
      }
    }
  }
}

__device__ __forceinline__ double chunks_to_double_b(const unsigned long long* acc)
{
  uint64_t w[4] = {0, 0, 0, 0};
  for (int j = 0; j < 6; ++j) {
    const int64_t a = static_cast<int64_t>(acc[j]);
    uint64_t t[5]   = {0, 0, 0, 0, 0};
    const int sh = 32 * j, li = sh >> 6, bi = sh & 63;
    const uint64_t lo  = static_cast<uint64_t>(a);
    const uint64_t ext = a < 0 ? ~0ull : 0ull;
    t[li]              = lo << bi;
    t[li + 1]          = bi ? (lo >> (64 - bi)) | (ext << bi) : ext;
    for (int q = li + 2; q < 5; ++q) t[q] = ext;
    uint64_t carry = 0;
    for (int q = 0; q < 4; ++q) {
      const uint64_t x  = w[q] + t[q];
      const uint64_t c1 = x < w[q] ? 1 : 0;
      const uint64_t y  = x + carry;
      const uint64_t c2 = y < x ? 1 : 0;
      w[q]              = y;
      carry             = c1 + c2;
    }
  }
  const bool neg = static_cast<int64_t>(w[3]) < 0;
  if (neg) {
    uint64_t c = 1;
    for (int q = 0; q < 4; ++q) {
      w[q] = ~w[q] + c;
      c    = (c && w[q] == 0) ? 1 : 0;
    }
  }
  int msb = -1;
  for (int q = 3; q >= 0; --q)
    if (w[q]) {
      msb = 64 * q + 63 - __clzll(w[q]);
      break;
    }
  if (msb < 0) return 0.0;
  const int lo = msb - 63;
  uint64_t top, sticky = 0;
  if (lo <= 0) {
    top = w[0] << (-lo);
  } else {
    const int li = lo >> 6, bi = lo & 63;
    top = w[li] >> bi;
    if (bi && li + 1 < 4) top |= w[li + 1] << (64 - bi);
    for (int i = 0; i < li; ++i) sticky |= w[i];
    if (bi) sticky |= w[li] & ((1ull << bi) - 1);
  }
  double d = __ull2double_rn(top | (sticky ? 1ull : 0ull));
  d        = scalbn(d, lo - 96);
  return neg ? -d : d;
}

__global__ void __launch_bounds__(kBThreads) batch_emit_kernel(BatchArgs a)
{
  const int nit = *a.nitems;
  for (int it = blockIdx.x; it < nit; it += gridDim.x) {
    const ItemD w = a.items[it];
    const BReq& q = a.reqs[w.req];
    unsigned long long* cursor = reinterpret_cast<unsigned long long*>(q.status);
    if (q.kind == RQ_GROUPBY) {
      const int st = gb_stride(q.vtype);
      // table slots [begin, end) (the extra slot cap is in the last item)
      for (int64_t base = w.begin; base < w.end; base += blockDim.x) {
        const int64_t i   = base + threadIdx.x;
        bool used         = false;
        uint64_t key      = 0;
        const unsigned long long* s = nullptr;
        if (i < w.end) {
          s   = q.table + i * st;
          key = s[0];
          used = (i < static_cast<int64_t>(q.cap)) ? key != kEmptyKey : key != kEmptyKey;
          if (i == static_cast<int64_t>(q.cap)) key = kEmptyKey;  // the extra slot's key value
        }
        const unsigned long long pos = warp_claim(cursor, used);
        if (!used) continue;
        if (pos >= static_cast<unsigned long long>(q.out_cap)) {
          atomicExch(reinterpret_cast<unsigned long long*>(q.status + 1), 1ull);
          continue;
        }
        q.o0[pos] = static_cast<long long>(key);
        q.o2[pos] = static_cast<long long>(s[1]);
        if (q.vtype == V_INT64) static_cast<long long*>(q.o1)[pos] = static_cast<long long>(s[2]);
        else static_cast<double*>(q.o1)[pos] = chunks_to_double_b(s + 2);
      }
    } else {
      // probe rows [begin, end): emit every match
      for (int64_t base = w.begin; base < w.end; base += blockDim.x) {
        const int64_t r = base + threadIdx.x;
        const bool live = r < w.end;
        const uint64_t key = live ? static_cast<uint64_t>(__ldg(q.k1 + r)) : 0;
        uint64_t idx       = live ? __umul64hi(bmix(key), q.cap) : 0;
        bool more          = live;
        int probe          = 0;
        while (__any_sync(__activemask(), more)) {
          bool hit     = false;
          uint64_t brw = 0;
          if (more) {
            const unsigned long long* s = q.table + 2 * idx;
            const uint64_t row          = s[1];
            if (row == kEmptyRow) {
              more = false;
            } else if (++probe > kMaxProbeB) {
              more = false;
              atomicExch(reinterpret_cast<unsigned long long*>(q.status + 1), 1ull);
            } else {
              hit = s[0] == key;
              brw = row;
              idx = idx + 1 == q.cap ? 0 : idx + 1;
            }
          }
          const unsigned long long pos = warp_claim(cursor, hit);
          if (hit) {
            if (pos < static_cast<unsigned long long>(q.out_cap)) {
              q.o0[pos]                               = static_cast<long long>(key);
              static_cast<long long*>(q.o1)[pos]      = __ldg(static_cast<const long long*>(q.v1) + r);
              q.o2[pos]                               = static_cast<long long>(key);
              q.o3[pos]                               = __ldg(q.v2 + brw);
            } else {
              atomicExch(reinterpret_cast<unsigned long long*>(q.status + 1), 1ull);
            }
          }
        }
      }
    }
  }
}

}  // namespace

// ---- host engine ------------------------------------------------------------
struct BatchEngine {
  int max_reqs, max_items;
  int64_t tile_rows;
  cudaStream_t stream;
  int grid;
  // pinned host + device descriptors: [reqs | items x3 | counts x3 | err]
  BReq* h_reqs;
  ItemD* h_items;  // 3 lists of max_items
  int* h_counts;   // 3 counts
  unsigned long long* h_status;  // [max_reqs][2] results, then the error word
  BReq* d_reqs;
  ItemD* d_items;
  int* d_counts;
  int* d_err;
  unsigned long long* d_status;  // status words live here (BReq.status points into it)
  cudaGraphExec_t exec = nullptr;
  cudaGraph_t graph    = nullptr;
};

}  // namespace ldf


namespace ldf {
void set_last_error(const std::string& msg);
}

namespace {
template <typename F>
int bguard(F&& f)
{
  ldf::set_last_error("");
  try {
    f();
    return LDF_OK;
  } catch (const ldf::LdfError& e) {
    ldf::set_last_error(e.what());
    return e.code;
  } catch (const std::exception& e) {
    ldf::set_last_error(e.what());
    return LDF_ERR_INTERNAL;
  }
}
}  // namespace

extern "C" int ldf_b200_batch_create(int32_t max_reqs, int32_t max_items, int64_t tile_rows, int32_t ctas_per_sm,
                                     void* stream, void** engine)
{
  return bguard([&] {
    LDF_REQUIRE(max_reqs > 0 && max_items > 0 && tile_rows >= 256 && ctas_per_sm > 0 && engine, "bad engine config");
    auto* e      = new ldf::BatchEngine{};
    e->max_reqs  = max_reqs;
    e->grid      = ldf::num_sms() * ctas_per_sm;
    // adaptive tiles give at most ~2 items per CTA plus one partial tile per request
    e->max_items = std::max<int>(max_items, 2 * e->grid + 2 * max_reqs + 16);
    e->tile_rows = tile_rows;
    e->stream    = static_cast<cudaStream_t>(stream);
    LDF_CUDA(cudaHostAlloc(&e->h_reqs, sizeof(ldf::BReq) * max_reqs, cudaHostAllocMapped));
    LDF_CUDA(cudaHostAlloc(&e->h_items, sizeof(ldf::ItemD) * e->max_items * 3, cudaHostAllocMapped));
    LDF_CUDA(cudaHostAlloc(&e->h_counts, sizeof(int) * 4, cudaHostAllocMapped));
    LDF_CUDA(cudaMallocHost(&e->h_status, sizeof(unsigned long long) * (2 * max_reqs + 1)));
    LDF_CUDA(cudaMalloc(&e->d_reqs, sizeof(ldf::BReq) * max_reqs));
    LDF_CUDA(cudaMalloc(&e->d_items, sizeof(ldf::ItemD) * e->max_items * 3));
    LDF_CUDA(cudaMalloc(&e->d_counts, sizeof(int) * 4));
    LDF_CUDA(cudaMalloc(&e->d_err, sizeof(int)));
    LDF_CUDA(cudaMalloc(&e->d_status, sizeof(unsigned long long) * 2 * max_reqs));
    LDF_CUDA(cudaMemset(e->d_err, 0, sizeof(int)));
    // capture: upload descriptors, 3 persistent kernels, download statuses
    cudaStream_t cs;
    LDF_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    LDF_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    ldf::StageArgs sa{};
    LDF_CUDA(cudaHostGetDevicePointer(reinterpret_cast<void**>(const_cast<ldf::BReq**>(&sa.h_reqs)), e->h_reqs, 0));
    LDF_CUDA(cudaHostGetDevicePointer(reinterpret_cast<void**>(const_cast<ldf::ItemD**>(&sa.h_items)), e->h_items, 0));
    LDF_CUDA(cudaHostGetDevicePointer(reinterpret_cast<void**>(const_cast<int**>(&sa.h_counts)), e->h_counts, 0));
    sa.d_reqs    = e->d_reqs;
    sa.d_items   = e->d_items;
    sa.d_counts  = e->d_counts;
    sa.max_items = e->max_items;
    ldf::BatchArgs a0{e->d_reqs, e->d_items, e->d_counts + 0, e->d_err};
    ldf::BatchArgs a1{e->d_reqs, e->d_items + e->max_items, e->d_counts + 1, e->d_err};
    ldf::BatchArgs a2{e->d_reqs, e->d_items + 2 * e->max_items, e->d_counts + 2, e->d_err};
    ldf::batch_stage_kernel<<<ldf::num_sms(), ldf::kBThreads, 0, cs>>>(sa);
    ldf::batch_init_kernel<<<e->grid, ldf::kBThreads, 0, cs>>>(a0);
    ldf::batch_build_kernel<<<e->grid, ldf::kBThreads, 0, cs>>>(a1);
    ldf::batch_emit_kernel<<<e->grid, ldf::kBThreads, 0, cs>>>(a2);
    cudaMemcpyAsync(e->h_status, e->d_status, sizeof(unsigned long long) * 2 * max_reqs, cudaMemcpyDeviceToHost, cs);
    cudaMemcpyAsync(e->h_status + 2 * max_reqs, e->d_err, sizeof(int), cudaMemcpyDeviceToHost, cs);
    cudaError_t ce = cudaStreamEndCapture(cs, &e->graph);
    cudaStreamDestroy(cs);
    LDF_CUDA(ce);
    LDF_CUDA(cudaGraphInstantiate(&e->exec, e->graph, 0));
    *engine = e;
  });
}

extern "C" int ldf_b200_batch_run(void* engine, const ldf_batch_request* reqs, int32_t nreq)
{
  return bguard([&] {
    auto* e = static_cast<ldf::BatchEngine*>(engine);
    LDF_REQUIRE(e && nreq >= 0 && nreq <= e->max_reqs, "batch larger than the engine's request capacity");
    LDF_REQUIRE(nreq == 0 || reqs != nullptr, "null request array");
    // units of work of each kernel: table slots (init), build rows, emit units
    auto units = [](const ldf_batch_request& r, int list) -> int64_t {
      const int64_t slots = r.kind == 0 ? static_cast<int64_t>(r.cap) + 1 : static_cast<int64_t>(r.cap);
      if (list == 0) return slots;
      if (list == 1) return r.kind == 0 ? r.n : r.m;
      return r.kind == 0 ? slots : r.n;
    };
    int64_t tile[3];
    for (int l = 0; l < 3; ++l) {
      int64_t total = 0;
      for (int i = 0; i < nreq; ++i) total += units(reqs[i], l);
      // about two tiles per CTA of the persistent grid, between kMinTile and tile_rows rows
      int64_t t = (total + 2 * e->grid - 1) / (2 * e->grid);
      t         = (t + 255) / 256 * 256;
      tile[l]   = std::max<int64_t>(std::min<int64_t>(t, e->tile_rows), std::min<int64_t>(ldf::kMinTile, e->tile_rows));
    }
    int cnt[3] = {0, 0, 0};
    auto push  = [&](int list, int req, int64_t en) {
      for (int64_t s = 0; s < en; s += tile[list]) {
        LDF_REQUIRE(cnt[list] < e->max_items, "batch larger than the engine's work-item capacity");
        e->h_items[list * e->max_items + cnt[list]++] = ldf::ItemD{req, list, s, std::min<int64_t>(en, s + tile[list])};
      }
    };
    for (int i = 0; i < nreq; ++i) {
      const ldf_batch_request& r = reqs[i];
      LDF_REQUIRE(r.kind == 0 || r.kind == 1, "unknown batch request kind");
      LDF_REQUIRE(r.cap >= 2 && r.table != nullptr, "request without a hash table");
      LDF_REQUIRE(r.n >= 0 && r.m >= 0 && r.out_cap >= 0, "negative request size");
      LDF_REQUIRE(r.n == 0 || (r.k1 != nullptr && r.v1 != nullptr), "request without lhs columns");
      LDF_REQUIRE(r.kind == 0 || r.m == 0 || (r.k2 != nullptr && r.v2 != nullptr), "join without rhs columns");
      LDF_REQUIRE(r.kind == 1 || r.vtype == 0 || r.vtype == 1, "unknown groupby value type");
      LDF_REQUIRE(r.kind == 0 || r.cap > static_cast<uint64_t>(r.m), "join multimap smaller than the build side");
      LDF_REQUIRE(r.out_cap == 0 || (r.o0 && r.o1 && r.o2 && (r.kind == 0 || r.o3)), "missing output buffer");
      ldf::BReq q{};
      q.kind    = r.kind;
      q.vtype   = r.vtype;
      q.n       = r.n;
      q.m       = r.m;
      q.k1      = reinterpret_cast<const long long*>(r.k1);
      q.v1      = r.v1;
      q.k2      = reinterpret_cast<const long long*>(r.k2);
      q.v2      = reinterpret_cast<const long long*>(r.v2);
      q.vvalid  = r.vvalid;
      q.table   = reinterpret_cast<unsigned long long*>(r.table);
      q.cap     = r.cap;
      q.o0      = static_cast<long long*>(r.o0);
      q.o1      = r.o1;
      q.o2      = static_cast<long long*>(r.o2);
      q.o3      = static_cast<long long*>(r.o3);
      q.out_cap = r.out_cap;
      q.status  = e->d_status + 2 * i;
      e->h_reqs[i] = q;
      // groupby tables carry one extra slot (index cap) for the empty-marker key
      for (int l = 0; l < 3; ++l) push(l, i, units(r, l));
    }
    e->h_counts[0] = cnt[0];
    e->h_counts[1] = cnt[1];
    e->h_counts[2] = cnt[2];
    e->h_counts[3] = nreq;
    LDF_CUDA(cudaGraphLaunch(e->exec, e->stream));
    ldf::prof::count_launches(4);  // stage, init, build, emit
  });
}

extern "C" int ldf_b200_batch_wait(void* engine, uint64_t* out_rows, int32_t* overflow)
{
  return bguard([&] {
    auto* e = static_cast<ldf::BatchEngine*>(engine);
    LDF_CUDA(cudaStreamSynchronize(e->stream));
    int err = 0;
    std::memcpy(&err, e->h_status + 2 * e->max_reqs, sizeof(int));
    if (err) ldf::fail(LDF_ERR_TIMEOUT, "batch kernel reported a device error");
    for (int i = 0; i < e->max_reqs; ++i) {
      if (out_rows) out_rows[i] = e->h_status[2 * i];
      if (overflow) overflow[i] = e->h_status[2 * i + 1] != 0 ? 1 : 0;
    }
  });
}

extern "C" int ldf_b200_batch_destroy(void* engine)
{
  return bguard([&] {
    auto* e = static_cast<ldf::BatchEngine*>(engine);
    if (!e) return;
    if (e->exec) cudaGraphExecDestroy(e->exec);
    if (e->graph) cudaGraphDestroy(e->graph);
    cudaFreeHost(e->h_reqs);
    cudaFreeHost(e->h_items);
    cudaFreeHost(e->h_counts);
    cudaFreeHost(e->h_status);
    cudaFree(e->d_reqs);
    cudaFree(e->d_items);
    cudaFree(e->d_counts);
    cudaFree(e->d_err);
    cudaFree(e->d_status);
    delete e;
  });
}
