// Host runtime pieces shared by all ops: allocator contract, SM count,
// device-wide scans, error-word checks, launch counting and the optional
// per-kernel CUDA-event profile.
#include <atomic>
#include <map>
#include <mutex>

#include "scan.cuh"

namespace ldf {
void set_last_error(const std::string& msg);

// ---------------------------------------------------------------------------
// Launch accounting.  When profiling is on, each launch is bracketed by two
// CUDA events recorded on the launch's stream; ldf_b200_profile_report()
// waits for them and returns per-kernel counts and summed device times.
// ---------------------------------------------------------------------------
namespace prof {
namespace {
std::atomic<unsigned long long> g_launches{0};
std::atomic<int> g_enabled{0};
struct Pending {
  std::string name;
  cudaEvent_t a, b;
};
std::mutex g_mu;
std::vector<Pending> g_pending;
std::map<std::string, std::pair<unsigned long long, double>> g_totals;
thread_local cudaEvent_t t_begin = nullptr;
}  // namespace

void begin(const char*, cudaStream_t s)
{
  g_launches.fetch_add(1, std::memory_order_relaxed);
  if (!g_enabled.load(std::memory_order_relaxed)) return;
  LDF_CUDA(cudaEventCreate(&t_begin));
  LDF_CUDA(cudaEventRecord(t_begin, s));
}

void count_launches(unsigned long long n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

void end(const char* name, cudaStream_t s)
{
  if (!g_enabled.load(std::memory_order_relaxed) || t_begin == nullptr) return;
  cudaEvent_t e;
  LDF_CUDA(cudaEventCreate(&e));
  LDF_CUDA(cudaEventRecord(e, s));
  std::lock_guard<std::mutex> g(g_mu);
  g_pending.push_back(Pending{name, t_begin, e});
  t_begin = nullptr;
}

void collect()
{
  std::lock_guard<std::mutex> g(g_mu);
  for (auto& p : g_pending) {
    cudaEventSynchronize(p.b);
    float ms = 0;
    cudaEventElapsedTime(&ms, p.a, p.b);
    auto& t = g_totals[p.name];
    t.first += 1;
    t.second += ms;
    cudaEventDestroy(p.a);
    cudaEventDestroy(p.b);
  }
  g_pending.clear();
}
}  // namespace prof

int num_sms()
{
  static thread_local int dev_cached = -1;
  static thread_local int sms        = 0;
  int dev                            = 0;
  LDF_CUDA(cudaGetDevice(&dev));
  if (dev != dev_cached) {
    LDF_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    dev_cached = dev;
  }
  return sms;
}

cudaStream_t staging_stream()
{
  constexpr int kMaxDevices = 64;
  static std::mutex mu;
  static cudaStream_t streams[kMaxDevices] = {};
  int dev = 0;
  LDF_CUDA(cudaGetDevice(&dev));
  LDF_REQUIRE(dev >= 0 && dev < kMaxDevices, "device ordinal out of range");
  std::lock_guard<std::mutex> g(mu);
  if (streams[dev] == nullptr) LDF_CUDA(cudaStreamCreateWithFlags(&streams[dev], cudaStreamNonBlocking));
  return streams[dev];
}

void* Allocator::allocate(size_t nbytes) const
{
  if (nbytes == 0) nbytes = 16;
  // Round to 256 B so vectorised accesses never cross an allocation end.
  nbytes = (nbytes + 255) & ~size_t(255);
  void* p = nullptr;
  if (a_ && a_->allocate) {
    p = a_->allocate(a_->ctx, nbytes, static_cast<void*>(s_));
  } else {
    if (cudaMallocAsync(&p, nbytes, s_) != cudaSuccess) {
      cudaGetLastError();
      p = nullptr;
    }
  }
  if (p == nullptr)
    fail(LDF_ERR_OUT_OF_MEMORY, "device allocation of " + std::to_string(nbytes) + " bytes failed");
  return p;
}

void Allocator::deallocate(void* p, size_t nbytes) const
{
  if (p == nullptr) return;
  if (nbytes == 0) nbytes = 16;
  nbytes = (nbytes + 255) & ~size_t(255);
  if (a_ && a_->deallocate) {
    a_->deallocate(a_->ctx, p, nbytes, static_cast<void*>(s_));
  } else {
    cudaFreeAsync(p, s_);
  }
}

void* Allocator::allocate_scratch(size_t nbytes) const
{
  if (nbytes == 0) nbytes = 16;
  nbytes = (nbytes + 255) & ~size_t(255);
  if (nbytes > kSmallScratch) return allocate(nbytes);
  if (left_ < nbytes) {
    bump_ = static_cast<char*>(allocate(kScratchChunk));
    chunks_.push_back(bump_);
    left_ = kScratchChunk;
  }
  void* p = bump_;
  bump_ += nbytes;
  left_ -= nbytes;
  return p;
}

void Allocator::deallocate_scratch(void* p, size_t nbytes) const
{
  if (p == nullptr) return;
  if (nbytes == 0) nbytes = 16;
  nbytes = (nbytes + 255) & ~size_t(255);
  if (nbytes > kSmallScratch) deallocate(p, nbytes);
  // small scratch lives until its chunk is returned
}

Allocator::~Allocator()
{
  for (void* c : chunks_) deallocate(c, kScratchChunk);
}

OpContext::OpContext(const ldf_allocator* a, cudaStream_t s) : alloc_(a, s)
{
  err_ = Buffer<int>(alloc_, 1);
  LDF_CUDA(cudaMemsetAsync(err_.get(), 0, sizeof(int), s));
}

static void raise_device_error(int h)
{
  if (h == LDF_ERR_TIMEOUT)
    fail(LDF_ERR_TIMEOUT, "a bounded device-side wait expired (look-back did not complete)");
  if (h != 0) fail(LDF_ERR_INTERNAL, "device kernel reported error " + std::to_string(h));
}

int64_t OpContext::read_i64(const int64_t* d) const
{
  int64_t h[1] = {0};
  int e        = 0;
  LDF_CUDA(cudaMemcpyAsync(h, d, sizeof(int64_t), cudaMemcpyDeviceToHost, stream()));
  LDF_CUDA(cudaMemcpyAsync(&e, err_.get(), sizeof(int), cudaMemcpyDeviceToHost, stream()));
  LDF_CUDA(cudaStreamSynchronize(stream()));
  raise_device_error(e);
  return h[0];
}

void OpContext::finish() const
{
  int e = 0;
  LDF_CUDA(cudaMemcpyAsync(&e, err_.get(), sizeof(int), cudaMemcpyDeviceToHost, stream()));
  LDF_CUDA(cudaStreamSynchronize(stream()));
  raise_device_error(e);
}

// ---------------------------------------------------------------------------
// Single-pass exclusive scan with decoupled look-back.  256 threads x 16 items
// per tile; the input is read once and the output written once, both
// coalesced: item i of a thread is element i * 32 + lane of its warp's
// 512-element segment, so each warp scans its segment as 16 warp-wide scans
// with a running carry.  Warp 0 does the look-back over a window of 32
// predecessor tiles per round trip.
// ---------------------------------------------------------------------------
namespace {
constexpr int kScanThreads = 256;
constexpr int kScanItems   = 16;
constexpr int kScanWarps   = kScanThreads / 32;
constexpr int kScanTile    = kScanThreads * kScanItems;

// Exclusive prefix of `tile` over the tile aggregates before it; every lane
// of one warp calls it.  Publishes the tile's aggregate first and its
// inclusive prefix at the end.  A predecessor that has not published after
// `spin_limit` polls sets LDF_ERR_TIMEOUT in *err and ends the wait.
__device__ __forceinline__ uint64_t warp_lookback(uint64_t* status, int64_t tile, uint64_t aggregate, int* err,
                                                  uint32_t spin_limit)
{
  const int lane = threadIdx.x & 31;
  if (tile == 0) {
    if (lane == 0) st_release_u64(&status[0], kFlagPrefix | aggregate);
    return 0;
  }
  if (lane == 0) st_release_u64(&status[tile], kFlagAgg | aggregate);
  uint64_t excl  = 0;
  int64_t j      = tile - 1;  // the window covers tiles j, j - 1, ..., j - 31 (lane order)
  uint32_t spins = 0;
  for (;;) {
    const int64_t t  = j - lane;
    const uint64_t v = t >= 0 ? ld_volatile_u64(&status[t]) : kFlagPrefix;
    const uint64_t f = v & ~kValueMask;
    const uint32_t not_ready = __ballot_sync(0xffffffffu, f == 0);
    const uint32_t prefix    = __ballot_sync(0xffffffffu, f == kFlagPrefix);
    const int first_prefix   = prefix ? __ffs(prefix) - 1 : 32;
    const int first_waiting  = not_ready ? __ffs(not_ready) - 1 : 32;
    if (first_waiting < first_prefix) {  // a tile before the nearest prefix has not published yet
      if (++spins > spin_limit) {
        if (lane == 0) atomicExch(err, LDF_ERR_TIMEOUT);
        break;
      }
      __nanosleep(32);
      continue;
    }
    excl += warp_reduce_sum<uint64_t>(lane <= first_prefix ? (v & kValueMask) : 0);
    if (first_prefix < 32) break;
    j -= 32;
  }
  if (lane == 0) st_release_u64(&status[tile], kFlagPrefix | (excl + aggregate));
  return excl;
}

// One tile per block.  The tile is loaded coalesced into shared memory, where
// thread t then owns kScanItems consecutive elements (runs padded by one word
// so that neither the coalesced nor the per-thread accesses conflict on
// banks): a serial sum per thread, one warp scan of the thread sums, the
// block's warp totals and the look-back in warp 0, then the per-thread runs
// written back to shared memory and stored coalesced.
template <typename TIn>
__global__ void __launch_bounds__(kScanThreads)
  scan_kernel(const TIn* in, int64_t* out, int64_t n, uint64_t* status,
              unsigned long long* counter, int64_t* total, int* err, uint32_t spin_limit)
{
  constexpr int kPad = kScanItems + 1;
  __shared__ int64_t s_x[kScanThreads * kPad];
  __shared__ int64_t s_warp[kScanWarps + 1];
  __shared__ int64_t s_tile;
  __shared__ uint64_t s_prefix;
  const int64_t tile  = next_tile_id(counter, &s_tile);
  const int warp      = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t tbase = tile * kScanTile;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    const int e     = i * kScanThreads + threadIdx.x;
    const int64_t r = tbase + e;
    s_x[(e / kScanItems) * kPad + e % kScanItems] = r < n ? static_cast<int64_t>(in[r]) : 0;
  }
  __syncthreads();
  int64_t v[kScanItems];
  int64_t sum = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    v[k] = s_x[threadIdx.x * kPad + k];
    sum += v[k];
  }
  const int64_t inc = warp_inclusive_scan(sum);
  if (lane == 31) s_warp[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    const int64_t w    = lane < kScanWarps ? s_warp[lane] : 0;
    const int64_t winc = warp_inclusive_scan(w);
    if (lane < kScanWarps) s_warp[lane] = winc - w;
    const int64_t tile_total = __shfl_sync(0xffffffffu, winc, kScanWarps - 1);
    const uint64_t excl = warp_lookback(status, tile, static_cast<uint64_t>(tile_total), err, spin_limit);
    if (lane == 0) {
      s_prefix = excl;
      if (tile == static_cast<int64_t>(gridDim.x) - 1) *total = static_cast<int64_t>(excl) + tile_total;
    }
  }
  __syncthreads();
  int64_t run = static_cast<int64_t>(s_prefix) + s_warp[warp] + inc - sum;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    s_x[threadIdx.x * kPad + k] = run;
    run += v[k];
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    const int e     = i * kScanThreads + threadIdx.x;
    const int64_t r = tbase + e;
    if (r < n) out[r] = s_x[(e / kScanItems) * kPad + e % kScanItems];
  }
}

template <typename TIn>
void exclusive_scan_impl(const TIn* in, int64_t* out, int64_t n, int64_t* d_total,
                         const OpContext& ctx)
{
  const Allocator& alloc = ctx.alloc();
  cudaStream_t s         = ctx.stream();
  if (n == 0) {
    LDF_CUDA(cudaMemsetAsync(d_total, 0, sizeof(int64_t), s));
    return;
  }
  const int64_t tiles = ceil_div(n, kScanTile);
  Buffer<uint64_t> status(alloc, tiles + 2);
  unsigned long long* counter = reinterpret_cast<unsigned long long*>(status.get() + tiles);
  LDF_CUDA(cudaMemsetAsync(status.get(), 0, (tiles + 2) * sizeof(uint64_t), s));
  launch("scan", scan_kernel<TIn>, static_cast<unsigned>(tiles), kScanThreads, 0, s, in, out, n, status.get(),
         counter, d_total, ctx.err(), kSpinLimit);
  LDF_CHECK_LAUNCH();
}
}  // namespace

// The scan kernel of exclusive_scan_i64 launched as one block that takes
// tile 1 of a two-tile input, so the look-back waits on tile 0, whose status
// word nothing writes: the wait ends after `spin_limit` polls with
// LDF_ERR_TIMEOUT in the error word, which finish() turns into the op's
// error.  Exercises the timeout path of every look-back without a hang.
void stalled_lookback(uint32_t spin_limit, const OpContext& ctx)
{
  cudaStream_t s = ctx.stream();
  Buffer<int64_t> io(ctx.alloc(), 4 * kScanTile + 1);  // input, output, total
  Buffer<uint64_t> status(ctx.alloc(), 4);
  LDF_CUDA(cudaMemsetAsync(io.get(), 0, (4 * kScanTile + 1) * sizeof(int64_t), s));
  LDF_CUDA(cudaMemsetAsync(status.get(), 0, 4 * sizeof(uint64_t), s));
  static const unsigned long long kFirstTile = 1;  // the block takes tile 1
  LDF_CUDA(cudaMemcpyAsync(status.get() + 2, &kFirstTile, sizeof(kFirstTile), cudaMemcpyHostToDevice, s));
  launch("scan", scan_kernel<int64_t>, 1u, kScanThreads, 0, s, static_cast<const int64_t*>(io.get()),
         io.get() + 2 * kScanTile, static_cast<int64_t>(2 * kScanTile), status.get(),
         reinterpret_cast<unsigned long long*>(status.get() + 2), io.get() + 4 * kScanTile, ctx.err(), spin_limit);
  LDF_CHECK_LAUNCH();
  ctx.finish();
}

void exclusive_scan_i64(const int64_t* in, int64_t* out, int64_t n, int64_t* d_total,
                        const OpContext& ctx)
{
  exclusive_scan_impl<int64_t>(in, out, n, d_total, ctx);
}
void exclusive_scan_u32(const uint32_t* in, int64_t* out, int64_t n, int64_t* d_total,
                        const OpContext& ctx)
{
  exclusive_scan_impl<uint32_t>(in, out, n, d_total, ctx);
}

}  // namespace ldf

extern "C" {
int ldf_b200_test_stalled_lookback(uint32_t spin_limit, const ldf_allocator* alloc, void* stream)
{
  ldf::set_last_error("");
  try {
    LDF_REQUIRE(spin_limit >= 1 && spin_limit <= ldf::kSpinLimit, "spin_limit must be in [1, kSpinLimit]");
    ldf::OpContext ctx(alloc, static_cast<cudaStream_t>(stream));
    ldf::stalled_lookback(spin_limit, ctx);
    return LDF_OK;
  } catch (const ldf::LdfError& e) {
    ldf::set_last_error(e.what());
    return e.code;
  } catch (const std::exception& e) {
    ldf::set_last_error(e.what());
    return LDF_ERR_INTERNAL;
  }
}

void ldf_b200_profile_enable(int on)
{
  ldf::prof::collect();
  ldf::prof::g_enabled.store(on ? 1 : 0);
}

unsigned long long ldf_b200_launch_count(void) { return ldf::prof::g_launches.load(); }

int ldf_b200_profile_report(char* buf, size_t len, int reset)
{
  ldf::prof::collect();
  std::string out;
  {
    std::lock_guard<std::mutex> g(ldf::prof::g_mu);
    for (auto& kv : ldf::prof::g_totals)
      out += kv.first + " " + std::to_string(kv.second.first) + " " + std::to_string(kv.second.second) + "\n";
    if (reset) ldf::prof::g_totals.clear();
  }
  if (buf && len) {
    size_t n = std::min(len - 1, out.size());
    std::memcpy(buf, out.data(), n);
    buf[n] = 0;
  }
  return static_cast<int>(out.size());
}
}
