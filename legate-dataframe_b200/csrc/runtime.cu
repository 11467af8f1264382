// Host runtime pieces shared by all ops: allocator contract, SM count,
// device-wide scans, error-word checks, launch counting and the optional
// per-kernel CUDA-event profile.
#include <atomic>
#include <map>
#include <mutex>

#include "scan.cuh"

namespace ldf {

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
// Single-pass exclusive scan with decoupled look-back.  256 threads x 8 items
// per tile; the input is read once and the output written once.
// ---------------------------------------------------------------------------
namespace {
constexpr int kScanThreads = 256;
constexpr int kScanItems   = 8;
constexpr int kScanTile    = kScanThreads * kScanItems;

template <typename TIn>
__global__ void __launch_bounds__(kScanThreads)
  scan_kernel(const TIn* in, int64_t* out, int64_t n, uint64_t* status,
              unsigned long long* counter, int64_t* total, int* err)
{
  __shared__ int64_t s_scan[kScanThreads / 32 + 1];
  __shared__ int64_t s_tile;
  __shared__ uint64_t s_prefix;
  const int64_t tile = next_tile_id(counter, &s_tile);
  const int64_t base = tile * kScanTile + static_cast<int64_t>(threadIdx.x) * kScanItems;
  int64_t v[kScanItems];
  int64_t sum = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    int64_t r = base + i;
    v[i]      = r < n ? static_cast<int64_t>(in[r]) : 0;
    sum += v[i];
  }
  int64_t tile_total;
  int64_t excl = block_exclusive_scan<int64_t, kScanThreads>(sum, s_scan, &tile_total);
  if (threadIdx.x == 0) {
    s_prefix = lookback_exclusive(status, tile, static_cast<uint64_t>(tile_total), err);
    if (tile == static_cast<int64_t>(gridDim.x) - 1) *total = static_cast<int64_t>(s_prefix) + tile_total;
  }
  __syncthreads();
  int64_t run = static_cast<int64_t>(s_prefix) + excl;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    int64_t r = base + i;
    if (r < n) out[r] = run;
    run += v[i];
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
  launch("scan", scan_kernel<TIn>, static_cast<unsigned>(tiles), kScanThreads, 0, s, 
    in, out, n, status.get(), counter, d_total, ctx.err());
  LDF_CHECK_LAUNCH();
}
}  // namespace

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
