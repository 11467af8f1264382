// Hash partition that allocates no device memory.
//
// Some callers cannot allocate device memory themselves: a legate task body
// that runs concurrently with other tasks on the same GPU must not call
// cudaMalloc (it synchronizes the device and can deadlock with those tasks),
// and an embedding host may have handed all device memory to its own pool.
// ldf_b200_hash_partition_noalloc serves them: the caller passes the input
// and the output buffers, and all scratch lives in one fixed-size array in the
// library's device image, created when the library is loaded on a GPU and
// held until the process exits.
//
// Limits: fixed-width columns only, at most LDF_B200_NOALLOC_MAX_ROWS rows and
// 256 buckets (one stable radix pass over the bucket id).  Every call shares
// the one scratch array and leaves its contents behind; each call clears what
// must start at zero.  Calls whose work overlaps on the GPU (different
// streams, or different host threads) race on the scratch: serialize them.
#include <mutex>

#include "radix.cuh"

namespace ldf {
void radix_histogram_raw(cudaStream_t s, const RadixPass& p, int64_t n, uint32_t* d_hist);
int64_t radix_status_words(int64_t n);
void onesweep_gather_pass_raw(cudaStream_t s, const RadixPass& p, int64_t n, int32_t* rows_out,
                              const uint64_t* d_bases, uint64_t* status, int* err);
}  // namespace ldf

namespace {

constexpr int64_t kMaxRows = LDF_B200_NOALLOC_MAX_ROWS;
constexpr int64_t kTileRows = ldf::kRadixTile;  // rows per onesweep tile

// Scratch layout (bytes): row permutation, look-back status words, bucket
// histogram, digit bases, error word.
constexpr size_t kPermBytes   = static_cast<size_t>(kMaxRows) * 4;
constexpr size_t kStatusWords = static_cast<size_t>((kMaxRows + kTileRows - 1) / kTileRows) * 256 + 2;
constexpr size_t kOffPerm     = 0;
constexpr size_t kOffStatus   = kPermBytes;
constexpr size_t kOffHist     = kOffStatus + kStatusWords * 8;
constexpr size_t kOffBases    = kOffHist + 256 * 4;
constexpr size_t kOffErr      = kOffBases + 256 * 8;
constexpr size_t kScratchBytes = kOffErr + 256;

// The scratch array.  In host code this name is only a host-side stand-in:
// its device address comes from cudaGetSymbolAddress (below).
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// Device address of g_noalloc_scratch for each device, looked up on the first
// call made with that device current and kept for the life of the process
// (so the entry point must not be called again on a device after a
// cudaDeviceReset of it).
std::mutex g_mu;
void* g_addr[256] = {};

void* scratch_address()
{
  int dev = 0;
  LDF_CUDA(cudaGetDevice(&dev));
  LDF_REQUIRE(dev >= 0 && dev < 256, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_mu);
  if (g_addr[dev] == nullptr) {
    void* p          = nullptr;
    cudaError_t e    = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr) {
      cudaGetLastError();
      ldf::fail(LDF_ERR_CUDA, std::string("cudaGetSymbolAddress of the no-alloc scratch failed: ") +
                                cudaGetErrorString(e));
    }
    g_addr[dev] = p;
  }
  return g_addr[dev];
}

// Output row i takes input row rows[i].  When the radix pass gave up on a
// bounded wait (err set), some rows[] entries were never written and still
// hold row ids of an earlier call: the kernel then copies nothing, and any
// entry outside [0, n) is skipped, so no read leaves the input columns.
__global__ void gather_rows_kernel(ldf::DCol src, const int32_t* rows, int64_t n, void* dst, uint8_t* dst_valid,
                                   const int* err)
{
  if (*reinterpret_cast<const volatile int*>(err) != 0) return;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = rows[i];
    if (r < 0 || r >= n) continue;
    ldf::copy_fixed(dst, i, src.data, r, src.width);
    if (dst_valid) dst_valid[i] = ldf::dvalid(src, r) ? 1 : 0;
  }
}

}  // namespace

namespace ldf {
void set_last_error(const std::string& msg);
}

extern "C" int ldf_b200_hash_partition_noalloc(const ldf_column* table, int32_t ncols, const int32_t* keys,
                                               int32_t nkeys, int32_t nparts, ldf_column* out, int64_t* offsets,
                                               void* stream)
{
  ldf::set_last_error("");
  try {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    LDF_REQUIRE(ncols >= 1 && table != nullptr && out != nullptr && offsets != nullptr, "bad arguments");
    LDF_REQUIRE(nparts >= 1 && nparts <= 256, "the no-alloc hash partition supports 1 to 256 buckets");
    const int64_t n = table[0].size;
    if (n > kMaxRows)
      ldf::fail(LDF_ERR_INVALID_ARGUMENT, "the no-alloc hash partition takes at most " + std::to_string(kMaxRows) +
                                            " rows, got " + std::to_string(n));
    for (int j = 0; j < ncols; ++j) {
      LDF_REQUIRE(table[j].size == n, "columns differ in length");
      LDF_REQUIRE(table[j].type != LDF_STRING, "the no-alloc hash partition takes fixed-width columns only");
      ldf::type_width(table[j].type);
      LDF_REQUIRE(n == 0 || (table[j].data != nullptr && out[j].data != nullptr), "column without data buffer");
      LDF_REQUIRE(table[j].valid == nullptr || n == 0 || out[j].valid != nullptr,
                  "a nullable column needs an output validity buffer");
    }
    ldf::KeyCols k = ldf::make_keys(table, ncols, keys, nkeys);

    unsigned char* base = static_cast<unsigned char*>(scratch_address());
    int32_t* perm       = reinterpret_cast<int32_t*>(base + kOffPerm);
    uint64_t* status    = reinterpret_cast<uint64_t*>(base + kOffStatus);
    uint32_t* hist      = reinterpret_cast<uint32_t*>(base + kOffHist);
    uint64_t* bases     = reinterpret_cast<uint64_t*>(base + kOffBases);
    int* err            = reinterpret_cast<int*>(base + kOffErr);

    ldf::RadixPass p{};
    p.src       = ldf::DigitSrc::BUCKET;
    p.shift     = 0;
    p.hash_keys = k;
    p.nparts    = static_cast<uint32_t>(nparts);

    // bucket histogram -> host -> digit bases
    uint32_t h[256];
    ldf::radix_histogram_raw(s, p, n, hist);
    LDF_CUDA(cudaMemcpyAsync(h, hist, sizeof(h), cudaMemcpyDeviceToHost, s));
    LDF_CUDA(cudaStreamSynchronize(s));
    uint64_t b[256];
    uint64_t acc = 0;
    for (int d = 0; d < 256; ++d) {
      b[d] = acc;
      acc += h[d];
    }
    for (int bkt = 0; bkt < nparts; ++bkt) offsets[bkt] = static_cast<int64_t>(b[bkt]);
    offsets[nparts] = static_cast<int64_t>(acc);

    if (n > 0) {
      LDF_CUDA(cudaMemcpyAsync(bases, b, sizeof(b), cudaMemcpyHostToDevice, s));
      LDF_CUDA(cudaMemsetAsync(status, 0, static_cast<size_t>(ldf::radix_status_words(n)) * 8, s));
      LDF_CUDA(cudaMemsetAsync(err, 0, sizeof(int), s));
      ldf::onesweep_gather_pass_raw(s, p, n, perm, bases, status, err);
      for (int j = 0; j < ncols; ++j) {
        ldf::DCol src = ldf::make_dcol(table[j]);
        uint8_t* ov   = table[j].valid ? out[j].valid : nullptr;
        ldf::launch("gather_rows", gather_rows_kernel, 296u, 256u, 0, s, src, static_cast<const int32_t*>(perm), n,
                    out[j].data, ov, static_cast<const int*>(err));
      }
      int e = 0;
      LDF_CUDA(cudaMemcpyAsync(&e, err, sizeof(int), cudaMemcpyDeviceToHost, s));
      LDF_CUDA(cudaStreamSynchronize(s));
      if (e != 0) ldf::fail(LDF_ERR_TIMEOUT, "a bounded device-side wait expired in the no-alloc hash partition");
    }
    for (int j = 0; j < ncols; ++j) {
      out[j].type       = table[j].type;
      out[j].nullable   = table[j].valid != nullptr ? 1 : 0;
      out[j].size       = n;
      out[j].chars      = nullptr;
      out[j].chars_base = 0;
      out[j].num_chars  = 0;
      if (!table[j].valid) out[j].valid = nullptr;
    }
    return LDF_OK;
  } catch (const ldf::LdfError& e) {
    ldf::set_last_error(e.what());
    return e.code;
  } catch (const std::exception& e) {
    ldf::set_last_error(e.what());
    return LDF_ERR_INTERNAL;
  }
}
