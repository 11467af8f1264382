// Block-wide scans and the single-pass decoupled look-back used by every
// count-then-write kernel (join probe, compaction, radix-sort scatter).
#pragma once

#include "common.cuh"

namespace ldf {

// Warp inclusive scan (shuffle-up, 5 steps).
template <typename T>
__device__ __forceinline__ T warp_inclusive_scan(T v)
{
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    T n = __shfl_up_sync(0xffffffffu, v, d);
    if (lane >= d) v += n;
  }
  return v;
}

template <typename T>
__device__ __forceinline__ T warp_reduce_sum(T v)
{
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(0xffffffffu, v, d);
  return v;
}

// Block exclusive scan of one value per thread.  `smem` needs NWARPS + 1
// entries.  Returns the exclusive prefix; *total receives the block sum.
template <typename T, int NTHREADS>
__device__ __forceinline__ T block_exclusive_scan(T v, T* smem, T* total)
{
  constexpr int NW = NTHREADS / 32;
  const int lane   = threadIdx.x & 31;
  const int warp   = threadIdx.x >> 5;
  T inc            = warp_inclusive_scan(v);
  if (lane == 31) smem[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    T w  = lane < NW ? smem[lane] : T(0);
    T wi = warp_inclusive_scan(w);
    if (lane < NW) smem[lane] = wi - w;
    if (lane == NW - 1) smem[NW] = wi;
  }
  __syncthreads();
  T res  = smem[warp] + inc - v;
  *total = smem[NW];
  __syncthreads();
  return res;
}

// ---------------------------------------------------------------------------
// Decoupled look-back (single-pass prefix scan over tiles).  Tile status is one
// 64-bit word: bits 62-63 flag (0 = not ready, 1 = aggregate, 2 = inclusive
// prefix), bits 0-61 the value.  Tiles take their ids from an atomic counter in
// launch order, so a tile only waits on tiles that already run; the wait is
// bounded and reports LDF_ERR_TIMEOUT through *err instead of hanging.
// ---------------------------------------------------------------------------
constexpr uint64_t kFlagAgg    = 1ull << 62;
constexpr uint64_t kFlagPrefix = 2ull << 62;
constexpr uint64_t kValueMask  = (1ull << 62) - 1;

__device__ __forceinline__ uint64_t ld_volatile_u64(const uint64_t* p)
{
  uint64_t v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_u64(uint64_t* p, uint64_t v)
{
  asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Called by one thread of the tile.  Returns the exclusive prefix of `tile`.
__device__ __forceinline__ uint64_t lookback_exclusive(uint64_t* status, int64_t tile,
                                                       uint64_t aggregate, int* err)
{
  if (tile == 0) {
    st_release_u64(&status[0], kFlagPrefix | aggregate);
    return 0;
  }
  st_release_u64(&status[tile], kFlagAgg | aggregate);
  uint64_t excl = 0;
  int64_t j     = tile - 1;
  uint32_t spins = 0;
  while (j >= 0) {
    uint64_t s = ld_volatile_u64(&status[j]);
    uint64_t f = s & ~kValueMask;
    if (f == 0) {
      if (++spins > kSpinLimit) {
        atomicExch(err, LDF_ERR_TIMEOUT);
        break;
      }
      __nanosleep(32);
      continue;
    }
    excl += s & kValueMask;
    if (f == kFlagPrefix) break;
    --j;
  }
  __threadfence();
  st_release_u64(&status[tile], kFlagPrefix | (excl + aggregate));
  return excl;
}

// Dynamic tile id (launch order) for look-back kernels.
__device__ __forceinline__ int64_t next_tile_id(unsigned long long* counter, int64_t* smem_slot)
{
  if (threadIdx.x == 0) *smem_slot = static_cast<int64_t>(atomicAdd(counter, 1ull));
  __syncthreads();
  int64_t t = *smem_slot;
  __syncthreads();
  return t;
}

// ---------------------------------------------------------------------------
// Host helpers (scan.cu).
// ---------------------------------------------------------------------------
// Per-call context: allocator, stream and the call's device error word, which
// bounded waits set instead of trapping.  The word is checked whenever the host
// reads a result back (the only synchronisation points of an op).
class OpContext {
 public:
  OpContext(const ldf_allocator* a, cudaStream_t s);
  const Allocator& alloc() const { return alloc_; }
  cudaStream_t stream() const { return alloc_.stream(); }
  int* err() const { return err_.get(); }
  // Copy one device int64 to the host, wait, and check the error word.
  int64_t read_i64(const int64_t* d) const;
  // Wait for the stream and check the error word.
  void finish() const;

 private:
  Allocator alloc_;
  Buffer<int> err_;
};

// out[i] = sum(in[0..i)) for counts; *d_total (device) = sum(in).
void exclusive_scan_i64(const int64_t* in, int64_t* out, int64_t n, int64_t* d_total,
                        const OpContext& ctx);
void exclusive_scan_u32(const uint32_t* in, int64_t* out, int64_t n, int64_t* d_total,
                        const OpContext& ctx);

}  // namespace ldf
