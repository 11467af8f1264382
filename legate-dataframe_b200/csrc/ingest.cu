// Arrow buffers -> the legate device layout, converted on the device.
//
// A column read from Arrow (Parquet, CSV, in-memory tables) arrives with a
// validity bitmap (1 bit per row) and, for strings, offsets (4 or 8 bytes per
// row).  The legate layout wants one byte per row for the null mask and a
// 16-byte inclusive range per string.  Copying the Arrow buffers as they are
// and expanding them here moves 1/8 of the mask bytes and 1/4 (int32 offsets)
// of the range bytes across PCIe, and needs no host pass over the rows.  The
// kernels are the converse direction of the reference's move_into conversions
// (null_mask.cu:98-113 bitmask_to_bools, ranges.cu:109-138 offsets_to_ranges),
// applied to the column copy of PhysicalColumn::from_arrow (column.cpp:86-122).
#include "table_ops.cuh"

namespace ldf {
namespace {

// Thread t writes rows [8t, 8t + 8): bit (shift + 8t + j) of `bits`, which
// lies in bytes t and t + 1.  `aligned`: out is 8-byte aligned, so full
// groups of 8 rows go out as one 8-byte store.
__global__ void bits_to_bytes_kernel(const uint8_t* bits, int shift, int64_t nbytes, int64_t n, uint8_t* out,
                                     int aligned)
{
  const int64_t groups = (n + 7) >> 3;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < groups; t += (int64_t)gridDim.x * blockDim.x) {
    uint32_t w = bits[t];
    if (shift != 0 && t + 1 < nbytes) w |= static_cast<uint32_t>(bits[t + 1]) << 8;
    const uint32_t v = (w >> shift) & 0xffu;
    const int64_t i0 = t * 8;
    if (aligned && i0 + 8 <= n) {
      uint64_t o = 0;
#pragma unroll
      for (int j = 0; j < 8; ++j) o |= static_cast<uint64_t>((v >> j) & 1u) << (8 * j);
      *reinterpret_cast<uint64_t*>(out + i0) = o;
    } else {
      for (int j = 0; j < 8 && i0 + j < n; ++j) out[i0 + j] = static_cast<uint8_t>((v >> j) & 1u);
    }
  }
}

template <typename T>
__global__ void offsets_to_ranges_kernel(const T* off, int64_t n, ldf_range* out)
{
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = ldf_range{static_cast<int64_t>(off[i]), static_cast<int64_t>(off[i + 1]) - 1};
}

unsigned ingest_blocks(int64_t work)
{
  const int64_t b   = ceil_div(work, 256);
  const int64_t cap = static_cast<int64_t>(num_sms()) * 16;
  return static_cast<unsigned>(b < 1 ? 1 : (b > cap ? cap : b));
}

}  // namespace

void arrow_bits_to_bytes(const uint8_t* bits, int64_t bit_offset, int64_t n, uint8_t* out, cudaStream_t s)
{
  LDF_REQUIRE(n >= 0 && bit_offset >= 0, "negative size or bit offset");
  if (n == 0) return;
  LDF_REQUIRE(bits != nullptr && out != nullptr, "null buffer");
  const uint8_t* b   = bits + (bit_offset >> 3);
  const int shift    = static_cast<int>(bit_offset & 7);
  const int64_t nb   = (shift + n + 7) >> 3;
  const int aligned  = (reinterpret_cast<uintptr_t>(out) & 7) == 0 ? 1 : 0;
  launch("bits_to_bytes", bits_to_bytes_kernel, ingest_blocks((n + 7) >> 3), 256, 0, s, b, shift, nb, n, out,
         aligned);
}

void arrow_offsets_to_ranges(const void* offsets, int offset_bytes, int64_t n, ldf_range* out, cudaStream_t s)
{
  LDF_REQUIRE(n >= 0, "negative size");
  LDF_REQUIRE(offset_bytes == 4 || offset_bytes == 8, "offsets must be 4 or 8 bytes wide");
  if (n == 0) return;
  LDF_REQUIRE(offsets != nullptr && out != nullptr, "null buffer");
  if (offset_bytes == 4)
    launch("offsets_to_ranges", offsets_to_ranges_kernel<int32_t>, ingest_blocks(n), 256, 0, s,
           static_cast<const int32_t*>(offsets), n, out);
  else
    launch("offsets_to_ranges", offsets_to_ranges_kernel<int64_t>, ingest_blocks(n), 256, 0, s,
           static_cast<const int64_t*>(offsets), n, out);
}

}  // namespace ldf
