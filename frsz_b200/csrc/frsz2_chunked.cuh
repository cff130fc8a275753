// frsz2_chunked.cuh -- chunk geometry of the chunked kernels for exponent
// blocks of 17 to kChunkMaxEDecompress values (frsz2_chunked_ct.cuh), and
// chunk_copy, the 16-byte copy between a chunk in global memory and its
// image in shared memory that those kernels and the blockwise kernels use.
#pragma once

#include "frsz2_fast.cuh"

namespace frsz2b {

constexpr int kChunkValues = 2048;             // values per chunk at most
// Largest block size the chunked kernels take (a chunk then still holds 16
// blocks); larger blocks go to the warp-per-block kernels.
constexpr int kChunkMaxEDecompress = 128;

// Copy `bytes` bytes between global memory at g and shared memory at
// s + (g mod 16) (s 16-byte aligned), so both sides share their 16-byte
// boundaries: single bytes up to g's first boundary and after its last one,
// 16-byte accesses between.  All threads of the CTA take part.
template<bool TO_GLOBAL>
__device__ __forceinline__ void chunk_copy(std::uint8_t* g, std::uint8_t* s, std::uint32_t bytes)
{
  const std::uint32_t h = (std::uint32_t)(reinterpret_cast<std::uintptr_t>(g) & 15u);
  const std::uint32_t head = h == 0 ? 0u : min(16u - h, bytes);
  const std::uint32_t n16 = (bytes - head) >> 4;
  const std::uint32_t tail0 = head + (n16 << 4);
  std::uint8_t* sb = s + h;
  for (std::uint32_t i = threadIdx.x; i < head; i += blockDim.x) {
    if (TO_GLOBAL)
      g[i] = sb[i];
    else
      sb[i] = __ldg(g + i);
  }
  uint4* g16 = reinterpret_cast<uint4*>(g + head);
  uint4* s16 = reinterpret_cast<uint4*>(sb + head);
  for (std::uint32_t i = threadIdx.x; i < n16; i += blockDim.x) {
    if (TO_GLOBAL)
      __stcs(g16 + i, s16[i]);
    else
      s16[i] = __ldg(g16 + i);
  }
  for (std::uint32_t i = tail0 + threadIdx.x; i < bytes; i += blockDim.x) {
    if (TO_GLOBAL)
      g[i] = sb[i];
    else
      sb[i] = __ldg(g + i);
  }
}

} // namespace frsz2b
