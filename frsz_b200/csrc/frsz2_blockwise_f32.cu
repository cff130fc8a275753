// fp32 instances of the one-thread-per-block kernels
// (frsz2_blockwise.cuh), bits 4..32.
#include "frsz2_blockwise_ce.cuh"

#include <array>
#include <utility>

namespace frsz2b {

cudaError_t launch_blockwise_f32(int bits, bool compress, const Job& j, cudaStream_t s)
{
  static constexpr auto table = make_blockwise_table<float, 4>(std::make_integer_sequence<int, 29>{});
  if (bits < 4 || bits > 32) return cudaErrorNotSupported;
  // block sizes with compile-time instances first
  if (bwc_has(j.E)) return launch_bwc(false, j.E, bits, compress, j, s);
  return table[bits - 4](compress, j, s);
}

} // namespace frsz2b
