// fp64 instances of the one-thread-per-block kernels
// (frsz2_blockwise.cuh), bits 4..64.
#include "frsz2_blockwise_ce.cuh"

#include <array>
#include <utility>

namespace frsz2b {

cudaError_t launch_blockwise_f64(int bits, bool compress, const Job& j, cudaStream_t s)
{
  static constexpr auto table = make_blockwise_table<double, 4>(std::make_integer_sequence<int, 61>{});
  if (bits < 4 || bits > 64) return cudaErrorNotSupported;
  // block sizes with compile-time instances first
  if (bwc_has(j.E)) return launch_bwc(true, j.E, bits, compress, j, s);
  return table[bits - 4](compress, j, s);
}

} // namespace frsz2b
