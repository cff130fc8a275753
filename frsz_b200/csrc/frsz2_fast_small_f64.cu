// fp64 instances of the compile-time-width kernels for exponent blocks of
// 1 or 2 values (fewer than the 4 values a lane holds), bits 4..64.
#include "frsz2_fast_dispatch.hpp"

namespace frsz2b {

cudaError_t launch_fast_small_f64(int bits, int E, bool compress, const Job& j, cudaStream_t s, unsigned grid)
{
  using seq = std::make_integer_sequence<int, 61>;
  static constexpr auto t1 = make_small_table<double, 1, 4>(seq{});
  static constexpr auto t2 = make_small_table<double, 2, 4>(seq{});
  if (bits < 4 || bits > 64) return cudaErrorNotSupported;
  switch (E) {
    case 1: return t1[bits - 4](compress, j, s, grid);
    case 2: return t2[bits - 4](compress, j, s, grid);
    default: return cudaErrorNotSupported;
  }
}

} // namespace frsz2b
