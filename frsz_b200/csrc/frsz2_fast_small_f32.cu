// fp32 instances of the compile-time-width kernels for exponent blocks of
// 1, 2 or 4 values (fewer than the 8 values a lane holds), bits 4..32.
#include "frsz2_fast_dispatch.hpp"

namespace frsz2b {

cudaError_t launch_fast_small_f32(int bits, int E, bool compress, const Job& j, cudaStream_t s, unsigned grid)
{
  using seq = std::make_integer_sequence<int, 29>;
  static constexpr auto t1 = make_small_table<float, 1, 4>(seq{});
  static constexpr auto t2 = make_small_table<float, 2, 4>(seq{});
  static constexpr auto t4 = make_small_table<float, 4, 4>(seq{});
  if (bits < 4 || bits > 32) return cudaErrorNotSupported;
  switch (E) {
    case 1: return t1[bits - 4](compress, j, s, grid);
    case 2: return t2[bits - 4](compress, j, s, grid);
    case 4: return t4[bits - 4](compress, j, s, grid);
    default: return cudaErrorNotSupported;
  }
}

} // namespace frsz2b
