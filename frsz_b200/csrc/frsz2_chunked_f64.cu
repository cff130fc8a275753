// fp64 instances of the compile-time-width chunked kernels
// (frsz2_chunked_ct.cuh), bits 4..64.
#include "frsz2_chunked_ct.cuh"

namespace frsz2b {

cudaError_t launch_chunked_ct_f64(int bits, bool compress, const Job& j, cudaStream_t s)
{
  static constexpr auto table = make_chunked_ct_table<double, 4>(std::make_integer_sequence<int, 61>{});
  if (bits < 4 || bits > 64) return cudaErrorNotSupported;
  return table[bits - 4](compress, j, s);
}

} // namespace frsz2b
