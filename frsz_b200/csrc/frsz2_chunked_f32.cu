// fp32 instances of the compile-time-width chunked kernels
// (frsz2_chunked_ct.cuh), bits 4..32.
#include "frsz2_chunked_ct.cuh"

namespace frsz2b {

cudaError_t launch_chunked_ct_f32(int bits, bool compress, const Job& j, cudaStream_t s)
{
  static constexpr auto table = make_chunked_ct_table<float, 4>(std::make_integer_sequence<int, 29>{});
  if (bits < 4 || bits > 32) return cudaErrorNotSupported;
  return table[bits - 4](compress, j, s);
}

} // namespace frsz2b
