// fp64 instances of the one-thread-per-block compress kernel with 16-byte
// global loads (frsz2_blockvec.cuh), bits 4..32.
#include "frsz2_blockvec.cuh"

namespace frsz2b {

cudaError_t launch_blockvec_f64(int bits, const Job& j, std::uint64_t nb_full, cudaStream_t s)
{
  static constexpr auto table = make_blockvec_table<double, 4>(std::make_integer_sequence<int, 29>{});
  if (bits < 4 || bits > 32) return cudaErrorNotSupported;
  return table[bits - 4](j, nb_full, s);
}

} // namespace frsz2b
