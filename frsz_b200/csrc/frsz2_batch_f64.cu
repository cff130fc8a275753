// fp64 instances of the batched persistent kernel.
#include "frsz2_batch_kernels.cuh"

#include <array>
#include <utility>

namespace frsz2b {

template<int LO, int... I>
constexpr auto f64_shape0(std::integer_sequence<int, I...>)
{
  return std::array<batch_entry, sizeof...(I)>{ batch_entry{ &launch_batch_class<double, LO + I, 256, 2>,
                                                             &batch_class_occupancy<double, LO + I, 256, 2>,
                                                             &launch_batch_tiles<double, LO + I, 256, 2> }... };
}

batch_entry batch_class_f64(int bits, int shape)
{
  static constexpr auto s0 = f64_shape0<4>(std::make_integer_sequence<int, 61>{});
  if (bits < 4 || bits > 64) return { nullptr, nullptr };
  if (shape == 0) return s0[bits - 4];
  switch (bits * 4 + shape) {
#define TUNED(B)                                                                                                   \
  case B * 4 + 1: return { &launch_batch_class<double, B, 128, 2>, &batch_class_occupancy<double, B, 128, 2> };      \
  case B * 4 + 2: return { &launch_batch_class<double, B, 512, 1>, &batch_class_occupancy<double, B, 512, 1> };
    FRSZ2_TUNED_WIDTHS(TUNED)
#undef TUNED
    default: return { nullptr, nullptr };
  }
}

} // namespace frsz2b
