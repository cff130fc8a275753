// fp32 instances of the compile-time-width kernels (bits 4..32).
#include "frsz2_fast_dispatch.hpp"

namespace frsz2b {
FRSZ2_FAST_TABLE(float, 4, 32, launch_fast_f32)
} // namespace frsz2b
