// fp64 instances of the compile-time-width kernels (bits 4..64).
#include "frsz2_fast_dispatch.hpp"

namespace frsz2b {
FRSZ2_FAST_TABLE(double, 4, 64, launch_fast_f64)
} // namespace frsz2b
