// fp64 instances of the fast kernels for a values pointer off the
// 32-byte layout (aligned to the element size), bits 4..64.
#include "frsz2_fast_dispatch.hpp"

namespace frsz2b {
FRSZ2_FAST_MIS_TABLE(double, 4, 64, launch_fast_mis_f64)
} // namespace frsz2b
