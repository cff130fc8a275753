// fp32 instances of the fast kernels for a values pointer off the
// 32-byte layout (aligned to the element size), bits 4..32.
#include "frsz2_fast_dispatch.hpp"

namespace frsz2b {
FRSZ2_FAST_MIS_TABLE(float, 4, 32, launch_fast_mis_f32)
} // namespace frsz2b
