// fp32 instances of the fast decompress kernel for block sizes that are a
// multiple of a lane's values but not a power of two (bits 4..32).
#include "frsz2_fast_dispatch.hpp"

namespace frsz2b {
FRSZ2_FAST_GEN_TABLE(float, 4, 32, launch_fast_gen_f32)
} // namespace frsz2b
