// fp64 instances of the fast decompress kernel for block sizes that are a
// multiple of a lane's values but not a power of two (bits 4..64).
#include "frsz2_fast_dispatch.hpp"

namespace frsz2b {
FRSZ2_FAST_GEN_TABLE(double, 4, 64, launch_fast_gen_f64)
} // namespace frsz2b
