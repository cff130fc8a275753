// fp32 instances of the compile-time block-size kernels
// (frsz2_blockwise_ce.cuh) for blocks of 7 values, bits 4..32.
#include "frsz2_blockwise_ce.cuh"

FRSZ2_BWC_DEFINE(f32, float, 7, 4, 29)
