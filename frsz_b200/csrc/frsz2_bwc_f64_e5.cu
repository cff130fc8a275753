// fp64 instances of the compile-time block-size kernels
// (frsz2_blockwise_ce.cuh) for blocks of 5 values, bits 4..64.
#include "frsz2_blockwise_ce.cuh"

FRSZ2_BWC_DEFINE(f64, double, 5, 4, 61)
