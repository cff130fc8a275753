// Test library for the device accessor frsz::frsz2_compressor::
// decompress_gpu_element: one kernel per (bits, block size, float type)
// instance reads values at given indices from inside device code.
#include "frsz2_b200.hpp"

#include <cstdint>

template<int B, int E, class T>
__global__ void k_read(frsz::frsz2_compressor<B, E, T> view, const std::uint64_t* idx, std::uint64_t count, T* out)
{
  for (std::uint64_t t = (std::uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < count;
       t += (std::uint64_t)gridDim.x * blockDim.x)
    out[t] = view.decompress_gpu_element(idx[t]);
}

template<int B, int E, class T>
static int run(const void* buf, std::uint64_t n, const std::uint64_t* idx, std::uint64_t count, void* out,
               cudaStream_t s)
{
  frsz::frsz2_compressor<B, E, T> view(static_cast<std::uint8_t*>(const_cast<void*>(buf)), n);
  const unsigned grid = (unsigned)((count + 255) / 256 < 4096 ? (count + 255) / 256 : 4096);
  k_read<B, E, T><<<grid > 0 ? grid : 1, 256, 0, s>>>(view, idx, count, static_cast<T*>(out));
  return (int)cudaGetLastError();
}

// Instances: every storage width, exact and padded blocks, block sizes that
// are not powers of two, one-value blocks, int8 exponents of fp64.
#define FRSZ2_ACCESSOR_CASES(X)                                                                                    \
  X(float, 16, 32) X(float, 15, 8) X(float, 9, 4) X(float, 9, 5) X(float, 32, 32) X(float, 21, 16) X(float, 4, 8)  \
  X(float, 8, 1) X(float, 32, 1) X(float, 13, 100) X(double, 16, 32) X(double, 21, 32) X(double, 21, 64)           \
  X(double, 9, 5) X(double, 33, 32) X(double, 64, 1) X(double, 52, 16) X(double, 64, 32) X(double, 7, 32)           \
  X(double, 12, 1024) X(double, 40, 4)

// -1: no instance for (is64, bits, E); otherwise the launch's cudaError_t.
extern "C" int frsz2_accessor_test_decode(int is64, int bits, int E, const void* buf, std::uint64_t n,
                                         const std::uint64_t* idx, std::uint64_t count, void* out, void* stream)
{
#define CASE(T, B, EE)                                                                                             \
  if (is64 == (sizeof(T) == 8) && bits == B && E == EE)                                                            \
    return run<B, EE, T>(buf, n, idx, count, out, static_cast<cudaStream_t>(stream));
  FRSZ2_ACCESSOR_CASES(CASE)
#undef CASE
  return -1;
}

extern "C" int frsz2_accessor_test_cases(int* is64, int* bits, int* E, int cap)
{
  int k = 0;
#define CASE(T, B, EE)                                                                                             \
  if (k < cap) {                                                                                                   \
    is64[k] = sizeof(T) == 8;                                                                                      \
    bits[k] = B;                                                                                                   \
    E[k] = EE;                                                                                                     \
  }                                                                                                                \
  ++k;
  FRSZ2_ACCESSOR_CASES(CASE)
#undef CASE
  return k;
}
