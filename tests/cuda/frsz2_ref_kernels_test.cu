// Test library for the drop-in launchable kernels frsz::compress_gpu /
// frsz::decompress_gpu (include/frsz2_b200.hpp): each instance launches them
// with the reference test's own launch shapes (test/test_frsz_gpu.cu:323-330):
// compress <<<ceil(n / 4E), 4E>>>, decompress
// <<<ceil(n / (max(1, 512/E) E)), max(1, 512/E) E>>>.
#include "frsz2_b200.hpp"

#include <cstdint>

template<int B, int E, class T>
static int run(const void* x, std::uint64_t n, void* buf, void* out, cudaStream_t s)
{
  using comp = frsz::frsz2_compressor<B, E, T>;
  comp view(static_cast<std::uint8_t*>(buf), n);
  constexpr int blocks_per_tb = 512 / E > 1 ? 512 / E : 1;
  constexpr int comp_threads = 4 * E;
  const int comp_blocks = (int)((n + comp_threads - 1) / comp_threads);
  constexpr int decomp_threads = blocks_per_tb * E;
  const int decomp_blocks = (int)((n + decomp_threads - 1) / decomp_threads);
  if (comp_blocks > 0)
    frsz::compress_gpu<comp, comp_threads><<<comp_blocks, comp_threads, 0, s>>>(static_cast<const T*>(x), view);
  if (cudaError_t e = cudaGetLastError()) return (int)e;
  if (decomp_blocks > 0) frsz::decompress_gpu<comp><<<decomp_blocks, decomp_threads, 0, s>>>(static_cast<T*>(out), view);
  return (int)cudaGetLastError();
}

// The reference test's end-to-end instances (test/test_frsz_gpu.cu:392-408),
// its E = 1 lossless case (:422-441), and a few more: padded blocks, a block
// size over 32, int8 exponents of fp64, 64-bit words.
#define FRSZ2_REFK_CASES(X)                                                                                        \
  X(double, 32, 32) X(double, 16, 32) X(double, 16, 8) X(double, 15, 8) X(double, 9, 8) X(double, 9, 4)             \
  X(double, 9, 5) X(float, 16, 8) X(float, 15, 8) X(float, 9, 4) X(float, 9, 5) X(float, 32, 1) X(double, 21, 32)   \
  X(float, 13, 100) X(double, 7, 32) X(double, 64, 1) X(double, 47, 16) X(float, 21, 64)

// -1: no instance for (is64, bits, E); otherwise the launches' cudaError_t.
extern "C" int frsz2_refk_test_run(int is64, int bits, int E, const void* x, std::uint64_t n, void* buf, void* out,
                                  void* stream)
{
#define CASE(T, B, EE)                                                                                             \
  if (is64 == (sizeof(T) == 8) && bits == B && E == EE)                                                            \
    return run<B, EE, T>(x, n, buf, out, static_cast<cudaStream_t>(stream));
  FRSZ2_REFK_CASES(CASE)
#undef CASE
  return -1;
}

extern "C" int frsz2_refk_test_cases(int* is64, int* bits, int* E, int cap)
{
  int k = 0;
#define CASE(T, B, EE)                                                                                             \
  if (k < cap) {                                                                                                   \
    is64[k] = sizeof(T) == 8;                                                                                      \
    bits[k] = B;                                                                                                   \
    E[k] = EE;                                                                                                     \
  }                                                                                                                \
  ++k;
  FRSZ2_REFK_CASES(CASE)
#undef CASE
  return k;
}
