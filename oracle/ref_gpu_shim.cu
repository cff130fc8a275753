// ref_gpu_shim.cu -- C entry points over the reference's own GPU kernels
// frsz::compress_gpu / frsz::decompress_gpu (include/frsz2.hpp:1258-1290),
// compiled unmodified from the reference header for sm_100a.
//
// TEST INFRASTRUCTURE ONLY: tests/test_gpu_reference_speed.py times these
// kernels beside this repository's on the same inputs (the reference's GPU
// kernels are the GPU speed bar; they are not the oracle -- their decode of
// zero codes differs from the reference CPU codec).  Launch shapes follow the
// reference's own test (test/test_frsz_gpu.cu:323-330, 340-341, 369-370).
#include "frsz2.hpp"

#include <cstdint>

namespace {

template<int B, int E, class T>
int run(bool compress, const void* in, std::size_t n, void* out, cudaStream_t s)
{
  using C = frsz::frsz2_compressor<B, E, T>;
  if (compress) {
    C c(static_cast<std::uint8_t*>(out), n);
    constexpr int threads = 4 * E;
    const int blocks = (int)((n + threads - 1) / threads);
    frsz::compress_gpu<C, threads><<<blocks, threads, 0, s>>>(static_cast<const T*>(in), c);
  } else {
    C c(const_cast<std::uint8_t*>(static_cast<const std::uint8_t*>(in)), n);
    constexpr int threads = (512 / E > 1 ? 512 / E : 1) * E;
    const int blocks = (int)((n + threads - 1) / threads);
    frsz::decompress_gpu<C><<<blocks, threads, 0, s>>>(static_cast<T*>(out), c);
  }
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

} // namespace

// Instances: the benchmark configurations the reference kernels compile for
// (its aligned path, bits == word width, requires E <= 32).
extern "C" int frsz2ref_gpu(int is_f64, int bits, int E, int compress, const void* in, std::size_t n, void* out,
                            void* stream)
{
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int key = is_f64 * 100000 + bits * 1000 + E;
  switch (key) {
    case 16 * 1000 + 32: return run<16, 32, float>(compress, in, n, out, s);
    case 32 * 1000 + 32: return run<32, 32, float>(compress, in, n, out, s);
    case 100000 + 16 * 1000 + 32: return run<16, 32, double>(compress, in, n, out, s);
    case 100000 + 21 * 1000 + 32: return run<21, 32, double>(compress, in, n, out, s);
    case 100000 + 32 * 1000 + 32: return run<32, 32, double>(compress, in, n, out, s);
    case 100000 + 21 * 1000 + 64: return run<21, 64, double>(compress, in, n, out, s);
    default: return 2;
  }
}
