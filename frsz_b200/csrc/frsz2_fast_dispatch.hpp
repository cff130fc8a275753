// frsz2_fast_dispatch.hpp -- per-width launch table of the fast kernels.
#pragma once

#include "frsz2_fast.cuh"

#include <array>
#include <utility>

namespace frsz2b {

// Enqueue the fast compress / decompress kernel for a compile-time width.
template<class T, int BITS>
cudaError_t launch_fast_one(bool compress, const Job& j, cudaStream_t s, unsigned grid)
{
  if constexpr (!fast_cfg<T, BITS>::ALIGNED) {
    if (job_padded(j)) {
      if (compress)
        k_compress_fast<T, BITS, kNT, 2, true><<<grid, kNT, 0, s>>>(j);
      else
        k_decompress_fast<T, BITS, kNT, 2, true><<<grid, kNT, 0, s>>>(j);
      return cudaGetLastError();
    }
  }
  if (compress)
    k_compress_fast<T, BITS><<<grid, kNT, 0, s>>>(j);
  else
    k_decompress_fast<T, BITS><<<grid, kNT, 0, s>>>(j);
  return cudaGetLastError();
}

using fast_fn = cudaError_t (*)(bool, const Job&, cudaStream_t, unsigned);

template<class T, int LO, int... I>
constexpr auto make_fast_table(std::integer_sequence<int, I...>)
{
  return std::array<fast_fn, sizeof...(I)>{ &launch_fast_one<T, LO + I>... };
}

// Returns cudaErrorNotSupported when `bits` has no instance.
#define FRSZ2_FAST_TABLE(T, LO, HI, NAME)                                                                           \
  cudaError_t NAME(int bits, bool compress, const Job& j, cudaStream_t s, unsigned grid)                          \
  {                                                                                                                \
    static constexpr auto table = make_fast_table<T, LO>(std::make_integer_sequence<int, HI - LO + 1>{});          \
    if (bits < LO || bits > HI) return cudaErrorNotSupported;                                                      \
    return table[bits - LO](compress, j, s, grid);                                                                 \
  }

cudaError_t launch_fast_f32(int bits, bool compress, const Job& j, cudaStream_t s, unsigned grid);
cudaError_t launch_fast_f64(int bits, bool compress, const Job& j, cudaStream_t s, unsigned grid);

// The same kernels for a values pointer off the 32-byte layout (MIS).
template<class T, int BITS>
cudaError_t launch_fast_mis_one(bool compress, const Job& j, cudaStream_t s, unsigned grid)
{
  if constexpr (!fast_cfg<T, BITS>::ALIGNED) {
    if (job_padded(j)) {
      if (compress)
        k_compress_fast<T, BITS, kNT, 2, true, 0, true><<<grid, kNT, 0, s>>>(j);
      else
        k_decompress_fast<T, BITS, kNT, 2, true, 0, true><<<grid, kNT, 0, s>>>(j);
      return cudaGetLastError();
    }
  }
  if (compress)
    k_compress_fast<T, BITS, kNT, 2, false, 0, true><<<grid, kNT, 0, s>>>(j);
  else
    k_decompress_fast<T, BITS, kNT, 2, false, 0, true><<<grid, kNT, 0, s>>>(j);
  return cudaGetLastError();
}

template<class T, int LO, int... I>
constexpr auto make_fast_mis_table(std::integer_sequence<int, I...>)
{
  return std::array<fast_fn, sizeof...(I)>{ &launch_fast_mis_one<T, LO + I>... };
}

#define FRSZ2_FAST_MIS_TABLE(T, LO, HI, NAME)                                                                       \
  cudaError_t NAME(int bits, bool compress, const Job& j, cudaStream_t s, unsigned grid)                          \
  {                                                                                                                \
    static constexpr auto table = make_fast_mis_table<T, LO>(std::make_integer_sequence<int, HI - LO + 1>{});      \
    if (bits < LO || bits > HI) return cudaErrorNotSupported;                                                      \
    return table[bits - LO](compress, j, s, grid);                                                                 \
  }

cudaError_t launch_fast_mis_f32(int bits, bool compress, const Job& j, cudaStream_t s, unsigned grid);
cudaError_t launch_fast_mis_f64(int bits, bool compress, const Job& j, cudaStream_t s, unsigned grid);

// Blocks of E < P values (E = 1, 2 or 4 for fp32; 1 or 2 for fp64): one
// instance per (width, E).
template<class T, int BITS, int ESM>
cudaError_t launch_small_one(bool compress, const Job& j, cudaStream_t s, unsigned grid)
{
  if (compress)
    k_compress_fast<T, BITS, kNT, 2, false, ESM><<<grid, kNT, 0, s>>>(j);
  else
    k_decompress_fast<T, BITS, kNT, 2, false, ESM><<<grid, kNT, 0, s>>>(j);
  return cudaGetLastError();
}

template<class T, int ESM, int LO, int... I>
constexpr auto make_small_table(std::integer_sequence<int, I...>)
{
  return std::array<fast_fn, sizeof...(I)>{ &launch_small_one<T, LO + I, ESM>... };
}

// Returns cudaErrorNotSupported when (bits, E) has no instance.
cudaError_t launch_fast_small_f32(int bits, int E, bool compress, const Job& j, cudaStream_t s, unsigned grid);
cudaError_t launch_fast_small_f64(int bits, int E, bool compress, const Job& j, cudaStream_t s, unsigned grid);

} // namespace frsz2b
