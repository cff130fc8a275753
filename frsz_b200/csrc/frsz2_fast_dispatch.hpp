// frsz2_fast_dispatch.hpp -- per-width launch table of the fast kernels.
#pragma once

#include "frsz2_fast.cuh"

#include <algorithm>
#include <array>
#include <utility>

namespace frsz2b {

// Launch shape of the decompress kernel for a width whose lane segments are
// not word-aligned (bit 1: 128 threads per CTA instead of 256; bit 0:
// registers capped for 2048 resident threads per SM), measured per width on
// B200 at 2^28 (fp64) / 2^29 (fp32) values, blocks of 32 and 64: a shape other
// than 0 where it gained at least 1 % (up to 29 %, fp32 at 7 bits).  Aligned
// widths (multiples of 4 bits for fp32, of 8 for fp64) do not use the table.
template<class T, int BITS>
constexpr int unaligned_decompress_shape()
{
  constexpr signed char f32[33] = { 0, 0, 0, 0, 0, 0, 0, 3, 0, 0, 0, 3, 0, 2, 2, 3, 0,
                                    2, 2, 3, 0, 0, 3, 2, 0, 2, 2, 2, 0, 2, 2, 2, 0 };
  constexpr signed char f64[65] = { 0, 0, 0, 0, 1, 3, 3, 3, 0, 0, 0, 3, 0, 3, 3, 3, 0, 0, 0, 3, 0, 3,
                                    3, 3, 0, 0, 0, 3, 0, 3, 3, 3, 0, 2, 2, 2, 2, 2, 2, 2, 0, 2, 2, 2,
                                    2, 0, 2, 2, 0, 2, 2, 2, 2, 2, 2, 2, 0, 2, 2, 2, 2, 0, 0, 0, 0 };
  return sizeof(T) == 8 ? f64[BITS] : f32[BITS];
}

template<class T, int BITS, int SH>
cudaError_t launch_decompress_unaligned(const Job& j, cudaStream_t s, unsigned grid)
{
  constexpr int NT = (SH & 2) ? 128 : kNT;
  constexpr int TE = fast_tile_values((int)sizeof(T), NT, 2);
  Job t = j;
  if constexpr (NT != kNT) {
    // tiles of NT / 32 * 2 rows (the caller checked E <= TE)
    t.tile_blocks = (std::uint32_t)(TE / j.E);
    t.tiles = (j.n + TE - 1) / TE;
    grid = (unsigned)std::min<std::uint64_t>(t.tiles, 1u << 30);
  }
  const bool pad = job_padded(j);
  if constexpr ((SH & 1) != 0) {
    if (pad)
      k_decompress_fast_occ<T, BITS, NT, true><<<grid, NT, 0, s>>>(t);
    else
      k_decompress_fast_occ<T, BITS, NT, false><<<grid, NT, 0, s>>>(t);
  } else {
    if (pad)
      k_decompress_fast<T, BITS, NT, 2, true><<<grid, NT, 0, s>>>(t);
    else
      k_decompress_fast<T, BITS, NT, 2, false><<<grid, NT, 0, s>>>(t);
  }
  return cudaGetLastError();
}

// Enqueue the fast compress / decompress kernel for a compile-time width.
template<class T, int BITS>
cudaError_t launch_fast_one(bool compress, const Job& j, cudaStream_t s, unsigned grid)
{
  if constexpr (!fast_cfg<T, BITS>::ALIGNED) {
    if (!compress) {
      constexpr int sh = unaligned_decompress_shape<T, BITS>();
      if ((sh & 2) == 0 || j.E <= fast_tile_values((int)sizeof(T), 128, 2))
        return launch_decompress_unaligned<T, BITS, sh>(j, s, grid);
      return launch_decompress_unaligned<T, BITS, sh & 1>(j, s, grid);
    }
    if (job_padded(j)) {
      if (compress)
        k_compress_fast<T, BITS, kNT, 2, true><<<grid, kNT, 0, s>>>(j);
      else
        k_decompress_fast<T, BITS, kNT, 2, true><<<grid, kNT, 0, s>>>(j);
      return cudaGetLastError();
    }
  }
  if (compress && j.E == 64 * fast_cfg<T, BITS>::P) {
    // blocks of two warp rows (fp32 512, fp64 256 values): each warp's two rows
    // are consecutive, so a block's maximum needs no barrier (measured: fp64 12
    // bits 0.85 -> 1.01, fp32 8 bits 0.87 -> 1.03 of HBM; 32 / 64 bits even)
    k_compress_fast<T, BITS, kNT, 2, false, 0, false, false, false, true><<<grid, kNT, 0, s>>>(j);
    return cudaGetLastError();
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

// Blocks whose size is a multiple of a lane's values, or of half of them, but
// not a power of two (fast_gen_tile_blocks; the caller sets the Job's
// whole-block tiles).  cudaErrorNotSupported sends the job to the other
// kernels.
template<class T, int BITS>
cudaError_t launch_fast_gen_one(bool compress, const Job& j, cudaStream_t s, unsigned grid)
{
  const bool pad = job_padded(j);
  if (j.E % fast_cfg<T, BITS>::P != 0) {
    // a multiple of half a lane, blocks without padding: two exponents per
    // lane; compress reads up to 32 half-lane maxima per block, and blocks of
    // up to 16 values keep the one-thread-per-block kernels (measured faster:
    // fp64 16 bits E 6 1.04 against 0.67 of HBM, fp32 16 bits E 12 0.82 / 0.69)
    if (pad) return cudaErrorNotSupported;
    if (compress) {
      if (j.E <= 16 || j.E > 16 * fast_cfg<T, BITS>::P) return cudaErrorNotSupported;
      k_compress_fast<T, BITS, kNT, 2, false, 0, false, true, true><<<grid, kNT, 0, s>>>(j);
    } else {
      k_decompress_fast<T, BITS, kNT, 2, false, 0, false, true, true><<<grid, kNT, 0, s>>>(j);
    }
    return cudaGetLastError();
  }
  if (compress) {
    // a lane reads its block's E / P lane maxima: up to 32 of them; padded
    // blocks keep the other kernels
    if (pad || j.E > 32 * fast_cfg<T, BITS>::P) return cudaErrorNotSupported;
    k_compress_fast<T, BITS, kNT, 2, false, 0, false, true><<<grid, kNT, 0, s>>>(j);
  } else if (pad) {
    // padded blocks: lanes place their bits by stream position (unaligned widths)
    if constexpr (fast_cfg<T, BITS>::ALIGNED)
      return cudaErrorNotSupported;
    else
      k_decompress_fast<T, BITS, kNT, 2, true, 0, false, true><<<grid, kNT, 0, s>>>(j);
  } else {
    k_decompress_fast<T, BITS, kNT, 2, false, 0, false, true><<<grid, kNT, 0, s>>>(j);
  }
  return cudaGetLastError();
}

template<class T, int LO, int... I>
constexpr auto make_fast_gen_table(std::integer_sequence<int, I...>)
{
  return std::array<fast_fn, sizeof...(I)>{ &launch_fast_gen_one<T, LO + I>... };
}

#define FRSZ2_FAST_GEN_TABLE(T, LO, HI, NAME)                                                                       \
  cudaError_t NAME(int bits, bool compress, const Job& j, cudaStream_t s, unsigned grid)                          \
  {                                                                                                                \
    static constexpr auto table = make_fast_gen_table<T, LO>(std::make_integer_sequence<int, HI - LO + 1>{});      \
    if (bits < LO || bits > HI) return cudaErrorNotSupported;                                                      \
    return table[bits - LO](compress, j, s, grid);                                                                 \
  }

cudaError_t launch_fast_gen_f32(int bits, bool compress, const Job& j, cudaStream_t s, unsigned grid);
cudaError_t launch_fast_gen_f64(int bits, bool compress, const Job& j, cudaStream_t s, unsigned grid);

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
