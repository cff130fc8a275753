// frsz2_blockvec.cuh -- compile-time-width compress kernel for exponent
// blocks of 17 to kBvMaxE values whose bytes fall on 16-byte boundaries: one
// thread per block, straight from global memory with 16-byte loads.
//
// Taken when E * sizeof(T) is a multiple of 16 (fp32 E divisible by 4, fp64
// by 2), the block bytes are a multiple of 4, bits <= 32 and both pointers
// are 16-byte aligned.  The kernel covers the array's whole blocks; the
// caller runs a partial last block on the generic kernel.
//
// A thread reads its block's values twice with 16-byte loads (the second
// pass mostly from L1 / L2): the block maximum, then the codes, which are
// added into 32-bit words at compile-time bit positions (a block's W-bit words
// are the same little-endian bit stream as 32-bit words when the block starts
// on a 4-byte boundary) and stored as each word -- or, when the block bytes
// are a multiple of 16, each group of four words -- completes.  The per-value
// arithmetic is the fast kernels', so the bytes are the reference's bit for
// bit.  (A decompress counterpart, one thread per block storing its values
// with 16-byte stores, measured slower on B200 than the chunked kernel's
// shared-memory staging: fp32 b16 E48 0.25 vs 0.33 of HBM, fp64 b32 E48 0.24
// vs 0.52.)
#pragma once

#include "frsz2_fast.cuh"
#include "frsz2_launch.hpp"

#include <algorithm>
#include <array>
#include <utility>

namespace frsz2b {

constexpr int kBvMinE = 17; // smaller blocks go to the blockwise kernels
constexpr int kBvMaxE = 64; // largest block size
constexpr int kBvThreads = 256;

template<class T, int BITS>
__global__ void __launch_bounds__(kBvThreads) k_compress_blockvec(Job j, std::uint64_t nb_full)
{
  static_assert(BITS <= 32, "codes of at most 32 bits");
  using Cfg = fast_cfg<T, BITS>;
  using U = typename Cfg::U;
  using K = key_of<T>;
  constexpr int W = Cfg::W;
  constexpr int VPL = 16 / (int)sizeof(T); // values per 16-byte load
  const int E = j.E;
  const std::uint32_t BB = j.block_bytes;
  const bool v4 = BB % 16 == 0;
  const std::uint64_t stride = (std::uint64_t)gridDim.x * kBvThreads;
  for (std::uint64_t b = (std::uint64_t)blockIdx.x * kBvThreads + threadIdx.x; b < nb_full; b += stride) {
    const uint4* __restrict__ xv = reinterpret_cast<const uint4*>(static_cast<const T*>(j.values_in) + b * E);
    auto value = [&](const uint4& v, int i) -> U { // i compile-time after unrolling
      if constexpr (sizeof(T) == 4)
        return i == 0 ? v.x : i == 1 ? v.y : i == 2 ? v.z : v.w;
      else
        return i == 0 ? ((std::uint64_t)v.y << 32) | v.x : ((std::uint64_t)v.w << 32) | v.z;
    };
    // pass 1: the block maximum of the raw keys, doubled (sign shifted out)
    std::uint32_t kr2 = 0;
#pragma unroll
    for (int q = 0; q < kBvMaxE / VPL; ++q) {
      if (q * VPL >= E) break;
      const uint4 v = __ldg(xv + q);
#pragma unroll
      for (int i = 0; i < VPL; ++i) {
        const U u = value(v, i);
        const std::uint32_t hi = sizeof(T) == 4 ? (std::uint32_t)u : (std::uint32_t)((std::uint64_t)u >> 32);
        kr2 = max(kr2, hi * 2u);
      }
    }
    const std::uint32_t kr = kr2 >> 1;
    // block exponent: the largest non-NaN magnitude's (std::max semantics)
    std::uint32_t kc = kr;
    if (kr >= K::SPECIAL) {
      kc = 0;
      for (int q = 0; q * VPL < E; ++q) {
        const uint4 v = __ldg(xv + q);
#pragma unroll
        for (int i = 0; i < VPL; ++i) kc = max(kc, K::clean(value(v, i)));
      }
    }
    const std::int64_t ex = exponent_of_field<T>((int)(kc >> K::FSHIFT));
    const std::int64_t be = wrap_signed(ex, W);
    const bool plain = kr < K::SPECIAL && be == ex && plain_exponent<T>(be);
    const T scale = pow2<T>(plain ? BITS - 2 - (int)be : 0);
    std::uint32_t* __restrict__ dst = reinterpret_cast<std::uint32_t*>(j.words + b * (std::uint64_t)BB);

    // pass 2: codes into 32-bit words, stored as they complete (in groups of
    // four when the block bytes allow 16-byte stores).  The block's last word
    // has index BB / 4 - 1 (BB * 8 - E * BITS < W <= 32), which ends a group
    // of four when BB is a multiple of 16.
    auto pack = [&](auto encode) {
      std::uint32_t cur = 0, grp[4] = { 0, 0, 0, 0 };
      uint4 v = make_uint4(0, 0, 0, 0);
      auto emit = [&](int wi, std::uint32_t word) { // wi compile-time after unrolling
        if (v4) {
          grp[wi % 4] = word;
          if (wi % 4 == 3) reinterpret_cast<uint4*>(dst)[wi / 4] = make_uint4(grp[0], grp[1], grp[2], grp[3]);
        } else {
          dst[wi] = word;
        }
      };
#pragma unroll
      for (int k = 0; k <= kBvMaxE; ++k) {
        const int p = k * BITS, wi = p / 32, o = p % 32;
        if (k == kBvMaxE || k >= E) {
          if (o != 0) emit(wi, cur); // the last, partial word (pad bits zero)
          break;
        }
        if (k % VPL == 0) v = __ldg(xv + k / VPL);
        const std::uint32_t c = encode(value(v, k % VPL));
        cur = c * (1u << o) + cur; // the bits do not overlap: the sum is the OR
        if (o + BITS >= 32) {
          emit(wi, cur);
          cur = o + BITS > 32 ? c >> (32 - o) : 0u;
        }
      }
    };
    if (plain)
      pack([&](U u) { return (std::uint32_t)encode_plain<T, BITS>(u, scale); });
    else
      pack([&](U u) { return (std::uint32_t)to_code<T>(u, (std::int16_t)be, BITS); });
    store_word(j.exps + b * (std::uint64_t)(W / 8), (std::uint64_t)be, W);
  }
}

// Whether the blockvec kernel takes a compress job (the caller runs a partial
// last block elsewhere).
inline bool blockvec_eligible(const Job& j, int es, const void* values, const void* words)
{
  if (j.E < kBvMinE || j.E > kBvMaxE || j.bits > 32) return false;
  if (((std::uint64_t)j.E * (std::uint64_t)es) % 16 != 0 || j.block_bytes % 4 != 0) return false;
  return reinterpret_cast<std::uintptr_t>(values) % 16 == 0 && reinterpret_cast<std::uintptr_t>(words) % 16 == 0;
}

template<class T, int BITS>
cudaError_t launch_blockvec_one(const Job& j, std::uint64_t nb_full, cudaStream_t s)
{
  if (nb_full == 0) return cudaSuccess;
  const std::uint64_t ctas = (nb_full + kBvThreads - 1) / kBvThreads;
  const unsigned grid = (unsigned)std::min<std::uint64_t>(ctas, (std::uint64_t)sm_count() * 32);
  k_compress_blockvec<T, BITS><<<grid, kBvThreads, 0, s>>>(j, nb_full);
  return cudaGetLastError();
}

using blockvec_fn = cudaError_t (*)(const Job&, std::uint64_t, cudaStream_t);

template<class T, int LO, int... I>
constexpr auto make_blockvec_table(std::integer_sequence<int, I...>)
{
  return std::array<blockvec_fn, sizeof...(I)>{ &launch_blockvec_one<T, LO + I>... };
}

cudaError_t launch_blockvec_f32(int bits, const Job& j, std::uint64_t nb_full, cudaStream_t s);
cudaError_t launch_blockvec_f64(int bits, const Job& j, std::uint64_t nb_full, cudaStream_t s);

} // namespace frsz2b
