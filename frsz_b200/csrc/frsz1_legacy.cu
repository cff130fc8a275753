// frsz1_legacy.cu -- the reference's legacy "frsz" codec (the LibPressio
// plugin of src/frsz.cc:15-165): values quantized with step 2*epsilon, stored
// as int16 differences to the previous quantized value within blocks of 256
// values; decoding is a running sum per block.
//
// Bit-exact with the reference's arithmetic (src/frsz.cc:113-148):
//   compress   q[i] = (T) round((double) x[i] * (1 / (2 eps)))   (half away from 0)
//              d[i] = q[i] - (i % 256 ? q[i-1] : 0)                (in T)
//              out[i] = int16 saturate(d[i])   (truncation; NaN -> 0 as on x86)
//   decompress y[256b] = (T)((double)(T)in[256b] * 2eps)
//              y[256b+i] = (T)((double)(T)in[k] * 2eps + (double) y[256b+i-1])
// with k = i (the reference reads block 0's deltas for every block) or, with
// FRSZ1_OWN_DELTAS, k = 256b + i.  Multiplies and adds are separate
// round-to-nearest operations (no contraction), as in the reference's build.
//
// compress is elementwise: a thread takes 8 (fp32) or 4 (fp64) consecutive
// values with one 32-byte load, its left neighbour's quantized value by a
// shuffle, and writes 16 or 8 bytes.  decompress runs one thread per block of
// 256 values (the sum is sequential and rounds at every step); 64 blocks per
// CTA go out through shared memory 16 values at a time, so the stores are
// coalesced.
#include "frsz2_fast.cuh"
#include "frsz2_launch.hpp"

#include "../../include/frsz2_b200.h"

#include <algorithm>
#include <cmath>

namespace frsz2b {
namespace {

constexpr int kLegacyBlock = 256; // src/frsz.cc:103, 132

#ifndef FRSZ1_MAGIC_ROUNDING
#define FRSZ1_MAGIC_ROUNDING 1
#endif

// std::round (half away from zero) of a double with additions only, by the
// magic-constant method for rounding to an integer (Muller et al., Handbook
// of Floating-Point Arithmetic, 2nd ed., sec. 5.1): adding 2^52 rounded
// toward zero to v = |p| + 0.5 leaves floor(v) + 2^52, from which 2^52 is
// subtracted exactly.  v itself is rounded, but for 0.5 <= |p| < 2^52 that
// rounding never carries it across an integer: |p| and 0.5 are multiples of
// ulp(|p|), so v is exact unless it has moved into the next binade, and a
// binade starts at a power of two, which is an integer with no other integer
// within 0.5 above it.  Below 0.5 it can: |p| = 0.5 - 2^-54 (the double just
// below 0.5) gives v = 1 - 2^-54, which rounds to 1.0, where std::round gives
// 0.  So |p| < 0.5 is 0 by a select.  The sign is copied back (so -0.4 gives
// -0.0 as std::round does).  |p| >= 2^52 (already an integer), Inf and NaN
// are returned as they are.
__device__ __forceinline__ double round_half_away(double p)
{
  constexpr double TWO52 = 4503599627370496.0;
  const double a = fabs(p);
  const double t = a < 0.5 ? 0.0 : __dsub_rn(__dadd_rz(__dadd_rn(a, 0.5), TWO52), TWO52);
  return copysign(a < TWO52 ? t : a, p);
}

template<class T>
__device__ __forceinline__ T legacy_quantize(T x, double inv)
{
  const double p = __dmul_rn((double)x, inv);
  // fp32 (conversion-bound: 0.76 -> 0.98 of HBM) only; fp64 measured even
  const double q = FRSZ1_MAGIC_ROUNDING && sizeof(T) == 4 ? round_half_away(p) : round(p);
  if constexpr (sizeof(T) == 4)
    return __double2float_rn(q);
  else
    return q;
}

// saturate<int16_t> (src/frsz.cc:97-101).  d is a difference of two
// integer-valued floats, so it is itself integer-valued (or +-Inf / NaN):
// clamped to [-32768, 32767] it converts exactly.  For fp32 that is done by
// adding 1.5 * 2^23 and reading the integer from the low bits of the sum (the
// same magic-constant method) instead of a conversion instruction.
template<class T>
__device__ __forceinline__ std::int16_t legacy_saturate(T d)
{
  if (d != d) return 0;
  if (!FRSZ1_MAGIC_ROUNDING || sizeof(T) == 8) {
    if (d < (T)-32768) return (std::int16_t)-32768;
    if (d > (T)32767) return (std::int16_t)32767;
    if constexpr (sizeof(T) == 4)
      return (std::int16_t)__float2int_rz(d);
    else
      return (std::int16_t)__double2int_rz(d);
  }
  const float c = fminf(fmaxf((float)d, -32768.0f), 32767.0f);
  return (std::int16_t)(__float_as_int(__fadd_rn(c, 12582912.0f)) - 0x4B400000);
}

template<class T>
__device__ __forceinline__ T legacy_sub(T a, T b)
{
  if constexpr (sizeof(T) == 4)
    return __fsub_rn(a, b);
  else
    return __dsub_rn(a, b);
}

template<class T>
__global__ void __launch_bounds__(256) k_frsz1_compress(const T* __restrict__ x, std::uint64_t n, double inv,
                                                        std::int16_t* __restrict__ out, bool vec)
{
  constexpr int V = 32 / (int)sizeof(T);
  const int lane = threadIdx.x & 31;
  const std::uint64_t i0 = ((std::uint64_t)blockIdx.x * blockDim.x + threadIdx.x) * V;
  T q[V];
  if (vec && i0 + V <= n) {
    std::uint32_t v[8];
    ld256_stream(x + i0, v);
#pragma unroll
    for (int k = 0; k < V; ++k) {
      T xv;
      if constexpr (sizeof(T) == 4)
        xv = __uint_as_float(v[k]);
      else
        xv = __longlong_as_double((long long)(((std::uint64_t)v[2 * k + 1] << 32) | v[2 * k]));
      q[k] = legacy_quantize<T>(xv, inv);
    }
  } else {
#pragma unroll
    for (int k = 0; k < V; ++k) q[k] = i0 + k < n ? legacy_quantize<T>(x[i0 + k], inv) : (T)0;
  }
  // the quantized value before this thread's first: the previous lane's last
  T prev = __shfl_up_sync(0xFFFFFFFFu, q[V - 1], 1);
  if (lane == 0 && i0 > 0 && i0 - 1 < n) prev = legacy_quantize<T>(x[i0 - 1], inv);
  std::int16_t d[V];
#pragma unroll
  for (int k = 0; k < V; ++k) {
    const T p = k == 0 ? prev : q[k - 1];
    d[k] = legacy_saturate<T>(((i0 + k) % kLegacyBlock == 0) ? legacy_sub<T>(q[k], (T)0) : legacy_sub<T>(q[k], p));
  }
  if (i0 + V <= n && vec) {
    if constexpr (V == 8) {
      uint4 w;
      w.x = (std::uint16_t)d[0] | ((std::uint32_t)(std::uint16_t)d[1] << 16);
      w.y = (std::uint16_t)d[2] | ((std::uint32_t)(std::uint16_t)d[3] << 16);
      w.z = (std::uint16_t)d[4] | ((std::uint32_t)(std::uint16_t)d[5] << 16);
      w.w = (std::uint16_t)d[6] | ((std::uint32_t)(std::uint16_t)d[7] << 16);
      __stcs(reinterpret_cast<uint4*>(out + i0), w);
    } else {
      uint2 w;
      w.x = (std::uint16_t)d[0] | ((std::uint32_t)(std::uint16_t)d[1] << 16);
      w.y = (std::uint16_t)d[2] | ((std::uint32_t)(std::uint16_t)d[3] << 16);
      __stcs(reinterpret_cast<uint2*>(out + i0), w);
    }
  } else {
#pragma unroll
    for (int k = 0; k < V; ++k)
      if (i0 + k < n) out[i0 + k] = d[k];
  }
}

constexpr int kDecBlocks = 64; // blocks of 256 values per CTA (one thread each)
constexpr int kDecChunk = 16;  // values per block staged at a time

template<class T>
__device__ __forceinline__ T legacy_step(std::int16_t q, double ebx2, T prev)
{
  const double t = __dadd_rn(__dmul_rn((double)(T)q, ebx2), (double)prev);
  if constexpr (sizeof(T) == 4)
    return __double2float_rn(t);
  else
    return t;
}

template<class T, bool OWN>
__global__ void __launch_bounds__(kDecBlocks) k_frsz1_decompress(const std::int16_t* __restrict__ in, std::uint64_t n,
                                                                  double ebx2, T* __restrict__ y, bool vec)
{
  // block 0's differences (the reference reads them for every block)
  __shared__ std::int16_t s_d0[OWN ? 1 : kLegacyBlock];
  __shared__ T s_out[kDecBlocks][kDecChunk + 1];
  const int tid = threadIdx.x;
  const std::uint64_t b0 = (std::uint64_t)blockIdx.x * kDecBlocks; // first block of the CTA
  const std::uint64_t v0 = b0 * kLegacyBlock;
  if constexpr (!OWN) {
    const std::uint64_t n0 = n < (std::uint64_t)kLegacyBlock ? n : (std::uint64_t)kLegacyBlock;
    for (std::uint64_t i = tid; i < n0; i += kDecBlocks) s_d0[i] = in[i];
  }
  __syncthreads();
  const std::uint64_t g0 = v0 + (std::uint64_t)tid * kLegacyBlock; // this thread's block
  const int len = g0 < n ? (int)((n - g0) < (std::uint64_t)kLegacyBlock ? n - g0 : (std::uint64_t)kLegacyBlock) : 0;
  T acc = (T)0;
  // own codes: two 16-byte loads per chunk, issued one chunk ahead so their
  // latency overlaps the previous chunk's sums
  uint4 pa = make_uint4(0, 0, 0, 0), pb = pa;
  auto fetch = [&](int c) {
    if (OWN && vec && c + kDecChunk <= len) {
      const uint4* p = reinterpret_cast<const uint4*>(in + g0 + c);
      pa = __ldg(p);
      pb = __ldg(p + 1);
    }
  };
  fetch(0);
  for (int c = 0; c < kLegacyBlock; c += kDecChunk) {
    // this chunk's codes: the block's own or block 0's
    std::int16_t qc[kDecChunk];
    if constexpr (OWN) {
      if (vec && c + kDecChunk <= len) {
        const uint4 a = pa, b = pb;
        if (c + kDecChunk < kLegacyBlock) fetch(c + kDecChunk);
        const std::uint32_t w[8] = { a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w };
#pragma unroll
        for (int k = 0; k < kDecChunk; ++k) qc[k] = (std::int16_t)(w[k / 2] >> (16 * (k % 2)));
      } else {
#pragma unroll
        for (int k = 0; k < kDecChunk; ++k) qc[k] = c + k < len ? in[g0 + c + k] : (std::int16_t)0;
      }
    } else {
#pragma unroll
      for (int k = 0; k < kDecChunk; ++k) qc[k] = (c + k == 0) ? (len > 0 ? in[g0] : (std::int16_t)0) : s_d0[c + k];
    }
#pragma unroll
    for (int k = 0; k < kDecChunk; ++k) {
      const int i = c + k;
      if (i < len) {
        if (i == 0) {
          const double t = __dmul_rn((double)(T)qc[0], ebx2);
          if constexpr (sizeof(T) == 4)
            acc = __double2float_rn(t);
          else
            acc = t;
        } else {
          acc = legacy_step<T>(qc[k], ebx2, acc);
        }
        s_out[tid][k] = acc;
      }
    }
    __syncthreads();
    // chunk c of every block: consecutive threads take consecutive values of
    // a block, then the next block
    for (int idx = tid; idx < kDecBlocks * kDecChunk; idx += kDecBlocks) {
      const int b = idx / kDecChunk, k = idx % kDecChunk;
      const std::uint64_t g = v0 + (std::uint64_t)b * kLegacyBlock + c + k;
      if (g < n) y[g] = s_out[b][k];
    }
    __syncthreads();
  }
}

template<class T>
int legacy_compress(double eps, const void* d_values, std::uint64_t n, void* d_out, cudaStream_t s)
{
  constexpr int V = 32 / (int)sizeof(T);
  const bool vec = reinterpret_cast<std::uintptr_t>(d_values) % 32 == 0 &&
                   reinterpret_cast<std::uintptr_t>(d_out) % (2 * V) == 0;
  const std::uint64_t threads = (n + V - 1) / V;
  const unsigned grid = (unsigned)std::max<std::uint64_t>(1, (threads + 255) / 256);
  k_frsz1_compress<T><<<grid, 256, 0, s>>>(static_cast<const T*>(d_values), n, 1.0 / (eps * 2.0),
                                          static_cast<std::int16_t*>(d_out), vec);
  return cuda_status(cudaGetLastError(), "legacy compress launch");
}

template<class T>
int legacy_decompress(double eps, const void* d_in, std::uint64_t n, void* d_values, bool own, cudaStream_t s)
{
  const std::uint64_t nb = (n + kLegacyBlock - 1) / kLegacyBlock;
  const unsigned grid = (unsigned)std::max<std::uint64_t>(1, (nb + kDecBlocks - 1) / kDecBlocks);
  const auto* q = static_cast<const std::int16_t*>(d_in);
  T* y = static_cast<T*>(d_values);
  const bool vec = reinterpret_cast<std::uintptr_t>(d_in) % 16 == 0;
  if (own)
    k_frsz1_decompress<T, true><<<grid, kDecBlocks, 0, s>>>(q, n, eps * 2, y, vec);
  else
    k_frsz1_decompress<T, false><<<grid, kDecBlocks, 0, s>>>(q, n, eps * 2, y, vec);
  return cuda_status(cudaGetLastError(), "legacy decompress launch");
}

int legacy_checks(int dtype, double epsilon, const void* a, const void* b, std::uint64_t n)
{
  if (dtype != FRSZ2_FLOAT && dtype != FRSZ2_DOUBLE)
    return set_error(FRSZ2_EDTYPE, "unsupported type: currently only floating point supported");
  if (!(epsilon > 0.0) || !std::isfinite(epsilon)) return set_error(FRSZ2_EFAIL, "epsilon must be positive and finite");
  if (n > 0 && (!a || !b)) return set_error(FRSZ2_EFAIL, "null pointer");
  return FRSZ2_OK;
}

} // namespace
} // namespace frsz2b

using namespace frsz2b;

extern "C" {

uint64_t frsz1_compressed_size(uint64_t n) { return n * sizeof(std::int16_t); }

int frsz1_compress(int dtype, double epsilon, const void* d_values, uint64_t n, void* d_out, void* stream)
{
  NvtxRange nvtx("frsz1_compress");
  if (int rc = legacy_checks(dtype, epsilon, d_values, d_out, n)) return rc;
  const std::size_t es = dtype == FRSZ2_FLOAT ? 4 : 8;
  if (reinterpret_cast<std::uintptr_t>(d_values) % es != 0 || reinterpret_cast<std::uintptr_t>(d_out) % 2 != 0)
    return set_error(FRSZ2_EFAIL, "misaligned pointer");
  if (n == 0) return FRSZ2_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  return dtype == FRSZ2_FLOAT ? legacy_compress<float>(epsilon, d_values, n, d_out, s)
                              : legacy_compress<double>(epsilon, d_values, n, d_out, s);
}

int frsz1_decompress(int dtype, double epsilon, const void* d_in, uint64_t n, void* d_values, int flags, void* stream)
{
  NvtxRange nvtx("frsz1_decompress");
  if (int rc = legacy_checks(dtype, epsilon, d_in, d_values, n)) return rc;
  const std::size_t es = dtype == FRSZ2_FLOAT ? 4 : 8;
  if (reinterpret_cast<std::uintptr_t>(d_values) % es != 0 || reinterpret_cast<std::uintptr_t>(d_in) % 2 != 0)
    return set_error(FRSZ2_EFAIL, "misaligned pointer");
  if (n == 0) return FRSZ2_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const bool own = (flags & FRSZ1_OWN_DELTAS) != 0;
  return dtype == FRSZ2_FLOAT ? legacy_decompress<float>(epsilon, d_in, n, d_values, own, s)
                              : legacy_decompress<double>(epsilon, d_in, n, d_values, own, s);
}

} // extern "C"
