// frsz2_common.cuh -- FRSZ2 layout algebra and bit-exact per-element arithmetic
// shared by every kernel of the B200 codec.
//
// The compressed byte layout is the reference's (robertu94/frsz
// include/frsz2.hpp:525-548):
//   [nb exponents, each a signed W-bit integer]
//   [pad to the next multiple of 256 bytes; a full 256 B when already aligned]
//   [nb blocks of ceil(E*bits/W) W-bit words; value k of a block occupies bits
//    [k*bits, (k+1)*bits) of the block's little-endian bit stream]
// with nb = ceil(n/E) and W = 8/16/32/64 for bits <= 8/16/32/64.
//
// Because the words are little-endian and packed LSB-first, a block's bytes
// ARE a little-endian bit stream whatever W is; the kernels exploit this by
// assembling 32-bit output chunks straight from the stream position.
#pragma once

#include <cstddef>
#include <cstdint>

#if defined(__CUDACC__)
#define FRSZ2_HD __host__ __device__ __forceinline__
#else
#define FRSZ2_HD inline
#endif

namespace frsz2b {

// ---------------------------------------------------------------- float traits

template<class T>
struct fp;

template<>
struct fp<float>
{
  using U = std::uint32_t;
  static constexpr int SIG = 23, EXPB = 8, BIAS = 127, UBITS = 32;
  static constexpr U SIGN = 0x80000000u, ABS = 0x7FFFFFFFu, INF = 0x7F800000u, SIGMASK = 0x007FFFFFu;
  static constexpr int EMASK = 0xFF;
};

template<>
struct fp<double>
{
  using U = std::uint64_t;
  static constexpr int SIG = 52, EXPB = 11, BIAS = 1023, UBITS = 64;
  static constexpr U SIGN = 0x8000000000000000ull, ABS = 0x7FFFFFFFFFFFFFFFull, INF = 0x7FF0000000000000ull,
                     SIGMASK = 0x000FFFFFFFFFFFFFull;
  static constexpr int EMASK = 0x7FF;
};

// ---------------------------------------------------------------- layout

// storage_t<bits> (frsz2.hpp:258-262): the word AND exponent width.
FRSZ2_HD int word_bits(int bits) { return bits <= 8 ? 8 : bits <= 16 ? 16 : bits <= 32 ? 32 : 64; }

// Geometry of one compressed array; all sizes follow frsz2.hpp:525-548.
struct Layout
{
  std::uint64_t n;           // elements
  std::uint64_t nb;          // exponent blocks, ceil(n / E)
  std::uint64_t exp_bytes;   // exponent region incl. the 256-byte pad
  std::uint64_t total_bytes; // compute_compressed_memory_size_byte(n)
  std::uint32_t block_bytes; // compressed_block_size_byte
  int bits, E, W;
};

FRSZ2_HD Layout make_layout(std::uint64_t n, int bits, int E)
{
  Layout L;
  L.n = n;
  L.bits = bits;
  L.E = E;
  L.W = word_bits(bits);
  L.nb = (n + (std::uint64_t)E - 1) / (std::uint64_t)E;
  const std::uint64_t words = ((std::uint64_t)E * (std::uint64_t)bits + (std::uint64_t)L.W - 1) / (std::uint64_t)L.W;
  L.block_bytes = (std::uint32_t)(words * (std::uint64_t)(L.W / 8));
  const std::uint64_t e = L.nb * (std::uint64_t)(L.W / 8);
  L.exp_bytes = e + 256 - e % 256;
  L.total_bytes = L.exp_bytes + L.nb * (std::uint64_t)L.block_bytes;
  return L;
}

// Bytes the reference writes into a block of `cnt` values: only the words
// 0 .. ceil(cnt*bits/W)-1 (compress_cpu_block, frsz2.hpp:1132-1178).
FRSZ2_HD std::uint32_t written_block_bytes(int cnt, int bits, int W)
{
  return (std::uint32_t)((((std::uint64_t)cnt * (std::uint64_t)bits + (std::uint64_t)W - 1) / (std::uint64_t)W) *
                         (std::uint64_t)(W / 8));
}

// Two's-complement narrowing to signed W bits (exp_type = make_signed_t<
// storage_t<bits>>, frsz2.hpp:510): fp64 exponents wrap when bits <= 8.
FRSZ2_HD std::int64_t wrap_signed(std::int64_t v, int w)
{
  if (w >= 64) return v;
  const std::uint64_t m = (1ull << w) - 1;
  std::uint64_t u = (std::uint64_t)v & m;
  if (u >> (w - 1)) u |= ~m;
  return (std::int64_t)u;
}

// ---------------------------------------------------------------- arithmetic

// float_traits<T>::exponent_t value of an exponent field (frsz2.hpp:312-320):
// int8_t for float, so the Inf/NaN field 255 reads as -128.
template<class T>
FRSZ2_HD int exponent_of_field(int field)
{
  if (sizeof(T) == 4) return field == 255 ? -128 : field - 127;
  return field - 1023;
}

// Exponent field of |x|, or 0 for NaN.  The block exponent is
// exponent(max |x|) with std::max skipping NaN (frsz2.hpp:1121-1125); the
// exponent field is monotone in |x|, so its max over the block is the field
// of the max.
template<class T>
FRSZ2_HD std::uint32_t max_field(typename fp<T>::U u)
{
  using F = fp<T>;
  const typename F::U a = u & F::ABS;
  return a > F::INF ? 0u : (std::uint32_t)(a >> F::SIG);
}

// floating_to_fixed (frsz2.hpp:352-376) followed by uint_fp_to_compressed
// (frsz2.hpp:555-558): the `bits`-bit code of one value for block exponent
// be16.  Truncating shifts, sign at the code's MSB.  Shifts of the word width
// or more (undefined in the reference; only reachable with +-Inf/NaN or
// wrapped int8 exponents) yield a zero magnitude.
template<class T>
FRSZ2_HD typename fp<T>::U to_code(typename fp<T>::U u, int be16, int bits)
{
  using F = fp<T>;
  using U = typename F::U;
  const int field = (int)((u >> F::SIG) & (U)F::EMASK);
  const int e = exponent_of_field<T>(field);
  const U m = (u & F::SIGMASK) | (field != 0 ? (U(1) << F::SIG) : U(0));
  const int shift = (F::EXPB - 1) - (be16 - e);
  U r;
  if (shift < -F::SIG) {
    r = 0;
  } else if (shift > 0) {
    r = shift >= F::UBITS ? U(0) : (U)(m << shift);
  } else {
    r = m >> (-shift);
  }
  r |= (u & F::SIGN);
  return r >> (F::UBITS - bits);
}

#if defined(__CUDACC__)
FRSZ2_HD int clz_u(std::uint32_t v)
{
#if defined(__CUDA_ARCH__)
  return __clz((int)v);
#else
  return v == 0 ? 32 : __builtin_clz(v);
#endif
}
FRSZ2_HD int clz_u(std::uint64_t v)
{
#if defined(__CUDA_ARCH__)
  return __clzll((long long)v);
#else
  return v == 0 ? 64 : __builtin_clzll(v);
#endif
}
#else
inline int clz_u(std::uint32_t v) { return v == 0 ? 32 : __builtin_clz(v); }
inline int clz_u(std::uint64_t v) { return v == 0 ? 64 : __builtin_clzll(v); }
#endif

template<class T>
FRSZ2_HD T from_bits(typename fp<T>::U u)
{
#if defined(__CUDA_ARCH__)
  if constexpr (sizeof(T) == 4)
    return __uint_as_float(u);
  else
    return __longlong_as_double((long long)u);
#else
  T x;
  __builtin_memcpy(&x, &u, sizeof(T));
  return x;
#endif
}

template<class T>
FRSZ2_HD typename fp<T>::U to_bits(T x)
{
#if defined(__CUDA_ARCH__)
  if constexpr (sizeof(T) == 4)
    return __float_as_uint(x);
  else
    return (std::uint64_t)__double_as_longlong(x);
#else
  typename fp<T>::U u;
  __builtin_memcpy(&u, &x, sizeof(T));
  return u;
#endif
}

// compressed_to_uint_fp (frsz2.hpp:550-553) + fixed_to_floating
// (frsz2.hpp:378-399) for a `bits`-bit code and block exponent be.
// countl_zero quirk (frsz2.hpp:180-186): a zero magnitude counts 32 leading
// zeros for BOTH widths (the LP64 unsigned-long overload), so z = 31 and the
// value decodes to +-2^(be-31) when be+bias >= 31.
template<class T>
FRSZ2_HD T from_code(typename fp<T>::U code, std::int64_t be, int bits)
{
  using F = fp<T>;
  using U = typename F::U;
  const U v = (U)(code << (F::UBITS - bits));
  const U f = v & F::ABS;
  const int z = f == 0 ? 31 : clz_u(f) - 1;
  const int t = (int)(be + F::BIAS);
  const int shift = -(z < t ? z : t);
  const U s = v & F::SIGN;
  const U e = (U)((U)((std::int64_t)shift + be + F::BIAS) << F::SIG);
  const int ms = F::EXPB - 1 + shift;
  U m;
  if (ms > 0)
    m = ms >= F::UBITS ? U(0) : (U)(f >> ms);
  else
    m = (U)(f << (-ms));
  m &= ~(U(1) << F::SIG);
  return from_bits<T>(s | e | m);
}

} // namespace frsz2b
