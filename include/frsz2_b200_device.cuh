// frsz2_b200_device.cuh -- device-side random access into an FRSZ2 buffer,
// for use inside the caller's own CUDA kernels (the role of the reference's
// frsz2_compressor::decompress_gpu_element, include/frsz2.hpp:1096-1104).
//
// frsz2_b200::device::decode_element<bits, E, T>(exponents, words, idx)
// returns value idx of an array compressed with `bits` bits per value and
// exponent blocks of E values, given the buffer's exponent section and its
// block section (the layout of include/frsz2.hpp:525-548).  The result equals
// the reference CPU decoder's value (decompress_cpu_element,
// include/frsz2.hpp:1199-1214) bit for bit -- including a zero code, which
// decodes to +-2^(e_b-31), and subnormal results -- which is also what the
// library's bulk kernels produce.  (The reference's own GPU accessor departs
// from its CPU decoder on exactly those two cases, include/frsz2.hpp:647-774.)
//
// Header only, no library calls: include it in a .cu file compiled for
// sm_100a.  frsz::frsz2_compressor (frsz2_b200.hpp) exposes it as the member
// decompress_gpu_element(idx).
#ifndef FRSZ2_B200_DEVICE_CUH
#define FRSZ2_B200_DEVICE_CUH

#include <cstddef>
#include <cstdint>
#include <type_traits>

namespace frsz2_b200 {
namespace device {

// IEEE-754 field sizes of float / double.
template<class T>
struct ieee;
template<>
struct ieee<float>
{
  using U = std::uint32_t;
  static constexpr int UBITS = 32, SIG = 23, EXPB = 8, BIAS = 127;
};
template<>
struct ieee<double>
{
  using U = std::uint64_t;
  static constexpr int UBITS = 64, SIG = 52, EXPB = 11, BIAS = 1023;
};

__device__ __forceinline__ int count_leading_zeros(std::uint32_t v) { return __clz((int)v); }
__device__ __forceinline__ int count_leading_zeros(std::uint64_t v) { return __clzll((long long)v); }

// The value of a `bits`-wide code in a block with exponent be: the code is
// the top `bits` bits of a sign-magnitude fixed-point number whose leading
// magnitude bit has weight 2^be (include/frsz2.hpp:550-558); normalising it
// follows fixed_to_floating (include/frsz2.hpp:378-399): leading zeros z of
// the magnitude (31 when the magnitude is zero, as the reference's count on a
// 64-bit unsigned long returns 32), exponent be - z clamped at the subnormal
// boundary, mantissa shifted into place, implicit bit dropped.
template<class T, int BITS>
__device__ __forceinline__ T decode_code(typename ieee<T>::U code, std::int64_t be)
{
  using F = ieee<T>;
  using U = typename F::U;
  constexpr U SIGN = U(1) << (F::UBITS - 1);
  const U v = (U)(code << (F::UBITS - BITS));
  const U f = v & ~SIGN;
  const int z = f == 0 ? 31 : count_leading_zeros(f) - 1;
  const std::int64_t t = be + F::BIAS;
  const int shift = -(int)(z < t ? z : t);
  const U e = (U)((U)((std::int64_t)shift + be + F::BIAS) << F::SIG);
  const int ms = F::EXPB - 1 + shift;
  U m;
  if (ms > 0)
    m = ms >= F::UBITS ? U(0) : (U)(f >> ms);
  else
    m = (U)(f << (-ms));
  m &= ~(U(1) << F::SIG);
  const U r = (v & SIGN) | e | m;
  if constexpr (sizeof(T) == 4)
    return __uint_as_float(r);
  else
    return __longlong_as_double((long long)r);
}

// Value idx of the array.  exponents: the buffer's first byte (nb signed
// exponents of the word width); words: the first block (the buffer plus the
// exponent section's size).  Word width and exponent width are both the
// storage word of `bits` (8, 16, 32 or 64 bits).
template<int BITS, int E, class T>
__device__ __forceinline__ T decode_element(const void* exponents, const void* words, std::size_t idx)
{
  static_assert(std::is_same<T, float>::value || std::is_same<T, double>::value, "float or double only");
  static_assert(4 <= BITS && BITS <= (int)sizeof(T) * 8, "4 <= bits <= width of the float type");
  static_assert(0 < E, "exponent block size must be positive");
  using Word = std::conditional_t<
    (BITS <= 8), std::uint8_t,
    std::conditional_t<(BITS <= 16), std::uint16_t, std::conditional_t<(BITS <= 32), std::uint32_t, std::uint64_t>>>;
  using Exp = std::make_signed_t<Word>;
  constexpr int W = (int)sizeof(Word) * 8;
  constexpr int BLOCK_WORDS = (E * BITS + W - 1) / W;
  const std::size_t b = idx / E;
  const int k = (int)(idx - b * E);
  const std::int64_t be = static_cast<const Exp*>(exponents)[b];
  const Word* wb = static_cast<const Word*>(words) + b * BLOCK_WORDS;
  const int p = k * BITS; // < 2^22
  const int w = p / W, o = p % W;
  // LSB-first packing (include/frsz2.hpp:565-644): the code starts at bit o
  // of word w and continues in the low bits of word w + 1
  std::uint64_t c = (std::uint64_t)wb[w] >> o;
  if (o + BITS > W) c |= (std::uint64_t)wb[w + 1] << (W - o);
  if constexpr (BITS < 64) c &= (1ull << BITS) - 1;
  return decode_code<T, BITS>((typename ieee<T>::U)c, be);
}

// ---------------------------------------------------------------- encode

// Unbiased exponent of x from its bit field, narrowed to the reference's
// exponent_t (int8 for float, so the Inf/NaN field gives -128; int16 for
// double); zero and subnormals give -bias (include/frsz2.hpp:312-320).
template<class T>
__device__ __forceinline__ int exponent_of(T x)
{
  using F = ieee<T>;
  typename F::U u;
  if constexpr (sizeof(T) == 4)
    u = __float_as_uint(x);
  else
    u = (std::uint64_t)__double_as_longlong(x);
  const int field = (int)((u >> F::SIG) & ((1u << F::EXPB) - 1));
  if constexpr (sizeof(T) == 4)
    return (int)(std::int8_t)(field - F::BIAS);
  else
    return (int)(std::int16_t)(field - F::BIAS);
}

// The `bits`-wide code of x in a block with exponent be: the sign-magnitude
// fixed-point value of x with the block maximum's leading bit at the top
// magnitude position (include/frsz2.hpp:352-376: significand with its
// implicit bit unless the exponent is -bias, shifted by (exponent bits - 1)
// - (be - e), truncated, no rounding; shifts that leave the word give 0),
// cut to its top `bits` bits (include/frsz2.hpp:555-558).
template<class T, int BITS>
__device__ __forceinline__ typename ieee<T>::U encode_value(T x, std::int16_t be)
{
  using F = ieee<T>;
  using U = typename F::U;
  U u;
  if constexpr (sizeof(T) == 4)
    u = __float_as_uint(x);
  else
    u = (std::uint64_t)__double_as_longlong(x);
  const int e = exponent_of(x);
  U m = u & ((U(1) << F::SIG) - 1);
  if (e != -F::BIAS) m |= U(1) << F::SIG;
  const int shift = F::EXPB - 1 - ((int)be - e);
  U r;
  if (shift < -F::SIG)
    r = 0;
  else if (shift > 0)
    r = shift >= F::UBITS ? U(0) : (U)(m << shift);
  else
    r = m >> (-shift);
  r |= u & (U(1) << (F::UBITS - 1));
  return r >> (F::UBITS - BITS);
}

// Compress exponent block b of an array into its exponent and its words
// (the layout of include/frsz2.hpp:525-548): x points at the block's first
// value and cnt (1..E) is its count.  The block exponent is the exponent of
// the largest magnitude, NaNs skipped as std::max skips them
// (include/frsz2.hpp:1121-1125), stored as the signed word-width exponent;
// codes are packed LSB-first (include/frsz2.hpp:565-644), and only the words
// the cnt values reach are written, as compress_cpu_block writes them
// (include/frsz2.hpp:1108-1179).
template<int BITS, int E, class T>
__device__ inline void encode_block(const T* x, std::size_t cnt, void* exponents, void* words, std::size_t b)
{
  using Word = std::conditional_t<
    (BITS <= 8), std::uint8_t,
    std::conditional_t<(BITS <= 16), std::uint16_t, std::conditional_t<(BITS <= 32), std::uint32_t, std::uint64_t>>>;
  using Exp = std::make_signed_t<Word>;
  constexpr int W = (int)sizeof(Word) * 8;
  constexpr std::size_t BLOCK_WORDS = ((std::size_t)E * BITS + W - 1) / W;
  T in_max = 0;
  for (std::size_t k = 0; k < cnt; ++k) {
    const T a = x[k] < T(0) ? -x[k] : x[k]; // a NaN stays a NaN
    in_max = in_max < a ? a : in_max;       // false for a NaN: skipped
  }
  const Exp be = (Exp)exponent_of(in_max);
  static_cast<Exp*>(exponents)[b] = be;
  Word* wb = static_cast<Word*>(words) + b * BLOCK_WORDS;
  Word cur = 0;
  std::size_t w = 0;
  for (std::size_t k = 0; k < cnt; ++k) {
    const std::uint64_t c = (std::uint64_t)encode_value<T, BITS>(x[k], (std::int16_t)be);
    const int o = (int)((k * BITS) % W);
    cur |= (Word)(c << o);
    if (o + BITS >= W) { // word w is complete
      wb[w++] = cur;
      cur = o + BITS > W ? (Word)(c >> (W - o)) : Word(0);
    }
  }
  if ((cnt * BITS) % W != 0) wb[w] = cur; // the partly filled last word
}

} // namespace device
} // namespace frsz2_b200

#endif
