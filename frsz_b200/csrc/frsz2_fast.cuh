// frsz2_fast.cuh -- compile-time-width FRSZ2 kernels (the hot path).
//
// One kernel instance per (float type, bits).  Lane mapping: each lane owns a
// contiguous run of P = 32 / sizeof(T) values (one 256-bit load / store), so
// its packed codes form one contiguous segment of L = P * bits stream bits;
// packing and unpacking are constant shifts, plus one neighbour shuffle when
// L is not a multiple of 32.  A warp row is 32 * P values; a 256-thread CTA
// handles a tile of 2 rows per warp (4096 fp32 / 2048 fp64 values).
//
// Arithmetic.  For blocks whose exponent lies in the "plain" domain (no
// Inf/NaN, e_b >= -95 for fp32 / >= -959 for fp64, no int8 exponent wrap)
// the reference's integer align-and-truncate (floating_to_fixed +
// uint_fp_to_compressed, include/frsz2.hpp:352-376, 555-558) equals
//     code = trunc(|x| * 2^(bits-2-e_b)) | sign << (bits-1)
// because scaling by a power of two is exact there, subnormal inputs
// truncate to 0 on both sides, and the code fits in bits-1 bits.  Likewise
// fixed_to_floating (include/frsz2.hpp:378-399) equals
//     x_hat = rz_convert(mag) * 2^(e_b-bits+2)   (mag != 0)
//     x_hat = 2^(e_b-31)                          (mag == 0, the clz quirk)
// with the sign or-ed in: rounding toward zero keeps the same 24 / 53 leading
// bits the reference's shift keeps, and every result is a normal number.
// Blocks outside the plain domain use the exact integer path of
// frsz2_common.cuh (a block-uniform branch), so results are bit-exact for
// every input.
#pragma once

#include "frsz2_kernels.cuh"

#include <type_traits>

namespace frsz2b {

// ESM = 0: exponent blocks of E >= P values (E a runtime power of two).
// ESM = 1, 2 or 4 (< P): blocks of exactly ESM values, so a lane holds P / ESM
// whole blocks, each padded to whole W-bit words; value i of a lane then sits
// at bit (i / ESM) * BBB + (i % ESM) * BITS of its segment.
template<class T, int BITS, int NT_ = kNT, int RPW_ = 2, int ESM_ = 0>
struct fast_cfg
{
  using U = typename fp<T>::U;
  using C = std::conditional_t<(BITS <= 32), std::uint32_t, std::uint64_t>;
  static constexpr int W = BITS <= 8 ? 8 : BITS <= 16 ? 16 : BITS <= 32 ? 32 : 64;
  static constexpr int B = BITS;                 // bits per value
  static constexpr int P = 32 / (int)sizeof(T);  // values per lane
  static constexpr int ESM = ESM_;
  static_assert(ESM == 0 || (ESM < P && (ESM & (ESM - 1)) == 0), "blocks smaller than a lane's values");
  static constexpr int BBB = ESM ? ((ESM * BITS + W - 1) / W) * W : 0; // bits of one small block
  static constexpr int L = ESM ? (P / ESM) * BBB : P * BITS;         // segment bits per lane
  static constexpr int NW = (L + 31) / 32;       // segment words
  static constexpr bool ALIGNED = (L % 32) == 0; // segments start on word boundaries
  static constexpr int ROW = 32 * P;             // values per warp row
  static constexpr int NT = NT_;                 // threads per CTA
  static constexpr int RPW = RPW_;               // rows per warp per tile
  static constexpr int WARPS = NT / 32;
  static constexpr int ROWS = WARPS * RPW;       // rows per tile
  static constexpr int TE = ROWS * ROW;          // values per tile
  // bit of a lane's segment where its value i starts
  __host__ __device__ static constexpr int pos(int i) { return ESM ? (i / ESM) * BBB + (i % ESM) * BITS : i * BITS; }
};

// Values per tile of the fast kernels for a CTA width and rows per warp.
__host__ __device__ constexpr int fast_tile_values(int dtype_bytes, int nt, int rpw)
{
  return (nt / 32) * rpw * 32 * (32 / dtype_bytes);
}

// ---------------------------------------------------------------- PTX helpers

__device__ __forceinline__ void ld256_stream(const void* p, std::uint32_t (&v)[8])
{
  asm volatile("ld.global.nc.L1::no_allocate.v8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
               : "l"(p));
}

__device__ __forceinline__ void st256_stream(void* p, const std::uint32_t (&v)[8])
{
  asm volatile("st.global.cs.v8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"l"(p), "r"(v[0]), "r"(v[1]), "r"(v[2]),
               "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7])
               : "memory");
}

// N consecutive 32-bit words at p, p aligned to 4 * (largest power of two
// dividing N), at most 32 bytes.
template<int N>
__device__ __forceinline__ void load_words(const std::uint32_t* p, std::uint32_t (&w)[N])
{
  constexpr int V = (N % 8 == 0) ? 8 : (N % 4 == 0) ? 4 : (N % 2 == 0) ? 2 : 1;
#pragma unroll
  for (int i = 0; i < N; i += V) {
    if constexpr (V == 8) {
      std::uint32_t t[8];
      asm volatile("ld.global.nc.L1::no_allocate.v8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                   : "=r"(t[0]), "=r"(t[1]), "=r"(t[2]), "=r"(t[3]), "=r"(t[4]), "=r"(t[5]), "=r"(t[6]), "=r"(t[7])
                   : "l"(p + i));
#pragma unroll
      for (int k = 0; k < 8; ++k) w[i + k] = t[k];
    } else if constexpr (V == 4) {
      const uint4 t = __ldg(reinterpret_cast<const uint4*>(p + i));
      w[i] = t.x;
      w[i + 1] = t.y;
      w[i + 2] = t.z;
      w[i + 3] = t.w;
    } else if constexpr (V == 2) {
      const uint2 t = __ldg(reinterpret_cast<const uint2*>(p + i));
      w[i] = t.x;
      w[i + 1] = t.y;
    } else {
      w[i] = __ldg(p + i);
    }
  }
}

template<int N>
__device__ __forceinline__ void store_words(std::uint32_t* p, const std::uint32_t (&w)[N])
{
  constexpr int V = (N % 8 == 0) ? 8 : (N % 4 == 0) ? 4 : (N % 2 == 0) ? 2 : 1;
#pragma unroll
  for (int i = 0; i < N; i += V) {
    if constexpr (V == 8) {
      std::uint32_t t[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) t[k] = w[i + k];
      st256_stream(p + i, t);
    } else if constexpr (V == 4) {
      __stcs(reinterpret_cast<uint4*>(p + i), make_uint4(w[i], w[i + 1], w[i + 2], w[i + 3]));
    } else if constexpr (V == 2) {
      __stcs(reinterpret_cast<uint2*>(p + i), make_uint2(w[i], w[i + 1]));
    } else {
      __stcs(reinterpret_cast<unsigned int*>(p + i), w[i]);
    }
  }
}

// Store one 32-bit stream word at tile byte offset `off`, keeping bytes at or
// beyond `limit` untouched (the unwritten tail of a partial last block).
__device__ __forceinline__ void store_word_bounded(std::uint8_t* base, std::uint32_t off, std::uint32_t limit,
                                                   std::uint32_t v)
{
  if (off + 4u <= limit) {
    *reinterpret_cast<std::uint32_t*>(base + off) = v;
  } else {
    for (std::uint32_t q = 0; off + q < limit; ++q) base[off + q] = (std::uint8_t)(v >> (8 * q));
  }
}

// ---------------------------------------------------------------- values off the 32-byte layout

// A lane's 32 bytes of values (8 words) when the values pointer sits kw
// words (1..7) past a 32-byte boundary: the lane loads its aligned segment
// a[0..8) (a = its values rounded down), takes the words after it from the
// next lane's segment by shuffles (lane 31, whose neighbour is in another
// row, loads them itself), and rotates by kw with one compile-time case per
// kw (kw is the same for every lane of a launch, so the switch does not
// diverge).  `first` marks the array's first lane, whose aligned segment
// would start before the array: it reads its own words one by one.  Every
// lane of the warp takes part.
template<bool EARLY>
__device__ __forceinline__ void ld_lane_mis(const std::uint32_t* a, int kw, bool first, std::uint32_t (&v)[8])
{
  const int lane = threadIdx.x & 31;
  std::uint32_t c0[8];
  if (!first) {
    ld256_stream(a, c0);
  } else {
#pragma unroll
    for (int i = 0; i < 8; ++i) c0[i] = 0;
  }
  // EARLY: lane 31's words past its segment are loaded together with the
  // segment rather than after the shuffles (which wait for the segment).
  // Measured on B200 with fp64 values off by 1-3 elements: compress 0.81 ->
  // 0.93 of HBM at 32 bits, 0.80 -> 0.84 at 16, but 0.73 -> 0.68 at 21, so
  // the caller enables it for the widths whose lane segments are word-aligned.
  std::uint32_t ext[7];
  if constexpr (EARLY) {
#pragma unroll
    for (int i = 0; i < 7; ++i) ext[i] = lane == 31 && i < kw ? __ldg(a + 8 + i) : 0u;
  }
  auto take = [&](auto kc) {
    constexpr int K = decltype(kc)::value;
    std::uint32_t c1[K];
#pragma unroll
    for (int i = 0; i < K; ++i) {
      const std::uint32_t nb = __shfl_down_sync(0xFFFFFFFFu, c0[i], 1);
      if constexpr (EARLY)
        c1[i] = lane == 31 ? ext[i] : nb;
      else
        c1[i] = lane == 31 ? __ldg(a + 8 + i) : nb;
    }
    if (first) {
#pragma unroll
      for (int i = 0; i < 8; ++i) v[i] = __ldg(a + K + i);
    } else {
#pragma unroll
      for (int i = 0; i < 8; ++i) v[i] = i + K < 8 ? c0[i + K] : c1[i + K - 8];
    }
  };
  switch (kw) {
    case 1: take(std::integral_constant<int, 1>{}); break;
    case 2: take(std::integral_constant<int, 2>{}); break;
    case 3: take(std::integral_constant<int, 3>{}); break;
    case 4: take(std::integral_constant<int, 4>{}); break;
    case 5: take(std::integral_constant<int, 5>{}); break;
    case 6: take(std::integral_constant<int, 6>{}); break;
    default: take(std::integral_constant<int, 7>{}); break;
  }
}

// The store counterpart: lane L's 8 words go to a[kw .. kw + 8) with a the
// lane's values rounded down to 32 bytes.  Lanes 1..31 store their aligned
// segment a[0..8) whole -- the previous lane's last kw words (by shuffles)
// and their own first 8 - kw; lane 0 stores its first 8 - kw words one by
// one (its segment starts in the previous row), lane 31 its last kw (they
// belong to the next row's first segment).  Every lane of the warp takes
// part.
__device__ __forceinline__ void st_lane_mis(std::uint32_t* a, int kw, const std::uint32_t (&v)[8])
{
  const int lane = threadIdx.x & 31;
  auto put = [&](auto kc) {
    constexpr int K = decltype(kc)::value;
    std::uint32_t seg[8];
#pragma unroll
    for (int i = 0; i < K; ++i) seg[i] = __shfl_up_sync(0xFFFFFFFFu, v[8 - K + i], 1);
#pragma unroll
    for (int i = K; i < 8; ++i) seg[i] = v[i - K];
    if (lane != 0) {
      st256_stream(a, seg);
    } else {
#pragma unroll
      for (int i = K; i < 8; ++i) a[i] = seg[i];
    }
    if (lane == 31) {
#pragma unroll
      for (int i = 0; i < K; ++i) a[8 + i] = v[8 - K + i];
    }
  };
  switch (kw) {
    case 1: put(std::integral_constant<int, 1>{}); break;
    case 2: put(std::integral_constant<int, 2>{}); break;
    case 3: put(std::integral_constant<int, 3>{}); break;
    case 4: put(std::integral_constant<int, 4>{}); break;
    case 5: put(std::integral_constant<int, 5>{}); break;
    case 6: put(std::integral_constant<int, 6>{}); break;
    default: put(std::integral_constant<int, 7>{}); break;
  }
}

// ---------------------------------------------------------------- bit fields

#ifndef FRSZ2_PUT_BITS_MAD
#define FRSZ2_PUT_BITS_MAD 1
#endif

// Insert the low NB bits of v (zero above NB) at stream bit POS of seg.  The
// bits at and above POS in seg are still zero, so adding v * 2^r equals
// OR-ing v << r, and the add runs as one integer multiply-add (on the FMA
// pipe) instead of a shift and an OR (both on the ALU pipe).
template<int POS, int NB, int N, class V>
__device__ __forceinline__ void put_bits(std::uint32_t (&seg)[N], V v)
{
  constexpr int q = POS / 32, r = POS % 32;
  if constexpr (sizeof(V) == 4) {
    if (FRSZ2_PUT_BITS_MAD)
      seg[q] = v * (1u << r) + seg[q];
    else
      seg[q] |= v << r;
    if constexpr (r != 0 && r + NB > 32) seg[q + 1] |= v >> (32 - r);
  } else {
    if (FRSZ2_PUT_BITS_MAD)
      seg[q] = (std::uint32_t)v * (1u << r) + seg[q];
    else
      seg[q] |= (std::uint32_t)(v << r);
    if constexpr (r + NB > 32) seg[q + 1] |= (std::uint32_t)(r == 0 ? (v >> 32) : (v >> (32 - r)));
    if constexpr (r + NB > 64) seg[q + 2] |= (std::uint32_t)(v >> (64 - r));
  }
}

// NB-bit field at stream bit POS of seg.
template<int POS, int NB, int N>
__device__ __forceinline__ auto get_bits(const std::uint32_t (&seg)[N])
{
  constexpr int q = POS / 32, r = POS % 32;
  if constexpr (NB <= 32) {
    constexpr std::uint32_t mask = NB == 32 ? 0xFFFFFFFFu : ((1u << NB) - 1u);
    if constexpr (r + NB <= 32)
      return (seg[q] >> r) & mask;
    else
      return __funnelshift_r(seg[q], seg[q + 1], r) & mask;
  } else {
    constexpr std::uint64_t mask = NB == 64 ? ~0ull : ((1ull << NB) - 1ull);
    const std::uint32_t lo = r == 0 ? seg[q] : __funnelshift_r(seg[q], seg[q + 1], r);
    std::uint32_t hi;
    if constexpr (r == 0)
      hi = seg[q + 1];
    else if constexpr (r + NB > 64)
      hi = __funnelshift_r(seg[q + 1], seg[q + 2], r);
    else
      hi = seg[q + 1] >> r;
    return ((((std::uint64_t)hi) << 32) | lo) & mask;
  }
}

template<int K, int BITS, int N, class C, int P>
__device__ __forceinline__ void pack_all(std::uint32_t (&seg)[N], const C (&c)[P])
{
  if constexpr (K < P) {
    put_bits<K * BITS, BITS>(seg, c[K]);
    pack_all<K + 1, BITS>(seg, c);
  }
}

template<int K, int BITS, int N, class C, int P>
__device__ __forceinline__ void unpack_all(const std::uint32_t (&seg)[N], C (&c)[P])
{
  if constexpr (K < P) {
    c[K] = (C)get_bits<K * BITS, BITS>(seg);
    unpack_all<K + 1, BITS>(seg, c);
  }
}

// pack_all / unpack_all at the positions of a lane configuration (Cfg::pos).
template<class Cfg, int K = 0, int N, class C, int P>
__device__ __forceinline__ void pack_lane(std::uint32_t (&seg)[N], const C (&c)[P])
{
  if constexpr (K < P) {
    put_bits<Cfg::pos(K), Cfg::B>(seg, c[K]);
    pack_lane<Cfg, K + 1>(seg, c);
  }
}

template<class Cfg, int K = 0, int N, class C, int P>
__device__ __forceinline__ void unpack_lane(const std::uint32_t (&seg)[N], C (&c)[P])
{
  if constexpr (K < P) {
    c[K] = (C)get_bits<Cfg::pos(K), Cfg::B>(seg);
    unpack_lane<Cfg, K + 1>(seg, c);
  }
}

// ---------------------------------------------------------------- encode / decode

template<class T, int BITS>
__device__ __forceinline__ typename fast_cfg<T, BITS>::C encode_plain(typename fp<T>::U u, T scale)
{
  using Cfg = fast_cfg<T, BITS>;
  using C = typename Cfg::C;
  const T x = from_bits<T>(u);
  if constexpr (sizeof(T) == 4) {
    const std::uint32_t mag = __float2uint_rz(fabsf(x) * scale);
    return mag | ((u >> (32 - BITS)) & (1u << (BITS - 1)));
  } else {
    const std::uint32_t hi = (std::uint32_t)(u >> 32);
    if constexpr (BITS <= 32) {
      const std::uint32_t mag = __double2uint_rz(fabs(x) * scale);
      return mag | ((hi >> (32 - BITS)) & (1u << (BITS - 1)));
    } else {
      const std::uint64_t mag = __double2ull_rz(fabs(x) * scale);
      return (C)(mag | ((std::uint64_t)(hi >> 31) << (BITS - 1)));
    }
  }
}

template<class T, int BITS>
__device__ __forceinline__ typename fp<T>::U decode_plain(typename fast_cfg<T, BITS>::C code, T inv,
                                                          typename fp<T>::U zero_bits)
{
  using U = typename fp<T>::U;
  using C = typename fast_cfg<T, BITS>::C;
  constexpr C MAGMASK = (C(1) << (BITS - 1)) - 1;
  const C mag = code & MAGMASK;
  U r;
  if constexpr (sizeof(T) == 4) {
    r = __float_as_uint(__uint2float_rz(mag) * inv);
  } else if constexpr (BITS <= 32) {
    r = (U)__double_as_longlong(__uint2double_rn(mag) * inv);
  } else {
    r = (U)__double_as_longlong(__ull2double_rz(mag) * inv);
  }
  r = mag == 0 ? zero_bits : r;
  return r | ((U)(code >> (BITS - 1)) << (fp<T>::UBITS - 1));
}

// ---------------------------------------------------------------- compress

#ifndef FRSZ2_STAGE_NW_MASK
#define FRSZ2_STAGE_NW_MASK (1u << 7)
#endif
// Word-aligned lane segments whose word count has no 8- or 16-byte store
// (7 words: fp32 at 28 bits, fp64 at 56) leave through shared memory as
// coalesced 16-byte stores; a lane's seven 4-byte stores 28 bytes apart
// measured 0.58-0.71 of HBM on compress (load/store queue throttled).
template<class Cfg>
__host__ __device__ constexpr bool staged_aligned()
{
  return Cfg::ALIGNED && Cfg::NW < 32 && ((FRSZ2_STAGE_NW_MASK >> Cfg::NW) & 1u) != 0;
}

// Shared-memory words a CTA needs to stage its warps' packed rows: only the
// unaligned widths and the staged aligned ones stage, one row per warp.  A row holds L words of codes plus,
// when exponent blocks are padded to whole W-bit words, under W bits of pad per
// block and at most 32 blocks per row (< 64 words); L + 64 keeps each warp's
// slice a multiple of 16 bytes.
template<class T, int BITS, int NT, int RPW, int ESM = 0>
struct stage_words
{
  using Cfg = fast_cfg<T, BITS, NT, RPW, ESM>;
  static constexpr int per_warp = Cfg::ALIGNED ? (staged_aligned<Cfg>() ? Cfg::L : 0) : Cfg::L + 64;
  static constexpr int value = per_warp ? Cfg::WARPS * per_warp : 4;
};

// Store / load the NBL consecutive W-bit exponents of one lane (blocks of
// fewer values than a lane holds).  p is aligned to their total size (at
// most 32 bytes); `present` (store) is how many of them exist.
template<int W, int NBL>
__device__ __forceinline__ void store_lane_exps(std::uint8_t* p, const std::int64_t (&e)[NBL], int present)
{
  constexpr int TBY = NBL * W / 8;
  if (present >= NBL) {
    if constexpr (TBY >= 4) {
      constexpr int NWD = TBY / 4;
      std::uint32_t wd[NWD];
#pragma unroll
      for (int k = 0; k < NWD; ++k) wd[k] = 0;
#pragma unroll
      for (int b = 0; b < NBL; ++b) {
        if constexpr (W == 64) {
          wd[2 * b] = (std::uint32_t)(std::uint64_t)e[b];
          wd[2 * b + 1] = (std::uint32_t)((std::uint64_t)e[b] >> 32);
        } else {
          constexpr std::uint32_t M = W == 32 ? 0xFFFFFFFFu : ((1u << W) - 1u);
          wd[(b * W) / 32] |= ((std::uint32_t)e[b] & M) << ((b * W) % 32);
        }
      }
      store_words<NWD>(reinterpret_cast<std::uint32_t*>(p), wd);
    } else if constexpr (TBY == 2) {
      *reinterpret_cast<std::uint16_t*>(p) = (std::uint16_t)(((std::uint32_t)e[0] & 0xFFu) | ((std::uint32_t)e[1] & 0xFFu) << 8);
    } else {
      *p = (std::uint8_t)e[0];
    }
  } else {
#pragma unroll
    for (int b = 0; b < NBL; ++b)
      if (b < present) store_word(p + b * (W / 8), (std::uint64_t)e[b], W);
  }
}

// All NBL exponents are read (the bytes past the last block belong to the
// buffer: the exponent section's pad or the first code words).
template<int W, int NBL>
__device__ __forceinline__ void load_lane_exps(const std::uint8_t* p, std::int64_t (&e)[NBL])
{
  constexpr int TBY = NBL * W / 8;
  if constexpr (TBY >= 4) {
    constexpr int NWD = TBY / 4;
    std::uint32_t wd[NWD];
    load_words<NWD>(reinterpret_cast<const std::uint32_t*>(p), wd);
#pragma unroll
    for (int b = 0; b < NBL; ++b) {
      if constexpr (W == 64)
        e[b] = (std::int64_t)(((std::uint64_t)wd[2 * b + 1] << 32) | wd[2 * b]);
      else if constexpr (W == 32)
        e[b] = (std::int32_t)wd[b];
      else if constexpr (W == 16)
        e[b] = (std::int16_t)(wd[(b * 16) / 32] >> ((b * 16) % 32));
      else
        e[b] = (std::int8_t)(wd[(b * 8) / 32] >> ((b * 8) % 32));
    }
  } else if constexpr (TBY == 2) {
    const std::uint16_t v = __ldg(reinterpret_cast<const unsigned short*>(p));
    e[0] = (std::int8_t)(v & 0xFFu);
    e[1] = (std::int8_t)(v >> 8);
  } else {
    e[0] = (std::int8_t)__ldg(p);
  }
}

// One tile of compress.  s_rmax: 2 * Cfg::ROWS words of shared memory (used
// only when an exponent block spans several warp rows); s_stage:
// stage_words<>::value words, 16-byte aligned.
// more_tiles: whether the CTA runs another tile after this one (the shared
// block maxima are then reused, so their readers must be done first).
// GEN: blocks of a multiple E of P values that is not a power of two, without
// block padding (as for fast_decompress_tile): tiles of j.tile_blocks whole
// blocks; each lane's maxima go to s_gmax (2 * ROWS * 32 words), and after
// one barrier a lane takes its block's maxima from its block's E / P lanes.
// HALF (with GEN): E a multiple of P / 2 but not of P; the same per half lane
// (s_gmax of 4 * ROWS * 32 words), each half encoding with its own exponent.
// WCR: blocks of exactly RPW warp rows (power-of-two E = RPW * 32 * P); a
// warp's rows are consecutive (row = warp * RPW + rr), so a block lies in one
// warp and its maximum needs no barrier.
template<class T, int BITS, int NT, int RPW_, bool PAD = false, int ESM = 0, bool MIS = false, bool GEN = false,
         bool HALF = false, bool WCR = false>
__device__ __forceinline__ void fast_compress_tile(const Job& j, std::uint64_t tile, std::uint32_t* s_rmax,
                                                   std::uint32_t* s_stage, bool more_tiles = true,
                                                   std::uint32_t* s_gmax = nullptr, std::uint32_t mE = 0)
{
  using Cfg = fast_cfg<T, BITS, NT, RPW_, ESM>;
  using U = typename Cfg::U;
  using C = typename Cfg::C;
  using K = key_of<T>;
  constexpr int P = Cfg::P, L = Cfg::L, NW = Cfg::NW, ROW = Cfg::ROW, RPW = Cfg::RPW, TE = Cfg::TE,
                W = Cfg::W;

  const T* __restrict__ x = static_cast<const T*>(j.values_in);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int E = j.E, log2E = j.log2E;
  const int G = E / P; // lanes per exponent block
  const int TB = (int)j.tile_blocks;

  {
    const int TV = GEN ? TB * E : TE; // values of a whole tile
    const std::uint64_t e0 = tile * (std::uint64_t)TV;
    const std::uint64_t rem64 = j.n - e0;
    const bool full = rem64 >= (std::uint64_t)TV;
    const int rem = full ? TV : (int)rem64;
    const int nbt = full ? TB : GEN ? (rem + E - 1) / E : ((rem + E - 1) >> log2E);
    const std::uint64_t b0 = tile * (std::uint64_t)TB;

    // MIS: values off the 32-byte layout by kw words (whole tiles only)
    const int kw = MIS ? (int)((reinterpret_cast<std::uintptr_t>(x) & 31u) >> 2) : 0;
    U u[RPW][P];
#pragma unroll
    for (int rr = 0; rr < RPW; ++rr) {
      const int idx = (WCR ? warp * RPW + rr : rr * Cfg::WARPS + warp) * ROW + lane * P;
      if (GEN ? idx + P <= rem : MIS ? full : (full || idx + P <= rem)) {
        std::uint32_t v[8];
        if constexpr (MIS)
          ld_lane_mis<Cfg::ALIGNED>(reinterpret_cast<const std::uint32_t*>(x + e0 + idx) - kw, kw, e0 + idx == 0, v);
        else
          ld256_stream(x + e0 + idx, v);
#pragma unroll
        for (int i = 0; i < P; ++i) {
          if constexpr (sizeof(T) == 4)
            u[rr][i] = v[i];
          else
            u[rr][i] = ((std::uint64_t)v[2 * i + 1] << 32) | v[2 * i];
        }
      } else {
#pragma unroll
        for (int i = 0; i < P; ++i) u[rr][i] = (idx + i < rem) ? to_bits<T>(x[e0 + idx + i]) : U(0);
      }
    }

    // block maxima: raw keys detect Inf/NaN, clean keys skip NaN like std::max
    // (blocks within a lane, ESM > 0: computed per block below)
    std::uint32_t km[RPW], kc[RPW];
    std::uint32_t kmh[RPW][2], kch[RPW][2]; // HALF: per half lane
    if constexpr (HALF) {
      constexpr int H = P / 2;
      const int G2 = E / H; // half lanes per block
#pragma unroll
      for (int rr = 0; rr < RPW; ++rr) {
        const int t = ((rr * Cfg::WARPS + warp) * 32 + lane) * 2;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          std::uint32_t m = K::raw(u[rr][h * H]);
#pragma unroll
          for (int i = 1; i < H; ++i) m = max(m, K::raw(u[rr][h * H + i]));
          std::uint32_t cm = m;
          if (m >= K::SPECIAL) {
            cm = K::clean(u[rr][h * H]);
#pragma unroll
            for (int i = 1; i < H; ++i) cm = max(cm, K::clean(u[rr][h * H + i]));
          }
          s_gmax[t + h] = m;
          s_gmax[2 * Cfg::ROWS * 32 + t + h] = cm;
        }
      }
      __syncthreads();
#pragma unroll
      for (int rr = 0; rr < RPW; ++rr) {
        const int idx = (rr * Cfg::WARPS + warp) * ROW + lane * P;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          std::uint32_t a = 0, bmax = 0;
          if (idx + h * H < rem) {
            const int l0 = (int)__umulhi((unsigned)(idx + h * H), mE) * G2;
            for (int q = 0; q < G2; ++q) a = max(a, s_gmax[l0 + q]);
            bmax = a;
            if (a >= K::SPECIAL) {
              bmax = 0;
              for (int q = 0; q < G2; ++q) bmax = max(bmax, s_gmax[2 * Cfg::ROWS * 32 + l0 + q]);
            }
          }
          kmh[rr][h] = a;
          kch[rr][h] = bmax;
        }
      }
      if (more_tiles) __syncthreads();
    } else if constexpr (ESM == 0) {
    bool any_special = false;
#pragma unroll
    for (int rr = 0; rr < RPW; ++rr) {
      std::uint32_t m = K::raw(u[rr][0]);
#pragma unroll
      for (int i = 1; i < P; ++i) m = max(m, K::raw(u[rr][i]));
      km[rr] = m;
      any_special |= m >= K::SPECIAL;
    }
    const bool warp_special = __any_sync(0xFFFFFFFFu, any_special);
#pragma unroll
    for (int rr = 0; rr < RPW; ++rr) {
      if (warp_special) {
        std::uint32_t m = K::clean(u[rr][0]);
#pragma unroll
        for (int i = 1; i < P; ++i) m = max(m, K::clean(u[rr][i]));
        kc[rr] = m;
      } else {
        kc[rr] = km[rr];
      }
    }
    if constexpr (WCR) {
      // the block is this warp's RPW rows
      std::uint32_t a = 0, c = 0;
#pragma unroll
      for (int rr = 0; rr < RPW; ++rr) {
        a = max(a, __reduce_max_sync(0xFFFFFFFFu, km[rr]));
        c = max(c, __reduce_max_sync(0xFFFFFFFFu, kc[rr]));
      }
#pragma unroll
      for (int rr = 0; rr < RPW; ++rr) {
        km[rr] = a;
        kc[rr] = c;
      }
    } else if constexpr (GEN) {
      // a block is G consecutive lanes of the tile, across warps and rows
#pragma unroll
      for (int rr = 0; rr < RPW; ++rr) {
        const int t = (rr * Cfg::WARPS + warp) * 32 + lane;
        s_gmax[t] = km[rr];
        s_gmax[Cfg::ROWS * 32 + t] = kc[rr];
      }
      __syncthreads();
#pragma unroll
      for (int rr = 0; rr < RPW; ++rr) {
        const int idx = (rr * Cfg::WARPS + warp) * ROW + lane * P;
        if (idx < rem) {
          const int l0 = (int)__umulhi((unsigned)idx, mE) * G;
          std::uint32_t a = 0;
          for (int q = 0; q < G; ++q) a = max(a, s_gmax[l0 + q]);
          // the clean maxima differ from the raw ones only in blocks with an Inf or NaN
          std::uint32_t b = a;
          if (a >= K::SPECIAL) {
            b = 0;
            for (int q = 0; q < G; ++q) b = max(b, s_gmax[Cfg::ROWS * 32 + l0 + q]);
          }
          km[rr] = a;
          kc[rr] = b;
        }
      }
      if (more_tiles) __syncthreads();
    } else if (G == 32) {
      // a block is one warp row: one warp-wide reduction per row
#pragma unroll
      for (int rr = 0; rr < RPW; ++rr) {
        km[rr] = __reduce_max_sync(0xFFFFFFFFu, km[rr]);
        kc[rr] = warp_special ? __reduce_max_sync(0xFFFFFFFFu, kc[rr]) : km[rr];
      }
    } else if (G < 32) {
      for (int s = 1; s < G; s <<= 1) {
#pragma unroll
        for (int rr = 0; rr < RPW; ++rr) km[rr] = max(km[rr], __shfl_xor_sync(0xFFFFFFFFu, km[rr], s));
        if (warp_special) {
#pragma unroll
          for (int rr = 0; rr < RPW; ++rr) kc[rr] = max(kc[rr], __shfl_xor_sync(0xFFFFFFFFu, kc[rr], s));
        }
      }
      if (!warp_special) {
#pragma unroll
        for (int rr = 0; rr < RPW; ++rr) kc[rr] = km[rr];
      }
    } else {
      // an exponent block spans G/32 whole rows of this tile
#pragma unroll
      for (int rr = 0; rr < RPW; ++rr) {
        const std::uint32_t a = __reduce_max_sync(0xFFFFFFFFu, km[rr]);
        const std::uint32_t b = __reduce_max_sync(0xFFFFFFFFu, kc[rr]);
        if (lane == 0) {
          s_rmax[rr * Cfg::WARPS + warp] = a;
          s_rmax[Cfg::ROWS + rr * Cfg::WARPS + warp] = b;
        }
      }
      __syncthreads();
      const int rpb = G / 32;
#pragma unroll
      for (int rr = 0; rr < RPW; ++rr) {
        const int row0 = ((rr * Cfg::WARPS + warp) / rpb) * rpb;
        std::uint32_t a = 0, b = 0;
        for (int q = 0; q < rpb; ++q) {
          a = max(a, s_rmax[row0 + q]);
          b = max(b, s_rmax[Cfg::ROWS + row0 + q]);
        }
        km[rr] = a;
        kc[rr] = b;
      }
      if (more_tiles) __syncthreads();
    }
    }

    // Unpadded blocks: a row is ROW * BITS / 8 bytes.  Padded blocks (E * BITS
    // not a multiple of W, so E <= 32 < ROW): a row is ROW / E whole blocks.
    // PAD is the caller's compile-time promise about E * BITS % W.
    const std::uint32_t blk_bits = 8u * j.block_bytes;
    const std::uint32_t pad_bits = blk_bits - (std::uint32_t)E * BITS;
    const std::uint32_t row_bytes = PAD ? (std::uint32_t)(ROW >> log2E) * j.block_bytes : (std::uint32_t)(4 * L);
    const int last_cnt = rem - (nbt - 1) * E;
    const std::uint32_t wb = full ? (std::uint32_t)TB * j.block_bytes
                                  : (std::uint32_t)(nbt - 1) * j.block_bytes + written_block_bytes(last_cnt, BITS, W);
    std::uint8_t* __restrict__ dst = j.words + b0 * (std::uint64_t)j.block_bytes;

#pragma unroll
    for (int rr = 0; rr < RPW; ++rr) {
      const int row = WCR ? warp * RPW + rr : rr * Cfg::WARPS + warp;
      const int idx = row * ROW + lane * P;
      const int bl = GEN ? (int)__umulhi((unsigned)idx, mE) : idx >> log2E;
      C c[P];
      if constexpr (HALF) {
        constexpr int H = P / 2;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int field = (int)(kch[rr][h] >> K::FSHIFT);
          const std::int64_t ex = exponent_of_field<T>(field);
          const std::int64_t be = wrap_signed(ex, W);
          const bool plain = kmh[rr][h] < K::SPECIAL && be == ex && plain_exponent<T>(be);
          if (plain) {
            const T scale = pow2<T>(BITS - 2 - (int)be);
#pragma unroll
            for (int i = h * H; i < (h + 1) * H; ++i) c[i] = encode_plain<T, BITS>(u[rr][i], scale);
          } else {
#pragma unroll
            for (int i = h * H; i < (h + 1) * H; ++i) c[i] = (C)to_code<T>(u[rr][i], (std::int16_t)be, BITS);
          }
          const int bh = (int)__umulhi((unsigned)(idx + h * H), mE);
          if (idx + h * H == bh * E && bh < nbt)
            store_word(j.exps + (b0 + (std::uint64_t)bh) * (std::uint64_t)(W / 8), (std::uint64_t)be, W);
        }
      } else if constexpr (ESM == 0) {
        const int field = (int)(kc[rr] >> K::FSHIFT);
        const std::int64_t ex = exponent_of_field<T>(field);
        const std::int64_t be = wrap_signed(ex, W);
        const bool plain = km[rr] < K::SPECIAL && be == ex && plain_exponent<T>(be);
        if (plain) {
          const T scale = pow2<T>(BITS - 2 - (int)be);
#pragma unroll
          for (int i = 0; i < P; ++i) c[i] = encode_plain<T, BITS>(u[rr][i], scale);
        } else {
#pragma unroll
          for (int i = 0; i < P; ++i) c[i] = (C)to_code<T>(u[rr][i], (std::int16_t)be, BITS);
        }
        if ((GEN ? idx == bl * E : (idx & (E - 1)) == 0) && bl < nbt)
          store_word(j.exps + (b0 + (std::uint64_t)bl) * (std::uint64_t)(W / 8), (std::uint64_t)be, W);
      } else {
        // the lane's P / ESM blocks, each with its own exponent
        constexpr int NBL = P / ESM;
        std::int64_t exb[NBL];
#pragma unroll
        for (int b = 0; b < NBL; ++b) {
          std::uint32_t mr = K::raw(u[rr][b * ESM]);
#pragma unroll
          for (int i = 1; i < ESM; ++i) mr = max(mr, K::raw(u[rr][b * ESM + i]));
          std::uint32_t mc = mr;
          if (mr >= K::SPECIAL) {
            mc = K::clean(u[rr][b * ESM]);
#pragma unroll
            for (int i = 1; i < ESM; ++i) mc = max(mc, K::clean(u[rr][b * ESM + i]));
          }
          const std::int64_t ex = exponent_of_field<T>((int)(mc >> K::FSHIFT));
          const std::int64_t be = wrap_signed(ex, W);
          const bool plain = mr < K::SPECIAL && be == ex && plain_exponent<T>(be);
          if (plain) {
            const T scale = pow2<T>(BITS - 2 - (int)be);
#pragma unroll
            for (int i = 0; i < ESM; ++i) c[b * ESM + i] = encode_plain<T, BITS>(u[rr][b * ESM + i], scale);
          } else {
#pragma unroll
            for (int i = 0; i < ESM; ++i) c[b * ESM + i] = (C)to_code<T>(u[rr][b * ESM + i], (std::int16_t)be, BITS);
          }
          exb[b] = be;
        }
        const int present = nbt - bl; // blocks of this lane inside the array
        if (present > 0)
          store_lane_exps<W, NBL>(j.exps + (b0 + (std::uint64_t)bl) * (std::uint64_t)(W / 8), exb, present);
      }

      std::uint32_t seg[NW + 3];
#pragma unroll
      for (int i = 0; i < NW + 3; ++i) seg[i] = 0;
      pack_lane<Cfg>(seg, c);

      // a row's stream bytes are contiguous and start on a 16-byte boundary
      const std::uint32_t row_byte = (std::uint32_t)row * row_bytes;
      if constexpr (staged_aligned<Cfg>()) {
        std::uint32_t* st = s_stage + warp * stage_words<T, BITS, NT, RPW_, ESM>::per_warp;
#pragma unroll
        for (int i = 0; i < NW; ++i) st[lane * NW + i] = seg[i]; // odd stride: no bank conflicts
        __syncwarp();
        const uint4* st4 = reinterpret_cast<const uint4*>(st);
        for (int q = lane; q < L / 4; q += 32) {
          const std::uint32_t off = row_byte + 16u * (std::uint32_t)q;
          const uint4 v = st4[q];
          if ((full && !GEN) || off + 16u <= wb) {
            __stcs(reinterpret_cast<uint4*>(dst + off), v);
          } else if (off < wb) {
            const std::uint32_t vw[4] = { v.x, v.y, v.z, v.w };
#pragma unroll
            for (int t = 0; t < 4; ++t)
              if (off + 4u * t < wb) store_word_bounded(dst, off + 4u * t, wb, vw[t]);
          }
        }
        __syncwarp(); // the next row reuses the buffer
      } else if constexpr (Cfg::ALIGNED) {
        const std::uint32_t off = row_byte + (std::uint32_t)lane * (std::uint32_t)(L / 8);
        std::uint32_t out[NW];
#pragma unroll
        for (int i = 0; i < NW; ++i) out[i] = seg[i];
        if ((full && !GEN) || off + 4u * NW <= wb) {
          store_words<NW>(reinterpret_cast<std::uint32_t*>(dst + off), out);
        } else {
#pragma unroll
          for (int i = 0; i < NW; ++i)
            if (off + 4u * i < wb) store_word_bounded(dst, off + 4u * i, wb, out[i]);
        }
      } else {
        // The lane writes the stream words whose first bit lies in [S, Sn):
        // S is its first stream bit, Sn the next lane's (S + L, plus the
        // block's pad after the last lane of a padded exponent block).  Bits
        // past the segment are zero pad, then the next lane's first bits,
        // which one shuffle brings.  The row's words go through shared memory
        // so they leave as coalesced 16-byte stores.
        const std::uint32_t h0 = __shfl_down_sync(0xFFFFFFFFu, seg[0], 1);
        std::uint32_t* st = s_stage + warp * stage_words<T, BITS, NT, RPW_, ESM>::per_warp;
        if constexpr (L < 32) {
          // segments shorter than a word (fp64 below 8 bits): up to three
          // lanes share a word, so each lane ORs its bits into the zeroed
          // row; pad bits stay zero
          const int nrw = PAD ? (int)(row_bytes >> 2) : L;
          for (int q = lane; q < nrw; q += 32) st[q] = 0u;
          __syncwarp();
          std::uint32_t S;
          if constexpr (PAD)
            S = (std::uint32_t)((lane * P) >> log2E) * blk_bits + (std::uint32_t)(lane & (G - 1)) * L;
          else
            S = (std::uint32_t)lane * L;
          const std::uint32_t w = S >> 5;
          const int o = (int)(S & 31u);
          atomicOr(&st[w], seg[0] << o);
          if (o + L > 32) atomicOr(&st[w + 1], seg[0] >> (32 - o));
        } else if constexpr (PAD) {
          const int g = lane & (G - 1);
          const std::uint32_t S = (std::uint32_t)((lane * P) >> log2E) * blk_bits + (std::uint32_t)g * L;
          const std::uint32_t Sn = S + L + (g == G - 1 ? pad_bits : 0u);
          const std::uint32_t f = (S + 31u) >> 5;
          const int d = (int)(f * 32u - S);
          const int k = (int)(((Sn + 31u) >> 5) - f);
          const int sh = (int)(Sn & 31u);
#pragma unroll
          for (int i = 0; i < NW + 2; ++i) {
            if (i < k) {
              std::uint32_t w = __funnelshift_r(seg[i], seg[i + 1], d);
              if (i == k - 1 && sh != 0) w |= h0 << sh;
              st[f + i] = w;
            }
          }
        } else {
          // unpadded: Sn = S + L at a compile-time offset within the segment
          constexpr int q = L / 32, r = L % 32;
          seg[q] |= h0 << r;
          seg[q + 1] = h0 >> (32 - r);
          const std::uint32_t S = (std::uint32_t)lane * L;
          const std::uint32_t f = (S + 31u) >> 5;
          const int d = (int)(f * 32u - S);
          const int k = (int)(((S + L + 31u) >> 5) - f);
#pragma unroll
          for (int i = 0; i < NW; ++i)
            if (i < k) st[f + i] = __funnelshift_r(seg[i], seg[i + 1], d);
        }
        __syncwarp();
        const uint4* st4 = reinterpret_cast<const uint4*>(st);
        for (int q = lane; q < (PAD ? (int)(row_bytes >> 4) : L / 4); q += 32) {
          const std::uint32_t off = row_byte + 16u * (std::uint32_t)q;
          const uint4 v = st4[q];
          if ((full && !GEN) || off + 16u <= wb) {
            __stcs(reinterpret_cast<uint4*>(dst + off), v);
          } else if (off < wb) {
            const std::uint32_t vw[4] = { v.x, v.y, v.z, v.w };
#pragma unroll
            for (int t = 0; t < 4; ++t)
              if (off + 4u * t < wb) store_word_bounded(dst, off + 4u * t, wb, vw[t]);
          }
        }
        __syncwarp(); // the next row reuses the buffer
      }
    }
  }
}

template<class T, int BITS, int NT = kNT, int RPW = 2, bool PAD = false, int ESM = 0, bool MIS = false,
         bool GEN = false, bool HALF = false, bool WCR = false>
__global__ void __launch_bounds__(NT) k_compress_fast(Job j)
{
  __shared__ std::uint32_t s_rmax[2 * fast_cfg<T, BITS, NT, RPW>::ROWS];
  __shared__ __align__(16) std::uint32_t s_stage[stage_words<T, BITS, NT, RPW, ESM>::value];
  __shared__ std::uint32_t s_gmax[GEN ? (HALF ? 4 : 2) * fast_cfg<T, BITS, NT, RPW>::ROWS * 32 : 1];
  const std::uint32_t mE = GEN ? 0xFFFFFFFFu / (std::uint32_t)j.E + 1u : 0u; // ceil(2^32 / E), E not a power of two
  for (std::uint64_t tile = blockIdx.x; tile < j.tiles; tile += gridDim.x)
    fast_compress_tile<T, BITS, NT, RPW, PAD, ESM, MIS, GEN, HALF, WCR>(j, tile, s_rmax, s_stage,
                                                                        tile + gridDim.x < j.tiles, s_gmax, mE);
}

// ---------------------------------------------------------------- decompress

// One tile of decompress.
// GEN: exponent blocks of any multiple E of a lane's P values (not a power of
// two): a tile is j.tile_blocks whole blocks (rows past them idle), a lane's P
// values lie in one block, found as idx / E with a multiply-high by
// mE = ceil(2^32 / E) (exact for idx, E < 2^12).  With PAD (unaligned widths
// only) a lane's stream bit is block * block bits + (idx - block * E) * BITS.
// HALF (with GEN, blocks without padding): E is a multiple of P / 2 but not of
// P, so a lane's two halves may lie in two blocks; each half takes its own
// exponent.
template<class T, int BITS, int NT, int RPW_, bool PAD = false, int ESM = 0, bool MIS = false, bool GEN = false,
         bool HALF = false>
__device__ __forceinline__ void fast_decompress_tile(const Job& j, std::uint64_t tile, std::uint32_t mE = 0)
{
  using Cfg = fast_cfg<T, BITS, NT, RPW_, ESM>;
  constexpr int NBL = ESM ? Cfg::P / ESM : HALF ? 2 : 1; // exponents per lane
  using U = typename Cfg::U;
  using C = typename Cfg::C;
  constexpr int P = Cfg::P, L = Cfg::L, NW = Cfg::NW, ROW = Cfg::ROW, RPW = Cfg::RPW, TE = Cfg::TE,
                W = Cfg::W;

  T* __restrict__ y = static_cast<T*>(j.values_out);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int E = j.E, log2E = j.log2E;
  const int TB = (int)j.tile_blocks;
  const std::uint32_t blk_bits = 8u * j.block_bytes;

  {
    const int TV = GEN ? TB * E : TE; // values of a whole tile
    const std::uint64_t e0 = tile * (std::uint64_t)TV;
    const std::uint64_t rem64 = j.n - e0;
    const bool full = rem64 >= (std::uint64_t)TV;
    const int rem = full ? TV : (int)rem64;
    const std::uint64_t b0 = tile * (std::uint64_t)TB;
    const std::uint32_t* __restrict__ src =
      reinterpret_cast<const std::uint32_t*>(j.words + b0 * (std::uint64_t)j.block_bytes);

    std::uint32_t wv[RPW][NW + 1];
    std::int64_t be[RPW][NBL];
#pragma unroll
    for (int rr = 0; rr < RPW; ++rr) {
      const int row = rr * Cfg::WARPS + warp;
      const int idx = row * ROW + lane * P;
      if ((GEN || !full) && idx >= rem) continue;
      const int bl = GEN ? (int)__umulhi((unsigned)idx, mE) : idx >> log2E;
      const std::uint8_t* ep = j.exps + (b0 + (std::uint64_t)bl) * (std::uint64_t)(W / 8);
      if constexpr (ESM == 0) {
        be[rr][0] = load_exp(ep, W);
        if constexpr (HALF) {
          const int bl1 = (int)__umulhi((unsigned)(idx + P / 2), mE);
          be[rr][1] = load_exp(j.exps + (b0 + (std::uint64_t)bl1) * (std::uint64_t)(W / 8), W);
        }
      } else {
        load_lane_exps<W, NBL>(ep, be[rr]);
      }
      // tile stream bit (blocks may end in pad bits when E * BITS is not a
      // multiple of W; only the unaligned widths take padded blocks; blocks
      // smaller than a lane are padded at compile-time positions)
      const std::uint32_t S = ESM ? (std::uint32_t)(idx / (ESM ? ESM : 1)) * Cfg::BBB
                              : (PAD && GEN) ? (std::uint32_t)bl * blk_bits + (std::uint32_t)(idx - bl * E) * BITS
                              : PAD ? (std::uint32_t)(idx >> log2E) * blk_bits + (std::uint32_t)(idx & (E - 1)) * BITS
                                    : (std::uint32_t)idx * BITS;
      if constexpr (Cfg::ALIGNED) {
        std::uint32_t t[NW];
        load_words<NW>(src + (S >> 5), t);
#pragma unroll
        for (int i = 0; i < NW; ++i) wv[rr][i] = t[i];
        wv[rr][NW] = 0;
      } else {
        const std::uint32_t w0 = S >> 5;
        const int o = (int)(S & 31u);
#pragma unroll
        for (int i = 0; i < NW; ++i) wv[rr][i] = __ldg(src + w0 + i);
        // the extra word only when the segment reaches into it
        wv[rr][NW] = (o + L > 32 * NW) ? __ldg(src + w0 + NW) : 0u;
      }
    }

#pragma unroll
    for (int rr = 0; rr < RPW; ++rr) {
      const int row = rr * Cfg::WARPS + warp;
      const int idx = row * ROW + lane * P;
      if ((GEN || !full) && idx >= rem) continue;
      std::uint32_t seg[NW + 1];
      if constexpr (Cfg::ALIGNED) {
#pragma unroll
        for (int i = 0; i <= NW; ++i) seg[i] = wv[rr][i];
      } else {
        const int blg = (PAD && GEN) ? (int)__umulhi((unsigned)idx, mE) : 0;
        const int o = (int)((ESM ? (std::uint32_t)(idx / (ESM ? ESM : 1)) * Cfg::BBB
                             : (PAD && GEN) ? (std::uint32_t)blg * blk_bits + (std::uint32_t)(idx - blg * E) * BITS
                             : PAD ? (std::uint32_t)(idx >> log2E) * blk_bits + (std::uint32_t)(idx & (E - 1)) * BITS
                                   : (std::uint32_t)idx * BITS) &
                            31u);
#pragma unroll
        for (int i = 0; i < NW; ++i) seg[i] = __funnelshift_r(wv[rr][i], wv[rr][i + 1], o);
        seg[NW] = 0;
      }
      C c[P];
      unpack_lane<Cfg>(seg, c);

      U outb[P];
      constexpr int PB = P / NBL; // values per exponent in this lane
#pragma unroll
      for (int q = 0; q < NBL; ++q) {
        const std::int64_t b = be[rr][q];
        if (plain_exponent<T>(b)) {
          const T inv = pow2<T>((int)b - BITS + 2);
          const U zero_bits = sizeof(T) == 4 ? (U)((std::uint32_t)(b + 96) << 23)
                                             : (U)((std::uint64_t)(b + 992) << 52);
#pragma unroll
          for (int i = q * PB; i < (q + 1) * PB; ++i) outb[i] = decode_plain<T, BITS>(c[i], inv, zero_bits);
        } else {
#pragma unroll
          for (int i = q * PB; i < (q + 1) * PB; ++i) outb[i] = to_bits<T>(from_code<T>((U)c[i], b, BITS));
        }
      }

      if (MIS ? full : (full || idx + P <= rem)) {
        std::uint32_t v[8];
#pragma unroll
        for (int i = 0; i < P; ++i) {
          if constexpr (sizeof(T) == 4) {
            v[i] = outb[i];
          } else {
            v[2 * i] = (std::uint32_t)outb[i];
            v[2 * i + 1] = (std::uint32_t)(outb[i] >> 32);
          }
        }
        if constexpr (MIS) {
          // values off the 32-byte layout by kw words (whole tiles only)
          const int kw = (int)((reinterpret_cast<std::uintptr_t>(y) & 31u) >> 2);
          st_lane_mis(reinterpret_cast<std::uint32_t*>(y + e0 + idx) - kw, kw, v);
        } else {
          st256_stream(y + e0 + idx, v);
        }
      } else {
        for (int i = 0; i < P && idx + i < rem; ++i) y[e0 + idx + i] = from_bits<T>(outb[i]);
      }
    }
  }
}

template<class T, int BITS, int NT = kNT, int RPW = 2, bool PAD = false, int ESM = 0, bool MIS = false,
         bool GEN = false, bool HALF = false>
__global__ void __launch_bounds__(NT) k_decompress_fast(Job j)
{
  const std::uint32_t mE = GEN ? 0xFFFFFFFFu / (std::uint32_t)j.E + 1u : 0u; // ceil(2^32 / E), E not a power of two
  for (std::uint64_t tile = blockIdx.x; tile < j.tiles; tile += gridDim.x)
    fast_decompress_tile<T, BITS, NT, RPW, PAD, ESM, MIS, GEN, HALF>(j, tile, mE);
}

// The same with registers capped so that 2048 / NT CTAs fit on an SM (more
// tiles' loads in flight per SM, at the price of some recomputation).
template<class T, int BITS, int NT, bool PAD>
__global__ void __launch_bounds__(NT, 2048 / NT) k_decompress_fast_occ(Job j)
{
  for (std::uint64_t tile = blockIdx.x; tile < j.tiles; tile += gridDim.x)
    fast_decompress_tile<T, BITS, NT, 2, PAD>(j, tile);
}

// Whether a job's exponent blocks end in pad bits (E * bits not a multiple of
// W); the fast kernels take such jobs only for widths with unaligned segments.
__host__ __device__ inline bool job_padded(const Job& j)
{
  return 8ull * j.block_bytes != (std::uint64_t)j.E * (std::uint64_t)j.bits;
}

// Requirements of the fast kernels for (dtype, bits, E) and pointers, beyond
// having an instance for `bits`.
__host__ inline bool fast_eligible(const Job& j, int dtype_is_f64, const void* values, const void* words)
{
  const int P = dtype_is_f64 ? 4 : 8;
  const int TE = dtype_is_f64 ? 2048 : 4096;
  const int E = j.E;
  if (E < P || E > TE || (E & (E - 1)) != 0) return false;
  // padded blocks (E * bits not a multiple of W) only for widths whose lane
  // segments are not word-aligned: those kernels place each lane's bits
  // by its stream position
  if (((std::uint64_t)E * (std::uint64_t)j.bits) % (std::uint64_t)j.W != 0 && (P * j.bits) % 32 == 0) return false;
  if (reinterpret_cast<std::uintptr_t>(values) % 32 != 0) return false;
  if (reinterpret_cast<std::uintptr_t>(words) % 32 != 0) return false;
  return true;
}

// Whole blocks per tile of the GEN instances, or 0 when they do not apply: a
// block size that is a multiple of half a lane's P values but not a power of two,
// at most a tile, 32-byte aligned pointers (padded blocks: decompress of the
// unaligned widths only, checked at launch).  The count is the most whole
// blocks a tile holds, rounded down so that every tile's words start on a
// 32-byte boundary.
__host__ inline std::uint32_t fast_gen_tile_blocks(const Job& j, int dtype_is_f64, const void* values,
                                                   const void* words)
{
  const int P = dtype_is_f64 ? 4 : 8;
  const int TE = dtype_is_f64 ? 2048 : 4096;
  const int E = j.E;
  if (E < P || E > TE || E % (P / 2) != 0 || (E & (E - 1)) == 0) return 0;
  if (reinterpret_cast<std::uintptr_t>(values) % 32 != 0) return 0;
  if (reinterpret_cast<std::uintptr_t>(words) % 32 != 0) return 0;
  std::uint32_t g = 32; // blocks per 32-byte period of the word stream
  for (std::uint32_t b = j.block_bytes; g > 1 && b % 2 == 0; b /= 2) g /= 2;
  // E a multiple of P / 2 only: an even block count keeps tiles whole lanes
  if (E % P != 0 && g < 2) g = 2;
  const std::uint32_t tb = (std::uint32_t)(TE / E) / g * g;
  return tb;
}

// Requirements of the MIS instances: those of the fast kernels, with the
// values pointer aligned to the element size but not to 32 bytes (the words
// pointer still 32-byte aligned).
__host__ inline bool fast_mis_eligible(const Job& j, int dtype_is_f64, const void* values, const void* words)
{
  const std::uintptr_t v = reinterpret_cast<std::uintptr_t>(values);
  if (v % 32 == 0 || v % (dtype_is_f64 ? 8 : 4) != 0) return false;
  const void* aligned = reinterpret_cast<const void*>(v - v % 32);
  return fast_eligible(j, dtype_is_f64, aligned, words);
}

// Requirements of the small-block instances (ESM = E < P values per lane):
// E in {1, 2, 4} below the lane's P, 32-byte aligned pointers.
__host__ inline bool small_block_eligible(const Job& j, int dtype_is_f64, const void* values, const void* words)
{
  const int P = dtype_is_f64 ? 4 : 8;
  const int E = j.E;
  if (E >= P || (E != 1 && E != 2 && E != 4)) return false;
  if (reinterpret_cast<std::uintptr_t>(values) % 32 != 0) return false;
  if (reinterpret_cast<std::uintptr_t>(words) % 32 != 0) return false;
  return true;
}

} // namespace frsz2b

namespace frsz2b {

// Raw words and block exponent of one lane's P values, loaded ahead of the
// decode so a consumer can keep several lanes' loads in flight.
template<class T, int BITS>
struct lane_words
{
  using Cfg = fast_cfg<T, BITS>;
  // 32-bit exponents for W <= 32 keep the record small; only W = 64 needs more
  using exp_t = std::conditional_t<(Cfg::W == 64), std::int64_t, std::int32_t>;
  std::uint32_t w[Cfg::ALIGNED ? Cfg::NW : Cfg::NW + 1];
  exp_t be;
  int o; // bit offset of the segment in w[0] (unaligned widths only)
};

template<class T, int BITS>
__device__ __forceinline__ void fast_load_lane(const std::uint8_t* __restrict__ exps,
                                               const std::uint8_t* __restrict__ words, int log2E, std::uint64_t idx,
                                               lane_words<T, BITS>& lw)
{
  using Cfg = fast_cfg<T, BITS>;
  constexpr int L = Cfg::L, NW = Cfg::NW, W = Cfg::W;
  lw.be = (typename lane_words<T, BITS>::exp_t)load_exp(exps + (idx >> log2E) * (std::uint64_t)(W / 8), W);
  const std::uint64_t S = idx * (std::uint64_t)BITS;
  const std::uint32_t* src = reinterpret_cast<const std::uint32_t*>(words) + (S >> 5);
  lw.o = (int)(S & 31u);
  if constexpr (Cfg::ALIGNED) {
    std::uint32_t t[NW];
    load_words<NW>(src, t);
#pragma unroll
    for (int i = 0; i < NW; ++i) lw.w[i] = t[i];
  } else {
#pragma unroll
    for (int i = 0; i < NW; ++i) lw.w[i] = __ldg(src + i);
    lw.w[NW] = (lw.o + L > 32 * NW) ? __ldg(src + NW) : 0u;
  }
}

// The P codes of a loaded lane, in value order.
template<class T, int BITS>
__device__ __forceinline__ void fast_codes_loaded(const lane_words<T, BITS>& lw,
                                                  typename fast_cfg<T, BITS>::C (&c)[fast_cfg<T, BITS>::P])
{
  using Cfg = fast_cfg<T, BITS>;
  constexpr int NW = Cfg::NW;
  std::uint32_t seg[NW + 1];
  if constexpr (Cfg::ALIGNED) {
#pragma unroll
    for (int i = 0; i < NW; ++i) seg[i] = lw.w[i];
    seg[NW] = 0;
  } else {
#pragma unroll
    for (int i = 0; i < NW; ++i) seg[i] = __funnelshift_r(lw.w[i], lw.w[i + 1], lw.o);
    seg[NW] = 0;
  }
  unpack_all<0, BITS>(seg, c);
}

template<class T, int BITS>
__device__ __forceinline__ void fast_decode_loaded(const lane_words<T, BITS>& lw, T (&out)[fast_cfg<T, BITS>::P])
{
  using Cfg = fast_cfg<T, BITS>;
  using U = typename Cfg::U;
  using C = typename Cfg::C;
  constexpr int P = Cfg::P;
  C c[P];
  fast_codes_loaded<T, BITS>(lw, c);
  const std::int64_t be = lw.be;
  if (plain_exponent<T>(be)) {
    const T inv = pow2<T>((int)be - BITS + 2);
    const U zero_bits =
      sizeof(T) == 4 ? (U)((std::uint32_t)(be + 96) << 23) : (U)((std::uint64_t)(be + 992) << 52);
#pragma unroll
    for (int i = 0; i < P; ++i) out[i] = from_bits<T>(decode_plain<T, BITS>(c[i], inv, zero_bits));
  } else {
#pragma unroll
    for (int i = 0; i < P; ++i) out[i] = from_code<T>((U)c[i], be, BITS);
  }
}

// Decode the P values of one array that start at element idx (a multiple of
// P), for consumers that use the values in registers (fused kernels).  The
// array's stream must be contiguous (E * bits a multiple of W, E a power of
// two >= P); values at or beyond the array's end come out as garbage and must
// be ignored by the caller.
template<class T, int BITS>
__device__ __forceinline__ void fast_decode_lane(const std::uint8_t* __restrict__ exps,
                                                 const std::uint8_t* __restrict__ words, int log2E,
                                                 std::uint64_t idx, T (&out)[fast_cfg<T, BITS>::P])
{
  using Cfg = fast_cfg<T, BITS>;
  using U = typename Cfg::U;
  using C = typename Cfg::C;
  constexpr int P = Cfg::P, L = Cfg::L, NW = Cfg::NW, W = Cfg::W;
  const std::int64_t be = load_exp(exps + (idx >> log2E) * (std::uint64_t)(W / 8), W);
  const std::uint64_t S = idx * (std::uint64_t)BITS;
  const std::uint32_t* src = reinterpret_cast<const std::uint32_t*>(words) + (S >> 5);
  std::uint32_t seg[NW + 1];
  if constexpr (Cfg::ALIGNED) {
    std::uint32_t t[NW];
    load_words<NW>(src, t);
#pragma unroll
    for (int i = 0; i < NW; ++i) seg[i] = t[i];
    seg[NW] = 0;
  } else {
    const int o = (int)(S & 31u);
    std::uint32_t wv[NW + 1];
#pragma unroll
    for (int i = 0; i < NW; ++i) wv[i] = __ldg(src + i);
    wv[NW] = (o + L > 32 * NW) ? __ldg(src + NW) : 0u;
#pragma unroll
    for (int i = 0; i < NW; ++i) seg[i] = __funnelshift_r(wv[i], wv[i + 1], o);
    seg[NW] = 0;
  }
  C c[P];
  unpack_all<0, BITS>(seg, c);
  if (plain_exponent<T>(be)) {
    const T inv = pow2<T>((int)be - BITS + 2);
    const U zero_bits =
      sizeof(T) == 4 ? (U)((std::uint32_t)(be + 96) << 23) : (U)((std::uint64_t)(be + 992) << 52);
#pragma unroll
    for (int i = 0; i < P; ++i) out[i] = from_bits<T>(decode_plain<T, BITS>(c[i], inv, zero_bits));
  } else {
#pragma unroll
    for (int i = 0; i < P; ++i) out[i] = from_code<T>((U)c[i], be, BITS);
  }
}

} // namespace frsz2b
