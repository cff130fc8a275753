// frsz2_blockwise_ce.cuh -- one-thread-per-block kernels with the block size
// as a template parameter, for the small block sizes that are not powers of
// two and that callers use most (the reference's own tests code blocks of 5
// values; 3, 6, 7 and 12 are the other common ones).
//
// Same structure as the run-time-E blockwise kernels (frsz2_blockwise.cuh):
// a persistent grid of CTAs, each taking chunks of NT * BPT whole blocks;
// a chunk's values (compress) or block images (decompress) come into shared
// memory with 16-byte loads, the next chunk's loads fly while the current
// chunk is coded, and the other side leaves with 16-byte streaming stores.
// With E known at compile time, a thread holds its block's values in
// registers, every code's word and bit position is a constant, the chunk
// geometry and every shared-memory offset are constants, and the
// per-value loop exits of the run-time-E kernels disappear; only the array's
// last block, when it is partial, takes a loop over its count.
//
// The per-value arithmetic is the fast kernels' (float scaling in the plain
// exponent range, the exact integer restatement elsewhere), so the bytes and
// values are the reference's bit for bit.  Needs values aligned to the
// element size and the compressed buffer to the word size (the C ABI checks
// both).
#pragma once

#include "frsz2_blockwise.cuh"

namespace frsz2b {

#ifndef FRSZ2_BWC_CHUNK_C
#define FRSZ2_BWC_CHUNK_C 20480
#endif
#ifndef FRSZ2_BWC_CHUNK_D
#define FRSZ2_BWC_CHUNK_D 16384
#endif
#ifndef FRSZ2_BWC_QUNROLL
#define FRSZ2_BWC_QUNROLL 8
#endif
// unroll factor of a thread's loop over its blocks in a chunk
constexpr int kBwcQUnroll = FRSZ2_BWC_QUNROLL;

template<class T, int BITS, int E, bool COMPRESS>
struct bwc_cfg
{
  static constexpr int NT = bw_threads<T>();
  static constexpr int W = fast_cfg<T, BITS>::W;
  static constexpr int WB = W / 8;
  static constexpr int NW = (E * BITS + W - 1) / W; // words per block
  static constexpr int BB = NW * WB;                // block bytes
  // values per chunk aimed at: about 20 KB and at most 8 blocks per thread
  // compressing (the per-chunk work is spread over more blocks than the
  // run-time-E kernels' 16 KB), 16 KB and at most 4 blocks per thread
  // decompressing (the next chunk's exponents are held in registers; 5 blocks
  // per thread at E 3 measured slower)
  static constexpr int BPT0 = (COMPRESS ? FRSZ2_BWC_CHUNK_C : FRSZ2_BWC_CHUNK_D) / (NT * E * (int)sizeof(T));
  static constexpr int BPT_MAX = COMPRESS ? 8 : 4;
  static constexpr int BPT = BPT0 < 1 ? 1 : (BPT0 > BPT_MAX ? BPT_MAX : BPT0); // blocks per thread
  static constexpr int NBC = NT * BPT;               // blocks per chunk
  static constexpr std::uint32_t VAL_BYTES = (std::uint32_t)NBC * E * (std::uint32_t)sizeof(T);
  static constexpr std::uint32_t IMG_BYTES = (std::uint32_t)NBC * BB;
  // 16-byte loads a thread makes of a chunk (values, or a block image)
  static constexpr int LOADS_V = (int)((VAL_BYTES / 16 + NT - 1) / NT);
  static constexpr int LOADS_I = (int)((IMG_BYTES / 16 + NT - 1) / NT);
};

// Block exponent and plain-domain flag of a block's raw bit patterns
// (std::max semantics: NaNs are skipped).
template<class T, int BITS, int CNT_MAX, bool FULL>
__device__ __forceinline__ std::int64_t bwc_block_exponent(const typename fp<T>::U (&u)[CNT_MAX], int cnt,
                                                           bool& plain)
{
  using K = key_of<T>;
  using U = typename fp<T>::U;
  constexpr int W = fast_cfg<T, BITS>::W;
  std::uint32_t kr2 = 0;
#pragma unroll
  for (int k = 0; k < CNT_MAX; ++k) {
    if (!FULL && k >= cnt) break;
    const std::uint32_t hi = sizeof(T) == 4 ? (std::uint32_t)u[k] : (std::uint32_t)((std::uint64_t)u[k] >> 32);
    kr2 = max(kr2, hi * 2u);
  }
  const std::uint32_t kr = kr2 >> 1;
  std::uint32_t kc = kr;
  if (kr >= K::SPECIAL) {
    kc = 0;
#pragma unroll
    for (int k = 0; k < CNT_MAX; ++k) {
      if (!FULL && k >= cnt) break;
      kc = max(kc, K::clean((U)u[k]));
    }
  }
  const std::int64_t ex = exponent_of_field<T>((int)(kc >> K::FSHIFT));
  const std::int64_t be = wrap_signed(ex, W);
  plain = kr < K::SPECIAL && be == ex && plain_exponent<T>(be);
  return be;
}

// encode_plain (the plain-exponent-range code of a value) with one fused
// multiply-add instead of a multiply and a float-to-integer conversion (a
// quarter-rate instruction): in the plain range |x| * scale < 2^(BITS-1), so
// for BITS <= 24 (fp32) or <= 53 (fp64) the exact product plus 2^23 (2^52),
// rounded toward zero once, is 2^23 + trunc(|x| * scale) -- the magnitude
// lands in the low bits of the sum (the magic-number method of rounding to an
// integer, Muller et al., Handbook of Floating-Point Arithmetic, sec. 5.1,
// here with the rounding toward zero that truncation asks for).  The sign
// goes in with one bit select: the magnitude's bits above BITS-2 are zero and
// the shifted bit pattern's bits below BITS-1 are dropped.
template<class T, int BITS>
__device__ __forceinline__ typename fast_cfg<T, BITS>::C encode_plain_fma(typename fp<T>::U u, T scale)
{
  using C = typename fast_cfg<T, BITS>::C;
  if constexpr (sizeof(T) == 4) {
    static_assert(BITS <= 24, "the magnitude must fit below 2^23");
    const std::uint32_t f = __float_as_uint(__fmaf_rz(fabsf(__uint_as_float(u)), scale, 8388608.0f));
    constexpr std::uint32_t M = (1u << (BITS - 1)) - 1u;
    return (f & M) | ((u >> (32 - BITS)) & ~M);
  } else if constexpr (BITS <= 32) {
    const double d = __fma_rz(fabs(__longlong_as_double((long long)u)), scale, 4503599627370496.0);
    const std::uint32_t f = (std::uint32_t)__double2loint(d);
    constexpr std::uint32_t M = (1u << (BITS - 1)) - 1u;
    return (f & M) | (((std::uint32_t)(u >> 32) >> (32 - BITS)) & ~M);
  } else {
    static_assert(BITS <= 53, "the magnitude must fit below 2^52");
    const double d = __fma_rz(fabs(__longlong_as_double((long long)u)), scale, 4503599627370496.0);
    const std::uint64_t f = (std::uint64_t)__double_as_longlong(d);
    constexpr std::uint64_t M = (1ull << (BITS - 1)) - 1ull;
    return (C)((f & M) | ((u >> (64 - BITS)) & ~M));
  }
}

// Whether encode_plain_fma serves this width.
template<class T, int BITS>
constexpr bool fma_encodes()
{
  return sizeof(T) == 4 ? BITS <= 24 : BITS <= 53;
}

// Codes of one block into its W-bit words at dst; a partial block (FULL
// false) writes only the words its cnt values reach.
// PLAIN: 1 the block is known to be in the plain range, 0 it is not, -1 test
// the plain flag.
template<class T, int BITS, int E, bool FULL, int PLAIN = -1>
__device__ __forceinline__ void bwc_pack_block(const typename fp<T>::U (&u)[E], int cnt, std::int64_t be, bool plain,
                                               bw_word_t<fast_cfg<T, BITS>::W>* __restrict__ dst)
{
  using Cfg = fast_cfg<T, BITS>;
  using C = typename Cfg::C;
  using U = typename fp<T>::U;
  constexpr int W = Cfg::W;
  using Word = bw_word_t<W>;
  using Acc = std::conditional_t<(W <= 32), std::uint32_t, std::uint64_t>;
  const T scale = pow2<T>(plain ? BITS - 2 - (int)be : 0);
  auto pack = [&](auto encode) {
    Acc cur = 0;
#pragma unroll
    for (int k = 0; k <= E; ++k) {
      const int p = k * BITS, w = p / W, o = p % W; // constants after unrolling
      if (k == E || (!FULL && k >= cnt)) {
        if (o != 0) dst[w] = (Word)cur;
        break;
      }
      const C c = encode(u[k]);
      if constexpr (W <= 32)
        cur = (std::uint32_t)c * (1u << o) + cur; // the bits do not overlap: the sum is the OR
      else
        cur |= (Acc)c << o;
      if (o + BITS >= W) {
        dst[w] = (Word)cur;
        cur = o + BITS > W ? (Acc)(c >> (W - o)) : Acc(0);
      }
    }
  };
  auto plain_code = [&](U v) {
    if constexpr (fma_encodes<T, BITS>())
      return encode_plain_fma<T, BITS>(v, scale);
    else
      return encode_plain<T, BITS>(v, scale);
  };
  if (PLAIN == 1 || (PLAIN == -1 && plain))
    pack(plain_code);
  else
    pack([&](U v) { return (C)to_code<T>(v, (std::int16_t)be, BITS); });
}

// Resident CTAs per SM the register budget must allow (0: ptxas's own
// choice).  Compress is held to 4 (56 registers for fp32 b16 E5; with a
// bound of 1, ptxas spends 90 on the unrolled blocks, measured 2-8 % slower);
// decompress keeps ptxas's choice (40 registers there; 72 with a bound of 1,
// measured slower).
#ifndef FRSZ2_BWC_MIN_CTAS_C
#define FRSZ2_BWC_MIN_CTAS_C 4
#endif
#ifndef FRSZ2_BWC_MIN_CTAS_D
#define FRSZ2_BWC_MIN_CTAS_D 0
#endif
#if FRSZ2_BWC_MIN_CTAS_C > 0
#define FRSZ2_BWC_BOUNDS_C(nt) __launch_bounds__(nt, FRSZ2_BWC_MIN_CTAS_C)
#else
#define FRSZ2_BWC_BOUNDS_C(nt) __launch_bounds__(nt)
#endif
#if FRSZ2_BWC_MIN_CTAS_D > 0
#define FRSZ2_BWC_BOUNDS_D(nt) __launch_bounds__(nt, FRSZ2_BWC_MIN_CTAS_D)
#else
#define FRSZ2_BWC_BOUNDS_D(nt) __launch_bounds__(nt)
#endif

// One block of cnt (1..E) values at sv, any exponent: block exponent, the
// per-block choice of plain-range or exact-integer codes, words to dst,
// exponent to *ep.  Out of line, so the kernels' registers are sized for
// their inline path (whole warps of plain-range blocks); this one runs for
// warps holding a block outside the plain range and for the array's last,
// partial chunk.
template<class T, int BITS, int E>
__device__ __noinline__ void bwc_compress_block_any(const typename fp<T>::U* sv, int cnt,
                                                    bw_word_t<fast_cfg<T, BITS>::W>* dst,
                                                    bw_word_t<fast_cfg<T, BITS>::W>* ep)
{
  using U = typename fp<T>::U;
  using Word = bw_word_t<fast_cfg<T, BITS>::W>;
  U u[E];
  bool plain;
  std::int64_t be;
  if (cnt == E) {
#pragma unroll
    for (int k = 0; k < E; ++k) u[k] = sv[k];
    be = bwc_block_exponent<T, BITS, E, true>(u, E, plain);
    bwc_pack_block<T, BITS, E, true>(u, E, be, plain, dst);
  } else {
#pragma unroll
    for (int k = 0; k < E; ++k) u[k] = k < cnt ? sv[k] : U(0);
    be = bwc_block_exponent<T, BITS, E, false>(u, cnt, plain);
    bwc_pack_block<T, BITS, E, false>(u, cnt, be, plain, dst);
  }
  *ep = (Word)be;
}

// Chunk staging for a full chunk whose global side starts on a 16-byte
// boundary (every chunk but an array's last, when the array's pointers are
// 16-byte aligned): BYTES / 16 whole 16-byte accesses, no head, no tail, the
// loop bounds and predicates compile-time constants.  The other chunks use
// bw_issue / bw_commit / chunk_copy.
template<int NT, int MAXI, std::uint32_t BYTES>
__device__ __forceinline__ void bwc_issue_full(const std::uint8_t* g, uint4 (&r)[MAXI])
{
  constexpr std::uint32_t N16 = BYTES / 16;
  static_assert(BYTES % 16 == 0 && N16 <= (std::uint32_t)(MAXI * NT), "chunk bytes");
  const uint4* g16 = reinterpret_cast<const uint4*>(g);
#pragma unroll
  for (int i = 0; i < MAXI; ++i) {
    const std::uint32_t k = threadIdx.x + (std::uint32_t)(i * NT);
    if (N16 % NT == 0 || k < N16) r[i] = __ldg(g16 + k);
  }
}

template<int NT, int MAXI, std::uint32_t BYTES>
__device__ __forceinline__ void bwc_commit_full(std::uint8_t* s, const uint4 (&r)[MAXI])
{
  constexpr std::uint32_t N16 = BYTES / 16;
  uint4* s16 = reinterpret_cast<uint4*>(s);
#pragma unroll
  for (int i = 0; i < MAXI; ++i) {
    const std::uint32_t k = threadIdx.x + (std::uint32_t)(i * NT);
    if (N16 % NT == 0 || k < N16) s16[k] = r[i];
  }
}

template<int NT, std::uint32_t BYTES>
__device__ __forceinline__ void bwc_store_full(std::uint8_t* g, const std::uint8_t* s)
{
  constexpr std::uint32_t N16 = BYTES / 16;
  static_assert(BYTES % 16 == 0, "chunk bytes");
  uint4* g16 = reinterpret_cast<uint4*>(g);
  const uint4* s16 = reinterpret_cast<const uint4*>(s);
#pragma unroll
  for (int i = 0; i < (int)((N16 + NT - 1) / NT); ++i) {
    const std::uint32_t k = threadIdx.x + (std::uint32_t)(i * NT);
    if (N16 % NT == 0 || k < N16) __stcs(g16 + k, s16[k]);
  }
}

template<class T, int BITS, int E>
__global__ void FRSZ2_BWC_BOUNDS_C(bw_threads<T>()) k_compress_bwc(Job j)
{
  using G = bwc_cfg<T, BITS, E, true>;
  using U = typename fp<T>::U;
  constexpr int NT = G::NT, W = G::W, BB = G::BB, NBC = G::NBC;
  using Word = bw_word_t<W>;
  __shared__ __align__(16) std::uint8_t s_val[G::VAL_BYTES + 16];
  __shared__ __align__(16) std::uint8_t s_img[G::IMG_BYTES + 16];

  const T* __restrict__ x = static_cast<const T*>(j.values_in);
  const int tid = threadIdx.x;
  const std::uint64_t nb = (j.n + (std::uint64_t)E - 1) / (std::uint64_t)E;
  const std::uint64_t nchunks = (nb + (std::uint64_t)NBC - 1) / (std::uint64_t)NBC;
  auto values_of = [&](std::uint64_t ch, int& nv) {
    const std::uint64_t v0 = ch * (std::uint64_t)NBC * (std::uint64_t)E;
    nv = (int)(j.n - v0 < (std::uint64_t)(NBC * E) ? j.n - v0 : (std::uint64_t)(NBC * E));
    return reinterpret_cast<const std::uint8_t*>(x + v0);
  };
  uint4 r[G::LOADS_V];
  // chunk starts are 16-byte multiples apart on both sides (NBC * E values,
  // NBC * BB bytes), so one test on the array's first chunk covers all
  static_assert((G::VAL_BYTES % 16) == 0 && (G::IMG_BYTES % 16) == 0, "chunk sizes");
  const bool aligned = ((reinterpret_cast<std::uintptr_t>(x) | reinterpret_cast<std::uintptr_t>(j.words)) & 15u) == 0;
  auto issue = [&](std::uint64_t c) {
    int nvc;
    const std::uint8_t* g = values_of(c, nvc);
    if (aligned && nvc == NBC * E)
      bwc_issue_full<NT, G::LOADS_V, G::VAL_BYTES>(g, r);
    else
      bw_issue<NT, G::LOADS_V>(g, (std::uint32_t)nvc * (std::uint32_t)sizeof(T), r);
  };
  std::uint64_t ch = blockIdx.x;
  if (ch < nchunks) issue(ch);
  for (; ch < nchunks; ch += gridDim.x) {
    const std::uint64_t b0 = ch * (std::uint64_t)NBC;
    int nv;
    const std::uint8_t* gin = values_of(ch, nv);
    const int nbk = (nv + E - 1) / E;
    std::uint8_t* gout = j.words + b0 * (std::uint64_t)BB;
    const std::uint32_t hv = (std::uint32_t)(reinterpret_cast<std::uintptr_t>(gin) & 15u);
    const std::uint32_t hw = (std::uint32_t)(reinterpret_cast<std::uintptr_t>(gout) & 15u);
    const bool fast = aligned && nv == NBC * E;
    if (fast)
      bwc_commit_full<NT, G::LOADS_V, G::VAL_BYTES>(s_val, r);
    else
      bw_commit<NT, G::LOADS_V>(gin, s_val, (std::uint32_t)nv * (std::uint32_t)sizeof(T), r);
    __syncthreads();
    if (ch + gridDim.x < nchunks) issue(ch + gridDim.x); // the next chunk's loads fly while this one is coded
    // Every chunk but the array's last is full: its blocks are all whole and
    // every thread has all its blocks, so that path needs no bounds checks,
    // and a warp vote sends whole warps down the plain-range encode (a warp
    // with any block outside that range runs the per-block choice).
    auto code_blocks = [&](auto full_chunk) {
      constexpr bool FC = decltype(full_chunk)::value;
#pragma unroll kBwcQUnroll
      for (int q = 0; q < G::BPT; ++q) {
        const int b = tid + q * NT;
        if (!FC && b >= nbk) break;
        const U* __restrict__ sv = reinterpret_cast<const U*>(s_val + hv) + b * E;
        Word* __restrict__ dst = reinterpret_cast<Word*>(s_img + hw + (std::uint32_t)b * BB);
        Word* ep = reinterpret_cast<Word*>(j.exps) + (b0 + (std::uint64_t)b);
        if (FC) {
          U u[E];
#pragma unroll
          for (int k = 0; k < E; ++k) u[k] = sv[k];
          bool plain;
          const std::int64_t be = bwc_block_exponent<T, BITS, E, true>(u, E, plain);
          if (__all_sync(0xffffffffu, plain)) {
            bwc_pack_block<T, BITS, E, true, 1>(u, E, be, true, dst);
            *ep = (Word)be;
          } else {
            bwc_compress_block_any<T, BITS, E>(sv, E, dst, ep);
          }
        } else {
          bwc_compress_block_any<T, BITS, E>(sv, min(E, nv - b * E), dst, ep);
        }
      }
    };
    if (nv == NBC * E)
      code_blocks(std::true_type{});
    else
      code_blocks(std::false_type{});
    __syncthreads();
    if (fast) {
      bwc_store_full<NT, G::IMG_BYTES>(gout, s_img);
    } else {
      const int last_cnt = nv - (nbk - 1) * E;
      const std::uint32_t out_bytes = (std::uint32_t)(nbk - 1) * BB + written_block_bytes(last_cnt, BITS, W);
      chunk_copy<true>(gout, s_img, out_bytes);
    }
    // no barrier here: the next chunk's commit writes the values region,
    // which every thread finished reading before the barrier above
  }
}

template<class T, int BITS, int E>
__global__ void FRSZ2_BWC_BOUNDS_D(bw_threads<T>()) k_decompress_bwc(Job j)
{
  using G = bwc_cfg<T, BITS, E, false>;
  using U = typename fp<T>::U;
  using Cfg = fast_cfg<T, BITS>;
  using C = typename Cfg::C;
  constexpr int NT = G::NT, W = G::W, BB = G::BB, NBC = G::NBC, NW = G::NW;
  constexpr int CBITS = 8 * (int)sizeof(C);
  constexpr C CMASK = BITS == CBITS ? ~C(0) : (C)((C(1) << (BITS % CBITS)) - C(1));
  using Word = bw_word_t<W>;
  using SWord = std::conditional_t<(W == 8), std::int8_t,
                                   std::conditional_t<(W == 16), std::int16_t,
                                                      std::conditional_t<(W == 32), std::int32_t, std::int64_t>>>;
  __shared__ __align__(16) std::uint8_t s_val[G::VAL_BYTES + 16];
  __shared__ __align__(16) std::uint8_t s_img[G::IMG_BYTES + 16];

  T* __restrict__ y = static_cast<T*>(j.values_out);
  const int tid = threadIdx.x;
  const std::uint64_t nb = (j.n + (std::uint64_t)E - 1) / (std::uint64_t)E;
  const std::uint64_t nchunks = (nb + (std::uint64_t)NBC - 1) / (std::uint64_t)NBC;
  auto blocks_of = [&](std::uint64_t ch, int& nv, int& nbk) {
    const std::uint64_t b0 = ch * (std::uint64_t)NBC;
    const std::uint64_t v0 = b0 * (std::uint64_t)E;
    nv = (int)(j.n - v0 < (std::uint64_t)(NBC * E) ? j.n - v0 : (std::uint64_t)(NBC * E));
    nbk = (nv + E - 1) / E;
    return b0;
  };
  uint4 r[G::LOADS_I];
  std::int64_t be[G::BPT];
  // chunk starts are 16-byte multiples apart on both sides, as in compress
  static_assert((G::VAL_BYTES % 16) == 0 && (G::IMG_BYTES % 16) == 0, "chunk sizes");
  const bool aligned = ((reinterpret_cast<std::uintptr_t>(y) | reinterpret_cast<std::uintptr_t>(j.words)) & 15u) == 0;
  auto issue = [&](std::uint64_t ch) {
    int nv, nbk;
    const std::uint64_t b0 = blocks_of(ch, nv, nbk);
#pragma unroll
    for (int q = 0; q < G::BPT; ++q) {
      const int b = tid + q * NT;
      if (b < nbk) be[q] = (std::int64_t)reinterpret_cast<const SWord*>(j.exps)[b0 + (std::uint64_t)b];
    }
    // whole blocks: the buffer holds every block in full
    if (aligned && nv == NBC * E)
      bwc_issue_full<NT, G::LOADS_I, G::IMG_BYTES>(j.words + b0 * (std::uint64_t)BB, r);
    else
      bw_issue<NT, G::LOADS_I>(j.words + b0 * (std::uint64_t)BB, (std::uint32_t)nbk * BB, r);
  };
  std::uint64_t ch = blockIdx.x;
  if (ch < nchunks) issue(ch);
  for (; ch < nchunks; ch += gridDim.x) {
    int nv, nbk;
    const std::uint64_t b0 = blocks_of(ch, nv, nbk);
    const std::uint8_t* gin = j.words + b0 * (std::uint64_t)BB;
    std::uint8_t* gout = reinterpret_cast<std::uint8_t*>(y + b0 * (std::uint64_t)E);
    const std::uint32_t hw = (std::uint32_t)(reinterpret_cast<std::uintptr_t>(gin) & 15u);
    const std::uint32_t hv = (std::uint32_t)(reinterpret_cast<std::uintptr_t>(gout) & 15u);
    const bool fast = aligned && nv == NBC * E;
    if (fast)
      bwc_commit_full<NT, G::LOADS_I, G::IMG_BYTES>(s_img, r);
    else
      bw_commit<NT, G::LOADS_I>(gin, s_img, (std::uint32_t)nbk * BB, r);
    std::int64_t ecur[G::BPT];
#pragma unroll
    for (int q = 0; q < G::BPT; ++q) ecur[q] = be[q];
    __syncthreads();
    if (ch + gridDim.x < nchunks) issue(ch + gridDim.x); // in flight while this chunk decodes
    // A thread's blocks, each decoded by its own exponent's arithmetic (a
    // warp vote and out-of-line rare paths, as compress uses, measured slower
    // here, and so did a conversion-free plain-range decode, the fused
    // multiply-add counterpart of compress's).  Full chunks skip the bounds
    // and partial-block tests.
    auto decode_blocks = [&](auto full_chunk) {
      constexpr bool FC = decltype(full_chunk)::value;
#pragma unroll
      for (int q = 0; q < G::BPT; ++q) {
        const int b = tid + q * NT;
        if (!FC && b >= nbk) break;
        const std::int64_t e = ecur[q];
        const Word* src = reinterpret_cast<const Word*>(s_img + hw + (std::uint32_t)b * BB);
        Word wd[NW];
#pragma unroll
        for (int w = 0; w < NW; ++w) wd[w] = src[w];
        U* sv = reinterpret_cast<U*>(s_val + hv) + b * E;
        const int cnt = FC ? E : min(E, nv - b * E);
        // full blocks store all E values; the array's last block, when
        // partial, only its cnt
        auto unpack = [&](auto decode, auto full) {
#pragma unroll
          for (int k = 0; k < E; ++k) {
            if (!decltype(full)::value && k >= cnt) break;
            const int p = k * BITS, w = p / W, o = p % W; // constants after unrolling
            C c = (C)((C)wd[w] >> o);
            if (o + BITS > W) c |= (C)((C)wd[w + 1] << (W - o));
            sv[k] = decode((C)(c & CMASK));
          }
        };
        auto run = [&](auto full) {
          if (plain_exponent<T>(e)) {
            const T inv = pow2<T>((int)e - BITS + 2);
            const U zero_bits =
              sizeof(T) == 4 ? (U)((std::uint32_t)(e + 96) << 23) : (U)((std::uint64_t)(e + 992) << 52);
            unpack([&](C c) { return decode_plain<T, BITS>(c, inv, zero_bits); }, full);
          } else {
            unpack([&](C c) { return to_bits<T>(from_code<T>((U)c, e, BITS)); }, full);
          }
        };
        if (FC || cnt == E)
          run(std::true_type{});
        else
          run(std::false_type{});
      }
    };
    if (nv == NBC * E)
      decode_blocks(std::true_type{});
    else
      decode_blocks(std::false_type{});
    __syncthreads();
    if (fast)
      bwc_store_full<NT, G::VAL_BYTES>(gout, s_val);
    else
      chunk_copy<true>(gout, s_val, (std::uint32_t)nv * (std::uint32_t)sizeof(T));
    // no barrier here: the next chunk's commit writes the image region,
    // which every thread finished reading before the barrier above
  }
}

// Launch of one (width, block size): a persistent grid of the resident CTAs,
// fewer when there are fewer chunks.
template<class T, int BITS, int E>
cudaError_t launch_bwc_one(bool compress, const Job& j, cudaStream_t s)
{
  using GC = bwc_cfg<T, BITS, E, true>;
  using GD = bwc_cfg<T, BITS, E, false>;
  static std::atomic<int> resident[2];
  std::atomic<int>& slot = resident[compress ? 0 : 1];
  int per_sm = slot.load(std::memory_order_relaxed);
  if (per_sm == 0) {
    int n = 0;
    const cudaError_t e = compress
                            ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_compress_bwc<T, BITS, E>, GC::NT, 0)
                            : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_decompress_bwc<T, BITS, E>, GD::NT, 0);
    if (e != cudaSuccess) return e;
    per_sm = n < 1 ? 1 : n;
    slot.store(per_sm, std::memory_order_relaxed);
  }
  const std::uint64_t nb = (j.n + (std::uint64_t)E - 1) / (std::uint64_t)E;
  const std::uint64_t ctas = (std::uint64_t)sm_count() * (std::uint64_t)per_sm;
  const std::uint64_t nbc = compress ? (std::uint64_t)GC::NBC : (std::uint64_t)GD::NBC;
  const unsigned grid = (unsigned)std::max<std::uint64_t>(1, std::min<std::uint64_t>((nb + nbc - 1) / nbc, ctas));
  if (compress)
    k_compress_bwc<T, BITS, E><<<grid, GC::NT, 0, s>>>(j);
  else
    k_decompress_bwc<T, BITS, E><<<grid, GD::NT, 0, s>>>(j);
  return cudaGetLastError();
}

template<class T, int E, int LO, int... I>
constexpr auto make_bwc_table(std::integer_sequence<int, I...>)
{
  return std::array<blockwise_fn, sizeof...(I)>{ &launch_bwc_one<T, LO + I, E>... };
}

// Block sizes with compile-time instances (every width of both float types).
#define FRSZ2_BWC_SIZES(X) X(3) X(5) X(6) X(7) X(12)

#define FRSZ2_BWC_DECL(E)                                                                                              \
  cudaError_t launch_bwc_f32_e##E(int bits, bool compress, const Job& j, cudaStream_t s);                              \
  cudaError_t launch_bwc_f64_e##E(int bits, bool compress, const Job& j, cudaStream_t s);
FRSZ2_BWC_SIZES(FRSZ2_BWC_DECL)
#undef FRSZ2_BWC_DECL

// The compile-time-E launch for (float type, E, bits), or cudaErrorNotSupported
// when E has no instance.
inline cudaError_t launch_bwc(bool is64, int E, int bits, bool compress, const Job& j, cudaStream_t s)
{
  switch (E) {
#define FRSZ2_BWC_CASE(EE)                                                                                             \
  case EE:                                                                                                             \
    return is64 ? launch_bwc_f64_e##EE(bits, compress, j, s) : launch_bwc_f32_e##EE(bits, compress, j, s);
    FRSZ2_BWC_SIZES(FRSZ2_BWC_CASE)
#undef FRSZ2_BWC_CASE
    default: return cudaErrorNotSupported;
  }
}

inline bool bwc_has(int E)
{
  switch (E) {
#define FRSZ2_BWC_HAS(EE) case EE:
    FRSZ2_BWC_SIZES(FRSZ2_BWC_HAS)
#undef FRSZ2_BWC_HAS
    return true;
    default: return false;
  }
}

} // namespace frsz2b

// Defines launch_bwc_<f32|f64>_e<E> over every width (one translation unit
// per float type and block size keeps the compile parallel).
#define FRSZ2_BWC_DEFINE(TNAME, T, E, LO, COUNT)                                                                      \
  namespace frsz2b {                                                                                                   \
  cudaError_t launch_bwc_##TNAME##_e##E(int bits, bool compress, const Job& j, cudaStream_t s)                         \
  {                                                                                                                    \
    static constexpr auto table = make_bwc_table<T, E, LO>(std::make_integer_sequence<int, COUNT>{});                 \
    if (bits < LO || bits >= LO + COUNT) return cudaErrorNotSupported;                                                 \
    return table[bits - LO](compress, j, s);                                                                           \
  }                                                                                                                    \
  }
