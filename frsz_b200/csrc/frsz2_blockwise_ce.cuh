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

template<class T, int BITS, int E>
struct bwc_cfg
{
  static constexpr int NT = bw_threads<T>();
  static constexpr int W = fast_cfg<T, BITS>::W;
  static constexpr int WB = W / 8;
  static constexpr int NW = (E * BITS + W - 1) / W; // words per block
  static constexpr int BB = NW * WB;                // block bytes
  static constexpr int BPT0 = bw_bytes<T>() / (NT * E * (int)sizeof(T));
  static constexpr int BPT = BPT0 < 1 ? 1 : (BPT0 > kBwMaxBpt ? kBwMaxBpt : BPT0); // blocks per thread
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

// Codes of one block into its W-bit words at dst; a partial block (FULL
// false) writes only the words its cnt values reach.
template<class T, int BITS, int E, bool FULL>
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
  if (plain)
    pack([&](U v) { return encode_plain<T, BITS>(v, scale); });
  else
    pack([&](U v) { return (C)to_code<T>(v, (std::int16_t)be, BITS); });
}

template<class T, int BITS, int E>
__global__ void __launch_bounds__(bw_threads<T>()) k_compress_bwc(Job j)
{
  using G = bwc_cfg<T, BITS, E>;
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
  std::uint64_t ch = blockIdx.x;
  if (ch < nchunks) {
    int nv0;
    const std::uint8_t* g0 = values_of(ch, nv0);
    bw_issue<NT, G::LOADS_V>(g0, (std::uint32_t)nv0 * (std::uint32_t)sizeof(T), r);
  }
  for (; ch < nchunks; ch += gridDim.x) {
    const std::uint64_t b0 = ch * (std::uint64_t)NBC;
    int nv;
    const std::uint8_t* gin = values_of(ch, nv);
    const int nbk = (nv + E - 1) / E;
    std::uint8_t* gout = j.words + b0 * (std::uint64_t)BB;
    const std::uint32_t hv = (std::uint32_t)(reinterpret_cast<std::uintptr_t>(gin) & 15u);
    const std::uint32_t hw = (std::uint32_t)(reinterpret_cast<std::uintptr_t>(gout) & 15u);
    bw_commit<NT, G::LOADS_V>(gin, s_val, (std::uint32_t)nv * (std::uint32_t)sizeof(T), r);
    __syncthreads();
    if (ch + gridDim.x < nchunks) { // the next chunk's loads fly while this one is coded
      int nvn;
      const std::uint8_t* gn = values_of(ch + gridDim.x, nvn);
      bw_issue<NT, G::LOADS_V>(gn, (std::uint32_t)nvn * (std::uint32_t)sizeof(T), r);
    }
#pragma unroll
    for (int q = 0; q < G::BPT; ++q) {
      const int b = tid + q * NT;
      if (b >= nbk) break;
      const U* __restrict__ sv = reinterpret_cast<const U*>(s_val + hv) + b * E;
      Word* __restrict__ dst = reinterpret_cast<Word*>(s_img + hw + (std::uint32_t)b * BB);
      U u[E];
      std::int64_t be;
      if ((b + 1) * E <= nv) {
#pragma unroll
        for (int k = 0; k < E; ++k) u[k] = sv[k];
        bool plain;
        be = bwc_block_exponent<T, BITS, E, true>(u, E, plain);
        bwc_pack_block<T, BITS, E, true>(u, E, be, plain, dst);
      } else { // the array's last block, partial
        const int cnt = nv - b * E;
#pragma unroll
        for (int k = 0; k < E; ++k) u[k] = k < cnt ? sv[k] : U(0);
        bool plain;
        be = bwc_block_exponent<T, BITS, E, false>(u, cnt, plain);
        bwc_pack_block<T, BITS, E, false>(u, cnt, be, plain, dst);
      }
      reinterpret_cast<Word*>(j.exps)[b0 + (std::uint64_t)b] = (Word)be;
    }
    __syncthreads();
    const int last_cnt = nv - (nbk - 1) * E;
    const std::uint32_t out_bytes = (std::uint32_t)(nbk - 1) * BB + written_block_bytes(last_cnt, BITS, W);
    chunk_copy<true>(gout, s_img, out_bytes);
    // no barrier here: the next chunk's commit writes the values region,
    // which every thread finished reading before the barrier above
  }
}

template<class T, int BITS, int E>
__global__ void __launch_bounds__(bw_threads<T>()) k_decompress_bwc(Job j)
{
  using G = bwc_cfg<T, BITS, E>;
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
  auto issue = [&](std::uint64_t ch) {
    int nv, nbk;
    const std::uint64_t b0 = blocks_of(ch, nv, nbk);
#pragma unroll
    for (int q = 0; q < G::BPT; ++q) {
      const int b = tid + q * NT;
      if (b < nbk) be[q] = (std::int64_t)reinterpret_cast<const SWord*>(j.exps)[b0 + (std::uint64_t)b];
    }
    // whole blocks: the buffer holds every block in full
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
    bw_commit<NT, G::LOADS_I>(gin, s_img, (std::uint32_t)nbk * BB, r);
    std::int64_t ecur[G::BPT];
#pragma unroll
    for (int q = 0; q < G::BPT; ++q) ecur[q] = be[q];
    __syncthreads();
    if (ch + gridDim.x < nchunks) issue(ch + gridDim.x); // in flight while this chunk decodes
#pragma unroll
    for (int q = 0; q < G::BPT; ++q) {
      const int b = tid + q * NT;
      if (b >= nbk) break;
      const std::int64_t e = ecur[q];
      const Word* src = reinterpret_cast<const Word*>(s_img + hw + (std::uint32_t)b * BB);
      Word wd[NW];
#pragma unroll
      for (int w = 0; w < NW; ++w) wd[w] = src[w];
      U* sv = reinterpret_cast<U*>(s_val + hv) + b * E;
      const int cnt = min(E, nv - b * E);
      // full blocks store all E values; the array's last block, when partial,
      // only its cnt
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
      if (cnt == E)
        run(std::true_type{});
      else
        run(std::false_type{});
    }
    __syncthreads();
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
  using G = bwc_cfg<T, BITS, E>;
  static std::atomic<int> resident[2];
  std::atomic<int>& slot = resident[compress ? 0 : 1];
  int per_sm = slot.load(std::memory_order_relaxed);
  if (per_sm == 0) {
    int n = 0;
    const cudaError_t e = compress
                            ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_compress_bwc<T, BITS, E>, G::NT, 0)
                            : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_decompress_bwc<T, BITS, E>, G::NT, 0);
    if (e != cudaSuccess) return e;
    per_sm = n < 1 ? 1 : n;
    slot.store(per_sm, std::memory_order_relaxed);
  }
  const std::uint64_t nb = (j.n + (std::uint64_t)E - 1) / (std::uint64_t)E;
  const std::uint64_t ctas = (std::uint64_t)sm_count() * (std::uint64_t)per_sm;
  const unsigned grid =
    (unsigned)std::max<std::uint64_t>(1, std::min<std::uint64_t>((nb + G::NBC - 1) / G::NBC, ctas));
  if (compress)
    k_compress_bwc<T, BITS, E><<<grid, G::NT, 0, s>>>(j);
  else
    k_decompress_bwc<T, BITS, E><<<grid, G::NT, 0, s>>>(j);
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
