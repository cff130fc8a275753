// frsz2_blockwise.cuh -- compile-time-width kernels for exponent blocks of
// up to kBwMaxE values of any size (such as the reference tests' 5): one
// thread per exponent block.
//
// A CTA takes a chunk of bw_threads * bpt whole blocks.  Compress: the chunk's
// values come into shared memory with 16-byte loads; each thread reads its
// block's values (at most kBwMaxE, unrolled, so every code lands at a
// compile-time bit position), takes the block exponent, encodes and packs
// the codes into W-bit words in registers and writes them to a second
// shared-memory region, the chunk's block image, which leaves with 16-byte
// stores; the exponents leave with one store per thread.  Decompress runs
// the other way.  The per-value arithmetic is the fast kernels' (float
// scaling in the plain exponent range, the exact integer restatement
// elsewhere), so the bytes and values are the reference's bit for bit.
//
// Needs values aligned to the element size and the compressed buffer to the
// word size (the C ABI checks both); any E from 1 to kBwMaxE.
#pragma once

#include "frsz2_chunked.cuh"
#include "frsz2_launch.hpp"

#include <algorithm>
#include <array>
#include <atomic>
#include <utility>

namespace frsz2b {

#ifndef FRSZ2_BW_BYTES_F32
#define FRSZ2_BW_BYTES_F32 16384
#endif
#ifndef FRSZ2_BW_PIPE_F32
#define FRSZ2_BW_PIPE_F32 1
#endif
#ifndef FRSZ2_BW_PIPE_F64
#define FRSZ2_BW_PIPE_F64 1
#endif
constexpr int kBwMaxE = 16;       // largest block size
constexpr int kBwMaxBpt = 4;      // blocks per thread per chunk at most

// Bytes of values per chunk aimed at.
template<class T>
constexpr int bw_bytes()
{
  return sizeof(T) == 4 ? FRSZ2_BW_BYTES_F32 : 16384;
}
// Whether a CTA loads the next chunk while it works on the current one.
template<class T>
constexpr bool bw_pipe()
{
  return sizeof(T) == 4 ? FRSZ2_BW_PIPE_F32 != 0 : FRSZ2_BW_PIPE_F64 != 0;
}

// Threads per CTA: 256 for fp32, 128 for fp64, so that a chunk's two regions
// stay within the default 48 KB of dynamic shared memory for every E.
template<class T>
constexpr int bw_threads()
{
  return sizeof(T) == 4 ? 256 : 128;
}

#ifndef FRSZ2_BW_MIN_CTAS_F32
#define FRSZ2_BW_MIN_CTAS_F32 1
#endif
#ifndef FRSZ2_BW_MIN_CTAS_F64
#define FRSZ2_BW_MIN_CTAS_F64 1
#endif
// Resident CTAs per SM the register budget must allow.
template<class T>
constexpr int bw_min_ctas()
{
  return sizeof(T) == 4 ? FRSZ2_BW_MIN_CTAS_F32 : FRSZ2_BW_MIN_CTAS_F64;
}

template<int W>
using bw_word_t = std::conditional_t<
  (W == 8), std::uint8_t,
  std::conditional_t<(W == 16), std::uint16_t, std::conditional_t<(W == 32), std::uint32_t, std::uint64_t>>>;

// Blocks per thread per chunk for block size E.
template<class T>
__host__ __device__ inline int bw_bpt(int E)
{
  const int b = bw_bytes<T>() / (bw_threads<T>() * E * (int)sizeof(T));
  return b < 1 ? 1 : (b > kBwMaxBpt ? kBwMaxBpt : b);
}

// Bytes of the values region (the block image region has the same size: a
// block's bytes never exceed its values' bytes, since W divides the float
// width).  Each region carries 16 bytes for the alignment offset.
template<class T>
__host__ __device__ inline std::uint32_t bw_region_bytes(int E)
{
  return (std::uint32_t)(bw_threads<T>() * bw_bpt<T>(E) * E) * (std::uint32_t)sizeof(T) + 16u;
}
template<class T>
__host__ __device__ inline std::size_t bw_smem_bytes(int E)
{
  return 2 * (std::size_t)bw_region_bytes<T>(E);
}
// The most any block size up to kBwMaxE needs: 32,800 bytes for both types.
template<class T>
constexpr std::size_t bw_smem_max()
{
  return 2 * ((std::size_t)bw_threads<T>() * kBwMaxE * sizeof(T) + 16);
}
static_assert(bw_smem_max<float>() <= 48 * 1024 && bw_smem_max<double>() <= 48 * 1024, "default shared memory");

// Largest chunk of values or block images in bytes, and the 16-byte loads a
// thread makes of one.
template<class T>
constexpr std::uint32_t bw_max_chunk_bytes()
{
  return (std::uint32_t)bw_threads<T>() * kBwMaxE * (std::uint32_t)sizeof(T) > (std::uint32_t)bw_bytes<T>()
           ? (std::uint32_t)bw_threads<T>() * kBwMaxE * (std::uint32_t)sizeof(T)
           : (std::uint32_t)bw_bytes<T>();
}
template<class T>
constexpr int bw_loads_per_thread()
{
  return (int)((bw_max_chunk_bytes<T>() / 16 + bw_threads<T>() - 1) / bw_threads<T>());
}

// Global -> shared copy of `bytes` (at most bw_max_chunk_bytes) from g to
// s + (g mod 16), as chunk_copy<false> does, in two steps: bw_issue starts a
// thread's 16-byte loads into registers, bw_commit stores them (and the odd
// bytes before g's first and after its last 16-byte boundary).  Issuing the
// next chunk's loads before working on the current one hides their latency.
template<int NT, int MAXI>
__device__ __forceinline__ void bw_issue(const std::uint8_t* g, std::uint32_t bytes, uint4 (&r)[MAXI])
{
  const std::uint32_t h = (std::uint32_t)(reinterpret_cast<std::uintptr_t>(g) & 15u);
  const std::uint32_t head = h == 0 ? 0u : min(16u - h, bytes);
  const std::uint32_t n16 = (bytes - head) >> 4;
  const uint4* g16 = reinterpret_cast<const uint4*>(g + head);
#pragma unroll
  for (int i = 0; i < MAXI; ++i) {
    const std::uint32_t k = threadIdx.x + (std::uint32_t)(i * NT);
    if (k < n16) r[i] = __ldg(g16 + k);
  }
}

template<int NT, int MAXI>
__device__ __forceinline__ void bw_commit(const std::uint8_t* g, std::uint8_t* s, std::uint32_t bytes,
                                          const uint4 (&r)[MAXI])
{
  const std::uint32_t tid = threadIdx.x;
  const std::uint32_t h = (std::uint32_t)(reinterpret_cast<std::uintptr_t>(g) & 15u);
  const std::uint32_t head = h == 0 ? 0u : min(16u - h, bytes);
  const std::uint32_t n16 = (bytes - head) >> 4;
  const std::uint32_t tail0 = head + (n16 << 4);
  std::uint8_t* sb = s + h;
  uint4* s16 = reinterpret_cast<uint4*>(sb + head);
#pragma unroll
  for (int i = 0; i < MAXI; ++i) {
    const std::uint32_t k = tid + (std::uint32_t)(i * NT);
    if (k < n16) s16[k] = r[i];
  }
  if (tid < head) sb[tid] = __ldg(g + tid);
  for (std::uint32_t i = tail0 + tid; i < bytes; i += NT) sb[i] = __ldg(g + i);
}

template<class T, int BITS>
__global__ void __launch_bounds__(bw_threads<T>(), bw_min_ctas<T>()) k_compress_blockwise(Job j)
{
  using Cfg = fast_cfg<T, BITS>;
  using U = typename Cfg::U;
  using C = typename Cfg::C;
  using K = key_of<T>;
  constexpr int W = Cfg::W;
  using Word = bw_word_t<W>;
  extern __shared__ __align__(16) std::uint8_t s_chunk[];

  const T* __restrict__ x = static_cast<const T*>(j.values_in);
  const int tid = threadIdx.x;
  const int E = j.E;
  const std::uint32_t BB = j.block_bytes;
  const int bpt = bw_bpt<T>(E);
  constexpr int NT = bw_threads<T>();
  const int nbc = NT * bpt;
  std::uint8_t* s_val = s_chunk;
  std::uint8_t* s_img = s_chunk + bw_region_bytes<T>(E);
  const std::uint64_t nb = (j.n + (std::uint64_t)E - 1) / (std::uint64_t)E;
  const std::uint64_t nchunks = (nb + (std::uint64_t)nbc - 1) / (std::uint64_t)nbc;

  constexpr int MAXI = bw_loads_per_thread<T>();
  // chunk ch: its first block, values and the global addresses of both sides
  auto values_of = [&](std::uint64_t ch, int& nv) {
    const std::uint64_t v0 = ch * (std::uint64_t)nbc * (std::uint64_t)E;
    nv = (int)(j.n - v0 < (std::uint64_t)(nbc * E) ? j.n - v0 : (std::uint64_t)(nbc * E));
    return reinterpret_cast<const std::uint8_t*>(x + v0);
  };
  uint4 r[MAXI];
  std::uint64_t ch = blockIdx.x;
  if (bw_pipe<T>() && ch < nchunks) {
    int nv0;
    const std::uint8_t* g0 = values_of(ch, nv0);
    bw_issue<NT, MAXI>(g0, (std::uint32_t)nv0 * (std::uint32_t)sizeof(T), r);
  }
  for (; ch < nchunks; ch += gridDim.x) {
    const std::uint64_t b0 = ch * (std::uint64_t)nbc;
    int nv;
    const std::uint8_t* gin = values_of(ch, nv);
    if (!bw_pipe<T>()) bw_issue<NT, MAXI>(gin, (std::uint32_t)nv * (std::uint32_t)sizeof(T), r);
    const int nbk = (nv + E - 1) / E;
    std::uint8_t* gout = j.words + b0 * (std::uint64_t)BB;
    const std::uint32_t hv = (std::uint32_t)(reinterpret_cast<std::uintptr_t>(gin) & 15u);
    const std::uint32_t hw = (std::uint32_t)(reinterpret_cast<std::uintptr_t>(gout) & 15u);
    bw_commit<NT, MAXI>(gin, s_val, (std::uint32_t)nv * (std::uint32_t)sizeof(T), r);
    __syncthreads();
    if (bw_pipe<T>() && ch + gridDim.x < nchunks) { // the next chunk's loads fly while this one is coded
      int nvn;
      const std::uint8_t* gn = values_of(ch + gridDim.x, nvn);
      bw_issue<NT, MAXI>(gn, (std::uint32_t)nvn * (std::uint32_t)sizeof(T), r);
    }
    for (int b = tid; b < nbk; b += NT) {
      const T* __restrict__ sv = reinterpret_cast<const T*>(s_val + hv) + b * E;
      const int cnt = min(E, nv - b * E);
      // Loops run to the block's count: fully unrolled (bit positions stay
      // compile-time) with a branch out after value cnt - 1, uniform across
      // the warp except in the array's last block.  Values are read from
      // shared memory in each pass instead of being held in registers.
      //
      // pass 1: the block maximum of the raw keys, doubled (the sign shifted
      // out: a multiply, not a mask)
      std::uint32_t kr2 = 0;
#pragma unroll
      for (int k = 0; k < kBwMaxE; ++k) {
        if (k >= cnt) break;
        const U u = to_bits<T>(sv[k]);
        const std::uint32_t hi = sizeof(T) == 4 ? (std::uint32_t)u : (std::uint32_t)((std::uint64_t)u >> 32);
        kr2 = max(kr2, hi * 2u);
      }
      const std::uint32_t kr = kr2 >> 1;
      // block exponent: the largest non-NaN magnitude's (std::max semantics)
      std::uint32_t kc = kr;
      if (kr >= K::SPECIAL) {
        kc = 0;
#pragma unroll
        for (int k = 0; k < kBwMaxE; ++k) {
          if (k >= cnt) break;
          kc = max(kc, K::clean(to_bits<T>(sv[k])));
        }
      }
      const std::int64_t ex = exponent_of_field<T>((int)(kc >> K::FSHIFT));
      const std::int64_t be = wrap_signed(ex, W);
      const bool plain = kr < K::SPECIAL && be == ex && plain_exponent<T>(be);
      const T scale = pow2<T>(plain ? BITS - 2 - (int)be : 0);
      Word* __restrict__ dst = reinterpret_cast<Word*>(s_img + hw + (std::uint32_t)b * BB);
      // pass 2: codes into words, each word stored once it is complete, the
      // last (partial) one after the block's last value -- so only the words
      // the block's values reach are written.  Words of up to 32 bits are
      // built in a 32-bit register (a narrower store keeps the low bits) and a
      // code is added at its position, c * 2^o + word, which equals the OR
      // since the bits do not overlap and runs as one multiply-add instead of
      // a shift and an OR.
      using Acc = std::conditional_t<(W <= 32), std::uint32_t, std::uint64_t>;
      auto pack = [&](auto encode) {
        Acc cur = 0;
#pragma unroll
        for (int k = 0; k <= kBwMaxE; ++k) {
          const int p = k * BITS, w = p / W, o = p % W; // compile-time after unrolling
          if (k == kBwMaxE || k >= cnt) {
            if (o != 0) dst[w] = (Word)cur;
            break;
          }
          const C c = encode(to_bits<T>(sv[k]));
          if constexpr (W <= 32)
            cur = (std::uint32_t)c * (1u << o) + cur;
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
      store_word(j.exps + (b0 + (std::uint64_t)b) * (std::uint64_t)(W / 8), (std::uint64_t)be, W);
    }
    __syncthreads();
    const int last_cnt = nv - (nbk - 1) * E;
    const std::uint32_t out_bytes = (std::uint32_t)(nbk - 1) * BB + written_block_bytes(last_cnt, BITS, W);
    chunk_copy<true>(gout, s_img, out_bytes);
    // no barrier here: the next chunk's commit writes the values region,
    // which every thread finished reading before the barrier above
  }
}

template<class T, int BITS>
__global__ void __launch_bounds__(bw_threads<T>(), bw_min_ctas<T>()) k_decompress_blockwise(Job j)
{
  using Cfg = fast_cfg<T, BITS>;
  using U = typename Cfg::U;
  using C = typename Cfg::C;
  constexpr int W = Cfg::W;
  using Word = bw_word_t<W>;
  constexpr int NWMAX = (kBwMaxE * BITS + W - 1) / W;
  constexpr int CBITS = 8 * (int)sizeof(C);
  constexpr C CMASK = BITS == CBITS ? ~C(0) : (C)((C(1) << (BITS % CBITS)) - C(1));
  extern __shared__ __align__(16) std::uint8_t s_chunk[];

  T* __restrict__ y = static_cast<T*>(j.values_out);
  const int tid = threadIdx.x;
  const int E = j.E;
  const std::uint32_t BB = j.block_bytes;
  const int nwb = (int)(BB / (W / 8));
  const int bpt = bw_bpt<T>(E);
  constexpr int NT = bw_threads<T>();
  const int nbc = NT * bpt;
  std::uint8_t* s_val = s_chunk;
  std::uint8_t* s_img = s_chunk + bw_region_bytes<T>(E);
  const std::uint64_t nb = (j.n + (std::uint64_t)E - 1) / (std::uint64_t)E;
  const std::uint64_t nchunks = (nb + (std::uint64_t)nbc - 1) / (std::uint64_t)nbc;

  constexpr int MAXI = bw_loads_per_thread<T>();
  // chunk ch's blocks and values, and the loads of its block image and
  // exponents
  auto blocks_of = [&](std::uint64_t ch, int& nv, int& nbk) {
    const std::uint64_t b0 = ch * (std::uint64_t)nbc;
    const std::uint64_t v0 = b0 * (std::uint64_t)E;
    nv = (int)(j.n - v0 < (std::uint64_t)(nbc * E) ? j.n - v0 : (std::uint64_t)(nbc * E));
    nbk = (nv + E - 1) / E;
    return b0;
  };
  uint4 r[MAXI];
  std::int64_t be[kBwMaxBpt];
  auto issue = [&](std::uint64_t ch) {
    int nv, nbk;
    const std::uint64_t b0 = blocks_of(ch, nv, nbk);
#pragma unroll
    for (int q = 0; q < kBwMaxBpt; ++q) {
      const int b = tid + q * NT;
      if (q < bpt && b < nbk) be[q] = load_exp(j.exps + (b0 + (std::uint64_t)b) * (std::uint64_t)(W / 8), W);
    }
    // whole blocks: the buffer holds every block in full
    bw_issue<NT, MAXI>(j.words + b0 * (std::uint64_t)BB, (std::uint32_t)nbk * BB, r);
  };
  std::uint64_t ch = blockIdx.x;
  if (bw_pipe<T>() && ch < nchunks) issue(ch);
  for (; ch < nchunks; ch += gridDim.x) {
    if (!bw_pipe<T>()) issue(ch);
    int nv, nbk;
    const std::uint64_t b0 = blocks_of(ch, nv, nbk);
    const std::uint8_t* gin = j.words + b0 * (std::uint64_t)BB;
    std::uint8_t* gout = reinterpret_cast<std::uint8_t*>(y + b0 * (std::uint64_t)E);
    const std::uint32_t hw = (std::uint32_t)(reinterpret_cast<std::uintptr_t>(gin) & 15u);
    const std::uint32_t hv = (std::uint32_t)(reinterpret_cast<std::uintptr_t>(gout) & 15u);
    bw_commit<NT, MAXI>(gin, s_img, (std::uint32_t)nbk * BB, r);
    std::int64_t ecur[kBwMaxBpt];
#pragma unroll
    for (int q = 0; q < kBwMaxBpt; ++q) ecur[q] = be[q];
    __syncthreads();
    if (bw_pipe<T>() && ch + gridDim.x < nchunks) issue(ch + gridDim.x); // in flight while this chunk decodes

#pragma unroll
    for (int q = 0; q < kBwMaxBpt; ++q) {
      const int b = tid + q * NT;
      if (q >= bpt || b >= nbk) break;
      const std::int64_t e = ecur[q];
      const Word* src = reinterpret_cast<const Word*>(s_img + hw + (std::uint32_t)b * BB);
      Word wd[NWMAX];
#pragma unroll
      for (int w = 0; w < NWMAX; ++w) {
        if (w >= nwb) break;
        wd[w] = src[w];
      }
      const int cnt = min(E, nv - b * E);
      T* sv = reinterpret_cast<T*>(s_val + hv) + b * E;
      // one loop per arithmetic, so only the block's own runs
      auto unpack = [&](auto decode) {
#pragma unroll
        for (int k = 0; k < kBwMaxE; ++k) {
          if (k >= cnt) break;
          const int p = k * BITS, w = p / W, o = p % W; // compile-time after unrolling
          C c = (C)((C)wd[w] >> o);
          if (o + BITS > W) c |= (C)((C)wd[w + 1] << (W - o));
          sv[k] = from_bits<T>(decode((C)(c & CMASK)));
        }
      };
      if (plain_exponent<T>(e)) {
        const T inv = pow2<T>((int)e - BITS + 2);
        const U zero_bits =
          sizeof(T) == 4 ? (U)((std::uint32_t)(e + 96) << 23) : (U)((std::uint64_t)(e + 992) << 52);
        unpack([&](C c) { return decode_plain<T, BITS>(c, inv, zero_bits); });
      } else {
        unpack([&](C c) { return to_bits<T>(from_code<T>((U)c, e, BITS)); });
      }
    }
    __syncthreads();
    chunk_copy<true>(gout, s_val, (std::uint32_t)nv * (std::uint32_t)sizeof(T));
    // no barrier here: the next chunk's commit writes the image region,
    // which every thread finished reading before the barrier above
  }
}

// Launch of one width: a persistent grid of the resident CTAs (each CTA
// overlaps the next chunk's loads with the current chunk's work), fewer when
// there are fewer chunks.
template<class T, int BITS>
cudaError_t launch_blockwise_one(bool compress, const Job& j, cudaStream_t s)
{
  const std::size_t smem = bw_smem_bytes<T>(j.E);
  // resident CTAs per SM by direction and block size, queried once (threads
  // racing on the first call all store the same value)
  static std::atomic<int> resident[2][kBwMaxE + 1];
  std::atomic<int>& slot = resident[compress ? 0 : 1][j.E];
  int per_sm = slot.load(std::memory_order_relaxed);
  if (per_sm == 0) {
    int n = 0;
    const cudaError_t e =
      compress ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_compress_blockwise<T, BITS>, bw_threads<T>(), smem)
               : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_decompress_blockwise<T, BITS>, bw_threads<T>(),
                                                               smem);
    if (e != cudaSuccess) return e;
    per_sm = n < 1 ? 1 : n;
    slot.store(per_sm, std::memory_order_relaxed);
  }
  const std::uint64_t nb = (j.n + (std::uint64_t)j.E - 1) / (std::uint64_t)j.E;
  const std::uint64_t nbc = (std::uint64_t)bw_threads<T>() * (std::uint64_t)bw_bpt<T>(j.E);
  const std::uint64_t ctas = (std::uint64_t)sm_count() * (std::uint64_t)per_sm;
  const unsigned grid = (unsigned)std::max<std::uint64_t>(1, std::min<std::uint64_t>((nb + nbc - 1) / nbc, ctas));
  if (compress)
    k_compress_blockwise<T, BITS><<<grid, bw_threads<T>(), smem, s>>>(j);
  else
    k_decompress_blockwise<T, BITS><<<grid, bw_threads<T>(), smem, s>>>(j);
  return cudaGetLastError();
}

using blockwise_fn = cudaError_t (*)(bool, const Job&, cudaStream_t);

template<class T, int LO, int... I>
constexpr auto make_blockwise_table(std::integer_sequence<int, I...>)
{
  return std::array<blockwise_fn, sizeof...(I)>{ &launch_blockwise_one<T, LO + I>... };
}

// Whether the blockwise kernels take a job: block sizes up to kBwMaxE (the
// C ABI has already checked the pointers' alignment).
inline bool blockwise_eligible(const Job& j) { return j.E >= 1 && j.E <= kBwMaxE; }

cudaError_t launch_blockwise_f32(int bits, bool compress, const Job& j, cudaStream_t s);
cudaError_t launch_blockwise_f64(int bits, bool compress, const Job& j, cudaStream_t s);

} // namespace frsz2b
