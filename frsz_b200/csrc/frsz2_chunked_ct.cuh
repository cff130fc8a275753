// frsz2_chunked_ct.cuh -- compile-time-width decompress for exponent blocks
// of 17 to kChunkMaxEDecompress values that the fast kernels do not take
// (block sizes that are not powers of two, pointers off the 32-byte layout).
//
// A persistent grid of CTAs; each takes chunks of kChunkValues / E whole
// blocks.  A chunk's block image comes into shared memory with 16-byte loads
// and its exponents into a per-block table (the scale 2^(e_b - BITS + 2) and
// the zero code's value 2^(e_b - 31) computed once per block, not per value);
// the next chunk's image and exponents are loaded into registers while the
// current chunk decodes.  Every thread decodes values at their stream
// positions -- value v of the chunk is code (v mod E) of block v / E -- and
// stores them with coalesced 4- or 8-byte stores.  With the width a template
// parameter, the masks and the code's word span are constants.  Plain-range
// blocks use the fast kernels' float arithmetic, the others the exact integer
// restatement, so the values are the reference's bit for bit.
#pragma once

#include "frsz2_blockwise.cuh"
#include "frsz2_chunked.cuh"

namespace frsz2b {

template<class T, int BITS>
struct chunk_ct_cfg
{
  static constexpr int W = fast_cfg<T, BITS>::W;
  static constexpr int WB = W / 8;
  static constexpr int MIN_E = 17;                             // smaller blocks go elsewhere
  static constexpr int MAX_BLOCKS = kChunkValues / MIN_E;      // blocks per chunk at most
  // a chunk's image: the values' bits plus each block's pad to whole words
  static constexpr std::uint32_t IMG_MAX = (std::uint32_t)((kChunkValues * BITS + 7) / 8 + MAX_BLOCKS * WB);
  static constexpr int LOADS = (int)((IMG_MAX / 16 + kNT - 1) / kNT); // 16-byte loads per thread
  static constexpr int VPT = kChunkValues / kNT;                // values per thread
  // every value before a thread's last lies inside any full chunk
  static_assert(kNT * (VPT - 1) <= kChunkValues - kChunkMaxEDecompress + 1, "full-chunk bound");
};

#ifndef FRSZ2_CHUNKED_UNROLL
#define FRSZ2_CHUNKED_UNROLL 2
#endif
// unroll factor of a thread's loop over its values in a chunk (fully
// unrolled, ptxas spends 76-102 registers on them)
constexpr int kChunkedUnroll = FRSZ2_CHUNKED_UNROLL;

template<class T, int BITS>
__global__ void __launch_bounds__(kNT) k_decompress_chunked_ct(Job j)
{
  using G = chunk_ct_cfg<T, BITS>;
  using Cfg = fast_cfg<T, BITS>;
  using U = typename Cfg::U;
  using C = typename Cfg::C;
  constexpr int W = G::W;
  constexpr int CBITS = 8 * (int)sizeof(C);
  constexpr C CMASK = BITS == CBITS ? ~C(0) : (C)((C(1) << (BITS % CBITS)) - C(1));
  using SWord = std::conditional_t<(W == 8), std::int8_t,
                                   std::conditional_t<(W == 16), std::int16_t,
                                                      std::conditional_t<(W == 32), std::int32_t, std::int64_t>>>;
  // image at its global start's offset modulo 16, plus guard words read (and
  // masked off) by the codes at the image's end
  __shared__ __align__(16) std::uint32_t s_img[(G::IMG_MAX + 16 + 16) / 4];
  // per block: the exponent, and the plain-range decode's scale and zero-code
  // value packed for one 8- (fp32) or 16-byte (fp64) load
  using Par = std::conditional_t<sizeof(T) == 4, uint2, ulonglong2>;
  __shared__ std::int32_t s_e[G::MAX_BLOCKS];
  __shared__ Par s_par[G::MAX_BLOCKS];

  T* __restrict__ y = static_cast<T*>(j.values_out);
  const int tid = threadIdx.x;
  const int E = j.E;
  const std::uint32_t BB = j.block_bytes, bb_bits = 8u * BB;
  const int nbc = kChunkValues / E;
  const std::uint64_t nb = (j.n + (std::uint64_t)E - 1) / (std::uint64_t)E;
  const std::uint64_t nchunks = (nb + (std::uint64_t)nbc - 1) / (std::uint64_t)nbc;
  auto blocks_of = [&](std::uint64_t ch, int& nv, int& nbk) {
    const std::uint64_t b0 = ch * (std::uint64_t)nbc;
    const std::uint64_t v0 = b0 * (std::uint64_t)E;
    nv = (int)(j.n - v0 < (std::uint64_t)(nbc * E) ? j.n - v0 : (std::uint64_t)(nbc * E));
    nbk = (nv + E - 1) / E;
    return b0;
  };

  uint4 r[G::LOADS];
  std::int64_t en = 0; // this thread's block exponent of the next chunk
  auto issue = [&](std::uint64_t ch) {
    int nv, nbk;
    const std::uint64_t b0 = blocks_of(ch, nv, nbk);
    if (tid < nbk) en = (std::int64_t)reinterpret_cast<const SWord*>(j.exps)[b0 + (std::uint64_t)tid];
    // whole blocks: the buffer holds every block in full
    bw_issue<kNT, G::LOADS>(j.words + b0 * (std::uint64_t)BB, (std::uint32_t)nbk * BB, r);
  };

  // value tid of a chunk: block b, code o; each further value is kNT later
  const int b_first = tid / E, o_first = tid - (tid / E) * E;
  const int step_b = kNT / E, step_o = kNT - (kNT / E) * E;

  std::uint64_t ch = blockIdx.x;
  if (ch < nchunks) issue(ch);
  for (; ch < nchunks; ch += gridDim.x) {
    int nv, nbk;
    const std::uint64_t b0 = blocks_of(ch, nv, nbk);
    const std::uint8_t* gin = j.words + b0 * (std::uint64_t)BB;
    const std::uint32_t h = (std::uint32_t)(reinterpret_cast<std::uintptr_t>(gin) & 15u);
    bw_commit<kNT, G::LOADS>(gin, reinterpret_cast<std::uint8_t*>(s_img), (std::uint32_t)nbk * BB, r);
    bool plain = true;
    if (tid < nbk) {
      const int e = (int)en;
      plain = plain_exponent<T>(e);
      s_e[tid] = e;
      Par par;
      if constexpr (sizeof(T) == 4) {
        par.x = __float_as_uint(pow2<float>(e - BITS + 2));
        par.y = (std::uint32_t)(e + 96) << 23;
      } else {
        par.x = (unsigned long long)__double_as_longlong(pow2<double>(e - BITS + 2));
        par.y = (unsigned long long)(e + 992) << 52;
      }
      if (plain) s_par[tid] = par;
    }
    // one decision per chunk: whether every block takes the plain-range decode
    const bool all_plain = __syncthreads_and(plain) != 0;
    if (ch + gridDim.x < nchunks) issue(ch + gridDim.x); // in flight while this chunk decodes

    const std::uint32_t bit0 = h * 8u;
    T* __restrict__ yv = y + b0 * (std::uint64_t)E + tid;
    // value tid + k * kNT: block b, code o, stream bit pos, advanced per step
    // (a block wrap moves pos over the block's pad bits)
    const std::uint32_t pos_step = (std::uint32_t)step_b * bb_bits + (std::uint32_t)(step_o * BITS);
    const std::uint32_t pos_wrap = bb_bits - (std::uint32_t)(E * BITS);
    auto decode_values = [&](auto full_chunk, auto plain_chunk) {
      constexpr bool FC = decltype(full_chunk)::value, PC = decltype(plain_chunk)::value;
      int b = b_first, o = o_first;
      std::uint32_t pos = bit0 + (std::uint32_t)b_first * bb_bits + (std::uint32_t)(o_first * BITS);
#pragma unroll kChunkedUnroll
      for (int k = 0; k < G::VPT; ++k) {
        // a full chunk holds nbc * E values, up to E - 1 fewer than
        // kChunkValues: only a thread's last value can pass its end
        if ((FC && k < G::VPT - 1) || tid + k * kNT < nv) {
          const int q = (int)(pos & 31u);
          const std::uint32_t* w = s_img + (pos >> 5);
          C c;
          if constexpr (BITS <= 32) {
            c = (C)__funnelshift_r(w[0], w[1], q);
          } else {
            const std::uint32_t lo = __funnelshift_r(w[0], w[1], q);
            const std::uint32_t hi = __funnelshift_r(w[1], w[2], q);
            c = (C)(((std::uint64_t)hi << 32) | lo);
          }
          c &= CMASK;
          U res;
          if (PC) {
            const Par par = s_par[b];
            if constexpr (sizeof(T) == 4)
              res = decode_plain<T, BITS>(c, __uint_as_float(par.x), (U)par.y);
            else
              res = decode_plain<T, BITS>(c, __longlong_as_double((long long)par.x), (U)par.y);
          } else {
            const int e = s_e[b];
            if (plain_exponent<T>(e)) {
              const Par par = s_par[b];
              if constexpr (sizeof(T) == 4)
                res = decode_plain<T, BITS>(c, __uint_as_float(par.x), (U)par.y);
              else
                res = decode_plain<T, BITS>(c, __longlong_as_double((long long)par.x), (U)par.y);
            } else {
              res = to_bits<T>(from_code<T>((U)c, e, BITS));
            }
          }
          yv[k * kNT] = from_bits<T>(res);
        }
        b += step_b;
        o += step_o;
        pos += pos_step;
        const bool wrap = o >= E;
        o -= wrap ? E : 0;
        b += wrap ? 1 : 0;
        pos += wrap ? pos_wrap : 0u;
      }
    };
    const bool full = nv == nbc * E;
    if (full && all_plain)
      decode_values(std::true_type{}, std::true_type{});
    else if (full)
      decode_values(std::true_type{}, std::false_type{});
    else
      decode_values(std::false_type{}, std::false_type{});
    __syncthreads(); // the next commit overwrites the image and the tables
  }
}

// Block exponent of cnt values at sv (std::max semantics: NaNs are skipped)
// and whether the block is in the plain range; four running maxima, so the
// loads of a thread's block overlap.
template<class T, int BITS>
__device__ __forceinline__ std::int64_t chunk_block_exponent(const typename fp<T>::U* sv, int cnt, bool& plain)
{
  using K = key_of<T>;
  constexpr int W = fast_cfg<T, BITS>::W;
  auto hi2 = [](typename fp<T>::U u) {
    return (sizeof(T) == 4 ? (std::uint32_t)u : (std::uint32_t)((std::uint64_t)u >> 32)) * 2u;
  };
  std::uint32_t m0 = 0, m1 = 0, m2 = 0, m3 = 0;
  int k = 0;
  for (; k + 4 <= cnt; k += 4) {
    m0 = max(m0, hi2(sv[k]));
    m1 = max(m1, hi2(sv[k + 1]));
    m2 = max(m2, hi2(sv[k + 2]));
    m3 = max(m3, hi2(sv[k + 3]));
  }
  for (; k < cnt; ++k) m0 = max(m0, hi2(sv[k]));
  const std::uint32_t kr = max(max(m0, m1), max(m2, m3)) >> 1;
  std::uint32_t kc = kr;
  if (kr >= K::SPECIAL) {
    kc = 0;
    for (int i = 0; i < cnt; ++i) kc = max(kc, K::clean(sv[i]));
  }
  const std::int64_t ex = exponent_of_field<T>((int)(kc >> K::FSHIFT));
  const std::int64_t be = wrap_signed(ex, W);
  plain = kr < K::SPECIAL && be == ex && plain_exponent<T>(be);
  return be;
}

// Compress counterpart for the same block sizes.  A chunk's values come into
// shared memory with 16-byte loads (the next chunk's in flight while this one
// is coded); one thread per block takes the block exponent and stores it;
// then one thread per 32-bit word of the chunk's block image gathers the
// codes that overlap the word (a code may straddle two words, the pad bits
// that end a block stay zero), and the image leaves with 16-byte stores.
// Only the bytes the reference writes are written: a partial last block ends
// at the word its last value reaches.
template<class T, int BITS>
__global__ void __launch_bounds__(kNT) k_compress_chunked_ct(Job j)
{
  using G = chunk_ct_cfg<T, BITS>;
  using Cfg = fast_cfg<T, BITS>;
  using U = typename Cfg::U;
  using C = typename Cfg::C;
  constexpr int W = G::W;
  using Word = bw_word_t<W>;
  constexpr std::uint32_t VAL_MAX = (std::uint32_t)kChunkValues * (std::uint32_t)sizeof(T);
  constexpr int LOADS_V = (int)((VAL_MAX / 16 + kNT - 1) / kNT);
  __shared__ __align__(16) std::uint8_t s_val[VAL_MAX + 16];
  __shared__ __align__(16) std::uint32_t s_img[(G::IMG_MAX + 16 + 16) / 4];
  __shared__ std::int32_t s_be[G::MAX_BLOCKS];
  __shared__ T s_scale[G::MAX_BLOCKS];

  const T* __restrict__ x = static_cast<const T*>(j.values_in);
  const int tid = threadIdx.x;
  const int E = j.E;
  const std::uint32_t BB = j.block_bytes;
  const int bb_bits = (int)(8u * BB);
  // floor(p / bb_bits) for the image bits p of a chunk (< 2^18) by one
  // multiply-high: exact while p * bb_bits < 2^32
  const std::uint32_t inv_bb = (std::uint32_t)((0xFFFFFFFFull + (std::uint64_t)bb_bits) / (std::uint64_t)bb_bits);
  const int nbc = kChunkValues / E;
  const std::uint64_t nb = (j.n + (std::uint64_t)E - 1) / (std::uint64_t)E;
  const std::uint64_t nchunks = (nb + (std::uint64_t)nbc - 1) / (std::uint64_t)nbc;
  auto values_of = [&](std::uint64_t ch, int& nv) {
    const std::uint64_t v0 = ch * (std::uint64_t)nbc * (std::uint64_t)E;
    nv = (int)(j.n - v0 < (std::uint64_t)(nbc * E) ? j.n - v0 : (std::uint64_t)(nbc * E));
    return reinterpret_cast<const std::uint8_t*>(x + v0);
  };
  uint4 r[LOADS_V];
  std::uint64_t ch = blockIdx.x;
  if (ch < nchunks) {
    int nv0;
    const std::uint8_t* g0 = values_of(ch, nv0);
    bw_issue<kNT, LOADS_V>(g0, (std::uint32_t)nv0 * (std::uint32_t)sizeof(T), r);
  }
  for (; ch < nchunks; ch += gridDim.x) {
    const std::uint64_t b0 = ch * (std::uint64_t)nbc;
    int nv;
    const std::uint8_t* gin = values_of(ch, nv);
    const int nbk = (nv + E - 1) / E;
    std::uint8_t* gout = j.words + b0 * (std::uint64_t)BB;
    const std::uint32_t hv = (std::uint32_t)(reinterpret_cast<std::uintptr_t>(gin) & 15u);
    const std::uint32_t h = (std::uint32_t)(reinterpret_cast<std::uintptr_t>(gout) & 15u);
    bw_commit<kNT, LOADS_V>(gin, s_val, (std::uint32_t)nv * (std::uint32_t)sizeof(T), r);
    __syncthreads();
    if (ch + gridDim.x < nchunks) { // the next chunk's loads fly while this one is coded
      int nvn;
      const std::uint8_t* gn = values_of(ch + gridDim.x, nvn);
      bw_issue<kNT, LOADS_V>(gn, (std::uint32_t)nvn * (std::uint32_t)sizeof(T), r);
    }
    const U* __restrict__ sv = reinterpret_cast<const U*>(s_val + hv);
    // block exponents: one thread per block
    bool plain = true;
    if (tid < nbk) {
      const int cnt = min(E, nv - tid * E);
      const std::int64_t be = chunk_block_exponent<T, BITS>(sv + tid * E, cnt, plain);
      s_be[tid] = (std::int32_t)be;
      s_scale[tid] = plain ? pow2<T>(BITS - 2 - (int)be) : T(0); // 0: outside the plain range
      reinterpret_cast<Word*>(j.exps)[b0 + (std::uint64_t)tid] = (Word)be;
    }
    const bool all_plain = __syncthreads_and(plain) != 0;
    // image words: smem byte h + i holds image byte i
    const int last_cnt = nv - (nbk - 1) * E;
    const std::uint32_t out_bytes = (std::uint32_t)(nbk - 1) * BB + written_block_bytes(last_cnt, BITS, W);
    const int nwords = (int)((h + out_bytes + 3u) / 4u);
    auto code_words = [&](auto plain_chunk) {
      constexpr bool PC = decltype(plain_chunk)::value;
      for (int w = tid; w < nwords; w += kNT) {
        const int p0 = 32 * w - 8 * (int)h; // image bit at the word's bit 0
        const int lo = p0 > 0 ? p0 : 0;
        std::uint64_t acc = 0;
        for (int b = (int)__umulhi((std::uint32_t)lo, inv_bb); b < nbk && b * bb_bits < p0 + 32; ++b) {
          const int base = b * bb_bits;
          const int cnt = min(E, nv - b * E);
          const int rlo = p0 - base > 0 ? p0 - base : 0;
          const int rhi = min(p0 + 32 - base, cnt * BITS);
          const U* vb = sv + b * E;
          const T scale = s_scale[b];
          const int be = s_be[b];
          for (int k = rlo / BITS; k * BITS < rhi; ++k) {
            C c;
            if (PC || scale != T(0))
              c = encode_plain<T, BITS>(vb[k], scale);
            else
              c = (C)to_code<T>(vb[k], (std::int16_t)be, BITS);
            const int sh = base + k * BITS - p0; // the code's bit 0 relative to the word's
            acc |= sh >= 0 ? (std::uint64_t)c << sh : (std::uint64_t)c >> -sh;
          }
        }
        s_img[w] = (std::uint32_t)acc;
      }
    };
    if (all_plain)
      code_words(std::true_type{});
    else
      code_words(std::false_type{});
    __syncthreads();
    chunk_copy<true>(gout, reinterpret_cast<std::uint8_t*>(s_img), out_bytes);
    // no barrier here: the next chunk's commit writes the values region,
    // which every thread finished reading before the barrier above; its
    // image words are written after two more barriers
  }
}

// Launch of one width: a persistent grid of the resident CTAs, fewer when
// there are fewer chunks.
template<class T, int BITS>
cudaError_t launch_chunked_ct_one(bool compress, const Job& j, cudaStream_t s)
{
  static std::atomic<int> resident[2];
  std::atomic<int>& slot = resident[compress ? 0 : 1];
  int per_sm = slot.load(std::memory_order_relaxed);
  if (per_sm == 0) {
    int n = 0;
    const cudaError_t e =
      compress ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_compress_chunked_ct<T, BITS>, kNT, 0)
               : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_decompress_chunked_ct<T, BITS>, kNT, 0);
    if (e != cudaSuccess) return e;
    per_sm = n < 1 ? 1 : n;
    slot.store(per_sm, std::memory_order_relaxed);
  }
  const std::uint64_t nb = (j.n + (std::uint64_t)j.E - 1) / (std::uint64_t)j.E;
  const std::uint64_t nbc = (std::uint64_t)(kChunkValues / j.E);
  const std::uint64_t ctas = (std::uint64_t)sm_count() * (std::uint64_t)per_sm;
  const unsigned grid = (unsigned)std::max<std::uint64_t>(1, std::min<std::uint64_t>((nb + nbc - 1) / nbc, ctas));
  if (compress)
    k_compress_chunked_ct<T, BITS><<<grid, kNT, 0, s>>>(j);
  else
    k_decompress_chunked_ct<T, BITS><<<grid, kNT, 0, s>>>(j);
  return cudaGetLastError();
}

using chunked_ct_fn = cudaError_t (*)(bool, const Job&, cudaStream_t);

template<class T, int LO, int... I>
constexpr auto make_chunked_ct_table(std::integer_sequence<int, I...>)
{
  return std::array<chunked_ct_fn, sizeof...(I)>{ &launch_chunked_ct_one<T, LO + I>... };
}

// Whether the compile-time-width chunked kernels take a job.
inline bool chunked_ct_eligible(const Job& j)
{
  return j.E >= chunk_ct_cfg<float, 4>::MIN_E && j.E <= kChunkMaxEDecompress;
}

cudaError_t launch_chunked_ct_f32(int bits, bool compress, const Job& j, cudaStream_t s);
cudaError_t launch_chunked_ct_f64(int bits, bool compress, const Job& j, cudaStream_t s);

} // namespace frsz2b
