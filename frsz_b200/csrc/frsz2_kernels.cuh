// frsz2_kernels.cuh -- FRSZ2 compress / decompress kernels for sm_100a.
//
// Two kernel families, both bit-exact with the reference CPU codec
// (compress_cpu_impl / decompress_cpu_impl, include/frsz2.hpp:1181, 1242):
//
//  * tile kernels (the hot path).  A CTA of 256 threads owns a tile of
//    TE = 256 * 4 * (16 / sizeof(T)) consecutive values (4096 fp32 / 2048 fp64),
//    i.e. TE / E whole exponent blocks.  Compress: four 128-bit loads per
//    thread, per-vector max exponent field, xor-shuffle (or shared-memory)
//    segmented max over the E / V lanes of a block, the reference's integer
//    align/truncate per value, codes staged in shared memory, then each thread
//    assembles 32-bit chunks of the packed little-endian stream with funnel
//    shifts and writes them with coalesced stores.  Decompress: the tile's
//    packed bytes are staged in shared memory with 128-bit loads, each thread
//    extracts the codes of its vectors with a rolling 64-bit window, decodes
//    them with the reference's clz normalisation and writes 128-bit stores.
//    Requirements (checked on the host): E a power of two in [8, TE], block
//    bytes a multiple of 4, TE/E * block bytes a multiple of 16, 16-byte
//    aligned value and word pointers.
//
//  * generic kernels: one warp per exponent block, any E >= 1 and any
//    alignment the element/word types allow.  Used when the tile kernels'
//    requirements do not hold (E = 1, 2, 4, 5 ..., odd block byte counts).
//
// Neither family writes a byte the reference leaves untouched: the 256-byte
// pad and the unused tail words of a partial last block keep their contents.
#pragma once

#include "frsz2_common.cuh"

#include <cuda_runtime.h>

namespace frsz2b {

constexpr int kNT = 256; // threads per CTA
constexpr int kR = 4;    // 128-bit vectors per thread per tile

template<class T>
struct tile_shape
{
  static constexpr int V = 16 / (int)sizeof(T); // values per 128-bit vector
  static constexpr int TE = kNT * kR * V;       // values per tile
};

// One array (or a block-aligned slice of one): pointers are to the slice's
// first exponent and first block, so slices of one buffer can run on
// different streams.
struct Job
{
  const void* values_in; // compress: T input
  void* values_out;      // decompress: T output
  std::uint8_t* exps;    // exponent of block 0 of this slice
  std::uint8_t* words;   // words of block 0 of this slice
  std::uint64_t n;       // values in this slice
  std::uint64_t tiles;   // tile kernels: ceil(n / TE)
  std::uint32_t block_bytes;
  std::int32_t bits, E, W;
  std::int32_t log2E;
  std::uint32_t tile_blocks; // TE / E
  std::uint32_t m_bb;        // ceil(2^32 / block_bytes)
  std::uint32_t m_bits;      // ceil(2^32 / bits)
};

// ---------------------------------------------------------------- word I/O

__device__ __forceinline__ void store_word(std::uint8_t* p, std::uint64_t v, int W)
{
  switch (W) {
    case 8: *p = (std::uint8_t)v; break;
    case 16: *reinterpret_cast<std::uint16_t*>(p) = (std::uint16_t)v; break;
    case 32: *reinterpret_cast<std::uint32_t*>(p) = (std::uint32_t)v; break;
    default: *reinterpret_cast<std::uint64_t*>(p) = v; break;
  }
}

__device__ __forceinline__ std::uint64_t load_word(const std::uint8_t* p, int W)
{
  switch (W) {
    case 8: return *p;
    case 16: return *reinterpret_cast<const std::uint16_t*>(p);
    case 32: return *reinterpret_cast<const std::uint32_t*>(p);
    default: return *reinterpret_cast<const std::uint64_t*>(p);
  }
}

// Signed W-bit exponent, sign-extended (exp_type, frsz2.hpp:510).
__device__ __forceinline__ std::int64_t load_exp(const std::uint8_t* p, int W)
{
  switch (W) {
    case 8: return *reinterpret_cast<const std::int8_t*>(p);
    case 16: return *reinterpret_cast<const std::int16_t*>(p);
    case 32: return *reinterpret_cast<const std::int32_t*>(p);
    default: return *reinterpret_cast<const std::int64_t*>(p);
  }
}

template<class T>
__device__ __forceinline__ typename fp<T>::U load_bits(const T* p)
{
  return to_bits<T>(*p);
}

// Block exponent from the block's max exponent field: exponent() of the max
// |x| (frsz2.hpp:1125), stored as exp_type (frsz2.hpp:1128) and passed to
// floating_to_fixed as std::int16_t (frsz2.hpp:354).
template<class T>
__device__ __forceinline__ std::int64_t block_exponent(std::uint32_t field_max, int W)
{
  return wrap_signed(exponent_of_field<T>((int)field_max), W);
}

// ---------------------------------------------------------------- keys

// Block-max key of a value: the magnitude bits that decide the exponent
// field (all of |x| for fp32, the high word of |x| for fp64).  A key at or
// above KEY_SPECIAL means the block holds +-Inf or NaN.
template<class T>
struct key_of;
template<>
struct key_of<float>
{
  static constexpr std::uint32_t SPECIAL = 0x7F800000u;
  static constexpr int FSHIFT = 23;
  __device__ static std::uint32_t raw(std::uint32_t u) { return u & 0x7FFFFFFFu; }
  __device__ static std::uint32_t clean(std::uint32_t u)
  {
    const std::uint32_t a = u & 0x7FFFFFFFu;
    return a > 0x7F800000u ? 0u : a;
  }
};
template<>
struct key_of<double>
{
  static constexpr std::uint32_t SPECIAL = 0x7FF00000u;
  static constexpr int FSHIFT = 20;
  __device__ static std::uint32_t raw(std::uint64_t u) { return (std::uint32_t)(u >> 32) & 0x7FFFFFFFu; }
  __device__ static std::uint32_t clean(std::uint64_t u)
  {
    const std::uint64_t a = u & 0x7FFFFFFFFFFFFFFFull;
    return a > 0x7FF0000000000000ull ? 0u : (std::uint32_t)(a >> 32);
  }
};

// Exponent range in which the float-arithmetic formulas are exact.
template<class T>
__device__ __forceinline__ bool plain_exponent(std::int64_t be)
{
  if constexpr (sizeof(T) == 4)
    return be >= -95 && be <= 127;
  else
    return be >= -959 && be <= 1023;
}

template<class T>
__device__ __forceinline__ T pow2(int e) // 2^e, e within the normal range
{
  if constexpr (sizeof(T) == 4)
    return __uint_as_float((std::uint32_t)(e + 127) << 23);
  else
    return __longlong_as_double((long long)(e + 1023) << 52);
}

// trunc(|x| * scale) with the sign at bit `bits` - 1, for a runtime width
// (the plain-range arithmetic of encode_plain in frsz2_fast.cuh).
template<class T>
__device__ __forceinline__ std::uint64_t encode_plain_rt(typename fp<T>::U u, T scale, int bits)
{
  const T x = from_bits<T>(u);
  const std::uint64_t s = (std::uint64_t)(u >> (fp<T>::UBITS - 1)) << (bits - 1);
  if constexpr (sizeof(T) == 4)
    return (std::uint64_t)__float2uint_rz(fabsf(x) * scale) | s;
  else
    return (std::uint64_t)__double2ull_rz(fabs(x) * scale) | s;
}

// ======================================================================
// generic kernels: one warp per exponent block
// ======================================================================

template<class T>
__global__ void __launch_bounds__(kNT) k_compress_generic(Job j)
{
  using U = typename fp<T>::U;
  const T* __restrict__ x = static_cast<const T*>(j.values_in);
  const int lane = threadIdx.x & 31;
  const std::uint64_t warp = ((std::uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const std::uint64_t nwarps = ((std::uint64_t)gridDim.x * blockDim.x) >> 5;
  const std::uint64_t nb = (j.n + (std::uint64_t)j.E - 1) / (std::uint64_t)j.E;
  const int bits = j.bits, W = j.W, E = j.E;

  for (std::uint64_t b = warp; b < nb; b += nwarps) {
    const std::uint64_t base = b * (std::uint64_t)E;
    const int cnt = (int)((j.n - base) < (std::uint64_t)E ? (j.n - base) : (std::uint64_t)E);
    std::uint32_t fmax = 0, kraw = 0;
    for (int k = lane; k < cnt; k += 32) {
      const U u = load_bits(x + base + k);
      const std::uint32_t f = max_field<T>(u);
      fmax = f > fmax ? f : fmax;
      kraw = max(kraw, key_of<T>::raw(u));
    }
    fmax = __reduce_max_sync(0xFFFFFFFFu, fmax);
    kraw = __reduce_max_sync(0xFFFFFFFFu, kraw);
    const std::int64_t ex = exponent_of_field<T>((int)fmax);
    const std::int64_t be = block_exponent<T>(fmax, W);
    const int be16 = (std::int16_t)be;
    if (lane == 0) store_word(j.exps + b * (std::uint64_t)(W / 8), (std::uint64_t)be, W);
    // the float arithmetic where it is exact (no Inf / NaN, no exponent wrap,
    // plain range), else the integer restatement
    const bool plain = kraw < key_of<T>::SPECIAL && be == ex && plain_exponent<T>(be);
    const T scale = pow2<T>(plain ? bits - 2 - (int)be : 0);
    auto code = [&](int k) -> std::uint64_t {
      const U u = load_bits(x + base + k);
      return plain ? encode_plain_rt<T>(u, scale, bits) : (std::uint64_t)to_code<T>(u, be16, bits);
    };

    // word w holds stream bits [w*W, w*W + W); only the words the reference
    // writes for `cnt` values are stored
    const int nw = (int)(((std::int64_t)cnt * bits + W - 1) / W);
    std::uint8_t* wbase = j.words + b * (std::uint64_t)j.block_bytes;
    for (int w = lane; w < nw; w += 32) {
      const std::int64_t pos = (std::int64_t)w * W;
      int k = (int)(pos / bits);
      const int off = (int)(pos - (std::int64_t)k * bits);
      std::uint64_t acc = code(k) >> off;
      int have = bits - off;
      for (++k; have < W && k < cnt; ++k) {
        acc |= code(k) << have;
        have += bits;
      }
      store_word(wbase + (std::uint64_t)w * (W / 8), acc, W);
    }
  }
}

template<class T>
__global__ void __launch_bounds__(kNT) k_decompress_generic(Job j)
{
  using U = typename fp<T>::U;
  T* __restrict__ y = static_cast<T*>(j.values_out);
  const int lane = threadIdx.x & 31;
  const std::uint64_t warp = ((std::uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const std::uint64_t nwarps = ((std::uint64_t)gridDim.x * blockDim.x) >> 5;
  const std::uint64_t nb = (j.n + (std::uint64_t)j.E - 1) / (std::uint64_t)j.E;
  const int bits = j.bits, W = j.W, E = j.E;
  const std::uint64_t wmask = W == 64 ? ~0ull : ((1ull << W) - 1);

  for (std::uint64_t b = warp; b < nb; b += nwarps) {
    const std::uint64_t base = b * (std::uint64_t)E;
    const int cnt = (int)((j.n - base) < (std::uint64_t)E ? (j.n - base) : (std::uint64_t)E);
    const std::int64_t be = load_exp(j.exps + b * (std::uint64_t)(W / 8), W);
    const std::uint8_t* wbase = j.words + b * (std::uint64_t)j.block_bytes;
    for (int k = lane; k < cnt; k += 32) {
      // retrieve_shift_value (frsz2.hpp:589-603)
      const std::int64_t p = (std::int64_t)k * bits;
      const std::int64_t w = p / W;
      const int o = (int)(p - w * W);
      std::uint64_t res = load_word(wbase + w * (W / 8), W);
      if (W != bits) {
        res >>= o;
        if (o + bits > W) res |= load_word(wbase + (w + 1) * (W / 8), W) << (W - o);
        res &= wmask;
      }
      const U code = (U)(res & (bits == 64 ? ~0ull : ((1ull << bits) - 1)));
      y[base + k] = from_code<T>(code, be, bits);
    }
  }
}

// ======================================================================
// tile kernels
// ======================================================================

// 32-bit chunk c of the tile's packed stream (bytes 4c .. 4c+3 after the
// tile's first block): the OR of every code overlapping it, with the block's
// trailing pad bits zero (the reference's last word holds only value bits).
template<class CV>
__device__ __forceinline__ std::uint32_t build_chunk(const CV* __restrict__ s_cv, std::uint32_t c, const Job& j)
{
  const std::uint32_t byte = c * 4u;
  const std::uint32_t bb = __umulhi(byte, j.m_bb); // byte / block_bytes
  const std::uint32_t pb = (byte - bb * j.block_bytes) * 8u;
  const std::uint32_t k0 = __umulhi(pb, j.m_bits); // pb / bits
  if (k0 >= (std::uint32_t)j.E) return 0u;
  const int off = (int)(pb - k0 * (std::uint32_t)j.bits);
  const CV* cb = s_cv + bb * (std::uint32_t)j.E;
  std::uint64_t acc = (std::uint64_t)cb[k0] >> off;
  int have = j.bits - off;
  for (std::uint32_t k = k0 + 1; have < 32 && k < (std::uint32_t)j.E; ++k) {
    acc |= (std::uint64_t)cb[k] << have;
    have += j.bits;
  }
  return (std::uint32_t)acc;
}

template<class T>
__device__ __forceinline__ void load_vec(const T* p, typename fp<T>::U (&u)[16 / sizeof(T)])
{
  const uint4 q = __ldcs(reinterpret_cast<const uint4*>(p));
  if constexpr (sizeof(T) == 4) {
    u[0] = q.x;
    u[1] = q.y;
    u[2] = q.z;
    u[3] = q.w;
  } else {
    u[0] = ((std::uint64_t)q.y << 32) | q.x;
    u[1] = ((std::uint64_t)q.w << 32) | q.z;
  }
}

template<class T, class CV>
__device__ __forceinline__ void compress_tile(const Job& j, std::uint64_t tile, unsigned char* smem)
{
  using U = typename fp<T>::U;
  constexpr int V = tile_shape<T>::V;
  constexpr int TE = tile_shape<T>::TE;
  CV* s_cv = reinterpret_cast<CV*>(smem);
  std::uint32_t* s_wmax = reinterpret_cast<std::uint32_t*>(smem + TE * sizeof(CV));
  const T* __restrict__ x = static_cast<const T*>(j.values_in);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int E = j.E, bits = j.bits, W = j.W;
  const int TB = (int)j.tile_blocks;
  const int G = E / V; // vectors per exponent block

  const std::uint64_t e0 = tile * (std::uint64_t)TE;
  const std::uint64_t rem64 = j.n - e0;
  const bool full = rem64 >= (std::uint64_t)TE;
  const int rem = full ? TE : (int)rem64;
  const int nbt = full ? TB : ((rem + E - 1) >> j.log2E);
  const std::uint64_t b0 = tile * (std::uint64_t)TB;

  U u[kR][V];
#pragma unroll
  for (int r = 0; r < kR; ++r) {
    const int idx = (r * kNT + tid) * V;
    if (full || idx + V <= rem) {
      load_vec<T>(x + e0 + idx, u[r]);
    } else {
#pragma unroll
      for (int i = 0; i < V; ++i) u[r][i] = (idx + i < rem) ? load_bits(x + e0 + idx + i) : U(0);
    }
  }

  std::uint32_t f[kR];
#pragma unroll
  for (int r = 0; r < kR; ++r) {
    std::uint32_t m = max_field<T>(u[r][0]);
#pragma unroll
    for (int i = 1; i < V; ++i) {
      const std::uint32_t g = max_field<T>(u[r][i]);
      m = g > m ? g : m;
    }
    f[r] = m;
  }
  if (G <= 32) {
    for (int s = 1; s < G; s <<= 1) {
#pragma unroll
      for (int r = 0; r < kR; ++r) {
        const std::uint32_t g = __shfl_xor_sync(0xFFFFFFFFu, f[r], s);
        f[r] = g > f[r] ? g : f[r];
      }
    }
  } else {
#pragma unroll
    for (int r = 0; r < kR; ++r) {
      const std::uint32_t g = __reduce_max_sync(0xFFFFFFFFu, f[r]);
      if (lane == 0) s_wmax[r * (kNT / 32) + warp] = g;
    }
    __syncthreads();
    const int gw = G / 32; // warp-chunks per exponent block
#pragma unroll
    for (int r = 0; r < kR; ++r) {
      const int v = r * kNT + tid;
      const int wc0 = (v / G) * gw;
      std::uint32_t m = 0;
      for (int q = 0; q < gw; ++q) {
        const std::uint32_t g = s_wmax[wc0 + q];
        m = g > m ? g : m;
      }
      f[r] = m;
    }
  }

#pragma unroll
  for (int r = 0; r < kR; ++r) {
    const int idx = (r * kNT + tid) * V;
    const std::int64_t be = block_exponent<T>(f[r], W);
    const int be16 = (std::int16_t)be;
    CV c[V];
#pragma unroll
    for (int i = 0; i < V; ++i) c[i] = (CV)to_code<T>(u[r][i], be16, bits);
    if constexpr (sizeof(T) == 4) { // 4 x u32 codes
      *reinterpret_cast<uint4*>(s_cv + idx) = make_uint4((std::uint32_t)c[0], (std::uint32_t)c[1],
                                                         (std::uint32_t)c[2], (std::uint32_t)c[3]);
    } else if constexpr (sizeof(CV) == 4) { // 2 x u32 codes
      *reinterpret_cast<uint2*>(s_cv + idx) = make_uint2((std::uint32_t)c[0], (std::uint32_t)c[1]);
    } else { // 2 x u64 codes
      *reinterpret_cast<uint4*>(s_cv + idx) =
        make_uint4((std::uint32_t)c[0], (std::uint32_t)((std::uint64_t)c[0] >> 32), (std::uint32_t)c[1],
                   (std::uint32_t)((std::uint64_t)c[1] >> 32));
    }
    if ((idx & (E - 1)) == 0) {
      const int bl = idx >> j.log2E;
      if (bl < nbt) store_word(j.exps + (b0 + (std::uint64_t)bl) * (std::uint64_t)(W / 8), (std::uint64_t)be, W);
    }
  }
  __syncthreads();

  const int last_cnt = rem - (nbt - 1) * E;
  const std::uint32_t wb = full ? (std::uint32_t)TB * j.block_bytes
                                : (std::uint32_t)(nbt - 1) * j.block_bytes + written_block_bytes(last_cnt, bits, W);
  std::uint8_t* __restrict__ dst = j.words + b0 * (std::uint64_t)j.block_bytes;
  for (std::uint32_t c = tid; c * 4u < wb; c += kNT) {
    const std::uint32_t ch = build_chunk<CV>(s_cv, c, j);
    if (c * 4u + 4u <= wb) {
      __stcs(reinterpret_cast<unsigned int*>(dst + c * 4u), ch);
    } else {
      for (std::uint32_t q = 0; c * 4u + q < wb; ++q) dst[c * 4u + q] = (std::uint8_t)(ch >> (8 * q));
    }
  }
  __syncthreads(); // shared memory is reused by the next tile
}

template<class T, class CV>
__global__ void __launch_bounds__(kNT) k_compress_tile(Job j)
{
  extern __shared__ __align__(16) unsigned char smem[];
  for (std::uint64_t tile = blockIdx.x; tile < j.tiles; tile += gridDim.x) compress_tile<T, CV>(j, tile, smem);
}

template<class T>
__device__ __forceinline__ void store_vec(T* p, const T (&y)[16 / sizeof(T)])
{
  if constexpr (sizeof(T) == 4) {
    __stcs(reinterpret_cast<float4*>(p), make_float4(y[0], y[1], y[2], y[3]));
  } else {
    __stcs(reinterpret_cast<double2*>(p), make_double2(y[0], y[1]));
  }
}

// Shared memory of the decompress tile: packed words then block exponents.
template<class T>
__host__ __device__ constexpr std::uint32_t decompress_tile_exp_offset(std::uint32_t tile_bytes)
{
  return ((tile_bytes + 16u + 15u) / 16u) * 16u;
}

template<class T, class CV>
__device__ __forceinline__ void decompress_tile(const Job& j, std::uint64_t tile, unsigned char* smem)
{
  using U = typename fp<T>::U;
  constexpr int V = tile_shape<T>::V;
  constexpr int TE = tile_shape<T>::TE;
  T* __restrict__ y = static_cast<T*>(j.values_out);
  const int tid = threadIdx.x;
  const int E = j.E, bits = j.bits, W = j.W;
  const int TB = (int)j.tile_blocks;

  const std::uint64_t e0 = tile * (std::uint64_t)TE;
  const std::uint64_t rem64 = j.n - e0;
  const bool full = rem64 >= (std::uint64_t)TE;
  const int rem = full ? TE : (int)rem64;
  const int nbt = full ? TB : ((rem + E - 1) >> j.log2E);
  const std::uint64_t b0 = tile * (std::uint64_t)TB;

  const std::uint32_t tile_bytes = (std::uint32_t)TB * j.block_bytes;
  std::uint32_t* s_w = reinterpret_cast<std::uint32_t*>(smem);
  std::int64_t* s_exp = reinterpret_cast<std::int64_t*>(smem + decompress_tile_exp_offset<T>(tile_bytes));

  // stage the packed words of the tile's nbt blocks (whole blocks are always
  // inside the buffer) plus four zero words for the read-ahead window
  const std::uint32_t nbytes = (std::uint32_t)nbt * j.block_bytes;
  const std::uint8_t* __restrict__ src = j.words + b0 * (std::uint64_t)j.block_bytes;
  for (std::uint32_t g = tid; g * 16u < nbytes; g += kNT) {
    if (g * 16u + 16u <= nbytes) {
      *reinterpret_cast<uint4*>(s_w + 4 * g) = __ldcs(reinterpret_cast<const uint4*>(src + 16u * g));
    } else {
      for (std::uint32_t q = 0; g * 16u + 4u * q < nbytes; ++q)
        s_w[4 * g + q] = *reinterpret_cast<const std::uint32_t*>(src + 16u * g + 4u * q);
    }
  }
  if (tid < 4) s_w[nbytes / 4 + tid] = 0u;
  for (int bl = tid; bl < nbt; bl += kNT) s_exp[bl] = load_exp(j.exps + (b0 + (std::uint64_t)bl) * (W / 8), W);
  __syncthreads();

  const std::uint32_t block_bits = j.block_bytes * 8u;
  const CV cmask = bits == (int)(8 * sizeof(CV)) ? ~CV(0) : (CV)((CV(1) << bits) - 1);
#pragma unroll
  for (int r = 0; r < kR; ++r) {
    const int idx = (r * kNT + tid) * V;
    if (!full && idx >= rem) continue;
    const int bl = idx >> j.log2E;
    const int k = idx & (E - 1);
    const std::int64_t be = s_exp[bl];
    std::uint32_t p = (std::uint32_t)bl * block_bits + (std::uint32_t)(k * bits);
    std::uint32_t w = p >> 5;
    int o = (int)(p & 31u);
    std::uint32_t lo = s_w[w], hi = s_w[w + 1];
    std::uint32_t hi2 = 0;
    if constexpr (sizeof(CV) == 8) hi2 = s_w[w + 2];
    T out[V];
#pragma unroll
    for (int i = 0; i < V; ++i) {
      CV code;
      if constexpr (sizeof(CV) == 4) {
        code = __funnelshift_r(lo, hi, o) & cmask;
      } else {
        const std::uint32_t c0 = __funnelshift_r(lo, hi, o), c1 = __funnelshift_r(hi, hi2, o);
        code = (((std::uint64_t)c1 << 32) | c0) & cmask;
      }
      out[i] = from_code<T>((U)code, be, bits);
      if (i + 1 < V) {
        o += bits;
        while (o >= 32) { // at most twice (bits <= 64)
          o -= 32;
          ++w;
          lo = hi;
          if constexpr (sizeof(CV) == 8) {
            hi = hi2;
            hi2 = s_w[w + 2];
          } else {
            hi = s_w[w + 1];
          }
        }
      }
    }
    if (full || idx + V <= rem) {
      store_vec<T>(y + e0 + idx, out);
    } else {
      for (int i = 0; i < V && idx + i < rem; ++i) y[e0 + idx + i] = out[i];
    }
  }
  __syncthreads(); // shared memory is reused by the next tile
}

template<class T, class CV>
__global__ void __launch_bounds__(kNT) k_decompress_tile(Job j)
{
  extern __shared__ __align__(16) unsigned char smem[];
  for (std::uint64_t tile = blockIdx.x; tile < j.tiles; tile += gridDim.x) decompress_tile<T, CV>(j, tile, smem);
}

} // namespace frsz2b

namespace frsz2b {

// Random access decode (decompress_cpu_element, frsz2.hpp:1199-1214): one
// thread per requested index; indices >= n decode nothing and write nothing.
template<class T>
__global__ void __launch_bounds__(kNT)
  k_decompress_elements(Job j, const std::uint64_t* __restrict__ idx, std::uint64_t count, T* __restrict__ out)
{
  using U = typename fp<T>::U;
  const int bits = j.bits, W = j.W;
  const std::uint64_t wmask = W == 64 ? ~0ull : ((1ull << W) - 1);
  for (std::uint64_t t = (std::uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < count;
       t += (std::uint64_t)gridDim.x * blockDim.x) {
    const std::uint64_t g = idx[t];
    if (g >= j.n) continue;
    const std::uint64_t b = g / (std::uint64_t)j.E;
    const int k = (int)(g - b * (std::uint64_t)j.E);
    const std::int64_t be = load_exp(j.exps + b * (std::uint64_t)(W / 8), W);
    const std::uint8_t* wbase = j.words + b * (std::uint64_t)j.block_bytes;
    const std::int64_t p = (std::int64_t)k * bits;
    const std::int64_t w = p / W;
    const int o = (int)(p - w * W);
    std::uint64_t res = load_word(wbase + w * (W / 8), W);
    if (W != bits) {
      res >>= o;
      if (o + bits > W) res |= load_word(wbase + (w + 1) * (W / 8), W) << (W - o);
      res &= wmask;
    }
    out[t] = from_code<T>((U)res, be, bits);
  }
}

} // namespace frsz2b
