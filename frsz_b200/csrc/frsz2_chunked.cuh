// frsz2_chunked.cuh -- runtime-width kernels for small exponent blocks the
// compile-time-width kernels do not take: block sizes that are not powers of
// two (such as the reference tests' 5), padded blocks of aligned-segment
// widths, pointers off the 32-byte layout (compress up to kChunkMaxECompress
// values per block, decompress up to kChunkMaxEDecompress).
//
// A CTA owns a chunk of whole exponent blocks (at most kChunkValues values).
// Compress: values are read with coalesced loads into registers; their
// exponent fields go to shared memory, one thread (E <= 32) or one warp
// (larger E) takes each block's maximum; every thread then encodes its values
// and ORs each code into a zeroed shared-memory image of the chunk's blocks at
// its stream position; the image and the exponents leave with coalesced
// stores.  Decompress runs the other way.  Blocks in the "plain" exponent
// domain use the float-scaling arithmetic of the fast kernels; the others the
// exact integer restatement, so results are bit-exact for every input.
#pragma once

#include "frsz2_fast.cuh"

namespace frsz2b {

constexpr int kChunkValues = 2048;             // values per chunk at most
// Largest block sizes the chunked kernels take (above them the warp-per-block
// kernels were faster on B200: compress E 48 0.13 vs 0.14 of HBM, E 255 0.21
// vs 0.32; decompress E 255 0.38 vs 0.43).
constexpr int kChunkMaxECompress = 16;
constexpr int kChunkMaxEDecompress = 128;
constexpr int kChunkVPT = kChunkValues / kNT;  // values per thread
constexpr int kChunkBytes = kChunkValues * 16; // block image: < values * (bits + W) / 8

// Blocks per chunk for block size E (E <= kChunkValues).
__host__ __device__ inline int chunk_blocks(int E) { return kChunkValues / E; }

// Per-block record in shared memory: exponent (low 16 bits, signed) and
// whether the block is in the plain domain (bit 16).
__device__ __forceinline__ std::uint32_t blk_record(std::int64_t be, bool plain)
{
  return ((std::uint32_t)be & 0xFFFFu) | (plain ? 0x10000u : 0u);
}
__device__ __forceinline__ std::int64_t blk_exp(std::uint32_t r) { return (std::int16_t)(r & 0xFFFFu); }
__device__ __forceinline__ bool blk_plain(std::uint32_t r) { return (r >> 16) != 0; }

// Codes are C = uint32 for bits <= 32, uint64 above (one kernel instance
// each), so the common widths do 32-bit shifts and masks.

// trunc(|x| * scale) with the sign at bit `bits` - 1 (plain domain).
template<class T, class C>
__device__ __forceinline__ C encode_plain_rt(typename fp<T>::U u, T scale, int bits)
{
  const T x = from_bits<T>(u);
  const C s = (C)(u >> (fp<T>::UBITS - 1)) << (bits - 1);
  if constexpr (sizeof(T) == 4)
    return (C)__float2uint_rz(fabsf(x) * scale) | s;
  else if constexpr (sizeof(C) == 4)
    return (C)__double2uint_rz(fabs(x) * scale) | s;
  else
    return (C)__double2ull_rz(fabs(x) * scale) | s;
}

// Value of a code in the plain domain: rz(mag) * 2^(be-bits+2), a zero
// magnitude giving 2^(be-31) (zero_bits), the code's sign bit or-ed in.
template<class T, class C>
__device__ __forceinline__ typename fp<T>::U decode_plain_rt(C code, int bits, T inv, typename fp<T>::U zero_bits)
{
  using U = typename fp<T>::U;
  const C mag = code & ((C(1) << (bits - 1)) - C(1));
  U r;
  if constexpr (sizeof(T) == 4)
    r = __float_as_uint(__uint2float_rz((std::uint32_t)mag) * inv);
  else if constexpr (sizeof(C) == 4)
    r = (U)__double_as_longlong(__uint2double_rn(mag) * inv);
  else
    r = (U)__double_as_longlong(__ull2double_rz(mag) * inv);
  r = mag == 0 ? zero_bits : r;
  return r | ((U)(code >> (bits - 1)) << (fp<T>::UBITS - 1));
}

// Copy `bytes` bytes between global memory at g and shared memory at
// s + (g mod 16) (s 16-byte aligned), so both sides share their 16-byte
// boundaries: single bytes up to g's first boundary and after its last one,
// 16-byte accesses between.  All threads of the CTA take part.
template<bool TO_GLOBAL>
__device__ __forceinline__ void chunk_copy(std::uint8_t* g, std::uint8_t* s, std::uint32_t bytes)
{
  const std::uint32_t h = (std::uint32_t)(reinterpret_cast<std::uintptr_t>(g) & 15u);
  const std::uint32_t head = h == 0 ? 0u : min(16u - h, bytes);
  const std::uint32_t n16 = (bytes - head) >> 4;
  const std::uint32_t tail0 = head + (n16 << 4);
  std::uint8_t* sb = s + h;
  for (std::uint32_t i = threadIdx.x; i < head; i += blockDim.x) {
    if (TO_GLOBAL)
      g[i] = sb[i];
    else
      sb[i] = __ldg(g + i);
  }
  uint4* g16 = reinterpret_cast<uint4*>(g + head);
  uint4* s16 = reinterpret_cast<uint4*>(sb + head);
  for (std::uint32_t i = threadIdx.x; i < n16; i += blockDim.x) {
    if (TO_GLOBAL)
      __stcs(g16 + i, s16[i]);
    else
      s16[i] = __ldg(g16 + i);
  }
  for (std::uint32_t i = tail0 + threadIdx.x; i < bytes; i += blockDim.x) {
    if (TO_GLOBAL)
      g[i] = sb[i];
    else
      sb[i] = __ldg(g + i);
  }
}

template<class T, class C>
__global__ void __launch_bounds__(kNT) k_compress_chunked(Job j)
{
  using U = typename fp<T>::U;
  __shared__ std::uint16_t s_key[kChunkValues];     // exponent field | Inf/NaN flag (bit 15)
  __shared__ std::uint32_t s_blk[kChunkValues];     // per block: blk_record
  __shared__ __align__(16) std::uint32_t s_img[kChunkBytes / 4 + 4];
  const T* __restrict__ x = static_cast<const T*>(j.values_in);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int E = j.E, bits = j.bits, W = j.W, EB = W / 8;
  const std::uint32_t BB = j.block_bytes;
  const int nbc = chunk_blocks(E);
  const std::uint64_t nb = (j.n + (std::uint64_t)E - 1) / (std::uint64_t)E;
  const std::uint64_t nchunks = (nb + nbc - 1) / nbc;
  // this thread's first value's block and offset within it; later values
  // are kNT further on
  const int step_b = kNT / E, step_o = kNT % E;

  for (std::uint64_t ch = blockIdx.x; ch < nchunks; ch += gridDim.x) {
    const std::uint64_t b0 = ch * (std::uint64_t)nbc;
    const std::uint64_t v0 = b0 * (std::uint64_t)E;
    const int nv = (int)(j.n - v0 < (std::uint64_t)(nbc * E) ? j.n - v0 : (std::uint64_t)(nbc * E));
    const int nbk = (nv + E - 1) / E;
    std::uint8_t* gout = j.words + b0 * (std::uint64_t)BB;
    const std::uint32_t hb = (std::uint32_t)(reinterpret_cast<std::uintptr_t>(gout) & 15u); // image offset
    const std::uint32_t img_words = (hb + nbk * BB + 3) / 4;

    const T* __restrict__ xc = x + v0;
    U u[kChunkVPT];
#pragma unroll
    for (int k = 0; k < kChunkVPT; ++k) {
      const int v = tid + k * kNT;
      u[k] = v < nv ? load_bits(xc + v) : U(0);
      if (v < nv) {
        const U a = u[k] & fp<T>::ABS;
        s_key[v] = (std::uint16_t)(max_field<T>(u[k]) | (a >= fp<T>::INF ? 0x8000u : 0u));
      }
    }
    for (std::uint32_t i = tid; i < img_words; i += kNT) s_img[i] = 0u;
    __syncthreads();

    // block exponents: the exponent field of the largest non-NaN magnitude
    // (std::max semantics); plain if no Inf/NaN, no exponent wrap and the
    // float arithmetic is exact there
    auto finish_block = [&](int b, std::uint32_t fmax, std::uint32_t special) {
      const std::int64_t ex = exponent_of_field<T>((int)fmax);
      const std::int64_t be = wrap_signed(ex, W);
      const bool plain = !special && be == ex && plain_exponent<T>(be);
      s_blk[b] = blk_record(be, plain);
    };
    if (E <= 32) {
      for (int b = tid; b < nbk; b += kNT) {
        const int lo = b * E, hi = min(lo + E, nv);
        std::uint32_t fm = 0, sp = 0;
        for (int v = lo; v < hi; ++v) {
          const std::uint32_t kk = s_key[v];
          fm = max(fm, kk & 0x7FFFu);
          sp |= kk & 0x8000u;
        }
        finish_block(b, fm, sp);
      }
    } else {
      for (int b = warp; b < nbk; b += kNT / 32) {
        const int lo = b * E, hi = min(lo + E, nv);
        std::uint32_t fm = 0, sp = 0;
        for (int v = lo + lane; v < hi; v += 32) {
          const std::uint32_t kk = s_key[v];
          fm = max(fm, kk & 0x7FFFu);
          sp |= kk & 0x8000u;
        }
        fm = __reduce_max_sync(0xFFFFFFFFu, fm);
        sp = __reduce_or_sync(0xFFFFFFFFu, sp);
        if (lane == 0) finish_block(b, fm, sp);
      }
    }
    __syncthreads();

    // codes into the block image
    const std::uint32_t bit0 = hb * 8u, bb_bits = BB * 8u;
    int b = tid / E, o = tid - (tid / E) * E;
#pragma unroll
    for (int k = 0; k < kChunkVPT; ++k) {
      const int v = tid + k * kNT;
      if (v < nv) {
        const std::uint32_t r = s_blk[b];
        const int be = (int)blk_exp(r);
        C c;
        if (blk_plain(r))
          c = encode_plain_rt<T, C>(u[k], pow2<T>(bits - 2 - be), bits);
        else
          c = (C)to_code<T>(u[k], (std::int16_t)be, bits);
        const std::uint32_t pos = bit0 + (std::uint32_t)b * bb_bits + (std::uint32_t)(o * bits);
        const int q = (int)(pos & 31u);
        std::uint32_t* w = s_img + (pos >> 5);
        atomicOr(w, (std::uint32_t)(c << q));
        if (q + bits > 32) {
          if constexpr (sizeof(C) == 4) {
            atomicOr(w + 1, c >> (32 - q)); // q > 0 here
          } else {
            const std::uint64_t rest = c >> (32 - q);
            atomicOr(w + 1, (std::uint32_t)rest);
            if (q + bits > 64) atomicOr(w + 2, (std::uint32_t)(rest >> 32));
          }
        }
      }
      b += step_b;
      o += step_o;
      if (o >= E) {
        o -= E;
        ++b;
      }
    }
    __syncthreads();

    for (int bb = tid; bb < nbk; bb += kNT)
      store_word(j.exps + (b0 + (std::uint64_t)bb) * (std::uint64_t)EB, (std::uint64_t)blk_exp(s_blk[bb]), W);
    // the last block of the array: only the words its values reach
    const int last_cnt = nv - (nbk - 1) * E;
    const std::uint32_t out_bytes = (std::uint32_t)(nbk - 1) * BB + written_block_bytes(last_cnt, bits, W);
    chunk_copy<true>(gout, reinterpret_cast<std::uint8_t*>(s_img), out_bytes);
    __syncthreads(); // shared memory is reused by the next chunk
  }
}

template<class T, class C>
__global__ void __launch_bounds__(kNT) k_decompress_chunked(Job j)
{
  using U = typename fp<T>::U;
  __shared__ std::int32_t s_exp[kChunkValues];
  __shared__ __align__(16) std::uint32_t s_img[kChunkBytes / 4 + 8];
  T* __restrict__ y = static_cast<T*>(j.values_out);
  const int tid = threadIdx.x;
  const int E = j.E, bits = j.bits, W = j.W, EB = W / 8;
  const std::uint32_t BB = j.block_bytes;
  const int nbc = chunk_blocks(E);
  const std::uint64_t nb = (j.n + (std::uint64_t)E - 1) / (std::uint64_t)E;
  const std::uint64_t nchunks = (nb + nbc - 1) / nbc;
  const int step_b = kNT / E, step_o = kNT % E;
  const C cmask = bits == (int)(8 * sizeof(C)) ? ~C(0) : ((C(1) << bits) - C(1));

  for (std::uint64_t ch = blockIdx.x; ch < nchunks; ch += gridDim.x) {
    const std::uint64_t b0 = ch * (std::uint64_t)nbc;
    const std::uint64_t v0 = b0 * (std::uint64_t)E;
    const int nv = (int)(j.n - v0 < (std::uint64_t)(nbc * E) ? j.n - v0 : (std::uint64_t)(nbc * E));
    const int nbk = (nv + E - 1) / E;
    for (int bb = tid; bb < nbk; bb += kNT)
      s_exp[bb] = (std::int32_t)load_exp(j.exps + (b0 + (std::uint64_t)bb) * (std::uint64_t)EB, W);
    // whole blocks: the buffer holds every block in full
    const std::uint8_t* gin = j.words + b0 * (std::uint64_t)BB;
    const std::uint32_t hb = (std::uint32_t)(reinterpret_cast<std::uintptr_t>(gin) & 15u); // image offset
    chunk_copy<false>(const_cast<std::uint8_t*>(gin), reinterpret_cast<std::uint8_t*>(s_img), (std::uint32_t)nbk * BB);
    if (tid < 4) s_img[(hb + nbk * BB + 3) / 4 + tid] = 0u; // words past the image read by the last codes
    __syncthreads();

    const std::uint32_t bit0 = hb * 8u, bb_bits = BB * 8u;
    T* __restrict__ yc = y + v0;
    int b = tid / E, o = tid - (tid / E) * E;
#pragma unroll
    for (int k = 0; k < kChunkVPT; ++k) {
      const int v = tid + k * kNT;
      if (v < nv) {
        const std::uint32_t pos = bit0 + (std::uint32_t)b * bb_bits + (std::uint32_t)(o * bits);
        const int q = (int)(pos & 31u);
        const std::uint32_t* w = s_img + (pos >> 5);
        C c;
        if constexpr (sizeof(C) == 4) {
          c = __funnelshift_r(w[0], w[1], q); // w[1] may be a guard word
        } else {
          c = (std::uint64_t)w[0] >> q;
          if (q + bits > 32) {
            c |= (std::uint64_t)w[1] << (32 - q);
            if (q + bits > 64) c |= (std::uint64_t)w[2] << (64 - q);
          }
        }
        c &= cmask;
        const int be = s_exp[b];
        U r;
        if (plain_exponent<T>(be)) {
          const T inv = pow2<T>(be - bits + 2);
          const U zero_bits = sizeof(T) == 4 ? (U)((std::uint32_t)(be + 96) << 23) : (U)((std::uint64_t)(be + 992) << 52);
          r = decode_plain_rt<T, C>(c, bits, inv, zero_bits);
        } else {
          r = to_bits<T>(from_code<T>((U)c, be, bits));
        }
        yc[v] = from_bits<T>(r);
      }
      b += step_b;
      o += step_o;
      if (o >= E) {
        o -= E;
        ++b;
      }
    }
    __syncthreads();
  }
}

} // namespace frsz2b
