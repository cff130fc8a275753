// frsz2_chunked.cuh -- runtime-width decompress kernel for exponent blocks of
// 17 to kChunkMaxEDecompress values that the compile-time-width kernels do not
// take (block sizes that are not powers of two, pointers off the 32-byte
// layout); smaller blocks go to the blockwise kernels.
//
// A CTA owns a chunk of whole exponent blocks (at most kChunkValues values):
// the chunk's block image comes into shared memory with 16-byte loads, every
// thread decodes values at their stream positions and writes them with
// coalesced stores.  Blocks in the "plain" exponent domain use the
// float-scaling arithmetic of the fast kernels; the others the exact integer
// restatement, so results are bit-exact for every input.  chunk_copy is also
// the blockwise kernels' copy-out.
#pragma once

#include "frsz2_fast.cuh"

namespace frsz2b {

constexpr int kChunkValues = 2048;             // values per chunk at most
// Largest block size the chunked kernel takes (above it the warp-per-block
// kernel was faster on B200: E 255 0.38 vs 0.43 of HBM).
constexpr int kChunkMaxEDecompress = 128;
constexpr int kChunkVPT = kChunkValues / kNT;  // values per thread
constexpr int kChunkBytes = kChunkValues * 16; // block image: < values * (bits + W) / 8

// Blocks per chunk for block size E (E <= kChunkValues).
__host__ __device__ inline int chunk_blocks(int E) { return kChunkValues / E; }

// Codes are C = uint32 for bits <= 32, uint64 above (one kernel instance
// each), so the common widths do 32-bit shifts and masks.

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
