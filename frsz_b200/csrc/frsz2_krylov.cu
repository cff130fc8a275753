// frsz2_krylov.cu -- decompress fused into its consumer: dot products and
// axpy over a basis of FRSZ2-compressed fp64 vectors (the compressed Krylov
// basis use of the reference's random-access decode,
// include/frsz2.hpp:1096-1104).  Values are decoded in registers straight into
// the FMAs and never written back.
//
//   frsz2_basis_dot:  h[j] = sum_i V_j[i] * w[i]           j < m
//   frsz2_basis_axpy: y[i] = y[i] + sum_j c[j] * V_j[i]     (j in order 0..m-1)
//
// dot: CTA b owns a contiguous element range; it stages its slice of w in
// shared memory once and streams every basis vector's slice through it (the
// basis and w are each read once).  Per-warp partial sums per vector go to
// shared memory; each CTA writes its m partials to the caller's workspace and
// the last CTA to finish (a ticket counter in the workspace) adds them in CTA
// order, so the result does not depend on scheduling.
#include "frsz2_fast.cuh"
#include "frsz2_launch.hpp"

#include "../../include/frsz2_b200.h"

#include <algorithm>
#include <string>

namespace frsz2b {
namespace {

constexpr int kMaxBasis = FRSZ2_MAX_BASIS;
constexpr int kKT = 256;            // threads per CTA
constexpr int kSub = 3072;          // w values staged per step (24 KiB)
#ifndef FRSZ2_KRYLOV_JB
#define FRSZ2_KRYLOV_JB 4
#endif
#ifndef FRSZ2_KRYLOV_MIN_CTAS
#define FRSZ2_KRYLOV_MIN_CTAS 4
#endif
// Basis vectors whose loads are in flight together, per kernel and width.
// Measured on B200 (100 vectors of 2^22 values, 4 CTAs per SM): the dot is
// fastest with 4 at 32 bits (0.89 of HBM against 0.83 with 6) and with 6 at 16
// and 24 bits (0.48 against 0.46, 0.68 against 0.66); the axpy with 6 at 16, 24
// and 32 bits (0.66 against 0.61, 0.87 against 0.82, 1.03 against 1.02).  At
// 21 bits 6 spills registers and halves the speed; 21, 48 and 64 bits keep
// FRSZ2_KRYLOV_JB.
constexpr int kJB = FRSZ2_KRYLOV_JB;
__host__ __device__ constexpr int jb_dot(int bits) { return bits == 16 || bits == 24 ? 6 : kJB; }
__host__ __device__ constexpr int jb_axpy(int bits) { return bits == 16 || bits == 24 || bits == 32 ? 6 : kJB; }
constexpr int kMinCtas = FRSZ2_KRYLOV_MIN_CTAS; // resident CTAs per SM the register budget must allow

struct BasisParams
{
  const std::uint8_t* buf[kMaxBasis]; // compressed vectors
};

struct BasisGeo
{
  std::uint64_t n;
  std::uint64_t exp_bytes;
  int log2E;
};

#ifndef FRSZ2_KRYLOV_NOCVT
#define FRSZ2_KRYLOV_NOCVT 1
#endif

// Values of widths up to 32 bits without an integer-to-double conversion,
// exactly the values fast_decode_loaded gives.  With t = code << (32 - BITS)
// (sign at bit 31) and m = max(t << 1, 1), a value is m * 2^(be-31): for a
// nonzero magnitude m = mag * 2^(33-BITS), so m * 2^(be-31) =
// mag * 2^(be-BITS+2); for a zero magnitude m = 1 gives the decoder's
// 2^(be-31).  m * 2^(be-31) = D - 2^(be+21) exactly, where D has exponent
// be+21 and m in the low 32 bits of its mantissa (m < 2^32; the subtraction
// of two doubles within a factor of 2 is exact).  Needs be+1044 to be a
// normal exponent field and be in the plain range: be in [-959, 1002].
// The value's sign goes onto the other factor of the product (sign_onto).
template<int BITS>
__device__ __forceinline__ bool nocvt_block(std::int64_t be)
{
  return FRSZ2_KRYLOV_NOCVT && BITS <= 32 && be >= -959 && be <= 1002;
}

__device__ __forceinline__ double nocvt_magnitude(std::uint32_t t, int hi, double base)
{
  const std::uint32_t m = max(t << 1, 1u);
  return __hiloint2double(hi, (int)m) - base;
}

__device__ __forceinline__ double sign_onto(double x, std::uint32_t t)
{
  return __hiloint2double(__double2hiint(x) ^ (int)(t & 0x80000000u), __double2loint(x));
}

// acc + sum over the lane's values of v[k] * wv[k], FMAs in value order.
template<int BITS>
__device__ __forceinline__ double lane_dot(const lane_words<double, BITS>& lw,
                                           const double (&wv)[fast_cfg<double, BITS>::P], double acc)
{
  constexpr int P = fast_cfg<double, BITS>::P;
  if constexpr (BITS <= 32) {
    const std::int64_t be = lw.be;
    if (nocvt_block<BITS>(be)) {
      std::uint32_t c[P];
      fast_codes_loaded<double, BITS>(lw, c);
      const int hi = (int)((std::uint32_t)(be + 1044) << 20);
      const double base = __hiloint2double(hi, 0);
#pragma unroll
      for (int k = 0; k < P; ++k) {
        const std::uint32_t t = c[k] << (32 - BITS);
        acc = fma(nocvt_magnitude(t, hi, base), sign_onto(wv[k], t), acc);
      }
      return acc;
    }
  }
  double v[P];
  fast_decode_loaded<double, BITS>(lw, v);
#pragma unroll
  for (int k = 0; k < P; ++k) acc = fma(v[k], wv[k], acc);
  return acc;
}

// acc[k] + cj * v[k] for the lane's values.
template<int BITS>
__device__ __forceinline__ void lane_axpy(const lane_words<double, BITS>& lw, double cj,
                                          double (&acc)[fast_cfg<double, BITS>::P])
{
  constexpr int P = fast_cfg<double, BITS>::P;
  if constexpr (BITS <= 32) {
    const std::int64_t be = lw.be;
    if (nocvt_block<BITS>(be)) {
      std::uint32_t c[P];
      fast_codes_loaded<double, BITS>(lw, c);
      const int hi = (int)((std::uint32_t)(be + 1044) << 20);
      const double base = __hiloint2double(hi, 0);
#pragma unroll
      for (int k = 0; k < P; ++k) {
        const std::uint32_t t = c[k] << (32 - BITS);
        acc[k] = fma(sign_onto(cj, t), nocvt_magnitude(t, hi, base), acc[k]);
      }
      return;
    }
  }
  double v[P];
  fast_decode_loaded<double, BITS>(lw, v);
#pragma unroll
  for (int k = 0; k < P; ++k) acc[k] = fma(cj, v[k], acc[k]);
}

template<int BITS>
__global__ void __launch_bounds__(kKT, kMinCtas)
  k_basis_dot(const __grid_constant__ BasisParams bp, int m, BasisGeo g, const double* __restrict__ w,
              std::uint64_t chunk, double* __restrict__ partials, unsigned int* __restrict__ ticket,
              double* __restrict__ h)
{
  constexpr int P = fast_cfg<double, BITS>::P;
  constexpr int JB = jb_dot(BITS);
  __shared__ double s_w[kSub];
  __shared__ double s_acc[kKT / 32][kMaxBasis];
  __shared__ bool s_last;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int j = lane; j < m; j += 32) s_acc[warp][j] = 0.0;

  const std::uint64_t c0 = (std::uint64_t)blockIdx.x * chunk;
  const std::uint64_t c1 = c0 + chunk < g.n ? c0 + chunk : g.n;
  for (std::uint64_t s0 = c0; s0 < c1; s0 += kSub) {
    const int len = (int)((c1 - s0) < (std::uint64_t)kSub ? (c1 - s0) : (std::uint64_t)kSub);
    __syncthreads(); // previous slice fully consumed
    for (int i = tid; i < len; i += kKT) s_w[i] = __ldg(w + s0 + i);
    __syncthreads();
    // JB vectors at a time: all their loads are issued before any decode
    for (int j0 = 0; j0 < m; j0 += JB) {
      double acc[JB];
#pragma unroll
      for (int jj = 0; jj < JB; ++jj) acc[jj] = 0.0;
      for (int i = tid * P; i < len; i += kKT * P) {
        lane_words<double, BITS> lw[JB];
#pragma unroll
        for (int jj = 0; jj < JB; ++jj)
          if (j0 + jj < m) {
            const std::uint8_t* buf = bp.buf[j0 + jj];
            fast_load_lane<double, BITS>(buf, buf + g.exp_bytes, g.log2E, s0 + (std::uint64_t)i, lw[jj]);
          }
        double wv[P];
#pragma unroll
        for (int k = 0; k < P; ++k) wv[k] = i + k < len ? s_w[i + k] : 0.0;
#pragma unroll
        for (int jj = 0; jj < JB; ++jj)
          if (j0 + jj < m) acc[jj] = lane_dot<BITS>(lw[jj], wv, acc[jj]);
      }
#pragma unroll
      for (int jj = 0; jj < JB; ++jj) {
        double a = acc[jj];
#pragma unroll
        for (int s = 16; s > 0; s >>= 1) a += __shfl_down_sync(0xFFFFFFFFu, a, s);
        if (lane == 0 && j0 + jj < m) s_acc[warp][j0 + jj] += a;
      }
    }
  }
  __syncthreads();
  for (int j = tid; j < m; j += kKT) {
    double p = 0.0;
#pragma unroll
    for (int q = 0; q < kKT / 32; ++q) p += s_acc[q][j];
    partials[(std::uint64_t)blockIdx.x * m + j] = p;
  }
  __threadfence();
  __syncthreads();
  if (tid == 0) s_last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  __syncthreads();
  if (s_last) {
    __threadfence();
    for (int j = tid; j < m; j += kKT) {
      double sum = 0.0;
      for (unsigned b = 0; b < gridDim.x; ++b) sum += __ldcg(partials + (std::uint64_t)b * m + j);
      h[j] = sum;
    }
    if (tid == 0) *ticket = 0u; // ready for the next call
  }
}

// Dot with work handed out at run time: an item is a group of vg vectors over
// a slice of kSub values; CTAs take items from a counter in the workspace, so
// SMs that run slower take fewer (a fixed split measured a 10 % spread of SM
// busy time), and write each (vector, slice) sum to its own place in
// partials; k_basis_dot_final adds them in slice order, so h does not depend
// on which CTA took which item, on the grid or on vg.
template<int BITS>
__global__ void __launch_bounds__(kKT, kMinCtas)
  k_basis_dot_dyn(const __grid_constant__ BasisParams bp, int m, BasisGeo g, const double* __restrict__ w,
                  unsigned int ns, int vg, double* __restrict__ partials, unsigned int* __restrict__ next_item)
{
  constexpr int P = fast_cfg<double, BITS>::P;
  constexpr int JB = jb_dot(BITS);
  __shared__ double s_w[kSub];
  __shared__ double s_acc[kKT / 32][kMaxBasis];
  __shared__ unsigned int s_item;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const unsigned int groups = (unsigned)((m + vg - 1) / vg);
  const unsigned int items = ns * groups;

  for (;;) {
    if (tid == 0) s_item = atomicAdd(next_item, 1u);
    __syncthreads(); // also: the previous item's s_w / s_acc are consumed
    const unsigned int it = s_item;
    if (it >= items) break;
    // an item: vectors [jb, je) over slice sl
    const unsigned int sl = it / groups;
    const int jb = (int)(it - sl * groups) * vg, je = min(jb + vg, m);
    const std::uint64_t s0 = (std::uint64_t)sl * kSub;
    const int len = (int)((g.n - s0) < (std::uint64_t)kSub ? (g.n - s0) : (std::uint64_t)kSub);
    for (int i = tid; i < len; i += kKT) s_w[i] = __ldg(w + s0 + i);
    __syncthreads();
    // JB vectors at a time: all their loads are issued before any decode
    for (int j0 = jb; j0 < je; j0 += JB) {
      double acc[JB];
#pragma unroll
      for (int jj = 0; jj < JB; ++jj) acc[jj] = 0.0;
      for (int i = tid * P; i < len; i += kKT * P) {
        lane_words<double, BITS> lw[JB];
#pragma unroll
        for (int jj = 0; jj < JB; ++jj)
          if (j0 + jj < je) {
            const std::uint8_t* buf = bp.buf[j0 + jj];
            fast_load_lane<double, BITS>(buf, buf + g.exp_bytes, g.log2E, s0 + (std::uint64_t)i, lw[jj]);
          }
        double wv[P];
#pragma unroll
        for (int k = 0; k < P; ++k) wv[k] = i + k < len ? s_w[i + k] : 0.0;
#pragma unroll
        for (int jj = 0; jj < JB; ++jj)
          if (j0 + jj < je) acc[jj] = lane_dot<BITS>(lw[jj], wv, acc[jj]);
      }
#pragma unroll
      for (int jj = 0; jj < JB; ++jj) {
        double a = acc[jj];
#pragma unroll
        for (int sh = 16; sh > 0; sh >>= 1) a += __shfl_down_sync(0xFFFFFFFFu, a, sh);
        if (lane == 0 && j0 + jj < je) s_acc[warp][j0 + jj] = a; // each (warp, vector) once per item
      }
    }
    __syncthreads();
    // this item's sums, vector-major: partials[j * ns + sl]
    for (int j = jb + tid; j < je; j += kKT) {
      double p = 0.0;
#pragma unroll
      for (int q = 0; q < kKT / 32; ++q) p += s_acc[q][j];
      partials[(std::uint64_t)j * ns + sl] = p;
    }
  }
}

// h[j] = sum over slices of partials[j * ns + slice], in a fixed order; one
// CTA per vector.  Leaves the slice counter at zero for the next call.
__global__ void __launch_bounds__(kKT)
  k_basis_dot_final(const double* __restrict__ partials, unsigned int ns, double* __restrict__ h,
                    unsigned int* __restrict__ next_slice)
{
  __shared__ double s_red[kKT / 32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const double* pj = partials + (std::uint64_t)blockIdx.x * ns;
  double sum = 0.0;
  for (unsigned int b = tid; b < ns; b += kKT) sum += __ldcg(pj + b);
#pragma unroll
  for (int sh = 16; sh > 0; sh >>= 1) sum += __shfl_down_sync(0xFFFFFFFFu, sum, sh);
  if (lane == 0) s_red[warp] = sum;
  __syncthreads();
  if (tid == 0) {
    double t = 0.0;
#pragma unroll
    for (int q = 0; q < kKT / 32; ++q) t += s_red[q];
    h[blockIdx.x] = t;
    if (blockIdx.x == 0) *next_slice = 0u;
  }
}

template<int BITS>
__global__ void __launch_bounds__(kKT, kMinCtas)
  k_basis_axpy(const __grid_constant__ BasisParams bp, int m, BasisGeo g, const double* __restrict__ coef,
               double* __restrict__ y)
{
  constexpr int P = fast_cfg<double, BITS>::P;
  constexpr int JB = jb_axpy(BITS);
  __shared__ double s_c[kMaxBasis];
  for (int j = threadIdx.x; j < m; j += kKT) s_c[j] = __ldg(coef + j);
  __syncthreads();
  const std::uint64_t stride = (std::uint64_t)gridDim.x * kKT * P;
  for (std::uint64_t idx = ((std::uint64_t)blockIdx.x * kKT + threadIdx.x) * P; idx < g.n; idx += stride) {
    const bool whole = idx + P <= g.n;
    double acc[P];
    if (whole) {
      std::uint32_t v[8];
      ld256_stream(y + idx, v);
#pragma unroll
      for (int k = 0; k < P; ++k) acc[k] = __longlong_as_double(((long long)v[2 * k + 1] << 32) | v[2 * k]);
    } else {
#pragma unroll
      for (int k = 0; k < P; ++k) acc[k] = idx + k < g.n ? y[idx + k] : 0.0;
    }
    for (int j0 = 0; j0 < m; j0 += JB) {
      lane_words<double, BITS> lw[JB];
#pragma unroll
      for (int jj = 0; jj < JB; ++jj)
        if (j0 + jj < m) {
          const std::uint8_t* buf = bp.buf[j0 + jj];
          fast_load_lane<double, BITS>(buf, buf + g.exp_bytes, g.log2E, idx, lw[jj]);
        }
#pragma unroll
      for (int jj = 0; jj < JB; ++jj)
        if (j0 + jj < m) lane_axpy<BITS>(lw[jj], s_c[j0 + jj], acc);
    }
    if (whole) {
      std::uint32_t v[8];
#pragma unroll
      for (int k = 0; k < P; ++k) {
        const unsigned long long b = (unsigned long long)__double_as_longlong(acc[k]);
        v[2 * k] = (std::uint32_t)b;
        v[2 * k + 1] = (std::uint32_t)(b >> 32);
      }
      st256_stream(y + idx, v);
    } else {
      for (int k = 0; k < P && idx + k < g.n; ++k) y[idx + k] = acc[k];
    }
  }
}

// widths with fused kernels (fp64 bases)
#define FRSZ2_KRYLOV_WIDTHS(X) X(16) X(21) X(24) X(32) X(48) X(64)

int basis_args(int dtype, int bits, int E, const void* const* basis, int m, std::uint64_t n, BasisParams* bp,
               BasisGeo* g)
{
  if (int rc = check_args(dtype, bits, E)) return rc;
  if (dtype != FRSZ2_DOUBLE) return set_error(FRSZ2_EFAIL, "fused basis kernels take fp64 bases");
  switch (bits) {
#define CASE(B) case B:
    FRSZ2_KRYLOV_WIDTHS(CASE)
#undef CASE
    break;
    default: return set_error(FRSZ2_EFAIL, "fused basis kernels have no instance for " + std::to_string(bits) + " bits");
  }
  if (E < 4 || E > 65536 || (E & (E - 1)) != 0 || ((std::uint64_t)E * bits) % word_bits(bits) != 0)
    return set_error(FRSZ2_EFAIL, "fused basis kernels need a power-of-two block size without block padding");
  if (m < 0 || m > kMaxBasis)
    return set_error(FRSZ2_EFAIL, "basis size must be in [0, " + std::to_string(kMaxBasis) + "]");
  if (m > 0 && !basis) return set_error(FRSZ2_EFAIL, "null basis");
  const Layout L = make_layout(n, bits, E);
  for (int j = 0; j < m; ++j) {
    if (!basis[j] || reinterpret_cast<std::uintptr_t>(basis[j]) % 32 != 0)
      return set_error(FRSZ2_EFAIL, "basis vector " + std::to_string(j) + " is null or not 32-byte aligned");
    bp->buf[j] = static_cast<const std::uint8_t*>(basis[j]);
  }
  g->n = n;
  g->exp_bytes = L.exp_bytes;
  int l = 0;
  while ((1 << l) < E) ++l;
  g->log2E = l;
  return FRSZ2_OK;
}

constexpr int kMaxCtasPerSm = 8; // bound used to size the workspace

// Values per CTA for `ctas` resident CTAs: a multiple of 256 (whole lanes).
std::uint64_t dot_chunk(std::uint64_t n, std::uint64_t ctas)
{
  std::uint64_t chunk = (n + ctas - 1) / ctas;
  return std::max<std::uint64_t>(256, ((chunk + 255) / 256) * 256);
}

// axpy grid: up to this many CTAs per SM (about 4 resident), the rest queue
// and start as others finish; measured on B200, 100 vectors of 2^22 values:
// 8 per SM 0.871 of HBM, 16 per SM 0.885, one CTA per 1,024 positions 0.887
// (32 bits; 21 bits 0.516 / 0.545 / 0.542).
#ifndef FRSZ2_AXPY_CTAS_PER_SM
#define FRSZ2_AXPY_CTAS_PER_SM 16
#endif

#ifndef FRSZ2_KRYLOV_DYNAMIC
#define FRSZ2_KRYLOV_DYNAMIC 1
#endif

template<int BITS>
int dyn_ctas_per_sm()
{
  int blocks = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k_basis_dot_dyn<BITS>, kKT, 0) != cudaSuccess ||
      blocks < 1)
    blocks = 1;
  return std::min(blocks, kMaxCtasPerSm);
}

template<int BITS>
int dot_ctas_per_sm()
{
  int blocks = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k_basis_dot<BITS>, kKT, 0) != cudaSuccess || blocks < 1)
    blocks = 1;
  return std::min(blocks, kMaxCtasPerSm);
}

} // namespace
} // namespace frsz2b

using namespace frsz2b;

extern "C" {

uint64_t frsz2_basis_workspace_size(int m, uint64_t n)
{
  if (m < 0) m = 0;
  const std::uint64_t grid = (std::uint64_t)sm_count() * kMaxCtasPerSm;
  const std::uint64_t slices = (n + kSub - 1) / kSub; // one row of m sums per slice
  return 256 + std::max(grid, slices) * (std::uint64_t)std::max(m, 1) * sizeof(double);
}

int frsz2_basis_dot(int dtype, int bits, int block_size, const void* const* basis, int m, uint64_t n,
                    const void* w, void* h, void* workspace, uint64_t workspace_bytes, void* stream)
{
  NvtxRange nvtx("frsz2_basis_dot");
  BasisParams bp{};
  BasisGeo g{};
  if (int rc = basis_args(dtype, bits, block_size, basis, m, n, &bp, &g)) return rc;
  if (m == 0) return FRSZ2_OK;
  if (!w || !h || !workspace) return set_error(FRSZ2_EFAIL, "null pointer");
  if (workspace_bytes < frsz2_basis_workspace_size(m, n))
    return set_error(FRSZ2_EFAIL, "workspace smaller than frsz2_basis_workspace_size()");
  if (reinterpret_cast<std::uintptr_t>(workspace) % 256 != 0)
    return set_error(FRSZ2_EFAIL, "workspace must be 256-byte aligned");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (n == 0) return cuda_status(cudaMemsetAsync(h, 0, (std::size_t)m * sizeof(double), s), "memset");
  if (FRSZ2_KRYLOV_DYNAMIC) {
    const std::uint64_t ns64 = (n + kSub - 1) / kSub;
    if (ns64 > 0xFFFFFFFFull) return set_error(FRSZ2_EFAIL, "basis vectors too long");
    const unsigned ns = (unsigned)ns64;
    auto* next_slice = static_cast<unsigned int*>(workspace);
    auto* rows = reinterpret_cast<double*>(static_cast<std::uint8_t*>(workspace) + 256);
    int per = 1;
    switch (bits) {
#define CASE(B)                                                                                                    \
  case B: per = dyn_ctas_per_sm<B>(); break;
      FRSZ2_KRYLOV_WIDTHS(CASE)
#undef CASE
    }
    const std::uint64_t ctas = (std::uint64_t)sm_count() * (std::uint64_t)per;
    // vectors per item: up to 32 vectors, all of them (whole slices); more,
    // about 8 items per CTA in multiples of jb_dot and at least 16 vectors (each
    // item stages its slice of w once).  Measured on B200 with 2^22-value
    // vectors, 32 bits: m = 100 0.76 of HBM with 32 vectors per item against
    // 0.74 with whole slices; m = 20 0.67 with whole slices against 0.62 with
    // 16 per item.
    std::uint64_t vg = (std::uint64_t)m;
    if (m > 32) {
      vg = ((std::uint64_t)m * ns + 8 * ctas - 1) / (8 * ctas);
      const std::uint64_t jb = (std::uint64_t)jb_dot(bits);
      vg = std::min<std::uint64_t>((std::uint64_t)m, std::max<std::uint64_t>(16, (vg + jb - 1) / jb * jb));
    }
    const std::uint64_t items = ns * (((std::uint64_t)m + vg - 1) / vg);
    if (items > 0xFFFFFFFFull) return set_error(FRSZ2_EFAIL, "basis vectors too long");
    const unsigned grid = (unsigned)std::max<std::uint64_t>(1, std::min<std::uint64_t>(items, ctas));
    switch (bits) {
#define CASE(B)                                                                                                    \
  case B:                                                                                                          \
    k_basis_dot_dyn<B><<<grid, kKT, 0, s>>>(bp, m, g, static_cast<const double*>(w), ns, (int)vg, rows,          \
                                            next_slice);                                                           \
    break;
      FRSZ2_KRYLOV_WIDTHS(CASE)
#undef CASE
    }
    if (int rc = cuda_status(cudaGetLastError(), "basis dot launch")) return rc;
    k_basis_dot_final<<<(unsigned)m, kKT, 0, s>>>(rows, ns, static_cast<double*>(h), next_slice);
    return cuda_status(cudaGetLastError(), "basis dot launch");
  }
  int per_sm = 1;
  switch (bits) {
#define CASE(B)                                                                                                    \
  case B: per_sm = dot_ctas_per_sm<B>(); break;
    FRSZ2_KRYLOV_WIDTHS(CASE)
#undef CASE
  }
  const std::uint64_t chunk = dot_chunk(n, (std::uint64_t)sm_count() * (std::uint64_t)per_sm);
  const unsigned grid = (unsigned)std::max<std::uint64_t>(1, (n + chunk - 1) / chunk);
  auto* ticket = static_cast<unsigned int*>(workspace);
  auto* partials = reinterpret_cast<double*>(static_cast<std::uint8_t*>(workspace) + 256);
  switch (bits) {
#define CASE(B)                                                                                                    \
  case B:                                                                                                          \
    k_basis_dot<B><<<grid, kKT, 0, s>>>(bp, m, g, static_cast<const double*>(w), chunk, partials, ticket,          \
                                        static_cast<double*>(h));                                                  \
    break;
    FRSZ2_KRYLOV_WIDTHS(CASE)
#undef CASE
  }
  return cuda_status(cudaGetLastError(), "basis dot launch");
}

int frsz2_basis_axpy(int dtype, int bits, int block_size, const void* const* basis, int m, uint64_t n,
                     const void* coef, void* y, void* stream)
{
  NvtxRange nvtx("frsz2_basis_axpy");
  BasisParams bp{};
  BasisGeo g{};
  if (int rc = basis_args(dtype, bits, block_size, basis, m, n, &bp, &g)) return rc;
  if (m == 0 || n == 0) return FRSZ2_OK;
  if (!coef || !y) return set_error(FRSZ2_EFAIL, "null pointer");
  if (reinterpret_cast<std::uintptr_t>(y) % 32 != 0) return set_error(FRSZ2_EFAIL, "y must be 32-byte aligned");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const std::uint64_t lanes = (n + 3) / 4;
  const unsigned grid = (unsigned)std::max<std::uint64_t>(
    1, std::min<std::uint64_t>((lanes + kKT - 1) / kKT, (std::uint64_t)sm_count() * FRSZ2_AXPY_CTAS_PER_SM));
  switch (bits) {
#define CASE(B)                                                                                                    \
  case B:                                                                                                          \
    k_basis_axpy<B><<<grid, kKT, 0, s>>>(bp, m, g, static_cast<const double*>(coef), static_cast<double*>(y));     \
    break;
    FRSZ2_KRYLOV_WIDTHS(CASE)
#undef CASE
  }
  return cuda_status(cudaGetLastError(), "basis axpy launch");
}

} // extern "C"
