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

// Place of value i of a slice of w in shared memory: 16-byte chunk q = i / 2
// at q ^ ((q >> 3) & 1).
__device__ __forceinline__ int dot_swz(int i) { return (((i >> 1) ^ ((i >> 4) & 1)) << 1) | (i & 1); }

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
    // 16-byte chunks of w swizzled (chunk q at q ^ ((q >> 3) & 1)), so the
    // 32-byte runs of a warp's lanes fall on distinct banks
    for (int i = tid; i < len; i += kKT) s_w[dot_swz(i)] = __ldg(w + s0 + i);
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
        if (i + P <= len) {
          const double2* wr = reinterpret_cast<const double2*>(s_w) + (i >> 1);
          const int f = (lane >> 2) & 1; // i >> 1 = 2 * tid + 512 * pass: chunk swizzle (tid >> 2) & 1
          const double2 wa = wr[f], wb = wr[1 - f];
          wv[0] = wa.x;
          wv[1] = wa.y;
          wv[2] = wb.x;
          wv[3] = wb.y;
        } else {
#pragma unroll
          for (int k = 0; k < P; ++k) wv[k] = i + k < len ? s_w[dot_swz(i + k)] : 0.0;
        }
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

// ---------------------------------------------------------------- dot over per-warp copy rings
//
// The register kernel above keeps each thread's next codes in registers, so
// the loads a warp has in flight are bounded by its register budget, and it
// waits on them (long scoreboard) for most of its time.  Here each warp
// streams its codes and exponents through its own ring of kRD shared-memory
// slots with bulk asynchronous copies (cp.async.bulk, completion counted on one
// mbarrier per slot): lane 0 issues a stage's copies kRD stages ahead of the
// warp's decode, so a stage's latency is covered by the stages before it and
// no register is held for a load in flight.
//
// Work is the same (slice, vector group) items as above, taken from a counter;
// the CTA claims each item two ahead, so a warp's ring runs on into the next
// item's stages while the CTA adds up the current one and stages the next
// slice of w.  Inside an item, a unit is a pair of vectors over a range of the
// slice's warp rows; warp k takes units k, k + 8, ... .  A stage is R warp rows
// (128 values each) of both vectors of a unit: their codes and the 16-byte
// aligned span of exponents that covers them.  Each unit's lane-summed result
// goes to its own place, and the item's sum per vector adds them in a fixed
// order, so h does not depend on scheduling.  w's slice sits in shared memory
// with its 16-byte chunks swizzled (chunk q at q ^ ((q >> 3) & 1)), so the
// 32-byte runs the lanes of a warp read fall on distinct banks.
//
// Every mbarrier wait is bounded (2 s): a wait that runs out sets an error
// flag in the workspace, the CTA stops at its next item boundary, and the
// dot then returns NaN for every h[j].

constexpr int kRW = 8;                 // warps per CTA
constexpr int kRT = kRW * 32;          // threads per CTA
constexpr int kRSlice = kSub;          // values per item (24 warp rows)
constexpr int kRRow = 128;             // values per warp row: 32 lanes x 4
constexpr int kRMaxGroup = 32;         // vectors per item at most
// Stages per warp ring.  Measured on B200 (100 vectors of 2^22 values, 64
// bits): the time does not change with 2, 3 or 4 stages of the same size and
// drops by a fifth when a stage doubles (1 -> 2 warp rows per vector); the
// shared memory of two stages of 2 rows keeps 2 CTAs per SM.
constexpr int kRD = 2;
constexpr int kRPart = 2 * kRMaxGroup; // unit sums per item, then the partial-row sums

template<int BITS>
struct ring_shape
{
  static constexpr int RB = 16 * BITS; // code bytes of one warp row (a multiple of 16)
  // warp rows per stage: two vectors' codes of a stage come to about 4 KiB
  static constexpr int R = BITS <= 16 ? 8 : BITS <= 24 ? 6 : BITS <= 32 ? 4 : 2;
  static constexpr int CODE = R * RB;  // code bytes per vector and stage
  static constexpr int W = fast_cfg<double, BITS>::W;
  static constexpr int Wb = W / 8;
};

// Bytes of one vector's exponent span in a slot: the 16-byte aligned span of
// exponents covering R warp rows that start at any row.
__host__ __device__ constexpr int ring_expw(int R, int log2E, int Wb)
{
  return ((((R * kRRow - 1) >> log2E) + 2) * Wb + 30 + 15) / 16 * 16;
}

__device__ __forceinline__ std::uint32_t smem_addr(const void* p)
{
  return (std::uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(std::uint64_t* bar, unsigned count)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(std::uint64_t* bar, unsigned bytes)
{
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(std::uint64_t* bar, unsigned parity)
{
  unsigned done;
  asm volatile("{\n\t.reg .pred p;\n\t"
               "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
               "selp.u32 %0, 1, 0, p;\n\t}"
               : "=r"(done)
               : "r"(smem_addr(bar)), "r"(parity)
               : "memory");
  return done != 0;
}

// Global -> shared bulk copy (no multicast), completion counted on `bar`.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, std::uint64_t* bar)
{
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                 smem_addr(dst)),
               "l"(src), "r"(bytes), "r"(smem_addr(bar))
               : "memory");
}

__device__ __forceinline__ std::uint64_t global_ns()
{
  std::uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Waits for a slot's phase, at most `limit_ns`; every lane of the warp gets
// the same answer.
__device__ __forceinline__ bool ring_wait(std::uint64_t* bar, unsigned parity, std::uint64_t limit_ns)
{
  bool done = mbar_try_wait(bar, parity);
  if (!done) {
    const std::uint64_t t0 = global_ns();
    while (!(done = mbar_try_wait(bar, parity)))
      if (global_ns() - t0 > limit_ns) break;
  }
  return __all_sync(0xFFFFFFFFu, done);
}

struct RingItem
{
  std::uint64_t s0; // first value of the slice
  int jb, G;        // vectors [jb, jb + G)
  int P, C, RC;     // vector pairs, row chunks per pair, warp rows per chunk
  int rows, len;    // whole warp rows in the slice, values in the slice
};

__device__ __forceinline__ RingItem ring_item(unsigned it, unsigned groups, int vg, int m, std::uint64_t n)
{
  RingItem r;
  const unsigned sl = it / groups;
  r.jb = (int)(it - sl * groups) * vg;
  r.G = min(vg, m - r.jb);
  r.s0 = (std::uint64_t)sl * kRSlice;
  const std::uint64_t rem = n - r.s0;
  r.len = rem < (std::uint64_t)kRSlice ? (int)rem : kRSlice;
  r.rows = r.len / kRRow;
  r.P = (r.G + 1) / 2;
  r.C = r.P >= kRW ? 1 : (kRW + r.P - 1) / r.P; // at least one unit per warp
  r.RC = (r.rows + r.C - 1) / r.C;
  return r;
}

// One lane's codes of a warp row held in shared memory.
template<int BITS>
__device__ __forceinline__ void ring_lane_words(const std::uint8_t* row, int lane, lane_words<double, BITS>& lw)
{
  using Cfg = fast_cfg<double, BITS>;
  constexpr int NW = Cfg::NW;
  if constexpr (Cfg::ALIGNED) {
    constexpr int LB = BITS / 2; // a lane's 4 codes in bytes
    const std::uint8_t* p = row + lane * LB;
    if constexpr (LB % 16 == 0) {
#pragma unroll
      for (int i = 0; i < NW / 4; ++i) {
        const uint4 v = reinterpret_cast<const uint4*>(p)[i];
        lw.w[4 * i] = v.x;
        lw.w[4 * i + 1] = v.y;
        lw.w[4 * i + 2] = v.z;
        lw.w[4 * i + 3] = v.w;
      }
    } else if constexpr (LB % 8 == 0) {
#pragma unroll
      for (int i = 0; i < NW / 2; ++i) {
        const uint2 v = reinterpret_cast<const uint2*>(p)[i];
        lw.w[2 * i] = v.x;
        lw.w[2 * i + 1] = v.y;
      }
    } else {
#pragma unroll
      for (int i = 0; i < NW; ++i) lw.w[i] = reinterpret_cast<const std::uint32_t*>(p)[i];
    }
    lw.o = 0;
  } else {
    const int S = lane * 4 * BITS;
    const std::uint32_t* q = reinterpret_cast<const std::uint32_t*>(row) + (S >> 5);
    lw.o = S & 31;
#pragma unroll
    for (int i = 0; i < NW; ++i) lw.w[i] = q[i];
    lw.w[NW] = (lw.o + 4 * BITS > 32 * NW) ? q[NW] : 0u;
  }
}

template<int BITS>
__global__ void __launch_bounds__(kRT, 2)
  k_basis_dot_ring(const __grid_constant__ BasisParams bp, int m, BasisGeo g, const double* __restrict__ w,
                   unsigned int ns, int vg, int expw, int slot_bytes, double* __restrict__ partials,
                   unsigned int* __restrict__ ctl)
{
  using S = ring_shape<BITS>;
  constexpr int R = S::R, RB = S::RB, CODE = S::CODE, Wb = S::Wb;
  extern __shared__ __align__(128) std::uint8_t smem[];
  double* s_w = reinterpret_cast<double*>(smem);              // kRSlice values, chunk-swizzled
  double* s_part = s_w + kRSlice;                             // kRPart
  std::uint64_t* s_bar = reinterpret_cast<std::uint64_t*>(s_part + kRPart);
  unsigned int* s_item = reinterpret_cast<unsigned int*>(s_bar + kRW * kRD); // 3 items, abort flag
  std::uint8_t* s_ring = smem + ((kRSlice + kRPart) * 8 + kRW * kRD * 8 + 16 + 127) / 128 * 128;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const unsigned int groups = (unsigned)((m + vg - 1) / vg);
  const unsigned int items = ns * groups;
  std::uint8_t* ring = s_ring + (std::size_t)warp * kRD * slot_bytes;
  std::uint64_t* bar = s_bar + warp * kRD;
  constexpr std::uint64_t kLimitNs = 2000000000ull;

  if (lane == 0)
    for (int s = 0; s < kRD; ++s) mbar_init(&bar[s], 1);
  if (tid == 0) {
    s_item[0] = atomicAdd(&ctl[0], 1u);
    s_item[1] = atomicAdd(&ctl[0], 1u);
    s_item[3] = 0u;
  }
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  __syncthreads();

  // w's slice of an item into s_w (zeros past the array), 16-byte chunks swizzled
  auto stage_w = [&](unsigned it) {
    const RingItem r = ring_item(it, groups, vg, m, g.n);
    double2* sw2 = reinterpret_cast<double2*>(s_w);
    for (int q = tid; q < kRSlice / 2; q += kRT) {
      const int i = 2 * q;
      const double a = i < r.len ? __ldg(w + r.s0 + i) : 0.0;
      const double b = i + 1 < r.len ? __ldg(w + r.s0 + i + 1) : 0.0;
      sw2[q ^ ((q >> 3) & 1)] = make_double2(a, b);
    }
  };
  if (s_item[0] < items) stage_w(s_item[0]);

  // ---- producer: the next stage of this warp's stream, kRD stages ahead.
  // Per unit it keeps the two vectors' buffers and the next stage's first
  // value; a stage then costs a few additions and lane 0's copies.
  unsigned int issued = 0, consumed = 0;
  int pk = 0;                           // item sequence number of the producer
  RingItem pi = ring_item(s_item[0], groups, vg, m, g.n);
  bool p_live = s_item[0] < items;      // the producer's item is a valid one
  int pu = warp;                        // unit
  int p_rows = 0;                       // warp rows of the unit not yet issued
  std::uint64_t p_pos = 0;              // first value of the next stage
  const std::uint8_t* p_buf0 = nullptr; // the unit's vectors
  const std::uint8_t* p_buf1 = nullptr;
  int p_nv = 0;
  int ck = 0;                           // item sequence number of the consumer
  bool ok = true;                       // no wait of this warp ran out
  unsigned int drain_from = 0;          // the first stage not known to have landed, after a wait ran out
  const int emask = (1 << g.log2E) - 1;

  auto p_unit = [&]() {
    if (pu >= pi.P * pi.C) {
      p_rows = 0;
      return;
    }
    const int c = pu % pi.C, pair = pu / pi.C;
    const int r0 = c * pi.RC;
    p_rows = max(0, min(pi.rows, r0 + pi.RC) - r0);
    p_pos = pi.s0 + (std::uint64_t)r0 * kRRow;
    const int j0 = pi.jb + 2 * pair;
    p_nv = min(2, pi.G - 2 * pair);
    p_buf0 = bp.buf[j0];
    p_buf1 = bp.buf[p_nv > 1 ? j0 + 1 : j0];
  };
  if (p_live) p_unit();

  // A stage to issue, moving over units and items; false when none is
  // allowed yet (item ck + 2 is announced at the end of item ck) or none is left.
  auto p_seek = [&]() -> bool {
    while (p_live) {
      if (p_rows > 0) return true;
      if (pu + kRW < pi.P * pi.C) {
        pu += kRW;
        p_unit();
        continue;
      }
      if (pk > ck) return false;
      ++pk;
      const unsigned int id = s_item[pk % 3];
      p_live = id < items;
      if (p_live) {
        pi = ring_item(id, groups, vg, m, g.n);
        pu = warp;
        p_unit();
      }
    }
    return false;
  };
  auto p_issue = [&]() {
    const int slot = (int)(issued % kRD);
    const int nr = min(R, p_rows);
    if (lane == 0) {
      const unsigned int cbytes = (unsigned)(nr * RB);
      const std::uint64_t e0 = (p_pos >> g.log2E) * Wb;
      const std::uint64_t e1 = (((p_pos + (std::uint64_t)nr * kRRow - 1) >> g.log2E) + 1) * Wb;
      const std::uint64_t ws = e0 & ~15ull;
      const unsigned int ebytes = (unsigned)(((e1 + 15) & ~15ull) - ws);
      std::uint8_t* sp = ring + (std::size_t)slot * slot_bytes;
      const std::uint64_t coff = g.exp_bytes + p_pos * (std::uint64_t)BITS / 8;
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      mbar_arrive_expect_tx(&bar[slot], (unsigned)p_nv * (cbytes + ebytes));
      bulk_g2s(sp, p_buf0 + coff, cbytes, &bar[slot]);
      bulk_g2s(sp + 2 * CODE, p_buf0 + ws, ebytes, &bar[slot]);
      if (p_nv > 1) {
        bulk_g2s(sp + CODE, p_buf1 + coff, cbytes, &bar[slot]);
        bulk_g2s(sp + 2 * CODE + expw, p_buf1 + ws, ebytes, &bar[slot]);
      }
    }
    ++issued;
    p_pos += (std::uint64_t)nr * kRRow;
    p_rows -= nr;
  };
  auto refill = [&]() {
    if (!ok) return;
    while (issued < consumed + kRD && p_seek()) p_issue();
  };
  __syncthreads(); // s_w of the first item

  const int f = (lane >> 2) & 1; // the lane's chunk swizzle in s_w
  for (;; ++ck) {
    refill();
    const unsigned int id = s_item[ck % 3];
    if (id >= items) break;
    const RingItem ci = ring_item(id, groups, vg, m, g.n);
    const double2* sw2 = reinterpret_cast<const double2*>(s_w) + 2 * lane;
    for (int u = warp; u < ci.P * ci.C; u += kRW) {
      const int c = u % ci.C, pair = u / ci.C;
      const int nv = min(2, ci.G - 2 * pair);
      const int ra = c * ci.RC, rb = min(ci.rows, ra + ci.RC);
      double acc0 = 0.0, acc1 = 0.0;
      for (int r0 = ra; r0 < rb; r0 += R) {
        const int slot = (int)(consumed % kRD);
        if (ok && !ring_wait(&bar[slot], (consumed / kRD) & 1u, kLimitNs)) {
          ok = false;
          drain_from = consumed;
          if (lane == 0) {
            atomicExch(&ctl[1], 1u);
            s_item[3] = 1u;
          }
        }
        const std::uint8_t* sp = ring + (std::size_t)slot * slot_bytes;
        const std::uint64_t pos0 = ci.s0 + (std::uint64_t)r0 * kRRow;
        // exponent offsets in the slot: block of value pos0 + d is
        // (pos0 >> log2E) + (((pos0 & emask) + d) >> log2E)
        const int ebase = (int)(((pos0 >> g.log2E) * Wb) & 15u);
        const int po = (int)(pos0 & (std::uint64_t)emask) + 4 * lane;
        const int nr = min(R, rb - r0);
#pragma unroll
        for (int rr = 0; rr < R; ++rr) {
          if (rr < nr) {
            const double2* wr = sw2 + (r0 + rr) * (kRRow / 2);
            const double2 wa = wr[f], wb = wr[1 - f]; // logical chunks 2 * lane and 2 * lane + 1
            const double wv[4] = { wa.x, wa.y, wb.x, wb.y };
            const int eoff = ebase + ((po + rr * kRRow) >> g.log2E) * Wb;
            lane_words<double, BITS> lw;
            ring_lane_words<BITS>(sp + rr * RB, lane, lw);
            lw.be = (typename lane_words<double, BITS>::exp_t)load_exp(sp + 2 * CODE + eoff, S::W);
            acc0 = lane_dot<BITS>(lw, wv, acc0);
            if (nv > 1) {
              lane_words<double, BITS> lw1;
              ring_lane_words<BITS>(sp + CODE + rr * RB, lane, lw1);
              lw1.be = (typename lane_words<double, BITS>::exp_t)load_exp(sp + 2 * CODE + expw + eoff, S::W);
              acc1 = lane_dot<BITS>(lw1, wv, acc1);
            }
          }
        }
        __syncwarp();
        ++consumed;
        refill();
      }
#pragma unroll
      for (int sh = 16; sh > 0; sh >>= 1) {
        acc0 += __shfl_down_sync(0xFFFFFFFFu, acc0, sh);
        acc1 += __shfl_down_sync(0xFFFFFFFFu, acc1, sh);
      }
      if (lane == 0) {
        const int t = 2 * pair;
        s_part[t * ci.C + c] = acc0;
        if (nv > 1) s_part[(t + 1) * ci.C + c] = acc1;
      }
    }
    // values past the slice's whole warp rows (the array's last, partial row)
    const bool tail = ci.len > ci.rows * kRRow;
    if (tail) {
      const std::uint64_t idx = ci.s0 + (std::uint64_t)ci.rows * kRRow + 4 * (std::uint64_t)lane;
      const int i = ci.rows * kRRow + 4 * lane;
      const double2* sw = reinterpret_cast<const double2*>(s_w);
      const int q0 = i / 2;
      const double2 wa = sw[q0 ^ ((q0 >> 3) & 1)], wb = sw[(q0 + 1) ^ (((q0 + 1) >> 3) & 1)];
      const double wv[4] = { wa.x, wa.y, wb.x, wb.y };
      for (int t = warp; t < ci.G; t += kRW) {
        double a = 0.0;
        if (idx < g.n) {
          const std::uint8_t* buf = bp.buf[ci.jb + t];
          lane_words<double, BITS> lw;
          fast_load_lane<double, BITS>(buf, buf + g.exp_bytes, g.log2E, idx, lw);
          a = lane_dot<BITS>(lw, wv, 0.0);
        }
#pragma unroll
        for (int sh = 16; sh > 0; sh >>= 1) a += __shfl_down_sync(0xFFFFFFFFu, a, sh);
        if (lane == 0) s_part[kRMaxGroup + t] = a;
      }
    }
    __syncthreads(); // the item's unit sums are in; s_w is free
    if (tid < ci.G) {
      double sum = 0.0;
      for (int c = 0; c < ci.C; ++c) sum += s_part[tid * ci.C + c];
      if (tail) sum += s_part[kRMaxGroup + tid];
      partials[(std::uint64_t)(ci.jb + tid) * ns + ci.s0 / kRSlice] = sum;
    }
    if (tid == 0) s_item[(ck + 2) % 3] = atomicAdd(&ctl[0], 1u);
    const unsigned int nid = s_item[(ck + 1) % 3];
    if (nid < items) stage_w(nid);
    __syncthreads(); // next slice of w, item ck + 2 and the abort flag visible
    if (s_item[3]) break;
  }
  // a stop after a wait ran out: let this warp's copies still in flight land
  // (bounded); after a normal end every issued stage has been consumed
  if (s_item[3])
    for (unsigned int q = ok ? consumed : drain_from; q < issued; ++q)
      ring_wait(&bar[q % kRD], (q / kRD) & 1u, 10000000ull);
}

// h[j] = sum over slices of partials[j * ns + slice], in a fixed order; one
// CTA per vector.  NaN for every h[j] when a ring wait ran out; the last CTA
// clears the item counter, the error flag and its own ticket for the next call.
__global__ void __launch_bounds__(kKT)
  k_basis_dot_ring_final(const double* __restrict__ partials, unsigned int ns, double* __restrict__ h,
                         unsigned int* __restrict__ ctl)
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
    h[blockIdx.x] = __ldcg(&ctl[1]) ? __longlong_as_double(0x7FF8000000000000ll) : t;
    __threadfence();
    if (atomicAdd(&ctl[2], 1u) == gridDim.x - 1) {
      ctl[0] = 0u;
      ctl[1] = 0u;
      ctl[2] = 0u;
    }
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

// Widths whose dot runs on the copy rings.  Measured on B200 (100 vectors of
// 2^22 values, E 32, of the HBM copy bandwidth; register kernel -> rings):
// 64 bits 0.78 -> 0.89; 48 bits 0.84 -> 0.65, 32 bits 0.89 -> 0.69, 24 bits
// 0.68 -> 0.55, 21 bits 0.53 -> 0.46, 16 bits 0.48 -> 0.39.  Below 64 bits a
// stage holds more values per byte, and the rings' decode, with half the
// resident warps of the register kernel, falls behind.
#define FRSZ2_RING_WIDTHS(X) X(64)

// The ring dot: items of up to kRMaxGroup vectors over a slice, one CTA per
// SM slot the shared memory allows, then the slice-ordered sums.
template<int BITS>
int launch_dot_ring(const BasisParams& bp, int m, const BasisGeo& g, const double* w, double* h,
                    void* workspace, cudaStream_t s)
{
  using S = ring_shape<BITS>;
  const std::uint64_t ns64 = (g.n + kRSlice - 1) / kRSlice;
  if (ns64 > 0xFFFFFFFFull) return set_error(FRSZ2_EFAIL, "basis vectors too long");
  const unsigned ns = (unsigned)ns64;
  const int vg = std::min(m, kRMaxGroup);
  const std::uint64_t items = ns64 * (std::uint64_t)((m + vg - 1) / vg);
  if (items > 0xFFFFFFF0ull) return set_error(FRSZ2_EFAIL, "basis vectors too long");
  const int expw = ring_expw(S::R, g.log2E, S::Wb);
  const int slot_bytes = (2 * S::CODE + 2 * expw + 127) / 128 * 128;
  const int smem = ((kRSlice + kRPart) * 8 + kRW * kRD * 8 + 16 + 127) / 128 * 128 + kRW * kRD * slot_bytes;
  int rc;
  if ((rc = cuda_status(cudaFuncSetAttribute(k_basis_dot_ring<BITS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             smem),
                        "dot shared memory")))
    return rc;
  int per = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_basis_dot_ring<BITS>, kRT, smem) != cudaSuccess ||
      per < 1)
    per = 1;
  const std::uint64_t ctas = (std::uint64_t)sm_count() * (std::uint64_t)per;
  const unsigned grid = (unsigned)std::max<std::uint64_t>(1, std::min<std::uint64_t>(items, ctas));
  auto* ctl = static_cast<unsigned int*>(workspace);
  auto* rows = reinterpret_cast<double*>(static_cast<std::uint8_t*>(workspace) + 256);
  k_basis_dot_ring<BITS><<<grid, kRT, smem, s>>>(bp, m, g, w, ns, vg, expw, slot_bytes, rows, ctl);
  if ((rc = cuda_status(cudaGetLastError(), "basis dot launch"))) return rc;
  k_basis_dot_ring_final<<<(unsigned)m, kKT, 0, s>>>(rows, ns, h, ctl);
  return cuda_status(cudaGetLastError(), "basis dot launch");
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
  switch (bits) {
#define CASE(B)                                                                                                    \
  case B: return launch_dot_ring<B>(bp, m, g, static_cast<const double*>(w), static_cast<double*>(h), workspace, s);
    FRSZ2_RING_WIDTHS(CASE)
#undef CASE
    default: break;
  }
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
