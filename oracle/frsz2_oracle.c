/*
 * frsz2_oracle.c -- CPU restatement of the reference FRSZ2 codec
 * (robertu94/frsz include/frsz2.hpp), runtime-parameterised over
 * bits-per-value, exponent block size and float type.
 *
 * TEST INFRASTRUCTURE ONLY: this is the checker for the CUDA kernels, never
 * the thing measured or shipped.  See frsz2_oracle.h for the parity pins.
 *
 * Behaviour outside the reference's defined domain: the reference shifts a
 * significand left by (exponent_bits-1) - (block_exp - e), which reaches the
 * word width or more only for blocks that hold +-Inf (fp32: the float
 * exponent_t wraps to -128, so every finite neighbour overshoots), for NaN
 * elements of fp64 blocks whose block exponent is far below 1024, and for fp64
 * values >= 2^128 at bits <= 8 (the int8 exponent wraps).  Those shifts are
 * undefined behaviour in C++; this restatement (and the CUDA kernels) define
 * them as a zero magnitude.  Parity is claimed on every other input.
 */
#include "frsz2_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

/* ---------------------------------------------------------------- bit casts
 * xstd::bit_cast (frsz2.hpp:129-139). */
static uint32_t f32_bits(float x) { uint32_t u; memcpy(&u, &x, 4); return u; }
static uint64_t f64_bits(double x) { uint64_t u; memcpy(&u, &x, 8); return u; }
static float bits_f32(uint32_t u) { float x; memcpy(&x, &u, 4); return x; }
static double bits_f64(uint64_t u) { double x; memcpy(&x, &u, 8); return x; }

/* Two's-complement narrowing to a signed `w`-bit integer (the reference's
 * implicit conversions to int8_t / int16_t; gcc and nvcc both wrap). */
static int64_t wrap_signed(int64_t v, int w)
{
  if (w >= 64) return v;
  const uint64_t m = (1ull << w) - 1;
  uint64_t u = (uint64_t)v & m;
  if (u >> (w - 1)) u |= ~m;
  return (int64_t)u;
}

/* ------------------------------------------------------------- size algebra */

/* storage_t<bits> (frsz2.hpp:258-262): the word type AND the exponent type
 * (exp_type = make_signed_t<storage_t<bits>>, frsz2.hpp:510). */
int frsz2o_word_bits(int bits)
{
  return bits <= 8 ? 8 : bits <= 16 ? 16 : bits <= 32 ? 32 : 64;
}

/* compressed_block_size_element_count / _byte (frsz2.hpp:526-529). */
size_t frsz2o_block_bytes(int bits, int block_size)
{
  const int w = frsz2o_word_bits(bits);
  const size_t words = ((size_t)block_size * (size_t)bits + (size_t)w - 1) / (size_t)w;
  return words * (size_t)(w / 8);
}

/* compute_exponent_block_size_byte (frsz2.hpp:534-540): the pad is added even
 * when the exponent array already ends on a 256-byte boundary. */
size_t frsz2o_exponent_bytes(int bits, int block_size, size_t n)
{
  const size_t nb = (n + (size_t)block_size - 1) / (size_t)block_size;
  const size_t e = nb * (size_t)(frsz2o_word_bits(bits) / 8);
  return e + 256 - e % 256;
}

/* compute_compressed_memory_size_byte (frsz2.hpp:542-548). */
size_t frsz2o_compressed_bytes(int bits, int block_size, size_t n)
{
  const size_t nb = (n + (size_t)block_size - 1) / (size_t)block_size;
  return frsz2o_exponent_bytes(bits, block_size, n) + nb * frsz2o_block_bytes(bits, block_size);
}

/* ------------------------------------------------------------- primitives */

/* detail::fp::exponent (frsz2.hpp:312-320): the unsigned field minus the bias,
 * narrowed to float_traits<T>::exponent_t (int8_t for float, so the Inf/NaN
 * field 255 becomes -128; int16_t for double). */
int frsz2o_exponent_f32(float x)
{
  const int field = (int)((f32_bits(x) >> 23) & 0xFFu);
  return (int)wrap_signed(field - 127, 8);
}
int frsz2o_exponent_f64(double x)
{
  const int field = (int)((f64_bits(x) >> 52) & 0x7FFu);
  return (int)wrap_signed(field - 1023, 16);
}

/* detail::fp::significand (frsz2.hpp:322-332): implicit 1 unless the exponent
 * equals -bias (zero or subnormal). */
uint32_t frsz2o_significand_f32(float x)
{
  uint32_t s = f32_bits(x) & 0x7FFFFFu;
  if (frsz2o_exponent_f32(x) != -127) s |= 1u << 23;
  return s;
}
uint64_t frsz2o_significand_f64(double x)
{
  uint64_t s = f64_bits(x) & ((1ull << 52) - 1);
  if (frsz2o_exponent_f64(x) != -1023) s |= 1ull << 52;
  return s;
}

/* detail::fp::sign (frsz2.hpp:334-338). */
int frsz2o_sign_f32(float x) { return (int)(f32_bits(x) >> 31); }
int frsz2o_sign_f64(double x) { return (int)(f64_bits(x) >> 63); }

/* detail::fp::floating_to_fixed (frsz2.hpp:352-376).  Truncation, no
 * rounding; the sign goes to the MSB of the 32/64-bit result. */
uint32_t frsz2o_floating_to_fixed_f32(float x, int16_t block_exponent)
{
  const int s = frsz2o_sign_f32(x);
  const int e = frsz2o_exponent_f32(x);
  const uint32_t m = frsz2o_significand_f32(x);
  const int shift = 8 - 1 - ((int)block_exponent - e);
  uint32_t r;
  if (-23 > shift) {
    r = 0;
  } else if (shift > 0) {
    r = shift >= 32 ? 0u : m << shift; /* >= 32: undefined in the reference */
  } else {
    r = m >> (-shift);
  }
  if (s) r |= 1u << 31;
  return r;
}
uint64_t frsz2o_floating_to_fixed_f64(double x, int16_t block_exponent)
{
  const int s = frsz2o_sign_f64(x);
  const int e = frsz2o_exponent_f64(x);
  const uint64_t m = frsz2o_significand_f64(x);
  const int shift = 11 - 1 - ((int)block_exponent - e);
  uint64_t r;
  if (-52 > shift) {
    r = 0;
  } else if (shift > 0) {
    r = shift >= 64 ? 0ull : m << shift; /* >= 64: undefined in the reference */
  } else {
    r = m >> (-shift);
  }
  if (s) r |= 1ull << 63;
  return r;
}

/* detail::fp::fixed_to_floating (frsz2.hpp:378-399).
 * countl_zero quirk (frsz2.hpp:180-186): on LP64 std::uint64_t is unsigned
 * long, whose overload returns CHAR_BIT*sizeof(unsigned int) = 32 for a zero
 * argument.  The 32-bit overload returns 32 as well, so a zero magnitude gives
 * z = 31 for both float types. */
float frsz2o_fixed_to_floating_f32(uint32_t fixed, int64_t block_exponent)
{
  const uint32_t f = fixed & 0x7FFFFFFFu;
  const int z = (f == 0 ? 32 : __builtin_clz(f)) - 1;
  const int t = (int)(block_exponent + 127);
  const int shift = -(z < t ? z : t);
  const uint32_t s = fixed & 0x80000000u;
  const uint32_t e = (uint32_t)((int64_t)shift + block_exponent + 127) << 23;
  const int ms = 8 - 1 + shift;
  uint32_t m = ms > 0 ? f >> ms : f << (-ms);
  m &= ~(1u << 23);
  return bits_f32(s | e | m);
}
double frsz2o_fixed_to_floating_f64(uint64_t fixed, int64_t block_exponent)
{
  const uint64_t f = fixed & 0x7FFFFFFFFFFFFFFFull;
  const int z = (f == 0 ? 32 : __builtin_clzll(f)) - 1;
  const int t = (int)(block_exponent + 1023);
  const int shift = -(z < t ? z : t);
  const uint64_t s = fixed & 0x8000000000000000ull;
  const uint64_t e = (uint64_t)((int64_t)shift + block_exponent + 1023) << 52;
  const int ms = 11 - 1 + shift;
  uint64_t m = ms > 0 ? f >> ms : f << (-ms);
  m &= ~(1ull << 52);
  return bits_f64(s | e | m);
}

/* ------------------------------------------------------------- word access */

static void store_word(uint8_t* p, int w, uint64_t v) { memcpy(p, &v, (size_t)(w / 8)); } /* little endian */
static uint64_t load_word(const uint8_t* p, int w)
{
  uint64_t v = 0;
  memcpy(&v, p, (size_t)(w / 8));
  return v;
}
static uint64_t word_mask(int w) { return w == 64 ? ~0ull : ((1ull << w) - 1); }

typedef struct {
  int is64, bits, E, W;
  size_t n, nb, block_bytes, exp_bytes;
} layout_t;

static int make_layout(layout_t* L, int is64, size_t n, int bits, int block_size)
{
  if (bits < 4 || bits > (is64 ? 64 : 32) || block_size <= 0) return 2;
  L->is64 = is64;
  L->bits = bits;
  L->E = block_size;
  L->W = frsz2o_word_bits(bits);
  L->n = n;
  L->nb = (n + (size_t)block_size - 1) / (size_t)block_size;
  L->block_bytes = frsz2o_block_bytes(bits, block_size);
  L->exp_bytes = frsz2o_exponent_bytes(bits, block_size, n);
  return 0;
}

/* compress_cpu_block (frsz2.hpp:1108-1179). */
static void compress_block(const layout_t* L, const void* data, size_t b, uint8_t* out)
{
  const size_t cnt = (L->n - b * (size_t)L->E) < (size_t)L->E ? (L->n - b * (size_t)L->E) : (size_t)L->E;
  const int W = L->W, bits = L->bits, U = L->is64 ? 64 : 32;
  const uint64_t mask = word_mask(W);
  uint8_t* words = out + L->exp_bytes + b * L->block_bytes;

  /* block max of |x|; std::max(a, b) = (a < b) ? b : a, so NaN is skipped */
  int ex;
  if (L->is64) {
    const double* x = (const double*)data + b * (size_t)L->E;
    double in_max = 0;
    for (size_t i = 0; i < cnt; ++i) {
      const double a = fabs(x[i]);
      in_max = (in_max < a) ? a : in_max;
    }
    ex = frsz2o_exponent_f64(in_max);
  } else {
    const float* x = (const float*)data + b * (size_t)L->E;
    float in_max = 0;
    for (size_t i = 0; i < cnt; ++i) {
      const float a = fabsf(x[i]);
      in_max = (in_max < a) ? a : in_max;
    }
    ex = frsz2o_exponent_f32(in_max);
  }
  /* exponents_[b] = max_exp, stored as exp_type (signed W-bit) */
  const int64_t be = wrap_signed(ex, W);
  store_word(out + b * (size_t)(W / 8), W, (uint64_t)be);
  const int16_t be16 = (int16_t)be; /* floating_to_fixed takes std::int16_t */

  uint64_t overlap = 0;
  for (size_t k = 0; k < cnt; ++k) {
    const int o = (int)((k * (size_t)bits) % (size_t)W);
    const size_t s = (k * (size_t)bits) / (size_t)W;
    uint64_t r = L->is64 ? frsz2o_floating_to_fixed_f64(((const double*)data)[b * (size_t)L->E + k], be16)
                         : frsz2o_floating_to_fixed_f32(((const float*)data)[b * (size_t)L->E + k], be16);
    const uint64_t cv = r >> (U - bits); /* uint_fp_to_compressed (frsz2.hpp:555-558) */
    /* write_shift_value (frsz2.hpp:565-576, 629-644) */
    uint64_t t0, t1;
    if (W == bits) {
      t0 = cv;
      t1 = 0;
    } else {
      t0 = (cv << o) & mask;
      t1 = (W < bits + o) ? ((cv >> (W - o)) & mask) : 0;
    }
    if (W == bits) {
      store_word(words + s * (size_t)(W / 8), W, t0);
    } else if (o == 0) {
      overlap = t0;
    } else if (o + bits < W) {
      overlap |= t0;
    } else {
      overlap |= t0;
      store_word(words + s * (size_t)(W / 8), W, overlap);
      overlap = t1;
    }
  }
  if (W != bits && cnt > 0) {
    const int lo = (int)(((cnt - 1) * (size_t)bits) % (size_t)W);
    const size_t ls = ((cnt - 1) * (size_t)bits) / (size_t)W;
    if (lo + bits != W) {
      const size_t idx = (lo + bits < W) ? ls : ls + 1;
      store_word(words + idx * (size_t)(W / 8), W, overlap);
    }
  }
}

/* retrieve_shift_value + compressed_to_uint_fp + fixed_to_floating for one
 * element (frsz2.hpp:550-553, 580-603, 1229-1239). */
static void decompress_one(const layout_t* L, const uint8_t* in, size_t b, size_t k, void* out_elem)
{
  const int W = L->W, bits = L->bits, U = L->is64 ? 64 : 32;
  const uint8_t* words = in + L->exp_bytes + b * L->block_bytes;
  const int64_t be = wrap_signed((int64_t)load_word(in + b * (size_t)(W / 8), W), W);
  const int o = (int)((k * (size_t)bits) % (size_t)W);
  const size_t byte_off = ((k * (size_t)bits) / (size_t)W) * (size_t)(W / 8);
  const uint64_t w0 = load_word(words + byte_off, W);
  uint64_t res;
  if (W == bits) {
    res = w0;
  } else {
    res = w0 >> o;
    if (W < bits + o) res |= load_word(words + byte_off + (size_t)(W / 8), W) << (W - o);
    res &= word_mask(W);
  }
  uint64_t local = res << (U - bits);
  if (!L->is64) local &= 0xFFFFFFFFull;
  if (L->is64)
    *(double*)out_elem = frsz2o_fixed_to_floating_f64(local, be);
  else
    *(float*)out_elem = frsz2o_fixed_to_floating_f32((uint32_t)local, be);
}

static void decompress_block(const layout_t* L, const uint8_t* in, size_t b, void* out)
{
  const size_t base = b * (size_t)L->E;
  const size_t cnt = (L->n - base) < (size_t)L->E ? (L->n - base) : (size_t)L->E;
  for (size_t k = 0; k < cnt; ++k) {
    if (L->is64)
      decompress_one(L, in, b, k, (double*)out + base + k);
    else
      decompress_one(L, in, b, k, (float*)out + base + k);
  }
}

/* ------------------------------------------------------------- whole array */

int frsz2o_compress_f32(const float* in, size_t n, int bits, int block_size, uint8_t* out)
{
  layout_t L;
  if (make_layout(&L, 0, n, bits, block_size)) return 2;
  for (size_t b = 0; b < L.nb; ++b) compress_block(&L, in, b, out);
  return 0;
}
int frsz2o_compress_f64(const double* in, size_t n, int bits, int block_size, uint8_t* out)
{
  layout_t L;
  if (make_layout(&L, 1, n, bits, block_size)) return 2;
  for (size_t b = 0; b < L.nb; ++b) compress_block(&L, in, b, out);
  return 0;
}
int frsz2o_decompress_f32(const uint8_t* in, size_t n, int bits, int block_size, float* out)
{
  layout_t L;
  if (make_layout(&L, 0, n, bits, block_size)) return 2;
  for (size_t b = 0; b < L.nb; ++b) decompress_block(&L, in, b, out);
  return 0;
}
int frsz2o_decompress_f64(const uint8_t* in, size_t n, int bits, int block_size, double* out)
{
  layout_t L;
  if (make_layout(&L, 1, n, bits, block_size)) return 2;
  for (size_t b = 0; b < L.nb; ++b) decompress_block(&L, in, b, out);
  return 0;
}

float frsz2o_decompress_element_f32(const uint8_t* in, size_t n, int bits, int block_size, size_t idx)
{
  layout_t L;
  float v = 0;
  if (make_layout(&L, 0, n, bits, block_size) || idx >= n) return v;
  decompress_one(&L, in, idx / (size_t)block_size, idx % (size_t)block_size, &v);
  return v;
}
double frsz2o_decompress_element_f64(const uint8_t* in, size_t n, int bits, int block_size, size_t idx)
{
  layout_t L;
  double v = 0;
  if (make_layout(&L, 1, n, bits, block_size) || idx >= n) return v;
  decompress_one(&L, in, idx / (size_t)block_size, idx % (size_t)block_size, &v);
  return v;
}

/* ------------------------------------------------------------- threaded */

typedef struct {
  const layout_t* L;
  const void* in;
  void* out;
  size_t b0, b1;
  int compress;
} job_t;

static void* run_job(void* p)
{
  const job_t* j = (const job_t*)p;
  for (size_t b = j->b0; b < j->b1; ++b) {
    if (j->compress)
      compress_block(j->L, j->in, b, (uint8_t*)j->out);
    else
      decompress_block(j->L, (const uint8_t*)j->in, b, j->out);
  }
  return NULL;
}

static int run_mt(const layout_t* L, const void* in, void* out, int threads, int compress)
{
  if (threads < 1) threads = 1;
  if (threads > 256) threads = 256;
  pthread_t tid[256];
  int created[256];
  job_t jobs[256];
  const size_t per = (L->nb + (size_t)threads - 1) / (size_t)threads;
  for (int t = 0; t < threads; ++t) {
    jobs[t].L = L;
    jobs[t].in = in;
    jobs[t].out = out;
    jobs[t].b0 = (size_t)t * per < L->nb ? (size_t)t * per : L->nb;
    jobs[t].b1 = jobs[t].b0 + per < L->nb ? jobs[t].b0 + per : L->nb;
    jobs[t].compress = compress;
    created[t] = pthread_create(&tid[t], NULL, run_job, &jobs[t]) == 0;
    if (!created[t]) run_job(&jobs[t]);
  }
  for (int t = 0; t < threads; ++t)
    if (created[t]) pthread_join(tid[t], NULL);
  return 0;
}

int frsz2o_compress_mt(int dtype_is_f64, const void* in, size_t n, int bits, int block_size, uint8_t* out, int threads)
{
  layout_t L;
  if (make_layout(&L, dtype_is_f64 ? 1 : 0, n, bits, block_size)) return 2;
  return run_mt(&L, in, out, threads, 1);
}
int frsz2o_decompress_mt(int dtype_is_f64, const uint8_t* in, size_t n, int bits, int block_size, void* out, int threads)
{
  layout_t L;
  if (make_layout(&L, dtype_is_f64 ? 1 : 0, n, bits, block_size)) return 2;
  return run_mt(&L, in, out, threads, 0);
}
