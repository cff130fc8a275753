/*
 * frsz1_oracle.c -- CPU restatement of the legacy "frsz" codec
 * (src/frsz.cc:103-150).  TEST INFRASTRUCTURE ONLY; see frsz1_oracle.h.
 * Compiled without floating-point contraction, as the reference's x86-64
 * build evaluates it (separate multiply and add, in double).
 */
#include "frsz1_oracle.h"

#include <math.h>

enum { FRSZ1_BLOCK = 256 }; /* src/frsz.cc:103, 132 (BLOCK = 256) */

/* saturate<int16_t> (src/frsz.cc:97-101): clamp, then truncate toward zero;
 * NaN (no comparison holds; the conversion is undefined in C++) -> 0, the
 * value x86 code produces (cvtt to int32 gives 0x80000000, low 16 bits 0). */
static int16_t saturate_i16(double d)
{
  if (d < -32768.0) return INT16_MIN;
  if (d > 32767.0) return INT16_MAX;
  if (d != d) return 0;
  return (int16_t)d;
}

/* src/frsz.cc:113-129: quantize, then the difference to the previous
 * quantized value within the block, both in T. */
void frsz1o_compress_f32(const float* x, size_t n, double epsilon, int16_t* out)
{
  const double inv = 1.0 / (epsilon * 2.0);
  float prev = 0.0f;
  for (size_t i = 0; i < n; ++i) {
    const float q = (float)round((double)x[i] * inv);
    const float delta = q - ((i % FRSZ1_BLOCK == 0) ? 0.0f : prev);
    out[i] = saturate_i16((double)delta);
    prev = q;
  }
}

void frsz1o_compress_f64(const double* x, size_t n, double epsilon, int16_t* out)
{
  const double inv = 1.0 / (epsilon * 2.0);
  double prev = 0.0;
  for (size_t i = 0; i < n; ++i) {
    const double q = round(x[i] * inv);
    const double delta = q - ((i % FRSZ1_BLOCK == 0) ? 0.0 : prev);
    out[i] = saturate_i16(delta);
    prev = q;
  }
}

/* src/frsz.cc:135-148: per block, the first value, then a running sum in
 * double rounded to T at every step.  The reference reads quantized[i] with i
 * the index within the block (so every block adds block 0's deltas);
 * own_deltas reads the block's own. */
void frsz1o_decompress_f32(const int16_t* in, size_t n, double epsilon, int own_deltas, float* y)
{
  const double ebx2 = epsilon * 2;
  for (size_t b = 0; b * FRSZ1_BLOCK < n; ++b) {
    const size_t g0 = b * FRSZ1_BLOCK;
    y[g0] = (float)((double)(float)in[g0] * ebx2);
    for (size_t i = 1; i < FRSZ1_BLOCK && g0 + i < n; ++i) {
      const size_t k = own_deltas ? g0 + i : i;
      y[g0 + i] = (float)((double)(float)in[k] * ebx2 + (double)y[g0 + i - 1]);
    }
  }
}

void frsz1o_decompress_f64(const int16_t* in, size_t n, double epsilon, int own_deltas, double* y)
{
  const double ebx2 = epsilon * 2;
  for (size_t b = 0; b * FRSZ1_BLOCK < n; ++b) {
    const size_t g0 = b * FRSZ1_BLOCK;
    y[g0] = (double)in[g0] * ebx2;
    for (size_t i = 1; i < FRSZ1_BLOCK && g0 + i < n; ++i) {
      const size_t k = own_deltas ? g0 + i : i;
      y[g0 + i] = (double)in[k] * ebx2 + y[g0 + i - 1];
    }
  }
}
