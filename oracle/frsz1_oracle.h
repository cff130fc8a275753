/*
 * frsz1_oracle.h -- CPU restatement of the reference's legacy "frsz" codec
 * (the LibPressio plugin of src/frsz.cc: epsilon quantization and int16
 * deltas within blocks of 256 values).
 *
 * TEST INFRASTRUCTURE ONLY, like frsz2_oracle.h: only tests/ (and bench.py's
 * baseline leg) may load it; the product never does.
 *
 * Parity: src/frsz.cc cannot be compiled here (it needs LibPressio), so this
 * restatement is pinned to the reference test's known answer
 * (test/test_frsz.cc:29-46) and otherwise follows the source line by line.
 *
 * compress (src/frsz.cc:103-130), T = float or double:
 *   q[i]  = (T) round_half_away((double) x[i] * (1.0 / (2 * epsilon)))
 *   d[i]  = q[i] - (i % 256 == 0 ? 0 : q[i - 1])        (in T)
 *   out[i] = int16 saturate(d[i]) (truncation; a NaN delta, undefined in
 *            the reference, gives 0 as its x86 builds do)
 * decompress (src/frsz.cc:132-150), per block b of 256 values:
 *   y[256b]     = (T) ((double)(T) in[256b] * (2 * epsilon))
 *   y[256b + i] = (T) ((double)(T) in[k] * (2 * epsilon) + (double) y[256b + i - 1])
 * with k = i in the reference (every block reads block 0's deltas, the
 * source's indexing) or k = 256b + i with `own_deltas` set.
 */
#ifndef FRSZ1_ORACLE_H
#define FRSZ1_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

void frsz1o_compress_f32(const float* x, size_t n, double epsilon, int16_t* out);
void frsz1o_compress_f64(const double* x, size_t n, double epsilon, int16_t* out);
void frsz1o_decompress_f32(const int16_t* in, size_t n, double epsilon, int own_deltas, float* y);
void frsz1o_decompress_f64(const int16_t* in, size_t n, double epsilon, int own_deltas, double* y);

#ifdef __cplusplus
}
#endif

#endif
