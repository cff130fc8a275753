/*
 * frsz2_oracle.h -- CPU restatement of the FRSZ2 fixed-rate codec.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA
 * implementation in frsz_b200/: only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py may load it.  The product library never links,
 * loads or calls it, and there is no CPU fallback built on it.
 *
 * Parity is pinned: tests/test_oracle.py checks this restatement byte-for-byte
 * against the reference's own frsz2.hpp compiled as oracle/_ref/libfrsz2_ref.so
 * (recipe: oracle/Makefile), and against the known answers of the reference's
 * tests (test/test_frsz_gpu.cu:88-158, 213-229, 276-301, 382-441).
 *
 * Every function mirrors frsz::frsz2_compressor<bits, E, T> from the
 * reference's include/frsz2.hpp, with bits / E / T as runtime arguments.
 *
 * Byte layout (include/frsz2.hpp:525-548):
 *   [nb exponents, each a signed W-bit integer]
 *   [pad to the next multiple of 256 bytes; a full 256 B when already aligned]
 *   [nb blocks of ceil(E*bits/W) W-bit words, LSB-first bit packing]
 * with nb = ceil(n/E) and W = 8/16/32/64 for bits <= 8/16/32/64.
 */
#ifndef FRSZ2_ORACLE_H
#define FRSZ2_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* W: storage word width in bits for a given bits-per-value (frsz2.hpp:258-262). */
int frsz2o_word_bits(int bits);
/* Compressed block size in bytes (frsz2.hpp:526-529). */
size_t frsz2o_block_bytes(int bits, int block_size);
/* Exponent region including the 256-byte pad (frsz2.hpp:534-540). */
size_t frsz2o_exponent_bytes(int bits, int block_size, size_t n);
/* Whole buffer (frsz2.hpp:542-548). */
size_t frsz2o_compressed_bytes(int bits, int block_size, size_t n);

/* Primitives (frsz2.hpp:312-399).  exponent() returns the reference's
 * float_traits<T>::exponent_t value widened to int. */
int frsz2o_exponent_f32(float x);
int frsz2o_exponent_f64(double x);
uint32_t frsz2o_significand_f32(float x);
uint64_t frsz2o_significand_f64(double x);
int frsz2o_sign_f32(float x);
int frsz2o_sign_f64(double x);
uint32_t frsz2o_floating_to_fixed_f32(float x, int16_t block_exponent);
uint64_t frsz2o_floating_to_fixed_f64(double x, int16_t block_exponent);
float frsz2o_fixed_to_floating_f32(uint32_t fixed, int64_t block_exponent);
double frsz2o_fixed_to_floating_f64(uint64_t fixed, int64_t block_exponent);

/* Whole-array codec (compress_cpu_impl frsz2.hpp:1181-1193,
 * decompress_cpu_impl frsz2.hpp:1242-1249).  `out` must hold
 * frsz2o_compressed_bytes(); bytes the reference never writes (the pad and the
 * unused tail words of a partial last block) are left untouched.
 * Return 0, or 2 for an unsupported bits / block size. */
int frsz2o_compress_f32(const float* in, size_t n, int bits, int block_size, uint8_t* out);
int frsz2o_compress_f64(const double* in, size_t n, int bits, int block_size, uint8_t* out);
int frsz2o_decompress_f32(const uint8_t* in, size_t n, int bits, int block_size, float* out);
int frsz2o_decompress_f64(const uint8_t* in, size_t n, int bits, int block_size, double* out);

/* Random access (decompress_cpu_element frsz2.hpp:1199-1214). */
float frsz2o_decompress_element_f32(const uint8_t* in, size_t n, int bits, int block_size, size_t idx);
double frsz2o_decompress_element_f64(const uint8_t* in, size_t n, int bits, int block_size, size_t idx);

/* Same codec, block ranges split over `threads` POSIX threads (bench.py's
 * cpu_baseline when the reference library is not present). */
int frsz2o_compress_mt(int dtype_is_f64, const void* in, size_t n, int bits, int block_size, uint8_t* out, int threads);
int frsz2o_decompress_mt(int dtype_is_f64, const uint8_t* in, size_t n, int bits, int block_size, void* out, int threads);

#ifdef __cplusplus
}
#endif

#endif
