/*
 * frsz2_b200.h -- C ABI of the B200 FRSZ2 fixed-rate codec (libfrsz2_b200.so).
 *
 * Plain pointers and sizes only.  `stream` is a cudaStream_t passed as void*
 * (NULL = the legacy default stream).  Every entry point returns a status:
 *
 *   FRSZ2_OK        0  success
 *   FRSZ2_EDTYPE    1  unsupported dtype            (src/frsz2.cc:164, 181: set_error(1, "unsupported dtype"))
 *   FRSZ2_EFAIL     2  unsupported bits / block size, bad argument or CUDA
 *                      failure                       (src/frsz2.cc:166-168, 183-185: set_error(2, what))
 *
 * and frsz2_last_error() gives the calling thread's last message, with the
 * reference's wording for unsupported values ("Unsupported number of bits: N",
 * "Unsupported exponent block size: N", include/frsz2.hpp:1300, 1326).
 *
 * The compressed format is byte-identical to the reference's
 * frsz::frsz2_compressor<bits, block_size, T> (include/frsz2.hpp:504-1256):
 *   [ceil(n/E) exponents, signed W-bit] [pad to next 256 B multiple, full 256 B
 *   if aligned] [ceil(n/E) blocks of ceil(E*bits/W) W-bit words, LSB-first]
 * with W = 8/16/32/64 for bits <= 8/16/32/64.  Bytes the reference never
 * writes (the pad, unused tail words of a partial last block) are left as the
 * caller's buffer had them.
 *
 * Valid arguments: dtype FRSZ2_FLOAT with 4 <= bits <= 32, FRSZ2_DOUBLE with
 * 4 <= bits <= 64 (static_asserts include/frsz2.hpp:511-517); 1 <= block_size
 * <= 65536.  Device pointers must be aligned to their element / word type.
 * Speed: power-of-two block sizes from 8 (fp32) / 4 (fp64) values up with a
 * 32-byte aligned buffer run at about the HBM bandwidth; values off the
 * 32-byte layout (a view such as x + 1) at 0.7-0.9 of it; block sizes 3, 5, 6,
 * 7 and 12 at 0.74-1.0, other block sizes up to 16 values at 0.4-0.8; block
 * sizes that are a multiple of 8 (fp32) / 4 (fp64) values without block
 * padding decompress at about the HBM bandwidth and compress at 0.75-1.0 (up
 * to 256 / 128 values), multiples of 4 / 2 decompress at about the HBM
 * bandwidth and compress at 0.55-0.7; other block sizes of 17-128 values decompress at
 * 0.33-0.89 and compress at 0.2-0.7; larger block sizes that are not powers of
 * two, or a buffer off the 32-byte layout, on slower general kernels.
 */
#ifndef FRSZ2_B200_H
#define FRSZ2_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FRSZ2_OK 0
#define FRSZ2_EDTYPE 1
#define FRSZ2_EFAIL 2

/* Element types: the two dtypes the plugin's compress/decompress switch
 * accepts (src/frsz2.cc:157-163, 174-179). */
#define FRSZ2_FLOAT 0
#define FRSZ2_DOUBLE 1

/* Replaces frsz.h:1 `extern "C" void register_frsz();` (empty body,
 * src/frsz.cc:11-13): a link anchor kept with the same name and signature. */
void register_frsz(void);

/* Library version; the plugin reports 0.0.2 (src/frsz2.cc:188-192). */
const char* frsz2_version(void);

/* Message for the calling thread's last non-zero status. */
const char* frsz2_last_error(void);

/* Replaces frsz2_compressor<bits,E,T>::compute_compressed_memory_size_byte
 * (include/frsz2.hpp:542-548) and compute_exponent_block_size_byte
 * (include/frsz2.hpp:534-540), with bits / E / T chosen at run time. */
int frsz2_compressed_size(int dtype, int bits, int block_size, uint64_t n, uint64_t* total_bytes);
int frsz2_exponent_size(int dtype, int bits, int block_size, uint64_t n, uint64_t* exponent_bytes);

/* Device buffers, stream-ordered, asynchronous.
 * Replaces frsz2_compressor<bits,E,T>::compress_cpu_impl (include/frsz2.hpp:1181-1193)
 * as reached from dispatch_frsz2_compression (include/frsz2.hpp:1346) and the
 * plugin's compress_impl (src/frsz2.cc:152-169), and the reference GPU kernel
 * compress_gpu (include/frsz2.hpp:1259-1274).  `d_compressed` holds
 * frsz2_compressed_size() bytes. */
int frsz2_compress(int dtype, int bits, int block_size, const void* d_values, uint64_t n, void* d_compressed,
                   void* stream);

/* Replaces decompress_cpu_impl (include/frsz2.hpp:1242-1249) via
 * dispatch_frsz2_decompression (include/frsz2.hpp:1347) and the plugin's
 * decompress_impl (src/frsz2.cc:171-186), and the reference GPU kernel
 * decompress_gpu (include/frsz2.hpp:1276-1288). */
int frsz2_decompress(int dtype, int bits, int block_size, const void* d_compressed, uint64_t n, void* d_values,
                     void* stream);

/* Host buffers: the same codec with the host<->device copies inside the call
 * (pinned memory recommended; pageable works).  Synchronous: returns when the
 * result is in host memory.  This is the drop-in for the reference's host-side
 * compress_cpu_impl / decompress_cpu_impl calls. */
int frsz2_compress_host(int dtype, int bits, int block_size, const void* h_values, uint64_t n, void* h_compressed,
                        void* stream);
int frsz2_decompress_host(int dtype, int bits, int block_size, const void* h_compressed, uint64_t n, void* h_values,
                          void* stream);

/* Blocks [block_begin, block_begin + block_count) of an array of n values,
 * written into / read from the WHOLE array's compressed buffer `d_compressed`
 * (its own exponent slots and block words, nothing else).  `d_values` points at
 * the value of the first block (block_begin * block_size).  The range analogue
 * of compress_cpu_block / decompress_cpu_block (include/frsz2.hpp:1108-1179,
 * 1217-1240): ranks or streams that own disjoint block ranges of one array can
 * work on it independently. */
int frsz2_compress_blocks(int dtype, int bits, int block_size, const void* d_values, uint64_t n, uint64_t block_begin,
                          uint64_t block_count, void* d_compressed, void* stream);
int frsz2_decompress_blocks(int dtype, int bits, int block_size, const void* d_compressed, uint64_t n,
                            uint64_t block_begin, uint64_t block_count, void* d_values, void* stream);

/* Random-access decode of `count` elements at device indices d_idx[0..count)
 * into d_out (device buffers), for host code.  The device-side accessor
 * decompress_gpu_element (include/frsz2.hpp:1096-1104) for use inside kernels
 * is include/frsz2_b200_device.cuh.  Values are bit-exact with the CPU decode
 * (decompress_cpu_element), including the zero code rule, which the reference
 * GPU element decode does not follow.  Indices >= n leave their output
 * untouched. */
int frsz2_decompress_elements(int dtype, int bits, int block_size, const void* d_compressed, uint64_t n,
                              const uint64_t* d_idx, uint64_t count, void* d_out, void* stream);

/* The same on HOST buffers: the compressed array, the indices and the outputs
 * in host memory (decompress_cpu_element, include/frsz2.hpp:1199-1214).  Only
 * the blocks that hold a requested index are copied to the GPU, decoded there
 * and the values copied back; the call returns when h_out is written.
 * Indices >= n leave their output untouched. */
int frsz2_decompress_elements_host(int dtype, int bits, int block_size, const void* h_compressed, uint64_t n,
                                   const uint64_t* h_idx, uint64_t count, void* h_out);

/* ---------------------------------------------------------------------------
 * Batched path: no counterpart in the reference (which compresses one array
 * per call).  Many arrays of mixed float types, widths, block sizes and sizes
 * run as one CUDA graph launch: a kernel per (float type, width) class present,
 * side by side, over its class's work list in device memory -- one CTA per
 * tile (the default) or a persistent grid.  The launch configuration (one CTA
 * per tile or persistent; threads per CTA, rows per warp, resident CTAs per SM;
 * classes side by side or one after another) comes from an autotuner that
 * times the candidates on the plan's own arrays, or from
 * frsz2_batch_configure.  Arrays the persistent
 * kernels cannot take (block sizes that are not powers of two, block padding,
 * misaligned pointers) get their own launch inside the same graph.  All
 * pointers are device pointers; a plan keeps its descriptors in device memory
 * until destroyed.
 */
typedef struct frsz2_batch_item {
  int dtype;              /* FRSZ2_FLOAT / FRSZ2_DOUBLE */
  int bits;
  int block_size;
  uint64_t n;
  const void* values;     /* compress input (may be NULL for a decompress-only plan) */
  void* decompressed;     /* decompress output (may be NULL for a compress-only plan; may equal values) */
  void* compressed;       /* frsz2_compressed_size() bytes */
} frsz2_batch_item;

typedef struct frsz2_batch frsz2_batch;

typedef struct frsz2_batch_stats {
  uint64_t arrays;            /* items in the plan */
  uint64_t persistent_arrays; /* items served by the persistent kernels */
  uint64_t separate_launches; /* items with their own launch in the graph */
  uint64_t classes;           /* (float type, width) classes = persistent kernels */
  uint64_t tiles[2];          /* persistent-kernel tiles [decompress, compress] */
  int threads_per_cta[2];
  int rows_per_warp[2];
  int ctas_per_sm[2];
  int side_by_side[2];        /* 1: classes run concurrently, 0: one after another */
  int tuned[2];
  int one_cta_per_tile[2];    /* 1: one CTA per tile, 0: persistent kernels per class */
} frsz2_batch_stats;

int frsz2_batch_create(const frsz2_batch_item* items, uint64_t count, frsz2_batch** plan);
int frsz2_batch_compress(frsz2_batch* plan, void* stream);
int frsz2_batch_decompress(frsz2_batch* plan, void* stream);
/* Times every launch shape on the plan's arrays for one direction (compress != 0
 * or decompress), keeps the fastest and rebuilds that direction's graph.  The
 * run writes the plan's outputs like a normal call.  *best_ms may be NULL. */
int frsz2_batch_autotune(frsz2_batch* plan, int compress, void* stream, float* best_ms);
/* Sets one direction's launch configuration by hand, as frsz2_batch_autotune
 * would (for instance a configuration tuned once offline): shape 0..2 (256 x 2,
 * 128 x 2, 512 x 1 threads x rows per warp), resident CTAs per SM, classes side
 * by side (1) or one after another (0), and one CTA per tile (1, shape 0 only)
 * instead of the persistent kernel per class (0).  Rebuilds that direction's
 * graph; returns 2 for a configuration the plan cannot run. */
int frsz2_batch_configure(frsz2_batch* plan, int compress, int shape, int ctas_per_sm, int side_by_side,
                          int one_cta_per_tile);
int frsz2_batch_info(const frsz2_batch* plan, frsz2_batch_stats* stats);
void frsz2_batch_destroy(frsz2_batch* plan);

/* Batched compress that allocates nothing (no counterpart in the reference).
 * For callers that may not allocate device memory at call time -- an
 * application whose allocator already owns the GPU's memory, or a request path
 * where a cudaMalloc is not allowed.  Same output as a plan built from the same
 * items and run with frsz2_batch_compress; `items` is host memory and the
 * `decompressed` fields are ignored.  The descriptor work list lives in a fixed
 * device array of the library (4096 arrays at most per call; larger calls
 * return 2), held by every GPU that loads the library until exit, shared by
 * all calls: calls whose work overlaps on the GPU (other streams or threads)
 * race; calls on one stream are ordered.  The descriptors reach the array
 * through kernel parameters, so no host copy is kept between calls.  The first
 * call on each device sets the array up (looks up its device address, which
 * is kept for the process); make it before any stream capture.  Calls after
 * cudaDeviceReset on that device are not supported. */
int frsz2_batch_compress_static(const frsz2_batch_item* items, uint64_t count, void* stream);

/* ---------------------------------------------------------------------------
 * Decompression fused into its consumer over a compressed basis of m fp64
 * vectors of n values (the Krylov-basis use of decompress_gpu_element,
 * include/frsz2.hpp:1096-1104, where a solver reads the basis through the
 * accessor): values are decoded in registers and fed to the FMAs.  `basis` is a
 * HOST array of m device pointers to compressed buffers (32-byte aligned), all
 * with the same bits / block_size / n.  Widths 16, 21, 24, 32, 48, 64; block
 * sizes that are powers of two without block padding; m <= FRSZ2_MAX_BASIS.
 *
 * frsz2_basis_dot:  h[j] = sum_i V_j[i] * w[i], j < m.  `workspace` is device
 *   memory of frsz2_basis_workspace_size(m, n) bytes (m sums per slice of
 *   3,072 values), 256-byte aligned, zero on first use (the call leaves it
 *   ready for the next one); the result does not depend on scheduling.  Calls
 *   sharing a workspace must not overlap.  At 64 bits the codes stream
 *   through shared memory by bulk asynchronous copies; a copy that has not
 *   landed after 2 s (a device fault, never normal operation) makes every
 *   h[j] of that call NaN.
 * frsz2_basis_axpy: y[i] += sum_j c[j] * V_j[i] (j in order), c and y device
 *   memory, y 32-byte aligned.
 */
#define FRSZ2_MAX_BASIS 256
uint64_t frsz2_basis_workspace_size(int m, uint64_t n);
int frsz2_basis_dot(int dtype, int bits, int block_size, const void* const* basis, int m, uint64_t n,
                    const void* w, void* h, void* workspace, uint64_t workspace_bytes, void* stream);
int frsz2_basis_axpy(int dtype, int bits, int block_size, const void* const* basis, int m, uint64_t n,
                     const void* coef, void* y, void* stream);

/* ---------------------------------------------------------------------------
 * Request server: no counterpart in the reference.  Compress / decompress
 * requests of any size arrive over time (arrival_ns, CLOCK_MONOTONIC as
 * returned by frsz2_now_ns; 0 = at submission).  A worker thread admits
 * eligible requests in arrival order into batches -- skipping, within a
 * bounded window, requests whose output does not fit the memory budget right
 * now -- and launches each batch on a free stream as soon as one exists, so
 * requests that arrive while others run overlap with them on the device.
 * Outputs go to the caller's `output` or, when it is NULL, to the server's
 * arena of `memory_budget` bytes, where they stay until frsz2_server_release
 * (or until completion with FRSZ2_REQ_RELEASE_ON_COMPLETION).  A request's
 * result is the same as a plain frsz2_compress / frsz2_decompress of it.
 * Completion statuses: 0 ok, 1 / 2 as elsewhere (including "request output
 * larger than the server's memory budget"), 3 cancelled before admission.
 */
#define FRSZ2_ECANCELLED 3
#define FRSZ2_OP_COMPRESS 0
#define FRSZ2_OP_DECOMPRESS 1
#define FRSZ2_REQ_RELEASE_ON_COMPLETION 1u
#define FRSZ2_REQ_ARRIVAL_RELATIVE 2u /* arrival_ns is an offset from the submit call */

typedef struct frsz2_server frsz2_server;

typedef struct frsz2_request {
  int op;               /* FRSZ2_OP_COMPRESS / FRSZ2_OP_DECOMPRESS */
  int dtype;
  int bits;
  int block_size;
  uint64_t n;           /* values */
  const void* input;    /* device: values (compress) or compressed buffer (decompress) */
  void* output;         /* device, or NULL to allocate from the server's arena */
  uint64_t arrival_ns;  /* eligible from this time on; 0 = at submission */
  uint32_t flags;       /* FRSZ2_REQ_* */
  uint32_t reserved;
} frsz2_request;

typedef struct frsz2_completion {
  uint64_t id;
  int status;
  int op;
  void* output;          /* where the result is */
  uint64_t output_bytes; /* arena bytes held until released (0 if none) */
  uint64_t bytes;        /* algorithmic bytes moved */
  uint64_t arrival_ns, admit_ns, done_ns;
} frsz2_completion;

typedef struct frsz2_server_counters {
  uint64_t completed, failed, batches, bytes, pending;
  uint64_t budget_bytes, arena_used_bytes, arena_peak_bytes;
  uint64_t max_batch, max_inflight_output_bytes;
} frsz2_server_counters;

uint64_t frsz2_now_ns(void);
int frsz2_server_create(uint64_t memory_budget, int max_batch, int streams, frsz2_server** server);
int frsz2_server_submit(frsz2_server* server, const frsz2_request* requests, uint64_t count, uint64_t* first_id);
int frsz2_server_cancel(frsz2_server* server, uint64_t id);
/* Up to `max` completions; waits up to wait_ms for the first one. */
int frsz2_server_poll(frsz2_server* server, frsz2_completion* out, uint64_t max, uint64_t* count, int wait_ms);
int frsz2_server_release(frsz2_server* server, uint64_t id);
int frsz2_server_stats(frsz2_server* server, frsz2_server_counters* stats);
void frsz2_server_destroy(frsz2_server* server);

/* ---------------------------------------------------------------------------
 * The reference's legacy "frsz" codec (the LibPressio plugin "frsz",
 * src/frsz.cc:15-165): values quantized with step 2*epsilon and stored as
 * int16 differences to the previous quantized value within blocks of 256
 * values; frsz1_compressed_size(n) = 2n bytes.  Device buffers,
 * stream-ordered.  compress / decompress follow compress_1d / decompress_1d
 * (src/frsz.cc:103-150) bit for bit; a NaN difference, undefined there, is
 * stored as 0.  dtype FRSZ2_FLOAT / FRSZ2_DOUBLE (else FRSZ2_EDTYPE with the
 * reference's message), epsilon > 0 (the plugin's "frsz:epsilon", default
 * 1e-4).  decompress as the reference adds block 0's differences in every
 * block (its decompress_1d reads quantized[i] with i the index within the
 * block); flags FRSZ1_OWN_DELTAS adds each block's own, the inverse of
 * compress.
 */
#define FRSZ1_OWN_DELTAS 1
uint64_t frsz1_compressed_size(uint64_t n);
int frsz1_compress(int dtype, double epsilon, const void* d_values, uint64_t n, void* d_out, void* stream);
int frsz1_decompress(int dtype, double epsilon, const void* d_compressed, uint64_t n, void* d_values, int flags,
                     void* stream);

#ifdef __cplusplus
}
#endif

#endif /* FRSZ2_B200_H */
