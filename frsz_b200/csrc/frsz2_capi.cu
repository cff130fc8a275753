// frsz2_capi.cu -- C ABI of libfrsz2_b200.so: argument checks, kernel choice,
// launch geometry, and the host-buffer path with pipelined copies.
#include "frsz2_blockvec.cuh"
#include "frsz2_blockwise.cuh"
#include "frsz2_chunked.cuh"
#include "frsz2_chunked_ct.cuh"
#include "frsz2_fast_dispatch.hpp"
#include "frsz2_kernels.cuh"
#include "frsz2_launch.hpp"

#include "../../include/frsz2_b200.h"

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

namespace frsz2b {

namespace {
thread_local std::string g_last_error;
}

int set_error(int code, const std::string& msg)
{
  g_last_error = msg;
  return code;
}

const char* last_error() { return g_last_error.c_str(); }

int cuda_status(cudaError_t e, const char* what)
{
  if (e == cudaSuccess) return FRSZ2_OK;
  return set_error(FRSZ2_EFAIL, std::string(what) + ": " + cudaGetErrorString(e));
}

int check_args(int dtype, int bits, int E)
{
  if (dtype != FRSZ2_FLOAT && dtype != FRSZ2_DOUBLE) return set_error(FRSZ2_EDTYPE, "unsupported dtype");
  const int max_bits = dtype == FRSZ2_FLOAT ? 32 : 64;
  if (bits < 4 || bits > max_bits) return set_error(FRSZ2_EFAIL, "Unsupported number of bits: " + std::to_string(bits));
  if (E < 1 || E > kMaxBlockSize)
    return set_error(FRSZ2_EFAIL, "Unsupported exponent block size: " + std::to_string(E));
  return FRSZ2_OK;
}

int sm_count()
{
  // per device, queried once (threads racing on the first call store the
  // same value)
  static std::atomic<int> cached[64];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
  int c = cached[dev].load(std::memory_order_relaxed);
  if (c == 0) {
    if (cudaDeviceGetAttribute(&c, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || c <= 0) c = 148;
    cached[dev].store(c, std::memory_order_relaxed);
  }
  return c;
}

static bool is_pow2(int x) { return x > 0 && (x & (x - 1)) == 0; }
static int ilog2(int x)
{
  int l = 0;
  while ((1 << l) < x) ++l;
  return l;
}

Job make_job(const Layout& L, int dtype)
{
  Job j{};
  j.n = L.n;
  j.block_bytes = L.block_bytes;
  j.bits = L.bits;
  j.E = L.E;
  j.W = L.W;
  j.log2E = is_pow2(L.E) ? ilog2(L.E) : -1;
  const int TE = dtype == FRSZ2_FLOAT ? tile_shape<float>::TE : tile_shape<double>::TE;
  j.tile_blocks = (L.E <= TE && is_pow2(L.E)) ? (std::uint32_t)(TE / L.E) : 0u;
  j.tiles = (L.n + (std::uint64_t)TE - 1) / (std::uint64_t)TE;
  j.m_bb = L.block_bytes >= 2 ? (std::uint32_t)((((1ull << 32) + L.block_bytes - 1) / L.block_bytes)) : 0u;
  j.m_bits = (std::uint32_t)((((1ull << 32) + (std::uint64_t)L.bits - 1) / (std::uint64_t)L.bits));
  return j;
}

bool tile_eligible(const Job& j, int dtype, const void* values, const void* words)
{
  const int V = dtype == FRSZ2_FLOAT ? tile_shape<float>::V : tile_shape<double>::V;
  const int TE = dtype == FRSZ2_FLOAT ? tile_shape<float>::TE : tile_shape<double>::TE;
  if (!is_pow2(j.E) || j.E < 8 || j.E > TE || j.E < V) return false;
  if (j.block_bytes % 4 != 0) return false;
  if (((std::uint64_t)j.tile_blocks * j.block_bytes) % 16 != 0) return false;
  if (reinterpret_cast<std::uintptr_t>(values) % 16 != 0) return false;
  if (reinterpret_cast<std::uintptr_t>(words) % 16 != 0) return false;
  return true;
}

template<class T>
static std::size_t compress_smem(int bits)
{
  constexpr int TE = tile_shape<T>::TE, V = tile_shape<T>::V;
  const std::size_t cv = (sizeof(T) == 8 && bits > 32) ? 8 : 4;
  return TE * cv + (TE / (32 * V)) * 4;
}

template<class T>
static std::size_t decompress_smem(const Job& j)
{
  const std::uint32_t tile_bytes = j.tile_blocks * j.block_bytes;
  return decompress_tile_exp_offset<T>(tile_bytes) + (std::size_t)j.tile_blocks * 8;
}

static unsigned grid_for(std::uint64_t work_items, std::uint64_t per_cta)
{
  const std::uint64_t need = (work_items + per_cta - 1) / per_cta;
  const std::uint64_t cap = (std::uint64_t)sm_count() * 64;
  return (unsigned)std::max<std::uint64_t>(1, std::min(need, cap));
}

// Compile-time-width kernels when an instance and the layout allow it;
// cudaErrorNotSupported means "use the runtime-width kernels".
template<class T>
static cudaError_t try_fast(bool compress, const Job& j, cudaStream_t s)
{
  const void* values = compress ? j.values_in : j.values_out;
  const unsigned grid = (unsigned)std::min<std::uint64_t>(j.tiles, 1u << 30);
  if (fast_eligible(j, sizeof(T) == 8, values, j.words))
    return sizeof(T) == 8 ? launch_fast_f64(j.bits, compress, j, s, grid)
                          : launch_fast_f32(j.bits, compress, j, s, grid);
  if (small_block_eligible(j, sizeof(T) == 8, values, j.words))
    return sizeof(T) == 8 ? launch_fast_small_f64(j.bits, j.E, compress, j, s, grid)
                          : launch_fast_small_f32(j.bits, j.E, compress, j, s, grid);
  if (fast_mis_eligible(j, sizeof(T) == 8, values, j.words))
    return sizeof(T) == 8 ? launch_fast_mis_f64(j.bits, compress, j, s, grid)
                          : launch_fast_mis_f32(j.bits, compress, j, s, grid);
  if (const std::uint32_t tb = fast_gen_tile_blocks(j, sizeof(T) == 8, values, j.words)) {
    // block sizes that are a multiple of a lane's values: tiles of tb whole blocks
    Job t = j;
    const std::uint64_t tv = (std::uint64_t)tb * (std::uint64_t)j.E;
    t.tile_blocks = tb;
    t.tiles = (j.n + tv - 1) / tv;
    const unsigned g = (unsigned)std::min<std::uint64_t>(t.tiles, 1u << 30);
    return sizeof(T) == 8 ? launch_fast_gen_f64(j.bits, compress, t, s, g)
                          : launch_fast_gen_f32(j.bits, compress, t, s, g);
  }
  return cudaErrorNotSupported;
}


// The blocks of a job from block b0 on (the generic kernel's share when the
// blockvec kernel takes the whole blocks).
static Job job_from_block(const Job& j, std::uint64_t b0, std::size_t es)
{
  Job t = j;
  const std::uint64_t e0 = b0 * (std::uint64_t)j.E;
  t.n = j.n - e0;
  if (j.values_in) t.values_in = static_cast<const std::uint8_t*>(j.values_in) + e0 * es;
  if (j.values_out) t.values_out = static_cast<std::uint8_t*>(j.values_out) + e0 * es;
  t.exps = j.exps + b0 * (std::uint64_t)(j.W / 8);
  t.words = j.words + b0 * (std::uint64_t)j.block_bytes;
  return t;
}

template<class T>
static int launch_compress_t(const Job& j, int dtype, cudaStream_t s, bool* used_tile)
{
  if (j.n == 0) return FRSZ2_OK;
  const cudaError_t fe = try_fast<T>(true, j, s);
  if (fe != cudaErrorNotSupported) {
    if (used_tile) *used_tile = true;
    return cuda_status(fe, "compress launch");
  }
  const bool tile = tile_eligible(j, dtype, j.values_in, j.words);
  if (used_tile) *used_tile = tile;
  if (tile) {
    const unsigned grid = (unsigned)std::min<std::uint64_t>(j.tiles, 1u << 30);
    if (sizeof(T) == 8 && j.bits > 32)
      k_compress_tile<T, std::uint64_t><<<grid, kNT, compress_smem<T>(j.bits), s>>>(j);
    else
      k_compress_tile<T, std::uint32_t><<<grid, kNT, compress_smem<T>(j.bits), s>>>(j);
  } else if (blockwise_eligible(j)) {
    return cuda_status(sizeof(T) == 8 ? launch_blockwise_f64(j.bits, true, j, s)
                                      : launch_blockwise_f32(j.bits, true, j, s),
                       "compress launch");
  } else if (blockvec_eligible(j, sizeof(T), j.values_in, j.words)) {
    const std::uint64_t full = j.n / (std::uint64_t)j.E;
    const cudaError_t e = sizeof(T) == 8 ? launch_blockvec_f64(j.bits, j, full, s)
                                         : launch_blockvec_f32(j.bits, j, full, s);
    if (e != cudaSuccess) return cuda_status(e, "compress launch");
    if (full * (std::uint64_t)j.E < j.n) k_compress_generic<T><<<1, kNT, 0, s>>>(job_from_block(j, full, sizeof(T)));
  } else if (chunked_ct_eligible(j)) {
    return cuda_status(sizeof(T) == 8 ? launch_chunked_ct_f64(j.bits, true, j, s)
                                      : launch_chunked_ct_f32(j.bits, true, j, s),
                       "compress launch");
  } else {
    const std::uint64_t nb = (j.n + (std::uint64_t)j.E - 1) / (std::uint64_t)j.E;
    k_compress_generic<T><<<grid_for(nb, kNT / 32), kNT, 0, s>>>(j);
  }
  return cuda_status(cudaGetLastError(), "compress launch");
}

template<class T>
static int launch_decompress_t(const Job& j, int dtype, cudaStream_t s, bool* used_tile)
{
  if (j.n == 0) return FRSZ2_OK;
  const cudaError_t fe = try_fast<T>(false, j, s);
  if (fe != cudaErrorNotSupported) {
    if (used_tile) *used_tile = true;
    return cuda_status(fe, "decompress launch");
  }
  const bool tile = tile_eligible(j, dtype, j.values_out, j.words);
  if (used_tile) *used_tile = tile;
  if (tile) {
    const unsigned grid = (unsigned)std::min<std::uint64_t>(j.tiles, 1u << 30);
    if (sizeof(T) == 8 && j.bits > 32)
      k_decompress_tile<T, std::uint64_t><<<grid, kNT, decompress_smem<T>(j), s>>>(j);
    else
      k_decompress_tile<T, std::uint32_t><<<grid, kNT, decompress_smem<T>(j), s>>>(j);
  } else if (blockwise_eligible(j)) {
    return cuda_status(sizeof(T) == 8 ? launch_blockwise_f64(j.bits, false, j, s)
                                      : launch_blockwise_f32(j.bits, false, j, s),
                       "decompress launch");
  } else if (chunked_ct_eligible(j)) {
    return cuda_status(sizeof(T) == 8 ? launch_chunked_ct_f64(j.bits, false, j, s)
                                      : launch_chunked_ct_f32(j.bits, false, j, s),
                       "decompress launch");
  } else {
    const std::uint64_t nb = (j.n + (std::uint64_t)j.E - 1) / (std::uint64_t)j.E;
    k_decompress_generic<T><<<grid_for(nb, kNT / 32), kNT, 0, s>>>(j);
  }
  return cuda_status(cudaGetLastError(), "decompress launch");
}

int launch_compress(const Job& j, int dtype, cudaStream_t s, bool* used_tile)
{
  return dtype == FRSZ2_FLOAT ? launch_compress_t<float>(j, dtype, s, used_tile)
                              : launch_compress_t<double>(j, dtype, s, used_tile);
}

int launch_decompress(const Job& j, int dtype, cudaStream_t s, bool* used_tile)
{
  return dtype == FRSZ2_FLOAT ? launch_decompress_t<float>(j, dtype, s, used_tile)
                              : launch_decompress_t<double>(j, dtype, s, used_tile);
}

static int check_alignment(int dtype, const Layout& L, const void* values, const void* buf)
{
  const std::size_t es = dtype == FRSZ2_FLOAT ? 4 : 8;
  if (reinterpret_cast<std::uintptr_t>(values) % es != 0)
    return set_error(FRSZ2_EFAIL, "value pointer is not aligned to the element size");
  if (reinterpret_cast<std::uintptr_t>(buf) % (std::size_t)(L.W / 8) != 0)
    return set_error(FRSZ2_EFAIL, "compressed pointer is not aligned to the word size");
  return FRSZ2_OK;
}

Job job_for_slice(const Layout& L, int dtype, std::uint64_t b0, std::uint64_t nblocks, const void* vin, void* vout,
                  std::uint8_t* buf)
{
  Layout S = L;
  const std::uint64_t e0 = b0 * (std::uint64_t)L.E;
  S.n = std::min<std::uint64_t>(L.n - e0, nblocks * (std::uint64_t)L.E);
  Job j = make_job(S, dtype);
  const std::size_t es = dtype == FRSZ2_FLOAT ? 4 : 8;
  j.values_in = vin ? static_cast<const std::uint8_t*>(vin) + e0 * es : nullptr;
  j.values_out = vout ? static_cast<std::uint8_t*>(vout) + e0 * es : nullptr;
  j.exps = buf + b0 * (std::uint64_t)(L.W / 8);
  j.words = buf + L.exp_bytes + b0 * (std::uint64_t)L.block_bytes;
  return j;
}

// ---------------------------------------------------------------- host path

namespace {

struct Staging
{
  std::mutex mu;
  void* d_values = nullptr;
  std::size_t values_cap = 0;
  void* d_buf = nullptr;
  std::size_t buf_cap = 0;
  cudaStream_t st[2] = { nullptr, nullptr };
  cudaEvent_t ev_start = nullptr;
  bool init = false;
};

Staging g_staging[64];

int ensure(void** p, std::size_t* cap, std::size_t want)
{
  if (*cap >= want) return FRSZ2_OK;
  if (*p) cudaFree(*p);
  *p = nullptr;
  *cap = 0;
  const std::size_t sz = std::max<std::size_t>(want, 1 << 20);
  int rc = cuda_status(cudaMalloc(p, sz), "staging allocation");
  if (rc) return rc;
  *cap = sz;
  return FRSZ2_OK;
}

// Streams and event of a device's staging (first use; caller holds S.mu).
int staging_init(Staging& S)
{
  if (S.init) return FRSZ2_OK;
  int rc;
  for (auto& s : S.st)
    if ((rc = cuda_status(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "stream create"))) return rc;
  if ((rc = cuda_status(cudaEventCreateWithFlags(&S.ev_start, cudaEventDisableTiming), "event create"))) return rc;
  S.init = true;
  return FRSZ2_OK;
}

// Values per host-path slice: smaller slices shorten the pipeline's fill and
// drain (an H2D with nothing to overlap at the start of a call, a D2H at its
// end); measured end to end on the 512^3 field over PCIe 5.0 x16: 64 MiB 76.1,
// 32 MiB 78.2, 16 MiB 78.8, 8 MiB 75.3 GB/s (the link's bidirectional copy
// rate is 81.4 GB/s).
#ifndef FRSZ2_HOST_SLICE_MIB
#define FRSZ2_HOST_SLICE_MIB 16
#endif

// Slices of whole tiles so every slice keeps the tile kernel's alignment.
std::uint64_t slice_blocks(const Layout& L, int dtype)
{
  const int TE = dtype == FRSZ2_FLOAT ? tile_shape<float>::TE : tile_shape<double>::TE;
  const std::uint64_t target_values =
    ((std::uint64_t)FRSZ2_HOST_SLICE_MIB << 20) / (dtype == FRSZ2_FLOAT ? 4 : 8); // values per slice
  std::uint64_t unit = (is_pow2(L.E) && L.E <= TE) ? (std::uint64_t)(TE / L.E) : 16; // blocks
  std::uint64_t blocks = std::max<std::uint64_t>(unit, (target_values / (std::uint64_t)L.E) / unit * unit);
  return blocks;
}

} // namespace

int host_codec(bool compress, int dtype, int bits, int E, const void* h_in, std::uint64_t n, void* h_out,
               cudaStream_t user)
{
  int rc = check_args(dtype, bits, E);
  if (rc) return rc;
  if ((!h_in || !h_out) && n > 0) return set_error(FRSZ2_EFAIL, "null pointer");
  const Layout L = make_layout(n, bits, E);
  if (n == 0) return FRSZ2_OK;
  int dev = 0;
  rc = cuda_status(cudaGetDevice(&dev), "cudaGetDevice");
  if (rc) return rc;
  if (dev < 0 || dev >= 64) return set_error(FRSZ2_EFAIL, "device index out of range");
  Staging& S = g_staging[dev];
  std::lock_guard<std::mutex> lock(S.mu);
  if ((rc = staging_init(S))) return rc;
  const std::size_t es = dtype == FRSZ2_FLOAT ? 4 : 8;
  if ((rc = ensure(&S.d_values, &S.values_cap, L.n * es))) return rc;
  if ((rc = ensure(&S.d_buf, &S.buf_cap, L.total_bytes))) return rc;
  std::uint8_t* d_buf = static_cast<std::uint8_t*>(S.d_buf);
  const std::uint8_t* hb_in = static_cast<const std::uint8_t*>(h_in);
  std::uint8_t* hb_out = static_cast<std::uint8_t*>(h_out);

  // order after prior work on the caller's stream
  if ((rc = cuda_status(cudaEventRecord(S.ev_start, user), "event record"))) return rc;
  for (auto& s : S.st)
    if ((rc = cuda_status(cudaStreamWaitEvent(s, S.ev_start, 0), "stream wait"))) return rc;

  const std::uint64_t per = slice_blocks(L, dtype);
  int k = 0;
  for (std::uint64_t b0 = 0; b0 < L.nb; b0 += per, ++k) {
    cudaStream_t s = S.st[k & 1];
    const std::uint64_t nbk = std::min(per, L.nb - b0);
    const std::uint64_t e0 = b0 * (std::uint64_t)E;
    const std::uint64_t ne = std::min<std::uint64_t>(L.n - e0, nbk * (std::uint64_t)E);
    const bool last = b0 + nbk == L.nb;
    const std::uint64_t exp_off = b0 * (std::uint64_t)(L.W / 8), exp_len = nbk * (std::uint64_t)(L.W / 8);
    const std::uint64_t w_off = L.exp_bytes + b0 * (std::uint64_t)L.block_bytes;
    // bytes the reference writes for this slice: whole blocks, except only
    // the written words of a partial last block
    const int last_cnt = (int)(ne - (nbk - 1) * (std::uint64_t)E);
    const std::uint64_t w_len =
      (nbk - 1) * (std::uint64_t)L.block_bytes +
      (last ? written_block_bytes(last_cnt, bits, L.W) : L.block_bytes);
    if (compress) {
      Job j = job_for_slice(L, dtype, b0, nbk, S.d_values, nullptr, d_buf);
      if ((rc = cuda_status(cudaMemcpyAsync(static_cast<std::uint8_t*>(S.d_values) + e0 * es, hb_in + e0 * es,
                                            ne * es, cudaMemcpyHostToDevice, s),
                            "H2D")))
        return rc;
      if ((rc = launch_compress(j, dtype, s, nullptr))) return rc;
      if ((rc = cuda_status(cudaMemcpyAsync(hb_out + exp_off, d_buf + exp_off, exp_len, cudaMemcpyDeviceToHost, s),
                            "D2H")))
        return rc;
      if ((rc = cuda_status(cudaMemcpyAsync(hb_out + w_off, d_buf + w_off, w_len, cudaMemcpyDeviceToHost, s), "D2H")))
        return rc;
    } else {
      Job j = job_for_slice(L, dtype, b0, nbk, nullptr, S.d_values, d_buf);
      if ((rc = cuda_status(cudaMemcpyAsync(d_buf + exp_off, hb_in + exp_off, exp_len, cudaMemcpyHostToDevice, s),
                            "H2D")))
        return rc;
      // whole blocks are read by the tile kernel; copy the full slice (the
      // buffer always holds whole blocks)
      if ((rc = cuda_status(cudaMemcpyAsync(d_buf + w_off, hb_in + w_off, nbk * (std::uint64_t)L.block_bytes,
                                            cudaMemcpyHostToDevice, s),
                            "H2D")))
        return rc;
      if ((rc = launch_decompress(j, dtype, s, nullptr))) return rc;
      if ((rc = cuda_status(cudaMemcpyAsync(hb_out + e0 * es, static_cast<std::uint8_t*>(S.d_values) + e0 * es,
                                            ne * es, cudaMemcpyDeviceToHost, s),
                            "D2H")))
        return rc;
    }
  }
  for (auto& s : S.st)
    if ((rc = cuda_status(cudaStreamSynchronize(s), "stream sync"))) return rc;
  return FRSZ2_OK;
}

} // namespace frsz2b

using namespace frsz2b;

extern "C" {

void register_frsz(void) {}

const char* frsz2_version(void) { return "0.0.2-b200"; }

const char* frsz2_last_error(void) { return frsz2b::last_error(); }

int frsz2_compressed_size(int dtype, int bits, int block_size, uint64_t n, uint64_t* total_bytes)
{
  int rc = check_args(dtype, bits, block_size);
  if (rc) return rc;
  if (!total_bytes) return set_error(FRSZ2_EFAIL, "null pointer");
  *total_bytes = make_layout(n, bits, block_size).total_bytes;
  return FRSZ2_OK;
}

int frsz2_exponent_size(int dtype, int bits, int block_size, uint64_t n, uint64_t* exponent_bytes)
{
  int rc = check_args(dtype, bits, block_size);
  if (rc) return rc;
  if (!exponent_bytes) return set_error(FRSZ2_EFAIL, "null pointer");
  *exponent_bytes = make_layout(n, bits, block_size).exp_bytes;
  return FRSZ2_OK;
}

int frsz2_compress(int dtype, int bits, int block_size, const void* d_values, uint64_t n, void* d_compressed,
                   void* stream)
{
  NvtxRange nvtx("frsz2_compress");
  int rc = check_args(dtype, bits, block_size);
  if (rc) return rc;
  if (n == 0) return FRSZ2_OK;
  if (!d_values || !d_compressed) return set_error(FRSZ2_EFAIL, "null pointer");
  const Layout L = make_layout(n, bits, block_size);
  if ((rc = check_alignment(dtype, L, d_values, d_compressed))) return rc;
  Job j = job_for_slice(L, dtype, 0, L.nb, d_values, nullptr, static_cast<std::uint8_t*>(d_compressed));
  return launch_compress(j, dtype, static_cast<cudaStream_t>(stream), nullptr);
}

int frsz2_decompress(int dtype, int bits, int block_size, const void* d_compressed, uint64_t n, void* d_values,
                     void* stream)
{
  NvtxRange nvtx("frsz2_decompress");
  int rc = check_args(dtype, bits, block_size);
  if (rc) return rc;
  if (n == 0) return FRSZ2_OK;
  if (!d_values || !d_compressed) return set_error(FRSZ2_EFAIL, "null pointer");
  const Layout L = make_layout(n, bits, block_size);
  if ((rc = check_alignment(dtype, L, d_values, d_compressed))) return rc;
  Job j = job_for_slice(L, dtype, 0, L.nb, nullptr, d_values,
                        const_cast<std::uint8_t*>(static_cast<const std::uint8_t*>(d_compressed)));
  return launch_decompress(j, dtype, static_cast<cudaStream_t>(stream), nullptr);
}

int frsz2_compress_host(int dtype, int bits, int block_size, const void* h_values, uint64_t n, void* h_compressed,
                        void* stream)
{
  NvtxRange nvtx("frsz2_compress_host");
  return host_codec(true, dtype, bits, block_size, h_values, n, h_compressed, static_cast<cudaStream_t>(stream));
}

int frsz2_decompress_host(int dtype, int bits, int block_size, const void* h_compressed, uint64_t n, void* h_values,
                          void* stream)
{
  NvtxRange nvtx("frsz2_decompress_host");
  return host_codec(false, dtype, bits, block_size, h_compressed, n, h_values, static_cast<cudaStream_t>(stream));
}

static int block_range_args(int dtype, int bits, int E, std::uint64_t n, std::uint64_t b0, std::uint64_t count,
                            const void* values, const void* buf, Layout* L)
{
  if (int rc = check_args(dtype, bits, E)) return rc;
  *L = make_layout(n, bits, E);
  if (b0 > L->nb || count > L->nb - b0) return set_error(FRSZ2_EFAIL, "block range outside the array");
  if (count == 0) return FRSZ2_OK;
  if (!values || !buf) return set_error(FRSZ2_EFAIL, "null pointer");
  return check_alignment(dtype, *L, values, buf);
}

int frsz2_compress_blocks(int dtype, int bits, int block_size, const void* d_values, uint64_t n, uint64_t block_begin,
                          uint64_t block_count, void* d_compressed, void* stream)
{
  NvtxRange nvtx("frsz2_compress_blocks");
  Layout L;
  if (int rc = block_range_args(dtype, bits, block_size, n, block_begin, block_count, d_values, d_compressed, &L))
    return rc;
  if (block_count == 0) return FRSZ2_OK;
  // job_for_slice offsets the value pointer by the range's first value itself
  const std::size_t es = dtype == FRSZ2_FLOAT ? 4 : 8;
  const void* base = static_cast<const std::uint8_t*>(d_values) - block_begin * (std::uint64_t)block_size * es;
  Job j = job_for_slice(L, dtype, block_begin, block_count, base, nullptr, static_cast<std::uint8_t*>(d_compressed));
  return launch_compress(j, dtype, static_cast<cudaStream_t>(stream), nullptr);
}

int frsz2_decompress_blocks(int dtype, int bits, int block_size, const void* d_compressed, uint64_t n,
                            uint64_t block_begin, uint64_t block_count, void* d_values, void* stream)
{
  NvtxRange nvtx("frsz2_decompress_blocks");
  Layout L;
  if (int rc = block_range_args(dtype, bits, block_size, n, block_begin, block_count, d_values, d_compressed, &L))
    return rc;
  if (block_count == 0) return FRSZ2_OK;
  const std::size_t es = dtype == FRSZ2_FLOAT ? 4 : 8;
  void* base = static_cast<std::uint8_t*>(d_values) - block_begin * (std::uint64_t)block_size * es;
  Job j = job_for_slice(L, dtype, block_begin, block_count, nullptr, base,
                        const_cast<std::uint8_t*>(static_cast<const std::uint8_t*>(d_compressed)));
  return launch_decompress(j, dtype, static_cast<cudaStream_t>(stream), nullptr);
}

int frsz2_decompress_elements(int dtype, int bits, int block_size, const void* d_compressed, uint64_t n,
                              const uint64_t* d_idx, uint64_t count, void* d_out, void* stream)
{
  NvtxRange nvtx("frsz2_decompress_elements");
  int rc = check_args(dtype, bits, block_size);
  if (rc) return rc;
  if (count == 0) return FRSZ2_OK;
  if (!d_compressed || !d_idx || !d_out) return set_error(FRSZ2_EFAIL, "null pointer");
  const Layout L = make_layout(n, bits, block_size);
  if ((rc = check_alignment(dtype, L, d_out, d_compressed))) return rc;
  Job j = job_for_slice(L, dtype, 0, L.nb, nullptr, nullptr,
                        const_cast<std::uint8_t*>(static_cast<const std::uint8_t*>(d_compressed)));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const unsigned grid = grid_for(count, kNT);
  if (dtype == FRSZ2_FLOAT)
    k_decompress_elements<float><<<grid, kNT, 0, s>>>(j, d_idx, count, static_cast<float*>(d_out));
  else
    k_decompress_elements<double><<<grid, kNT, 0, s>>>(j, d_idx, count, static_cast<double*>(d_out));
  return cuda_status(cudaGetLastError(), "element decode launch");
}

// Host-buffer random access (decompress_cpu_element, include/frsz2.hpp:1199-1214):
// the host gathers the exponent and block bytes of every block a valid index
// falls in into a small buffer laid out as an array of those blocks, which
// the element kernel decodes on the GPU.
int frsz2_decompress_elements_host(int dtype, int bits, int block_size, const void* h_compressed, uint64_t n,
                                   const uint64_t* h_idx, uint64_t count, void* h_out)
{
  NvtxRange nvtx("frsz2_decompress_elements_host");
  int rc = check_args(dtype, bits, block_size);
  if (rc) return rc;
  if (count == 0) return FRSZ2_OK;
  if (!h_compressed || !h_idx || !h_out) return set_error(FRSZ2_EFAIL, "null pointer");
  const Layout L = make_layout(n, bits, block_size);
  const std::uint64_t E = (std::uint64_t)block_size, EB = (std::uint64_t)(L.W / 8), BB = L.block_bytes;
  std::vector<std::uint64_t> blocks;
  blocks.reserve(count);
  for (std::uint64_t t = 0; t < count; ++t)
    if (h_idx[t] < n) blocks.push_back(h_idx[t] / E);
  if (blocks.empty()) return FRSZ2_OK; // every index out of range: outputs untouched
  std::sort(blocks.begin(), blocks.end());
  blocks.erase(std::unique(blocks.begin(), blocks.end()), blocks.end());
  const std::uint64_t m = blocks.size();
  const Layout M = make_layout(m * E, bits, block_size);
  const std::uint8_t* hb = static_cast<const std::uint8_t*>(h_compressed);
  std::vector<std::uint8_t> mini(M.total_bytes, 0);
  for (std::uint64_t k = 0; k < m; ++k) {
    std::memcpy(mini.data() + k * EB, hb + blocks[k] * EB, EB);
    std::memcpy(mini.data() + M.exp_bytes + k * BB, hb + L.exp_bytes + blocks[k] * BB, BB);
  }
  std::vector<std::uint64_t> mapped(count);
  for (std::uint64_t t = 0; t < count; ++t) {
    const std::uint64_t g = h_idx[t];
    if (g >= n) {
      mapped[t] = ~0ull; // the kernel skips it
      continue;
    }
    const std::uint64_t k = (std::uint64_t)(std::lower_bound(blocks.begin(), blocks.end(), g / E) - blocks.begin());
    mapped[t] = k * E + g % E;
  }

  int dev = 0;
  if ((rc = cuda_status(cudaGetDevice(&dev), "cudaGetDevice"))) return rc;
  if (dev < 0 || dev >= 64) return set_error(FRSZ2_EFAIL, "device index out of range");
  Staging& S = g_staging[dev];
  std::lock_guard<std::mutex> lock(S.mu);
  if ((rc = staging_init(S))) return rc;
  const std::size_t es = dtype == FRSZ2_FLOAT ? 4 : 8;
  const std::size_t idx_off = (M.total_bytes + 255) / 256 * 256;
  if ((rc = ensure(&S.d_buf, &S.buf_cap, idx_off + count * sizeof(std::uint64_t)))) return rc;
  if ((rc = ensure(&S.d_values, &S.values_cap, count * es))) return rc;
  std::uint8_t* d_buf = static_cast<std::uint8_t*>(S.d_buf);
  auto* d_idx = reinterpret_cast<std::uint64_t*>(d_buf + idx_off);
  cudaStream_t s = S.st[0];
  if ((rc = cuda_status(cudaMemcpyAsync(d_buf, mini.data(), M.total_bytes, cudaMemcpyHostToDevice, s), "H2D")) ||
      (rc = cuda_status(cudaMemcpyAsync(d_idx, mapped.data(), count * sizeof(std::uint64_t), cudaMemcpyHostToDevice,
                                        s),
                        "H2D")) ||
      (rc = cuda_status(cudaMemcpyAsync(S.d_values, h_out, count * es, cudaMemcpyHostToDevice, s), "H2D")))
    return rc;
  Job j = job_for_slice(M, dtype, 0, M.nb, nullptr, nullptr, d_buf);
  const unsigned grid = grid_for(count, kNT);
  if (dtype == FRSZ2_FLOAT)
    k_decompress_elements<float><<<grid, kNT, 0, s>>>(j, d_idx, count, static_cast<float*>(S.d_values));
  else
    k_decompress_elements<double><<<grid, kNT, 0, s>>>(j, d_idx, count, static_cast<double*>(S.d_values));
  if ((rc = cuda_status(cudaGetLastError(), "element decode launch"))) return rc;
  if ((rc = cuda_status(cudaMemcpyAsync(h_out, S.d_values, count * es, cudaMemcpyDeviceToHost, s), "D2H"))) return rc;
  return cuda_status(cudaStreamSynchronize(s), "stream synchronize");
}

} // extern "C"
