// frsz2_batch_static.cu -- batched compress that allocates nothing.
//
// For callers that cannot allocate device memory at call time: an
// application whose allocator already owns all of the GPU's memory (a
// serving process that reserved its whole budget up front, a framework with
// its own caching allocator), or a request path where a cudaMalloc -- which
// can synchronise the device and fail under memory pressure -- is not
// allowed.  frsz2_batch_create needs a cudaMalloc for the plan's descriptors;
// this entry point instead keeps the descriptor work list of the batched
// persistent kernels in a fixed device array that every GPU loading the
// library holds until the process exits.
//
// The work list reaches that array through the parameters of small upload
// kernels (up to kUploadItems descriptors per launch), so a call keeps no
// host-side copy of it: nothing a later call writes on the host can change
// what an earlier call's launches carry.
//
// Limits and sharing:
//  * at most kStaticItems (4096) arrays per call; larger batches are rejected
//    with status 2 and a message;
//  * the array is shared by every call on a device and keeps the last call's
//    contents.  Each call overwrites the prefix it uses before its kernels
//    read it, and nothing in it has to start at zero.  Calls on one stream
//    are ordered; calls whose work overlaps on the GPU (different streams, or
//    several host threads) race on the array;
//  * the first call on each device looks up the array's device address
//    (cudaGetSymbolAddress, with that device current) and keeps it for the
//    life of the process; make that first call before any stream capture.
//    After cudaDeviceReset on a device the kept address belongs to the
//    destroyed context, so calls after a reset are not supported.
#include "frsz2_batch_kernels.cuh"
#include "frsz2_launch.hpp"

#include "../../include/frsz2_b200.h"

#include <algorithm>
#include <mutex>
#include <string>

using namespace frsz2b;

namespace {

constexpr std::uint64_t kStaticItems = 4096;

// Device-side work list of the persistent kernels (352 KiB per device).
static __device__ __align__(256) BatchItem g_static_work[kStaticItems];

// Guards the per-device address table.
std::mutex g_mu;

// One upload launch: descriptors and their places in the work list, passed
// by value as the kernel's parameter (above the 4 KB of older CUDA releases,
// within the 32,764 bytes CUDA 12.1+ allows on every architecture).
constexpr int kUploadItems = 340;
struct StaticUpload
{
  BatchItem item[kUploadItems];
  std::uint32_t index[kUploadItems];
  int count;
};
static_assert(sizeof(StaticUpload) <= 32764, "kernel parameter too large");

__global__ void __launch_bounds__(128) k_static_upload(const StaticUpload up, BatchItem* __restrict__ work)
{
  for (int i = threadIdx.x; i < up.count; i += blockDim.x) work[up.index[i]] = up.item[i];
}

// Device address of g_static_work per device (set once per device).
BatchItem* g_work_ptr[64] = {};

constexpr int kClasses = 2 * 65; // (float type, width) keys: is64 * 65 + bits

int class_key(int dtype, int bits) { return (dtype == FRSZ2_DOUBLE ? 65 : 0) + bits; }

} // namespace

extern "C" int frsz2_batch_compress_static(const frsz2_batch_item* items, uint64_t count, void* stream)
{
  if (count > kStaticItems)
    return set_error(FRSZ2_EFAIL, "frsz2_batch_compress_static takes at most " + std::to_string(kStaticItems) +
                                    " arrays per call, got " + std::to_string(count));
  if (count > 0 && !items) return set_error(FRSZ2_EFAIL, "null items");
  cudaStream_t s = static_cast<cudaStream_t>(stream);

  int dev = 0;
  if (int rc = cuda_status(cudaGetDevice(&dev), "cudaGetDevice")) return rc;
  if (dev < 0 || dev >= 64) return set_error(FRSZ2_EFAIL, "device index out of range");
  BatchItem* d_work = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_work_ptr[dev]) {
      void* ptr = nullptr;
      if (int rc = cuda_status(cudaGetSymbolAddress(&ptr, g_static_work), "cudaGetSymbolAddress")) return rc;
      g_work_ptr[dev] = static_cast<BatchItem*>(ptr);
    }
    d_work = g_work_ptr[dev];
  }

  // validate, and count the persistent-kernel arrays of each class
  std::uint64_t per_class[kClasses] = {};
  for (std::uint64_t i = 0; i < count; ++i) {
    const frsz2_batch_item& it = items[i];
    if (int rc = check_args(it.dtype, it.bits, it.block_size)) return rc;
    if (it.n > 0 && (!it.values || !it.compressed))
      return set_error(FRSZ2_EFAIL, "null pointer in batch item " + std::to_string(i));
    const std::uintptr_t es = it.dtype == FRSZ2_DOUBLE ? 8 : 4;
    const std::uintptr_t ws = (std::uintptr_t)word_bits(it.bits) / 8;
    if (it.n > 0 && (reinterpret_cast<std::uintptr_t>(it.values) % es != 0 ||
                     reinterpret_cast<std::uintptr_t>(it.compressed) % ws != 0))
      return set_error(FRSZ2_EFAIL, "misaligned pointer in batch item " + std::to_string(i));
  }
  auto eligible = [](const frsz2_batch_item& it) {
    if (it.n == 0) return false;
    const bool is64 = it.dtype == FRSZ2_DOUBLE;
    const Layout L = make_layout(it.n, it.bits, it.block_size);
    const Job j =
      job_for_slice(L, it.dtype, 0, L.nb, it.values, nullptr, static_cast<std::uint8_t*>(it.compressed));
    const batch_entry e = is64 ? batch_class_f64(it.bits, 0) : batch_class_f32(it.bits, 0);
    const int tv = fast_tile_values(is64 ? 8 : 4, kShapes[0].nt, kShapes[0].rpw);
    return e.launch != nullptr && it.block_size <= tv && fast_eligible(j, is64, it.values, j.words);
  };
  for (std::uint64_t i = 0; i < count; ++i)
    if (eligible(items[i])) ++per_class[class_key(items[i].dtype, items[i].bits)];

  // class offsets in the work list
  std::uint64_t start[kClasses], fill[kClasses], tiles[kClasses] = {};
  std::uint64_t used = 0;
  for (int k = 0; k < kClasses; ++k) {
    start[k] = fill[k] = used;
    used += per_class[k];
  }
  // each descriptor goes to its class's next slot; the upload launches carry
  // them in item order (stream-ordered after earlier calls' kernels)
  StaticUpload up;
  up.count = 0;
  auto flush = [&]() -> int {
    if (up.count == 0) return FRSZ2_OK;
    k_static_upload<<<1, 128, 0, s>>>(up, d_work);
    up.count = 0;
    return cuda_status(cudaGetLastError(), "work list upload");
  };
  for (std::uint64_t i = 0; i < count; ++i) {
    const frsz2_batch_item& it = items[i];
    if (!eligible(it)) continue;
    const int k = class_key(it.dtype, it.bits);
    const int tv = fast_tile_values(it.dtype == FRSZ2_DOUBLE ? 8 : 4, kShapes[0].nt, kShapes[0].rpw);
    const Layout L = make_layout(it.n, it.bits, it.block_size);
    BatchItem& bi = up.item[up.count];
    bi.job = job_for_slice(L, it.dtype, 0, L.nb, it.values, nullptr, static_cast<std::uint8_t*>(it.compressed));
    bi.job.tiles = (it.n + (std::uint64_t)tv - 1) / (std::uint64_t)tv;
    bi.job.tile_blocks = (std::uint32_t)(tv / it.block_size);
    bi.tile_begin = tiles[k];
    tiles[k] += bi.job.tiles;
    up.index[up.count++] = (std::uint32_t)fill[k]++;
    if (up.count == kUploadItems)
      if (int rc = flush()) return rc;
  }
  if (int rc = flush()) return rc;

  for (int k = 0; k < kClasses; ++k) {
    if (per_class[k] == 0) continue;
    const bool is64 = k >= 65;
    const int bits = k - (is64 ? 65 : 0);
    const batch_entry e = is64 ? batch_class_f64(bits, 0) : batch_class_f32(bits, 0);
    const std::uint64_t ctas = (std::uint64_t)sm_count() * (std::uint64_t)e.occupancy(true);
    const unsigned grid = (unsigned)std::max<std::uint64_t>(1, std::min(ctas, tiles[k]));
    if (int rc = cuda_status(e.launch(true, d_work + start[k], (int)per_class[k], tiles[k], grid, s), "batch launch"))
      return rc;
  }
  // arrays the persistent kernels do not take: their own launch, no allocation
  for (std::uint64_t i = 0; i < count; ++i) {
    const frsz2_batch_item& it = items[i];
    if (it.n == 0 || eligible(it)) continue;
    const Layout L = make_layout(it.n, it.bits, it.block_size);
    const Job j =
      job_for_slice(L, it.dtype, 0, L.nb, it.values, nullptr, static_cast<std::uint8_t*>(it.compressed));
    if (int rc = launch_compress(j, it.dtype, s, nullptr)) return rc;
  }
  return FRSZ2_OK;
}
