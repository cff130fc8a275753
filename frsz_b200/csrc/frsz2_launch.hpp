// frsz2_launch.hpp -- internal host-side interface shared by the C ABI
// translation units (argument checks, error state, kernel launchers).
#pragma once

#include "frsz2_kernels.cuh"

#include <string>

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

namespace frsz2b {

constexpr int kMaxBlockSize = 65536;

// Record `msg` as the calling thread's last error and return `code`.
int set_error(int code, const std::string& msg);
const char* last_error();
int cuda_status(cudaError_t e, const char* what);

// FRSZ2_OK, or FRSZ2_EDTYPE / FRSZ2_EFAIL with the reference's messages.
int check_args(int dtype, int bits, int E);

int sm_count();

// NVTX range around a C-ABI call (visible in nsys / ncu timelines; a no-op
// without a tool attached).
struct NvtxRange
{
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

Job make_job(const Layout& L, int dtype);
bool tile_eligible(const Job& j, int dtype, const void* values, const void* words);

// Job over blocks [b0, b0 + nblocks) of an array with layout L whose buffer
// starts at `buf`; vin / vout point at the array's first value.
Job job_for_slice(const Layout& L, int dtype, std::uint64_t b0, std::uint64_t nblocks, const void* vin, void* vout,
                  std::uint8_t* buf);

// Enqueue the compress / decompress of one job on stream s.  *used_tile
// reports whether the tile kernel (rather than the generic one) was chosen.
int launch_compress(const Job& j, int dtype, cudaStream_t s, bool* used_tile);
int launch_decompress(const Job& j, int dtype, cudaStream_t s, bool* used_tile);

} // namespace frsz2b
