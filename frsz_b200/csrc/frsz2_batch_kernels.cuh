// frsz2_batch_kernels.cuh -- persistent kernel of the batched path.
//
// One instance per (float type, width, CTA shape, direction).  It walks the
// concatenated tile list of one class of arrays (same float type and width)
// with a grid stride; a tile's array is found by advancing a cursor through
// the class's descriptors (tiles of one CTA come in increasing order).  The
// tile bodies are the single-array fast kernels' own, so every array gets the
// same code and register budget.
#pragma once

#include "frsz2_fast.cuh"

namespace frsz2b {

struct BatchItem
{
  Job job;                  // geometry for the kernel's tile size
  std::uint64_t tile_begin; // first tile of this array within its class
};

template<class T, int BITS, int NT, int RPW, bool COMPRESS>
__global__ void __launch_bounds__(NT)
  k_batch_class(const BatchItem* __restrict__ items, int nitems, std::uint64_t total_tiles)
{
  __shared__ std::uint32_t s_rmax[2 * (NT / 32) * RPW];
  __shared__ __align__(16) std::uint32_t s_stage[stage_words<T, BITS, NT, RPW>::value];
  int cur = 0;
  for (std::uint64_t t = blockIdx.x; t < total_tiles; t += gridDim.x) {
    while (cur + 1 < nitems && items[cur + 1].tile_begin <= t) ++cur;
    const Job j = items[cur].job;
    const std::uint64_t lt = t - items[cur].tile_begin;
    if constexpr (!fast_cfg<T, BITS, NT, RPW>::ALIGNED) {
      if (job_padded(j)) {
        if (COMPRESS)
          fast_compress_tile<T, BITS, NT, RPW, true>(j, lt, s_rmax, s_stage);
        else
          fast_decompress_tile<T, BITS, NT, RPW, true>(j, lt);
        continue;
      }
    }
    if (COMPRESS)
      fast_compress_tile<T, BITS, NT, RPW>(j, lt, s_rmax, s_stage);
    else
      fast_decompress_tile<T, BITS, NT, RPW>(j, lt);
  }
}

// One CTA per tile of a class's concatenated tile list, the tile's array
// read from a per-tile index (one 4-byte load): the launch shape of the
// single-array kernels, which hardware CTA scheduling balances across SMs.
template<class T, int BITS, int NT, int RPW, bool COMPRESS>
__global__ void __launch_bounds__(NT)
  k_batch_tiles(const BatchItem* __restrict__ items, const std::uint32_t* __restrict__ tile_item)
{
  __shared__ std::uint32_t s_rmax[2 * (NT / 32) * RPW];
  __shared__ __align__(16) std::uint32_t s_stage[stage_words<T, BITS, NT, RPW>::value];
  const std::uint64_t t = blockIdx.x;
  const std::uint32_t it = __ldg(tile_item + t);
  const Job j = items[it].job;
  const std::uint64_t lt = t - items[it].tile_begin;
  if constexpr (!fast_cfg<T, BITS, NT, RPW>::ALIGNED) {
    if (job_padded(j)) {
      if (COMPRESS)
        fast_compress_tile<T, BITS, NT, RPW, true>(j, lt, s_rmax, s_stage, false);
      else
        fast_decompress_tile<T, BITS, NT, RPW, true>(j, lt);
      return;
    }
  }
  if (COMPRESS)
    fast_compress_tile<T, BITS, NT, RPW>(j, lt, s_rmax, s_stage, false);
  else
    fast_decompress_tile<T, BITS, NT, RPW>(j, lt);
}

using batch_tiles_fn = cudaError_t (*)(bool compress, const BatchItem* items, const std::uint32_t* tile_item,
                                       std::uint64_t tiles, cudaStream_t s);

template<class T, int BITS, int NT, int RPW>
cudaError_t launch_batch_tiles(bool compress, const BatchItem* items, const std::uint32_t* tile_item,
                               std::uint64_t tiles, cudaStream_t s)
{
  if (compress)
    k_batch_tiles<T, BITS, NT, RPW, true><<<(unsigned)tiles, NT, 0, s>>>(items, tile_item);
  else
    k_batch_tiles<T, BITS, NT, RPW, false><<<(unsigned)tiles, NT, 0, s>>>(items, tile_item);
  return cudaGetLastError();
}

// CTA shapes the autotuner chooses from: (threads, rows per warp).  Shape 0
// exists for every width; shapes 1 and 2 for the widths of FRSZ2_TUNED_WIDTHS.
struct Shape
{
  int nt, rpw;
};
constexpr Shape kShapes[] = { { 256, 2 }, { 128, 2 }, { 512, 1 } };
constexpr int kNumShapes = 3;

using batch_fn = cudaError_t (*)(bool compress, const BatchItem* items, int nitems, std::uint64_t tiles,
                                 unsigned grid, cudaStream_t s);

template<class T, int BITS, int NT, int RPW>
cudaError_t launch_batch_class(bool compress, const BatchItem* items, int nitems, std::uint64_t tiles, unsigned grid,
                               cudaStream_t s)
{
  if (compress)
    k_batch_class<T, BITS, NT, RPW, true><<<grid, NT, 0, s>>>(items, nitems, tiles);
  else
    k_batch_class<T, BITS, NT, RPW, false><<<grid, NT, 0, s>>>(items, nitems, tiles);
  return cudaGetLastError();
}

template<class T, int BITS, int NT, int RPW>
int batch_class_occupancy(bool compress)
{
  int blocks = 0;
  cudaError_t e = compress ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                               &blocks, k_batch_class<T, BITS, NT, RPW, true>, NT, 0)
                           : cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                               &blocks, k_batch_class<T, BITS, NT, RPW, false>, NT, 0);
  return (e == cudaSuccess && blocks > 0) ? blocks : 1;
}

// Launcher and occupancy query of a class, or nullptr when (bits, shape) has
// no instance.
struct batch_entry
{
  batch_fn launch;
  int (*occupancy)(bool);
  batch_tiles_fn launch_tiles; // one CTA per tile (shape 0 only)
};
batch_entry batch_class_f32(int bits, int shape);
batch_entry batch_class_f64(int bits, int shape);

// widths with all three shapes instantiated
#define FRSZ2_TUNED_WIDTHS(X) X(8) X(12) X(16) X(21) X(24) X(32)

} // namespace frsz2b
