// frsz2_b200.hpp -- C++ drop-in for the reference's frsz2 codec API
// (robertu94/frsz include/frsz2.hpp), executed by libfrsz2_b200.so on a B200.
//
// Replace `#include "frsz2.hpp"` with `#include "frsz2_b200.hpp"` and link
// -lfrsz2_b200 -lcudart.  The compressed format, the static size algebra and
// the runtime dispatch are the reference's; the work runs in sm_100a kernels.
//
//   frsz::frsz2_compressor<bits, E, T>  (include/frsz2.hpp:504-1256)
//     a non-owning view of one compressed buffer:
//       compress_cpu_impl / decompress_cpu_impl  -- HOST buffers (as in the
//           reference, include/frsz2.hpp:1181, 1242); copies to and from the
//           GPU happen inside the call
//       compress_gpu_impl / decompress_gpu_impl  -- DEVICE buffers, stream
//           ordered, asynchronous
//       decompress_gpu_elements                  -- random access from the
//           host: device indices in, device values out
//       decompress_gpu_element (device code)     -- random access inside the
//           caller's own kernels (include/frsz2.hpp:1096-1104); compiled
//           when the including file is built by nvcc
//   frsz::compress_gpu<Comp, block_size> / frsz::decompress_gpu<Comp>
//     (include/frsz2.hpp:1258-1288) -- the reference's launchable kernels,
//     same names, template and kernel parameters, any launch shape (the
//     reference tests launch <<<ceil(n / 4E), 4E>>> and
//     <<<ceil(n / (max(1, 512/E) E)), max(1, 512/E) E>>>), so code that
//     launches them compiles and produces the same bytes; nvcc only.  They
//     run simple one-thread-per-block / per-value device code; the
//     library's compress_gpu_impl / decompress_gpu_impl are the fast path.
//   frsz::int_list_t, frsz::dispatch_frsz2_compression /
//   dispatch_frsz2_decompression  (include/frsz2.hpp:1292-1347)
//     same signatures and std::runtime_error messages; host buffers.
//
// Errors from the library throw std::runtime_error with its message.
#ifndef FRSZ2_B200_HPP
#define FRSZ2_B200_HPP

#include "frsz2_b200.h"

#include <climits>
#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <type_traits>

#include <cuda_runtime_api.h>

#if defined(__CUDACC__)
#include "frsz2_b200_device.cuh"
#define FRSZ2_B200_HD __host__ __device__
#else
#define FRSZ2_B200_HD
#endif

namespace frsz {

namespace detail {

// storage_t<N> (include/frsz2.hpp:258-262): word AND exponent width.
template<std::size_t N>
using storage_t = std::conditional_t<
  (N <= 8), std::uint8_t,
  std::conditional_t<(N <= 16), std::uint16_t, std::conditional_t<(N <= 32), std::uint32_t, std::uint64_t>>>;

template<class T>
using scaled_t = std::conditional_t<sizeof(T) == 8, std::uint64_t, std::uint32_t>;

template<class T>
constexpr int dtype_code()
{
  static_assert(std::is_same<T, float>::value || std::is_same<T, double>::value, "float or double only");
  return std::is_same<T, float>::value ? FRSZ2_FLOAT : FRSZ2_DOUBLE;
}

inline void check(int rc)
{
  if (rc != FRSZ2_OK) throw std::runtime_error(frsz2_last_error());
}

template<class T>
constexpr T ceildiv(T a, T b)
{
  return a / b + (a % b != 0);
}

} // namespace detail

template<int bits_per_value_, int max_exp_block_size_, class FpType_>
struct frsz2_compressor
{
  constexpr static auto bits_per_value = bits_per_value_;
  constexpr static auto max_exp_block_size = max_exp_block_size_;
  using fp_type = FpType_;
  using exp_type = std::make_signed_t<detail::storage_t<bits_per_value>>;
  using uint_compressed_type = detail::storage_t<bits_per_value>;
  using uint_fp_type = detail::scaled_t<fp_type>;

  // the reference's compile-time constraints (include/frsz2.hpp:511-517)
  static_assert(bits_per_value <= sizeof(fp_type) * CHAR_BIT,
                "The number of bits per compressed value must be smaller (or equal to) the size of the "
                "original value type!");
  static_assert(0 < max_exp_block_size, "max_exp_block_size must be positive!");
  static_assert(4 <= bits_per_value, "Minimum bits per value is 4 (so at most 2 values share the same byte).");
  static_assert(bits_per_value <= 64, "maximum number for bits_per_value is 64.");
  // A narrowing of the reference, which only asks for 0 < E: the library's
  // kernels index bits within one block with 32-bit integers, so blocks are
  // capped at 65536 values (65536 * 64 bits < 2^31); the C ABI rejects larger
  // ones with status 2.
  static_assert(max_exp_block_size <= 65536, "this library supports exponent blocks of up to 65536 values");

  static constexpr int uint_compressed_size_bit = sizeof(uint_compressed_type) * CHAR_BIT;
  static constexpr int compressed_block_size_element_count =
    detail::ceildiv<int>(max_exp_block_size * bits_per_value, uint_compressed_size_bit);
  static constexpr int compressed_block_size_byte =
    compressed_block_size_element_count * sizeof(uint_compressed_type);

  // include/frsz2.hpp:534-540
  static constexpr std::size_t compute_exponent_block_size_byte(std::size_t number_elements)
  {
    const std::size_t e = detail::ceildiv<std::size_t>(number_elements, max_exp_block_size) * sizeof(exp_type);
    return e + 256 - e % 256;
  }

  // include/frsz2.hpp:542-548
  static constexpr std::size_t compute_compressed_memory_size_byte(std::size_t number_elements)
  {
    return compute_exponent_block_size_byte(number_elements) +
           detail::ceildiv<std::size_t>(number_elements, max_exp_block_size) * compressed_block_size_byte;
  }

  frsz2_compressor(std::uint8_t* data, std::size_t total_elements)
    : data_{ data }
    , exponents_{ reinterpret_cast<exp_type*>(data) }
    , compressed_{ reinterpret_cast<uint_compressed_type*>(data + compute_exponent_block_size_byte(total_elements)) }
    , total_elements_{ total_elements }
  {
  }

  FRSZ2_B200_HD uint_compressed_type* get_compressed_data() { return compressed_; }
  FRSZ2_B200_HD const uint_compressed_type* get_compressed_data() const { return compressed_; }
  FRSZ2_B200_HD const uint_compressed_type* get_const_compressed_data() const { return compressed_; }
  FRSZ2_B200_HD exp_type* get_exponent_data() { return exponents_; }
  FRSZ2_B200_HD const exp_type* get_exponent_data() const { return exponents_; }
  FRSZ2_B200_HD const exp_type* get_const_exponent_data() const { return exponents_; }
  FRSZ2_B200_HD std::size_t get_total_elements() const { return total_elements_; }

  // Host buffers (the view's buffer and `data` in host memory).
  int compress_cpu_impl(const fp_type* data)
  {
    detail::check(frsz2_compress_host(detail::dtype_code<fp_type>(), bits_per_value, max_exp_block_size, data,
                                      total_elements_, data_, nullptr));
    return 0;
  }
  int decompress_cpu_impl(fp_type* output) const
  {
    detail::check(frsz2_decompress_host(detail::dtype_code<fp_type>(), bits_per_value, max_exp_block_size, data_,
                                        total_elements_, output, nullptr));
    return 0;
  }

  // Value idx of a HOST buffer (include/frsz2.hpp:1199-1214): the block that
  // holds it is decoded on the GPU.
  fp_type decompress_cpu_element(const std::size_t idx) const
  {
    const std::uint64_t i = idx;
    fp_type v{};
    detail::check(frsz2_decompress_elements_host(detail::dtype_code<fp_type>(), bits_per_value, max_exp_block_size,
                                                 data_, total_elements_, &i, 1, &v));
    return v;
  }
  // Values at host indices idx[0..count) of a HOST buffer, in one call.
  void decompress_cpu_elements(const std::uint64_t* idx, std::size_t count, fp_type* output) const
  {
    detail::check(frsz2_decompress_elements_host(detail::dtype_code<fp_type>(), bits_per_value, max_exp_block_size,
                                                 data_, total_elements_, idx, count, output));
  }

  // Device buffers (the view's buffer and `data` in GPU memory).
  void compress_gpu_impl(const fp_type* d_data, cudaStream_t stream = nullptr)
  {
    detail::check(frsz2_compress(detail::dtype_code<fp_type>(), bits_per_value, max_exp_block_size, d_data,
                                 total_elements_, data_, stream));
  }
  void decompress_gpu_impl(fp_type* d_output, cudaStream_t stream = nullptr) const
  {
    detail::check(frsz2_decompress(detail::dtype_code<fp_type>(), bits_per_value, max_exp_block_size, data_,
                                   total_elements_, d_output, stream));
  }
  // Values at device indices d_idx[0..count) into d_output.
  void decompress_gpu_elements(const std::uint64_t* d_idx, std::size_t count, fp_type* d_output,
                               cudaStream_t stream = nullptr) const
  {
    detail::check(frsz2_decompress_elements(detail::dtype_code<fp_type>(), bits_per_value, max_exp_block_size, data_,
                                            total_elements_, d_idx, count, d_output, stream));
  }

#if defined(__CUDACC__)
  // Value idx, read in device code: pass the view to a kernel by value and
  // call this per index (the buffer must be device-accessible).  The result
  // equals decompress_cpu_impl's value idx bit for bit; idx must be below
  // get_total_elements().
  __device__ fp_type decompress_gpu_element(std::size_t idx) const
  {
    return frsz2_b200::device::decode_element<bits_per_value, max_exp_block_size, fp_type>(exponents_, compressed_,
                                                                                         idx);
  }
  // Compress exponent block `block` of the array `data` (device memory, all
  // get_total_elements() values) into the view's buffer: its exponent and
  // the words its values reach, the bytes compress_cpu_impl writes.
  __device__ void compress_gpu_block(std::size_t block, const fp_type* data)
  {
    const std::size_t first = block * (std::size_t)max_exp_block_size;
    const std::size_t left = total_elements_ - first;
    const std::size_t cnt = left < (std::size_t)max_exp_block_size ? left : (std::size_t)max_exp_block_size;
    frsz2_b200::device::encode_block<bits_per_value, max_exp_block_size, fp_type>(data + first, cnt, exponents_,
                                                                                compressed_, block);
  }
#endif

private:
  std::uint8_t* const data_;
  exp_type* const exponents_;
  uint_compressed_type* const compressed_;
  const std::size_t total_elements_;
};

#if defined(__CUDACC__)
// The reference's launchable kernels (include/frsz2.hpp:1258-1288), same
// names and parameters.  Any grid works: compress_gpu's threads take whole
// exponent blocks in a grid-stride loop (the reference's launch of one thread
// per value leaves the threads past the block count idle), decompress_gpu's
// threads take values as the reference's do.  The bytes written equal
// compress_cpu_impl's and the values decompress_cpu_impl's, bit for bit.
template<typename Frsz2Compressor, int block_size>
__global__ __launch_bounds__(block_size) void compress_gpu(const typename Frsz2Compressor::fp_type* __restrict__ data,
                                                           Frsz2Compressor compressor)
{
  constexpr std::size_t E = (std::size_t)Frsz2Compressor::max_exp_block_size;
  const std::size_t nb = (compressor.get_total_elements() + E - 1) / E;
  for (std::size_t b = (std::size_t)blockIdx.x * blockDim.x + threadIdx.x; b < nb;
       b += (std::size_t)gridDim.x * blockDim.x)
    compressor.compress_gpu_block(b, data);
}

template<typename Frsz2Compressor>
__global__ void decompress_gpu(typename Frsz2Compressor::fp_type* const __restrict__ output,
                               Frsz2Compressor compressor)
{
  for (std::size_t idx = (std::size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < compressor.get_total_elements();
       idx += (std::size_t)gridDim.x * blockDim.x)
    output[idx] = compressor.decompress_gpu_element(idx);
}
#endif

// ---------------------------------------------------------------- dispatch
// include/frsz2.hpp:1292-1347: recursive walk from runtime (bits, E) to a
// compile-time instance; unsupported values throw the reference's messages.

template<int... values>
struct int_list_t
{};

namespace detail {

template<int B, class T, class Op>
void dispatch_exp(int_list_t<>, int actual_exp, Op&&)
{
  throw std::runtime_error("Unsupported exponent block size: " + std::to_string(actual_exp));
}
template<int B, class T, class Op, int E0, int... Es>
void dispatch_exp(int_list_t<E0, Es...>, int actual_exp, Op&& op)
{
  if (E0 == actual_exp)
    op.template run<B, E0, T>();
  else
    dispatch_exp<B, T>(int_list_t<Es...>{}, actual_exp, op);
}
template<class T, class EL, class Op>
void dispatch_bits(int_list_t<>, int actual_bits, EL, int, Op&&)
{
  throw std::runtime_error("Unsupported number of bits: " + std::to_string(actual_bits));
}
template<class T, class EL, class Op, int B0, int... Bs>
void dispatch_bits(int_list_t<B0, Bs...>, int actual_bits, EL el, int actual_exp, Op&& op)
{
  if (B0 == actual_bits)
    dispatch_exp<B0, T>(el, actual_exp, op);
  else
    dispatch_bits<T>(int_list_t<Bs...>{}, actual_bits, el, actual_exp, op);
}

template<class T>
struct compress_op
{
  T* data;
  std::size_t n;
  std::uint8_t* out;
  template<int B, int E, class TT>
  void run()
  {
    frsz2_compressor<B, E, TT>(out, n).compress_cpu_impl(data);
  }
};
template<class T>
struct decompress_op
{
  T* data;
  std::size_t n;
  std::uint8_t* in;
  template<int B, int E, class TT>
  void run()
  {
    frsz2_compressor<B, E, TT>(in, n).decompress_cpu_impl(data);
  }
};

} // namespace detail

template<class FpType, int... bit_values, int... exp_block_sizes>
void dispatch_frsz2_compression(int_list_t<bit_values...> bl, int actual_bits_val, int_list_t<exp_block_sizes...> el,
                                int actual_exp_val, FpType* flt_mem, std::size_t total_elems, std::uint8_t* comp_mem)
{
  detail::dispatch_bits<FpType>(bl, actual_bits_val, el, actual_exp_val,
                                detail::compress_op<FpType>{ flt_mem, total_elems, comp_mem });
}

template<class FpType, int... bit_values, int... exp_block_sizes>
void dispatch_frsz2_decompression(int_list_t<bit_values...> bl, int actual_bits_val,
                                  int_list_t<exp_block_sizes...> el, int actual_exp_val, FpType* flt_mem,
                                  std::size_t total_elems, std::uint8_t* comp_mem)
{
  detail::dispatch_bits<FpType>(bl, actual_bits_val, el, actual_exp_val,
                                detail::decompress_op<FpType>{ flt_mem, total_elems, comp_mem });
}

} // namespace frsz

#undef FRSZ2_B200_HD

#endif // FRSZ2_B200_HPP
