// frsz2_b200_plugin.hpp -- the reference's LibPressio "frsz2" compressor
// plugin front end (robertu94/frsz src/frsz2.cc:25-208), header-only over
// libfrsz2_b200.so, usable without LibPressio.
//
// Same option keys and defaults ("frsz2:bits" = 32,
// "frsz2:max_exp_block_size" = 32, src/frsz2.cc:28-35, 58-64, 201-202), the
// same supported values (float bits 4..32, double bits 4..64, block sizes
// 2..1024 powers of two, src/frsz2.cc:83-134), the same configuration and
// documentation entries (src/frsz2.cc:38-56), the same error codes
// (1 "unsupported dtype", 2 with the dispatch's message, src/frsz2.cc:152-186)
// and version 0.0.2 / prefix "frsz2" (src/frsz2.cc:188-192).
//
// One deliberate difference: compress sizes its output with
// compute_compressed_memory_size_byte (the layout the codec writes), where
// the reference's output_size() (src/frsz2.cc:136-150) computes a smaller,
// legacy size and the codec then writes past the end of that buffer.
//
// Where LibPressio is available, a maintainer derives the LibPressio
// compressor plugin from this class: its options, configuration and
// documentation map one to one onto LibPressio's pressio_options entries.
#ifndef FRSZ2_B200_PLUGIN_HPP
#define FRSZ2_B200_PLUGIN_HPP

#include "frsz2_b200.h"

#include <cstddef>
#include <cstdint>
#include <map>
#include <string>
#include <vector>

#include <cuda_runtime_api.h>

namespace frsz2_b200 {

enum class dtype
{
  float32,
  float64,
  other
};

// A LibPressio-like data descriptor: element type, dimensions and a pointer
// to host or device memory.
struct data_view
{
  dtype type = dtype::other;
  void* ptr = nullptr;
  std::vector<std::size_t> dims;
  bool on_device = false;

  std::size_t num_elements() const
  {
    std::size_t n = dims.empty() ? 0 : 1;
    for (auto d : dims) n *= d;
    return n;
  }
};

class frsz2_plugin
{
public:
  std::map<std::string, std::uint64_t> get_options() const
  {
    return { { "frsz2:bits", bits }, { "frsz2:max_exp_block_size", max_exp_block_size } };
  }

  int set_options(const std::map<std::string, std::uint64_t>& options)
  {
    auto b = options.find("frsz2:bits");
    if (b != options.end()) bits = b->second;
    auto e = options.find("frsz2:max_exp_block_size");
    if (e != options.end()) max_exp_block_size = e->second;
    return 0;
  }

  std::map<std::string, std::string> get_configuration() const
  {
    return { { "pressio:thread_safe", "multiple" }, { "pressio:stability", "experimental" } };
  }

  std::map<std::string, std::string> get_documentation() const
  {
    return { { "pressio:description", "a fixed rate compressor which uses block exponents + rounding" },
             { "frsz2:bits", "the number of bits to use per symbol" },
             { "frsz2:max_exp_block_size",
               "the number of elements to have a common exponent. Supported values: 2, 4, 8, 16, 32, 64, 128, 256, "
               "512, 1024" } };
  }

  // Bytes compress() produces for `n` values of `type` with the current options.
  std::size_t compressed_size(dtype type, std::size_t n) const
  {
    std::uint64_t sz = 0;
    if (type == dtype::other || frsz2_compressed_size(code(type), (int)bits, (int)max_exp_block_size, n, &sz) != 0)
      return 0;
    return (std::size_t)sz;
  }

  // Compress into a buffer this call sizes and fills.  `input` may live on
  // the host or the device; `output` is host memory.
  int compress(const data_view& input, std::vector<std::uint8_t>& output)
  {
    if (input.type == dtype::other) return set_error(1, "unsupported dtype");
    if (int rc = check_supported(input.type)) return rc;
    const std::size_t n = input.num_elements();
    output.assign(compressed_size(input.type, n), 0);
    int rc;
    if (input.on_device) {
      void* d_out = nullptr;
      if (cudaMalloc(&d_out, output.size()) != cudaSuccess) return set_error(2, "device allocation failed");
      rc = frsz2_compress(code(input.type), (int)bits, (int)max_exp_block_size, input.ptr, n, d_out, nullptr);
      if (rc == 0 && cudaMemcpy(output.data(), d_out, output.size(), cudaMemcpyDeviceToHost) != cudaSuccess)
        rc = set_error(2, "copy of the compressed buffer failed");
      cudaFree(d_out);
    } else {
      rc = frsz2_compress_host(code(input.type), (int)bits, (int)max_exp_block_size, input.ptr, n, output.data(),
                               nullptr);
    }
    return rc ? set_error(2, frsz2_last_error()) : 0;
  }

  // Decompress into `output`, whose dtype and dims the caller sets
  // (src/frsz2.cc:171-186).  Host or device output memory.
  int decompress(const std::uint8_t* input, std::size_t input_bytes, data_view& output)
  {
    if (output.type == dtype::other) return set_error(1, "unsupported dtype");
    if (int rc = check_supported(output.type)) return rc;
    const std::size_t n = output.num_elements();
    const std::size_t need = compressed_size(output.type, n);
    if (input_bytes < need) return set_error(2, "compressed input is shorter than the format requires");
    int rc;
    if (output.on_device) {
      void* d_in = nullptr;
      if (cudaMalloc(&d_in, need) != cudaSuccess) return set_error(2, "device allocation failed");
      rc = cudaMemcpy(d_in, input, need, cudaMemcpyHostToDevice) == cudaSuccess
             ? frsz2_decompress(code(output.type), (int)bits, (int)max_exp_block_size, d_in, n, output.ptr, nullptr)
             : set_error(2, "copy of the compressed buffer failed");
      if (rc == 0 && cudaDeviceSynchronize() != cudaSuccess) rc = set_error(2, "decompress failed");
      cudaFree(d_in);
    } else {
      rc = frsz2_decompress_host(code(output.type), (int)bits, (int)max_exp_block_size, input, n, output.ptr,
                                 nullptr);
    }
    return rc ? set_error(2, frsz2_last_error()) : 0;
  }

  int error_code() const { return error_code_; }
  const std::string& error_msg() const { return error_msg_; }
  int major_version() const { return 0; }
  int minor_version() const { return 0; }
  int patch_version() const { return 2; }
  const char* version() const { return "0.0.2"; }
  const char* prefix() const { return "frsz2"; }

  std::uint64_t bits = 32;
  std::uint64_t max_exp_block_size = 32;

private:
  static int code(dtype t) { return t == dtype::float32 ? FRSZ2_FLOAT : FRSZ2_DOUBLE; }

  // The plugin's instantiated lists (src/frsz2.cc:83-134).
  int check_supported(dtype t)
  {
    const std::uint64_t max_bits = t == dtype::float32 ? 32 : 64;
    if (bits < 4 || bits > max_bits) return set_error(2, "Unsupported number of bits: " + std::to_string(bits));
    const std::uint64_t e = max_exp_block_size;
    if (e < 2 || e > 1024 || (e & (e - 1)) != 0)
      return set_error(2, "Unsupported exponent block size: " + std::to_string(e));
    return 0;
  }

  int set_error(int code, const std::string& msg)
  {
    error_code_ = code;
    error_msg_ = msg;
    return code;
  }

  int error_code_ = 0;
  std::string error_msg_;
};

} // namespace frsz2_b200

#endif // FRSZ2_B200_PLUGIN_HPP
