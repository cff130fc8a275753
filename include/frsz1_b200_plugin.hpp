// frsz1_b200_plugin.hpp -- the reference's LibPressio "frsz" compressor plugin
// front end (robertu94/frsz src/frsz.cc:17-161, the legacy epsilon codec),
// header-only over libfrsz2_b200.so, usable without LibPressio.
//
// Same option key and default ("frsz:epsilon" = 1e-4, src/frsz.cc:19-23, 42-46,
// 160), the same configuration and documentation entries (src/frsz.cc:25-39),
// the same error code and message for other dtypes (1, "unsupported type:
// currently only floating point supported", src/frsz.cc:57-58, 74-75), version
// 0.0.6 (the project version, CMakeLists.txt:3) and prefix "frsz".
//
// The number of values coded is the reference's normalized_dims(1).at(0)
// (src/frsz.cc:108, 139): LibPressio's pressio_data::normalized_dims drops the
// dimensions of extent 1 and cuts the list to its first entry, 0 when none is
// left.  A 1-D array codes all its values, a 2-D array its first extent only.
//
// The work runs in the library's CUDA kernels (frsz1_compress /
// frsz1_decompress), bit for bit the reference's compress_1d / decompress_1d;
// host data is copied to the current device and back.  Status 2 carries the
// library's message: a device failure, or epsilon <= 0, which the library
// rejects and the reference would code into saturated or zero differences.
#ifndef FRSZ1_B200_PLUGIN_HPP
#define FRSZ1_B200_PLUGIN_HPP

#include "frsz2_b200.h"
#include "frsz2_b200_plugin.hpp" // dtype, data_view

#include <cstddef>
#include <cstdint>
#include <map>
#include <string>
#include <vector>

#include <cuda_runtime_api.h>

namespace frsz2_b200 {

// The values a "frsz" compress or decompress codes for these dimensions.
inline std::size_t legacy_length(const std::vector<std::size_t>& dims)
{
  for (auto d : dims)
    if (d > 1) return d;
  return 0;
}

class frsz_plugin
{
public:
  std::map<std::string, double> get_options() const { return { { "frsz:epsilon", epsilon } }; }

  int set_options(const std::map<std::string, double>& options)
  {
    auto e = options.find("frsz:epsilon");
    if (e != options.end()) epsilon = e->second;
    return 0;
  }

  std::map<std::string, std::string> get_configuration() const
  {
    return { { "pressio:thread_safe", "multiple" }, { "pressio:stability", "experimental" } };
  }

  std::map<std::string, std::string> get_documentation() const
  {
    return { { "pressio:description", "a fixed rate version of the SZ Algorithm" },
             { "frsz:epsilon",
               "\"absolute error bound\" applied during quantization; because frsz does not store unpredictable "
               "values, this is not a true absolute error bound" } };
  }

  std::map<std::string, std::string> get_metrics_results() const { return {}; }

  // Bytes compress() produces for an input of these dimensions.
  std::size_t compressed_size(const std::vector<std::size_t>& dims) const
  {
    return (std::size_t)frsz1_compressed_size(legacy_length(dims));
  }

  // The int16 stream of `input` (host or device) into host bytes, two per
  // coded value (compress_1d, src/frsz.cc:105-135).
  int compress(const data_view& input, std::vector<std::uint8_t>& output)
  {
    if (input.type == dtype::other) return set_error(1, unsupported_type);
    const std::size_t n = legacy_length(input.dims);
    output.assign(compressed_size(input.dims), 0);
    if (n == 0) return 0;
    const std::size_t in_bytes = n * value_bytes(input.type);
    void* d_in = input.on_device ? input.ptr : nullptr;
    void* d_out = nullptr;
    int rc = 0;
    if (cudaMalloc(&d_out, output.size()) != cudaSuccess ||
        (!input.on_device && cudaMalloc(&d_in, in_bytes) != cudaSuccess))
      rc = set_error(2, "device allocation failed");
    if (rc == 0 && !input.on_device && cudaMemcpy(d_in, input.ptr, in_bytes, cudaMemcpyHostToDevice) != cudaSuccess)
      rc = set_error(2, "copy of the input failed");
    if (rc == 0 && frsz1_compress(code(input.type), epsilon, d_in, n, d_out, nullptr) != 0)
      rc = set_error(2, frsz2_last_error());
    if (rc == 0 && cudaMemcpy(output.data(), d_out, output.size(), cudaMemcpyDeviceToHost) != cudaSuccess)
      rc = set_error(2, "copy of the compressed buffer failed");
    if (!input.on_device) cudaFree(d_in);
    cudaFree(d_out);
    return rc;
  }

  // Fill the first legacy_length(output.dims) values of `output` (host or
  // device; its dtype and dims the caller sets) from host bytes, adding
  // block 0's differences in every block as the reference does
  // (decompress_1d, src/frsz.cc:137-158).
  int decompress(const std::uint8_t* input, std::size_t input_bytes, data_view& output)
  {
    if (output.type == dtype::other) return set_error(1, unsupported_type);
    const std::size_t n = legacy_length(output.dims);
    const std::size_t need = (std::size_t)frsz1_compressed_size(n);
    if (input_bytes < need) return set_error(2, "compressed input is shorter than the format requires");
    if (n == 0) return 0;
    const std::size_t out_bytes = n * value_bytes(output.type);
    void* d_in = nullptr;
    void* d_out = output.on_device ? output.ptr : nullptr;
    int rc = 0;
    if (cudaMalloc(&d_in, need) != cudaSuccess || (!output.on_device && cudaMalloc(&d_out, out_bytes) != cudaSuccess))
      rc = set_error(2, "device allocation failed");
    if (rc == 0 && cudaMemcpy(d_in, input, need, cudaMemcpyHostToDevice) != cudaSuccess)
      rc = set_error(2, "copy of the compressed buffer failed");
    if (rc == 0 && frsz1_decompress(code(output.type), epsilon, d_in, n, d_out, 0, nullptr) != 0)
      rc = set_error(2, frsz2_last_error());
    if (rc == 0) {
      const cudaError_t e = output.on_device ? cudaDeviceSynchronize()
                                             : cudaMemcpy(output.ptr, d_out, out_bytes, cudaMemcpyDeviceToHost);
      if (e != cudaSuccess) rc = set_error(2, "decompress failed");
    }
    if (!output.on_device) cudaFree(d_out);
    cudaFree(d_in);
    return rc;
  }

  int error_code() const { return error_code_; }
  const std::string& error_msg() const { return error_msg_; }
  int major_version() const { return 0; }
  int minor_version() const { return 0; }
  int patch_version() const { return 6; }
  const char* version() const { return "0.0.6"; }
  const char* prefix() const { return "frsz"; }

  double epsilon = 1e-4;

private:
  static constexpr const char* unsupported_type = "unsupported type: currently only floating point supported";

  static int code(dtype t) { return t == dtype::float32 ? FRSZ2_FLOAT : FRSZ2_DOUBLE; }
  static std::size_t value_bytes(dtype t) { return t == dtype::float32 ? 4 : 8; }

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

#endif // FRSZ1_B200_PLUGIN_HPP
