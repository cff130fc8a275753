// C++ API test: the reference-shaped template API (frsz2_b200.hpp) and the
// plugin front ends (frsz2_b200_plugin.hpp, frsz1_b200_plugin.hpp) over
// libfrsz2_b200.so.
//
// Usage: frsz2_api_test <out.bin>
// Writes, for each of the reference GPU test's end-to-end cases
// (test/test_frsz_gpu.cu:382-410), the 0xFF-canary buffer (+128 slack)
// produced by compress_cpu_impl, so the caller can compare it with the
// reference's bytes.  Exits non-zero on any failed check.
#include "frsz1_b200_plugin.hpp"
#include "frsz2_b200.hpp"
#include "frsz2_b200_plugin.hpp"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

static int failures = 0;
#define CHECK(c)                                                                                                     \
  do {                                                                                                               \
    if (!(c)) {                                                                                                      \
      std::fprintf(stderr, "CHECK failed %s:%d: %s\n", __FILE__, __LINE__, #c);                                      \
      ++failures;                                                                                                    \
    }                                                                                                                \
  } while (0)

// compile-time size algebra (include/frsz2.hpp:525-548)
static_assert(frsz::frsz2_compressor<32, 32, double>::compute_compressed_memory_size_byte(1 << 20) == 4325632, "");
static_assert(frsz::frsz2_compressor<21, 32, double>::compressed_block_size_byte == 84, "");
static_assert(frsz::frsz2_compressor<9, 5, float>::compressed_block_size_element_count == 3, "");
static_assert(std::is_same<frsz::frsz2_compressor<8, 32, double>::exp_type, std::int8_t>::value, "");
static_assert(frsz::frsz2_compressor<8, 1, float>::compute_exponent_block_size_byte(256) == 512, "");

template<class T>
static std::vector<T> pattern(std::size_t n)
{
  const double rep[9] = { 1., 2., 3., 4., .25, -.25, -.125, 1 / 32., .125 };
  std::vector<T> v(n);
  for (std::size_t i = 0; i < n; ++i) v[i] = (T)rep[i % 9];
  return v;
}

template<int B, int E, class T>
static void e2e_case(std::FILE* out, std::size_t n)
{
  using C = frsz::frsz2_compressor<B, E, T>;
  const auto x = pattern<T>(n);
  std::vector<std::uint8_t> buf(C::compute_compressed_memory_size_byte(n) + 128, 0xFF);
  C host(buf.data(), n);
  CHECK(host.compress_cpu_impl(x.data()) == 0);
  std::vector<T> y(n, (T)INFINITY);
  CHECK(host.decompress_cpu_impl(y.data()) == 0);
  CHECK(std::memcmp(x.data(), y.data(), n * sizeof(T)) == 0);

  // device buffers through the same view type
  T* dx = nullptr;
  T* dy = nullptr;
  std::uint8_t* db = nullptr;
  cudaMalloc((void**)&dx, n * sizeof(T));
  cudaMalloc((void**)&dy, n * sizeof(T));
  cudaMalloc((void**)&db, buf.size());
  cudaMemcpy(dx, x.data(), n * sizeof(T), cudaMemcpyHostToDevice);
  cudaMemset(db, 0xFF, buf.size());
  C dev(db, n);
  dev.compress_gpu_impl(dx);
  dev.decompress_gpu_impl(dy);
  std::vector<std::uint8_t> dbuf(buf.size());
  std::vector<T> y2(n);
  cudaMemcpy(dbuf.data(), db, buf.size(), cudaMemcpyDeviceToHost);
  cudaMemcpy(y2.data(), dy, n * sizeof(T), cudaMemcpyDeviceToHost);
  CHECK(dbuf == buf);
  CHECK(std::memcmp(x.data(), y2.data(), n * sizeof(T)) == 0);
  // random access
  std::vector<std::uint64_t> idx = { 0, 1, 7, n / 2, n - 1 };
  std::uint64_t* didx = nullptr;
  T* dv = nullptr;
  cudaMalloc((void**)&didx, idx.size() * 8);
  cudaMalloc((void**)&dv, idx.size() * sizeof(T));
  cudaMemcpy(didx, idx.data(), idx.size() * 8, cudaMemcpyHostToDevice);
  dev.decompress_gpu_elements(didx, idx.size(), dv);
  std::vector<T> v(idx.size());
  cudaMemcpy(v.data(), dv, idx.size() * sizeof(T), cudaMemcpyDeviceToHost);
  for (std::size_t i = 0; i < idx.size(); ++i) CHECK(v[i] == x[idx[i]]);
  // random access on the host buffer, one value and a batch
  for (std::size_t i = 0; i < idx.size(); ++i) CHECK(host.decompress_cpu_element(idx[i]) == x[idx[i]]);
  std::vector<T> hv(idx.size());
  host.decompress_cpu_elements(idx.data(), idx.size(), hv.data());
  for (std::size_t i = 0; i < idx.size(); ++i) CHECK(hv[i] == x[idx[i]]);
  cudaFree(dx);
  cudaFree(dy);
  cudaFree(db);
  cudaFree(didx);
  cudaFree(dv);

  const std::uint32_t hdr[4] = { (std::uint32_t)sizeof(T), (std::uint32_t)B, (std::uint32_t)E,
                                 (std::uint32_t)buf.size() };
  std::fwrite(hdr, sizeof(hdr), 1, out);
  std::fwrite(buf.data(), 1, buf.size(), out);
}

static void dispatch_checks()
{
  using bit_list = frsz::int_list_t<4, 8, 9, 15, 16, 21, 32>;
  using exp_list = frsz::int_list_t<2, 4, 8, 16, 32, 64>;
  const std::size_t n = 1000;
  auto x = pattern<double>(n);
  std::vector<std::uint8_t> a(frsz::frsz2_compressor<21, 32, double>::compute_compressed_memory_size_byte(n), 0);
  std::vector<std::uint8_t> b(a.size(), 0);
  frsz::dispatch_frsz2_compression<double>(bit_list{}, 21, exp_list{}, 32, x.data(), n, a.data());
  frsz::frsz2_compressor<21, 32, double>(b.data(), n).compress_cpu_impl(x.data());
  CHECK(a == b);
  std::vector<double> y(n);
  frsz::dispatch_frsz2_decompression<double>(bit_list{}, 21, exp_list{}, 32, y.data(), n, a.data());
  CHECK(std::memcmp(x.data(), y.data(), n * 8) == 0);
  bool thrown = false;
  try {
    frsz::dispatch_frsz2_compression<double>(bit_list{}, 17, exp_list{}, 32, x.data(), n, a.data());
  } catch (const std::runtime_error& e) {
    thrown = std::string(e.what()) == "Unsupported number of bits: 17";
  }
  CHECK(thrown);
  thrown = false;
  try {
    frsz::dispatch_frsz2_compression<double>(bit_list{}, 16, exp_list{}, 128, x.data(), n, a.data());
  } catch (const std::runtime_error& e) {
    thrown = std::string(e.what()) == "Unsupported exponent block size: 128";
  }
  CHECK(thrown);
}

static void plugin_checks()
{
  frsz2_b200::frsz2_plugin p;
  CHECK(p.get_options().at("frsz2:bits") == 32);
  CHECK(p.get_options().at("frsz2:max_exp_block_size") == 32);
  CHECK(std::string(p.prefix()) == "frsz2" && std::string(p.version()) == "0.0.2");
  CHECK(p.get_configuration().at("pressio:thread_safe") == "multiple");
  p.set_options({ { "frsz2:bits", 16 }, { "frsz2:max_exp_block_size", 8 } });
  auto x = pattern<float>(2160);
  frsz2_b200::data_view in{ frsz2_b200::dtype::float32, x.data(), { 2160 }, false };
  std::vector<std::uint8_t> comp;
  CHECK(p.compress(in, comp) == 0);
  CHECK((comp.size() == frsz::frsz2_compressor<16, 8, float>::compute_compressed_memory_size_byte(2160)));
  std::vector<float> y(2160);
  frsz2_b200::data_view out{ frsz2_b200::dtype::float32, y.data(), { 40, 54 }, false };
  CHECK(p.decompress(comp.data(), comp.size(), out) == 0);
  CHECK(std::memcmp(x.data(), y.data(), x.size() * 4) == 0);
  frsz2_b200::data_view bad{ frsz2_b200::dtype::other, x.data(), { 10 }, false };
  CHECK((p.compress(bad, comp) == 1 && p.error_msg() == "unsupported dtype"));
  p.set_options({ { "frsz2:max_exp_block_size", 48 } });
  CHECK((p.compress(in, comp) == 2 && p.error_msg() == "Unsupported exponent block size: 48"));
  p.set_options({ { "frsz2:max_exp_block_size", 32 }, { "frsz2:bits", 40 } });
  CHECK((p.compress(in, comp) == 2 && p.error_msg() == "Unsupported number of bits: 40"));
}

// The legacy "frsz" plugin: the reference test's known answer
// (test/test_frsz.cc:29-46), the block rules of compress_1d / decompress_1d
// (src/frsz.cc:105-158), the normalized_dims length rule, device data and the
// error surface.
static void legacy_plugin_checks()
{
  using frsz2_b200::data_view;
  using frsz2_b200::dtype;
  frsz2_b200::frsz_plugin p;
  CHECK(p.get_options().at("frsz:epsilon") == 1e-4);
  CHECK(std::string(p.prefix()) == "frsz" && std::string(p.version()) == "0.0.6" && p.patch_version() == 6);
  CHECK(p.get_configuration().at("pressio:stability") == "experimental");
  CHECK(p.get_documentation().at("pressio:description") == "a fixed rate version of the SZ Algorithm");
  p.set_options({ { "frsz:epsilon", 5.0 } });
  std::vector<float> f{ 10.f, 20.f, 30.f, 20.f, 10.f };
  data_view in{ dtype::float32, f.data(), { f.size() }, false };
  std::vector<std::uint8_t> comp;
  CHECK(p.compress(in, comp) == 0 && comp.size() == 10);
  std::int16_t q[5];
  std::memcpy(q, comp.data(), 10);
  CHECK(q[0] == 1 && q[1] == 1 && q[2] == 1 && q[3] == -1 && q[4] == -1);
  std::vector<float> g(5, -1.f);
  data_view out{ dtype::float32, g.data(), { 5 }, false };
  CHECK(p.decompress(comp.data(), comp.size(), out) == 0 && g == f);

  // 600 doubles 0, 2, 4, ... with step 1: block 1's first value is its own,
  // then the reference adds block 0's differences (2 each)
  p.set_options({ { "frsz:epsilon", 0.5 } });
  std::vector<double> x(600);
  for (std::size_t i = 0; i < x.size(); ++i) x[i] = 2.0 * (double)i;
  void* dx = nullptr;
  void* dy = nullptr;
  CHECK(cudaMalloc(&dx, 600 * 8) == cudaSuccess && cudaMalloc(&dy, 600 * 8) == cudaSuccess);
  CHECK(cudaMemcpy(dx, x.data(), 600 * 8, cudaMemcpyHostToDevice) == cudaSuccess);
  data_view din{ dtype::float64, dx, { 600 }, true };
  CHECK(p.compress(din, comp) == 0 && comp.size() == 1200);
  std::vector<std::int16_t> d(600);
  std::memcpy(d.data(), comp.data(), 1200);
  CHECK(d[0] == 0 && d[1] == 2 && d[255] == 2 && d[256] == 512 && d[512] == 1024);
  data_view dout{ dtype::float64, dy, { 600 }, true };
  CHECK(p.decompress(comp.data(), comp.size(), dout) == 0);
  std::vector<double> y(600);
  CHECK(cudaMemcpy(y.data(), dy, 600 * 8, cudaMemcpyDeviceToHost) == cudaSuccess);
  CHECK(y[255] == x[255] && y[256] == x[256] && y[257] == x[256] + 2.0 && y[599] == x[512] + 2.0 * 87);
  cudaFree(dx);
  cudaFree(dy);

  // a 2-D array codes its first extent only; a single value codes none
  std::vector<float> h(2160, 3.0f);
  data_view in2{ dtype::float32, h.data(), { 40, 54 }, false };
  CHECK(p.compress(in2, comp) == 0 && comp.size() == 80);
  data_view one{ dtype::float32, h.data(), { 1 }, false };
  CHECK(p.compress(one, comp) == 0 && comp.empty());

  data_view bad{ dtype::other, h.data(), { 10 }, false };
  CHECK((p.compress(bad, comp) == 1 && p.error_msg() == "unsupported type: currently only floating point supported"));
  CHECK(p.decompress(comp.data(), 0, out) == 2);
}

int main(int argc, char** argv)
{
  register_frsz();
  std::FILE* out = std::fopen(argc > 1 ? argv[1] : "/dev/null", "wb");
  if (!out) return 2;
  e2e_case<32, 32, double>(out, 2049);
  e2e_case<16, 32, double>(out, 2049);
  e2e_case<16, 8, double>(out, 2049);
  e2e_case<15, 8, double>(out, 2049);
  e2e_case<9, 8, double>(out, 2049);
  e2e_case<9, 4, double>(out, 2049);
  e2e_case<9, 5, double>(out, 2049);
  e2e_case<16, 8, float>(out, 2160);
  e2e_case<15, 8, float>(out, 2160);
  e2e_case<9, 4, float>(out, 2160);
  e2e_case<9, 5, float>(out, 2160);
  std::fclose(out);
  dispatch_checks();
  plugin_checks();
  legacy_plugin_checks();
  std::printf("%s (%d failures)\n", failures ? "FAILED" : "OK", failures);
  return failures ? 1 : 0;
}
