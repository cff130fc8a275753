// ref_shim.cpp -- C entry points over the UNMODIFIED reference codec.
//
// TEST INFRASTRUCTURE ONLY.  Built by oracle/Makefile against the reference's
// own include/frsz2.hpp (read where it lies, never copied) into
// oracle/_ref/libfrsz2_ref.so.  tests/ uses it to pin the C restatement
// (oracle/frsz2_oracle.c); bench.py times it as the reference CPU path.
//
// The runtime (bits, E) -> template dispatch below is this file's own; the
// codec work is done by the reference's frsz::frsz2_compressor methods
// compress_cpu_impl / decompress_cpu_impl (frsz2.hpp:1181, 1242),
// compress_cpu_block / decompress_cpu_block (frsz2.hpp:1108, 1217) and
// decompress_cpu_element (frsz2.hpp:1199), and the detail::fp primitives.
#include "frsz2.hpp"

#include <cstddef>
#include <cstdint>
#include <thread>
#include <vector>

namespace {

template<int... V>
struct ilist
{};

// Call f.template run<bits, E, T>() for the runtime (bits, E); return 2 when
// either value is not in the instantiated lists.
template<class T, class F, int B, int... E>
int walk_e(ilist<>, int, F&)
{
  return 2;
}
template<class T, class F, int B, int E0, int... Es>
int walk_e(ilist<E0, Es...>, int e, F& f)
{
  if (e == E0) {
    f.template run<B, E0, T>();
    return 0;
  }
  return walk_e<T, F, B>(ilist<Es...>{}, e, f);
}
template<class T, class F, class EL>
int walk_b(ilist<>, int, EL, int, F&)
{
  return 2;
}
template<class T, class F, class EL, int B0, int... Bs>
int walk_b(ilist<B0, Bs...>, int b, EL el, int e, F& f)
{
  if (b == B0) return walk_e<T, F, B0>(el, e, f);
  return walk_b<T, F>(ilist<Bs...>{}, b, el, e, f);
}

using e_list = ilist<1, 2, 4, 5, 8, 16, 32, 64, 128, 256, 512, 1024>;
using b32_list = ilist<4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16, 17, 18, 19, 20, 21, 22, 23, 24, 25, 26,
                       27, 28, 29, 30, 31, 32>;
using b64_list =
  ilist<4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16, 17, 18, 19, 20, 21, 22, 23, 24, 25, 26, 27, 28, 29, 30,
        31, 32, 33, 34, 35, 36, 37, 38, 39, 40, 41, 42, 43, 44, 45, 46, 47, 48, 49, 50, 51, 52, 53, 54, 55, 56,
        57, 58, 59, 60, 61, 62, 63, 64>;

template<class T>
struct bit_list_for;
template<>
struct bit_list_for<float>
{
  using type = b32_list;
};
template<>
struct bit_list_for<double>
{
  using type = b64_list;
};

template<class T, class F>
int dispatch(int bits, int e, F& f)
{
  return walk_b<T, F>(typename bit_list_for<T>::type{}, bits, e_list{}, e, f);
}

// Block range [b0, b1) handled by one thread, through the reference's own
// per-block methods.  Blocks are disjoint in both the exponent and the word
// regions, so threads never touch the same byte.
template<class T>
struct codec_job
{
  const void* in;
  void* out;
  std::size_t n;
  int threads;
  bool compress;
  std::size_t size_bytes = 0;

  template<int B, int E, class TT>
  void run()
  {
    using C = frsz::frsz2_compressor<B, E, TT>;
    size_bytes = C::compute_compressed_memory_size_byte(n);
    if (threads <= 1) {
      if (compress) {
        C c(static_cast<std::uint8_t*>(out), n);
        c.compress_cpu_impl(static_cast<const TT*>(in));
      } else {
        C c(const_cast<std::uint8_t*>(static_cast<const std::uint8_t*>(in)), n);
        c.decompress_cpu_impl(static_cast<TT*>(out));
      }
      return;
    }
    const std::size_t nb = (n + E - 1) / E;
    const std::size_t per = (nb + threads - 1) / threads;
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t) {
      const std::size_t b0 = std::min(nb, per * t), b1 = std::min(nb, b0 + per);
      pool.emplace_back([=]() {
        if (compress) {
          C c(static_cast<std::uint8_t*>(out), n);
          const TT* x = static_cast<const TT*>(in);
          for (std::size_t b = b0; b < b1; ++b)
            c.compress_cpu_block(b, x + b * E, std::min<std::size_t>(E, n - b * E));
        } else {
          const C c(const_cast<std::uint8_t*>(static_cast<const std::uint8_t*>(in)), n);
          TT* y = static_cast<TT*>(out);
          for (std::size_t b = b0; b < b1; ++b)
            c.decompress_cpu_block(b, y + b * E);
        }
      });
    }
    for (auto& th : pool) th.join();
  }
};

template<class T>
struct element_job
{
  const std::uint8_t* in;
  std::size_t n, idx;
  T value{};

  template<int B, int E, class TT>
  void run()
  {
    const frsz::frsz2_compressor<B, E, TT> c(const_cast<std::uint8_t*>(in), n);
    value = c.decompress_cpu_element(idx);
  }
};

struct size_job
{
  std::size_t n, size_bytes = 0, exp_bytes = 0;
  template<int B, int E, class TT>
  void run()
  {
    using C = frsz::frsz2_compressor<B, E, TT>;
    size_bytes = C::compute_compressed_memory_size_byte(n);
    exp_bytes = C::compute_exponent_block_size_byte(n);
  }
};

} // namespace

extern "C" {

int frsz2ref_compress(int is_f64, int bits, int e, const void* in, std::size_t n, void* out, int threads)
{
  if (is_f64) {
    codec_job<double> j{ in, out, n, threads, true };
    return dispatch<double>(bits, e, j);
  }
  codec_job<float> j{ in, out, n, threads, true };
  return dispatch<float>(bits, e, j);
}

int frsz2ref_decompress(int is_f64, int bits, int e, const void* in, std::size_t n, void* out, int threads)
{
  if (is_f64) {
    codec_job<double> j{ in, out, n, threads, false };
    return dispatch<double>(bits, e, j);
  }
  codec_job<float> j{ in, out, n, threads, false };
  return dispatch<float>(bits, e, j);
}

double frsz2ref_decompress_element_f64(int bits, int e, const void* in, std::size_t n, std::size_t idx)
{
  element_job<double> j{ static_cast<const std::uint8_t*>(in), n, idx };
  dispatch<double>(bits, e, j);
  return j.value;
}

float frsz2ref_decompress_element_f32(int bits, int e, const void* in, std::size_t n, std::size_t idx)
{
  element_job<float> j{ static_cast<const std::uint8_t*>(in), n, idx };
  dispatch<float>(bits, e, j);
  return j.value;
}

int frsz2ref_sizes(int is_f64, int bits, int e, std::size_t n, std::size_t* total, std::size_t* exps)
{
  size_job j{ n };
  const int rc = is_f64 ? dispatch<double>(bits, e, j) : dispatch<float>(bits, e, j);
  *total = j.size_bytes;
  *exps = j.exp_bytes;
  return rc;
}

// detail::fp primitives (frsz2.hpp:312-399), for the known-answer tests.
int frsz2ref_exponent_f32(float x) { return frsz::detail::fp::exponent(x); }
int frsz2ref_exponent_f64(double x) { return frsz::detail::fp::exponent(x); }
std::uint32_t frsz2ref_significand_f32(float x) { return frsz::detail::fp::significand(x); }
std::uint64_t frsz2ref_significand_f64(double x) { return frsz::detail::fp::significand(x); }
int frsz2ref_sign_f32(float x) { return frsz::detail::fp::sign(x); }
int frsz2ref_sign_f64(double x) { return frsz::detail::fp::sign(x); }
std::uint32_t frsz2ref_floating_to_fixed_f32(float x, std::int16_t e)
{
  return frsz::detail::fp::floating_to_fixed(x, e);
}
std::uint64_t frsz2ref_floating_to_fixed_f64(double x, std::int16_t e)
{
  return frsz::detail::fp::floating_to_fixed(x, e);
}
float frsz2ref_fixed_to_floating_f32(std::uint32_t v, std::int16_t e)
{
  return frsz::detail::fp::fixed_to_floating<float>(v, e);
}
double frsz2ref_fixed_to_floating_f64(std::uint64_t v, std::int16_t e)
{
  return frsz::detail::fp::fixed_to_floating<double>(v, e);
}

} // extern "C"
