// Times the fast convolution through the reference's public vsip API with the
// B200 plugin included: vsip::Matrix blocks in (pageable) host memory, the
// same call patterns as the reference benchmark, end to end as an OpenVSIP
// program sees them.
//
//   plugin_bench ROWS COLS LOOPS
// prints one JSON line with, per form, the wall seconds for LOOPS calls:
//   fused  : out = inv_fftm(vmmul<0>(replica, for_fftm(in)))  (by value;
//            benchmarks/fastconv.cpp Impl4vc, tests/fastconv.cpp:204): one
//            fused B200 pass per call through the plugin's be::fc_expr slot
//   phased : for_fftm(data, tmp); tmp = vmmul<0>(replica, tmp);
//            inv_fftm(tmp, data)  (by reference; benchmarks/fastconv.cpp:
//            100-106, Impl1op): two B200 Fftm calls, the vmmul on the host
//            (the plugin replaces Fftm, not vmmul)
#include "ovxx_fcb200.hpp"

#include <vsip/initfin.hpp>

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>

using namespace vsip;
typedef std::complex<float> cf;

int main(int argc, char **argv)
{
  vsipl init(argc, argv);
  if (argc != 4) { std::fprintf(stderr, "usage: plugin_bench ROWS COLS LOOPS\n"); return 2; }
  length_type rows = std::atol(argv[1]), cols = std::atol(argv[2]);
  long loops = std::atol(argv[3]);

  Matrix<cf> data(rows, cols), tmp(rows, cols), out(rows, cols);
  Vector<cf> replica(cols);
  for (index_type c = 0; c < cols; ++c)
    replica.put(c, cf(std::cos(0.001f * c * c), std::sin(0.001f * c * c)) / float(cols));
  for (index_type r = 0; r < rows; ++r)
    for (index_type c = 0; c < cols; ++c)
      data.put(r, c, cf(std::sin(0.1f * (r + c)), std::cos(0.07f * c)));

  typedef std::chrono::steady_clock clk;
  double fused_s = 0, phased_s = 0;
  {
    Fftm<cf, cf, row, fft_fwd, by_value> for_fftm(Domain<2>(rows, cols), 1.0);
    Fftm<cf, cf, row, fft_inv, by_value> inv_fftm(Domain<2>(rows, cols), 1.0);
    out = inv_fftm(vmmul<0>(replica, for_fftm(data)));  // warm-up: plans, staging, the fused plan
    clk::time_point t0 = clk::now();
    for (long l = 0; l < loops; ++l) out = inv_fftm(vmmul<0>(replica, for_fftm(data)));
    fused_s = std::chrono::duration<double>(clk::now() - t0).count();
  }
  {
    Fftm<cf, cf, row, fft_fwd, by_reference> for_fftm(Domain<2>(rows, cols), 1.0);
    Fftm<cf, cf, row, fft_inv, by_reference> inv_fftm(Domain<2>(rows, cols), 1.0);
    for_fftm(data, tmp);
    tmp = vmmul<0>(replica, tmp);
    inv_fftm(tmp, out);
    clk::time_point t0 = clk::now();
    for (long l = 0; l < loops; ++l)
    {
      for_fftm(data, tmp);
      tmp = vmmul<0>(replica, tmp);
      inv_fftm(tmp, out);
    }
    phased_s = std::chrono::duration<double>(clk::now() - t0).count();
  }
  double const samples = double(rows) * double(cols) * double(loops);
  std::printf("{\"rows\": %lu, \"cols\": %lu, \"loops\": %ld, \"fused_seconds\": %.6f, \"phased_seconds\": %.6f, "
              "\"fused_samples_per_s\": %.6e, \"phased_samples_per_s\": %.6e}\n",
              (unsigned long)rows, (unsigned long)cols, loops, fused_s, phased_s, samples / fused_s,
              samples / phased_s);
  return 0;
}
