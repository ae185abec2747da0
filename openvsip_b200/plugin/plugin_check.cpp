// Drives the fast-convolution path through the reference's public vsip API with
// the B200 plugin included, on data read from a file, and writes the results,
// so that a test can compare them with the FP64 oracle.
//
//   plugin_check ROWS COLS in.bin weights.bin out_prefix
// writes out_prefix.{phased,fused,fusedm,fusedm2,fusedm3}.bin: the phased Fftm -> vmmul -> Fftm
// form (benchmarks/fastconv.cpp:100-106), the fused by-value expression
// (tests/fastconv.cpp:204) and the matrix-of-coefficients expression with each
// row's weights equal to the vector times (1 + row/ROWS), called twice
// (fusedm, fusedm2: the second reuses the cached plan) and once more after
// the last row's last weight is doubled (fusedm3); and
// out_prefix.{fft2d,fft2d_rt}.bin: the 2-D vsip::Fft of the input and the
// inverse 2-D Fft (scale 1 / (ROWS COLS), by value) of that result.
#include "ovxx_fcb200.hpp"

#include <vsip/initfin.hpp>

#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

using namespace vsip;
typedef std::complex<float> cf;

static void save(std::string const &path, Matrix<cf> const &m)
{
  FILE *f = std::fopen(path.c_str(), "wb");
  for (index_type r = 0; r < m.size(0); ++r)
    for (index_type c = 0; c < m.size(1); ++c)
    {
      cf v = m.get(r, c);
      std::fwrite(&v, sizeof(cf), 1, f);
    }
  std::fclose(f);
}

int main(int argc, char **argv)
{
  vsipl init(argc, argv);
  if (argc != 6) { std::fprintf(stderr, "usage\n"); return 2; }
  length_type rows = std::atol(argv[1]), cols = std::atol(argv[2]);
  std::vector<cf> x(rows * cols), w(cols);
  FILE *f = std::fopen(argv[3], "rb");
  if (!f || std::fread(x.data(), sizeof(cf), x.size(), f) != x.size()) return 2;
  std::fclose(f);
  f = std::fopen(argv[4], "rb");
  if (!f || std::fread(w.data(), sizeof(cf), w.size(), f) != w.size()) return 2;
  std::fclose(f);
  std::string prefix = argv[5];

  Matrix<cf> in(rows, cols), tmp(rows, cols), out(rows, cols), wm(rows, cols);
  Vector<cf> wv(cols);
  for (index_type c = 0; c < cols; ++c) wv.put(c, w[c]);
  for (index_type r = 0; r < rows; ++r)
    for (index_type c = 0; c < cols; ++c)
    {
      in.put(r, c, x[r * cols + c]);
      wm.put(r, c, w[c] * (1.f + float(r) / float(rows)));
    }

  {
    Fftm<cf, cf, row, fft_fwd, by_reference> for_fftm(Domain<2>(rows, cols), 1.0);
    Fftm<cf, cf, row, fft_inv, by_reference> inv_fftm(Domain<2>(rows, cols), 1.0 / cols);
    for_fftm(in, tmp);
    tmp = vmmul<0>(wv, tmp);
    inv_fftm(tmp, out);
    save(prefix + ".phased.bin", out);
  }
  {
    Fftm<cf, cf, row, fft_fwd, by_value> for_fftm(Domain<2>(rows, cols), 1.0);
    Fftm<cf, cf, row, fft_inv, by_value> inv_fftm(Domain<2>(rows, cols), 1.0 / cols);
    out = inv_fftm(vmmul<0>(wv, for_fftm(in)));
    save(prefix + ".fused.bin", out);
    out = inv_fftm(wm * for_fftm(in));
    save(prefix + ".fusedm.bin", out);
    // the same weights again (the cached fused plan), then one weight changed
    out = inv_fftm(wm * for_fftm(in));
    save(prefix + ".fusedm2.bin", out);
    wm.put(rows - 1, cols - 1, wm.get(rows - 1, cols - 1) * 2.f);
    out = inv_fftm(wm * for_fftm(in));
    save(prefix + ".fusedm3.bin", out);
  }
  {
    Fft<const_Matrix, cf, cf, fft_fwd, by_reference> f2(Domain<2>(rows, cols), 1.0);
    Fft<const_Matrix, cf, cf, fft_inv, by_value> g2(Domain<2>(rows, cols), 1.0 / (rows * cols));
    f2(in, out);
    save(prefix + ".fft2d.bin", out);
    tmp = g2(out);
    save(prefix + ".fft2d_rt.bin", tmp);
  }
  return 0;
}
