// Test-infrastructure driver: runs the REFERENCE library's own public API
// (vsip::Fftm, vsip::vmmul) on inputs read from raw files, so that its outputs
// can pin the oracle and the GPU path.  It is compiled against the reference's
// headers and sources where they lie (see oracle/Makefile) and is never part of
// the product.  With the hand-written configuration in ref_config/ the
// reference's dispatcher selects its generic FP64-accumulating DFT backend
// (src/ovxx/signal/fft/dft.hpp:994-1085), because FFTW3 is not installed.
//
// Usage:
//   ref_driver fwd      ROWS COLS SCALE in.bin  -        out.bin
//   ref_driver inv      ROWS COLS SCALE in.bin  -        out.bin
//   ref_driver phased   ROWS COLS -     in.bin  rep.bin  out.bin
//   ref_driver fused    ROWS COLS -     in.bin  rep.bin  out.bin
//   ref_driver fusedm   ROWS COLS -     in.bin  repm.bin out.bin
//   ref_driver bench    ROWS COLS LOOPS
// Files hold raw interleaved complex<float>, row-major, ROWS x COLS
// (rep.bin: COLS values; repm.bin: ROWS x COLS values).
//
// The call patterns follow the reference benchmark and tests:
//   phased : benchmarks/fastconv.cpp:100-106  (Impl1op)
//   fused  : tests/fastconv.cpp:204            (fused_v_multi, Impl4vc)
//   fusedm : tests/fastconv.cpp:235            (fused_m_multi<0>, Impl4mc)

#include <vsip/initfin.hpp>
#include <vsip/support.hpp>
#include <vsip/math.hpp>
#include <vsip/signal.hpp>
#include <vsip/matrix.hpp>
#include <vsip/vector.hpp>

#include <chrono>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

using namespace vsip;
typedef std::complex<float> cf;

static std::vector<cf> read_file(char const *path, size_t n)
{
  std::vector<cf> v(n);
  FILE *f = std::fopen(path, "rb");
  if (!f) { std::fprintf(stderr, "cannot open %s\n", path); std::exit(2); }
  size_t got = std::fread(v.data(), sizeof(cf), n, f);
  std::fclose(f);
  if (got != n) { std::fprintf(stderr, "short read %s\n", path); std::exit(2); }
  return v;
}

static void write_file(char const *path, Matrix<cf> const &m)
{
  FILE *f = std::fopen(path, "wb");
  if (!f) { std::fprintf(stderr, "cannot open %s\n", path); std::exit(2); }
  for (index_type r = 0; r < m.size(0); ++r)
    for (index_type c = 0; c < m.size(1); ++c)
    {
      cf v = m.get(r, c);
      std::fwrite(&v, sizeof(cf), 1, f);
    }
  std::fclose(f);
}

static void fill(Matrix<cf> &m, std::vector<cf> const &v)
{
  for (index_type r = 0; r < m.size(0); ++r)
    for (index_type c = 0; c < m.size(1); ++c)
      m.put(r, c, v[r * m.size(1) + c]);
}

typedef Fftm<cf, cf, row, fft_fwd, by_reference> fwd_ref_t;
typedef Fftm<cf, cf, row, fft_inv, by_reference> inv_ref_t;
typedef Fftm<cf, cf, row, fft_fwd, by_value> fwd_val_t;
typedef Fftm<cf, cf, row, fft_inv, by_value> inv_val_t;

int main(int argc, char **argv)
{
  vsipl init(argc, argv);
  if (argc < 5) { std::fprintf(stderr, "bad usage\n"); return 2; }
  std::string mode = argv[1];
  length_type rows = std::atol(argv[2]);
  length_type cols = std::atol(argv[3]);

  if (mode == "bench")
  {
    // Phased fast convolution (benchmarks/fastconv.cpp:100-106) on a
    // deterministic input; prints wall seconds for LOOPS calls.
    long loops = std::atol(argv[4]);
    Matrix<cf> data(rows, cols), tmp(rows, cols);
    Vector<cf> replica(cols, cf(0.f, 0.f));
    replica.put(0, cf(1.f, 0.f));
    for (index_type r = 0; r < rows; ++r)
      for (index_type c = 0; c < cols; ++c)
        data.put(r, c, cf(std::sin(0.1f * (r + c)), std::cos(0.07f * c)));
    fwd_ref_t for_fftm(Domain<2>(rows, cols), 1.0);
    inv_ref_t inv_fftm(Domain<2>(rows, cols), 1.0 / cols);
    auto t0 = std::chrono::steady_clock::now();
    for (long l = 0; l < loops; ++l)
    {
      for_fftm(data, tmp);
      tmp = vmmul<0>(replica, tmp);
      inv_fftm(tmp, data);
    }
    auto t1 = std::chrono::steady_clock::now();
    double s = std::chrono::duration<double>(t1 - t0).count();
    std::printf("{\"seconds\": %.6f, \"samples\": %lu}\n", s,
                (unsigned long)(rows * cols * loops));
    return 0;
  }

  if (argc < 8) { std::fprintf(stderr, "bad usage\n"); return 2; }
  Matrix<cf> in(rows, cols), out(rows, cols);
  fill(in, read_file(argv[5], rows * cols));

  if (mode == "fwd" || mode == "inv")
  {
    double scale = std::atof(argv[4]);
    if (mode == "fwd")
    {
      fwd_ref_t f(Domain<2>(rows, cols), scale);
      f(in, out);
    }
    else
    {
      inv_ref_t f(Domain<2>(rows, cols), scale);
      f(in, out);
    }
  }
  else if (mode == "phased" || mode == "fused")
  {
    std::vector<cf> rv = read_file(argv[6], cols);
    Vector<cf> replica(cols);
    for (index_type c = 0; c < cols; ++c) replica.put(c, rv[c]);
    if (mode == "phased")
    {
      Matrix<cf> tmp(rows, cols);
      fwd_ref_t for_fftm(Domain<2>(rows, cols), 1.0);
      inv_ref_t inv_fftm(Domain<2>(rows, cols), 1.0 / cols);
      for_fftm(in, tmp);
      tmp = vmmul<0>(replica, tmp);
      inv_fftm(tmp, out);
    }
    else
    {
      fwd_val_t for_fftm(Domain<2>(rows, cols), 1.0);
      inv_val_t inv_fftm(Domain<2>(rows, cols), 1.0 / cols);
      out = inv_fftm(vmmul<0>(replica, for_fftm(in)));
    }
  }
  else if (mode == "fusedm")
  {
    Matrix<cf> w(rows, cols);
    fill(w, read_file(argv[6], rows * cols));
    fwd_val_t for_fftm(Domain<2>(rows, cols), 1.0);
    inv_val_t inv_fftm(Domain<2>(rows, cols), 1.0 / cols);
    out = inv_fftm(w * for_fftm(in));
  }
  else
  {
    std::fprintf(stderr, "unknown mode %s\n", mode.c_str());
    return 2;
  }
  write_file(argv[7], out);
  return 0;
}
