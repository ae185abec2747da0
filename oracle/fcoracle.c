/* CPU oracle for the fast-convolution path (TEST INFRASTRUCTURE ONLY; see
 * fcoracle.h).  Restates the reference's arithmetic:
 *
 *   - dft<1,complex,complex>::out_of_place  src/ovxx/signal/fft/dft.hpp:57-66
 *     (O(N^2), accumulate in double, twiddle exp(exponent*2*pi*j*k*w/N)).
 *     The angle's integer product k*w is reduced mod N before the multiply,
 *     which keeps the FP64 twiddle accurate for large N; the sum is the same.
 *   - dftm<complex,complex,row>             src/ovxx/signal/fft/dft.hpp:1040-1058
 *   - vmmul<0>                              src/ovxx/expr/vmmul.hpp:53-59
 *   - workspace scale pass                  src/ovxx/signal/fft/workspace.hpp:474-478
 *   - test::diff (error dB)                 support/test/diff.hpp:41-96
 *
 * The reference's production FFT is FFTW3 (not vendored, version unpinned;
 * call sites src/ovxx/fftw/fftw.cpp:73-95, 965-977).  Its published algorithm
 * is Cooley-Tukey; orc_fft_c64 restates radix-2 Cooley-Tukey in FP64 as the
 * fast oracle for large shapes. */
#include "fcoracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

static const double TWO_PI = 6.283185307179586476925286766559;

void orc_dft_c64(const double *in, long in_stride, double *out,
                 long out_stride, long n, int exponent, double scale)
{
  double *tmp = (double *)malloc(sizeof(double) * 2 * (size_t)n);
  for (long w = 0; w < n; ++w)
  {
    double sr = 0.0, si = 0.0;
    for (long k = 0; k < n; ++k)
    {
      long kw = (long)(((unsigned long long)k * (unsigned long long)w) % (unsigned long long)n);
      double phi = exponent * TWO_PI * (double)kw / (double)n;
      double c = cos(phi), s = sin(phi);
      double xr = in[2 * k * in_stride], xi = in[2 * k * in_stride + 1];
      sr += xr * c - xi * s;
      si += xr * s + xi * c;
    }
    tmp[2 * w] = sr * scale;
    tmp[2 * w + 1] = si * scale;
  }
  for (long w = 0; w < n; ++w)
  {
    out[2 * w * out_stride] = tmp[2 * w];
    out[2 * w * out_stride + 1] = tmp[2 * w + 1];
  }
  free(tmp);
}

static int is_pow2(long n) { return n > 0 && (n & (n - 1)) == 0; }

/* Iterative radix-2 decimation-in-time FFT, in place on a contiguous c64 array. */
static void fft_radix2_inplace(double *a, long n, int exponent)
{
  /* bit reversal */
  for (long i = 1, j = 0; i < n; ++i)
  {
    long bit = n >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j)
    {
      double tr = a[2 * i], ti = a[2 * i + 1];
      a[2 * i] = a[2 * j]; a[2 * i + 1] = a[2 * j + 1];
      a[2 * j] = tr; a[2 * j + 1] = ti;
    }
  }
  /* twiddles exp(exponent * 2 pi j k / n), k < n/2, computed directly */
  double *tw = (double *)malloc(sizeof(double) * (size_t)n);
  for (long k = 0; k < n / 2; ++k)
  {
    double phi = exponent * TWO_PI * (double)k / (double)n;
    tw[2 * k] = cos(phi);
    tw[2 * k + 1] = sin(phi);
  }
  for (long len = 2; len <= n; len <<= 1)
  {
    long half = len >> 1, step = n / len;
    for (long s = 0; s < n; s += len)
      for (long k = 0; k < half; ++k)
      {
        double wr = tw[2 * k * step], wi = tw[2 * k * step + 1];
        double *u = a + 2 * (s + k), *v = a + 2 * (s + k + half);
        double vr = v[0] * wr - v[1] * wi, vi = v[0] * wi + v[1] * wr;
        v[0] = u[0] - vr; v[1] = u[1] - vi;
        u[0] += vr; u[1] += vi;
      }
  }
  free(tw);
}

void orc_fft_c64(const double *in, double *out, long n, int exponent,
                 double scale)
{
  if (!is_pow2(n))
  {
    orc_dft_c64(in, 1, out, 1, n, exponent, scale);
    return;
  }
  if (out != in) memcpy(out, in, sizeof(double) * 2 * (size_t)n);
  fft_radix2_inplace(out, n, exponent);
  if (scale != 1.0)
    for (long i = 0; i < 2 * n; ++i) out[i] *= scale;
}

void orc_fftm_rows_c64(const double *in, long in_rs, double *out, long out_rs,
                       long rows, long cols, int exponent, double scale,
                       int method)
{
#pragma omp parallel for schedule(dynamic)
  for (long r = 0; r < rows; ++r)
  {
    if (method == 0)
      orc_dft_c64(in + 2 * r * in_rs, 1, out + 2 * r * out_rs, 1, cols,
                  exponent, scale);
    else
      orc_fft_c64(in + 2 * r * in_rs, out + 2 * r * out_rs, cols, exponent,
                  scale);
  }
}

void orc_vmmul_rows_c64(const double *v, const double *m, long m_rs,
                        double *out, long out_rs, long rows, long cols)
{
  for (long r = 0; r < rows; ++r)
    for (long c = 0; c < cols; ++c)
    {
      double vr = v[2 * c], vi = v[2 * c + 1];
      double mr = m[2 * (r * m_rs + c)], mi = m[2 * (r * m_rs + c) + 1];
      out[2 * (r * out_rs + c)] = vr * mr - vi * mi;
      out[2 * (r * out_rs + c) + 1] = vr * mi + vi * mr;
    }
}

void orc_fastconv_c64(const float *in, long rows, long cols, const float *rep,
                      long rep_rs, double *out, int method)
{
#pragma omp parallel
  {
    double *x = (double *)malloc(sizeof(double) * 2 * (size_t)cols);
    double *f = (double *)malloc(sizeof(double) * 2 * (size_t)cols);
    double *v = (double *)malloc(sizeof(double) * 2 * (size_t)cols);
#pragma omp for schedule(dynamic)
    for (long r = 0; r < rows; ++r)
    {
      for (long c = 0; c < 2 * cols; ++c) x[c] = (double)in[2 * r * cols + c];
      const float *rp = rep + 2 * r * rep_rs;
      for (long c = 0; c < 2 * cols; ++c) v[c] = (double)rp[c];
      if (method == 0) orc_dft_c64(x, 1, f, 1, cols, -1, 1.0);
      else orc_fft_c64(x, f, cols, -1, 1.0);
      orc_vmmul_rows_c64(v, f, cols, x, cols, 1, cols);
      if (method == 0) orc_dft_c64(x, 1, out + 2 * r * cols, 1, cols, +1, 1.0 / (double)cols);
      else orc_fft_c64(x, out + 2 * r * cols, cols, +1, 1.0 / (double)cols);
    }
    free(x); free(f); free(v);
  }
}

/* FP32 radix-2 FFT used by orc_fastconv_c32 (CPU speed baseline). */
static void fft_radix2_f32(float *a, long n, const float *tw, const long *rev)
{
  for (long i = 0; i < n; ++i)
  {
    long j = rev[i];
    if (i < j)
    {
      float tr = a[2 * i], ti = a[2 * i + 1];
      a[2 * i] = a[2 * j]; a[2 * i + 1] = a[2 * j + 1];
      a[2 * j] = tr; a[2 * j + 1] = ti;
    }
  }
  for (long len = 2; len <= n; len <<= 1)
  {
    long half = len >> 1, step = n / len;
    for (long s = 0; s < n; s += len)
      for (long k = 0; k < half; ++k)
      {
        float wr = tw[2 * k * step], wi = tw[2 * k * step + 1];
        float *u = a + 2 * (s + k), *v = a + 2 * (s + k + half);
        float vr = v[0] * wr - v[1] * wi, vi = v[0] * wi + v[1] * wr;
        v[0] = u[0] - vr; v[1] = u[1] - vi;
        u[0] += vr; u[1] += vi;
      }
  }
}

void orc_fastconv_c32(const float *in, long rows, long cols, const float *rep,
                      long rep_rs, float *out, int threads)
{
  if (!is_pow2(cols)) return;
  float *twf = (float *)malloc(sizeof(float) * (size_t)cols);
  float *twi = (float *)malloc(sizeof(float) * (size_t)cols);
  long *rev = (long *)malloc(sizeof(long) * (size_t)cols);
  for (long k = 0; k < cols / 2; ++k)
  {
    double phi = TWO_PI * (double)k / (double)cols;
    twf[2 * k] = (float)cos(phi); twf[2 * k + 1] = (float)-sin(phi);
    twi[2 * k] = (float)cos(phi); twi[2 * k + 1] = (float)sin(phi);
  }
  int bits = 0;
  while ((1L << bits) < cols) ++bits;
  for (long i = 0; i < cols; ++i)
  {
    long r = 0;
    for (int b = 0; b < bits; ++b) if (i & (1L << b)) r |= 1L << (bits - 1 - b);
    rev[i] = r;
  }
  float inv_n = 1.0f / (float)cols;
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#endif
#pragma omp parallel for schedule(static)
  for (long r = 0; r < rows; ++r)
  {
    float *a = out + 2 * r * cols;
    const float *rp = rep + 2 * r * rep_rs;
    memcpy(a, in + 2 * r * cols, sizeof(float) * 2 * (size_t)cols);
    fft_radix2_f32(a, cols, twf, rev);
    for (long c = 0; c < cols; ++c)
    {
      float xr = a[2 * c], xi = a[2 * c + 1], vr = rp[2 * c], vi = rp[2 * c + 1];
      a[2 * c] = (vr * xr - vi * xi) * inv_n;
      a[2 * c + 1] = (vr * xi + vi * xr) * inv_n;
    }
    fft_radix2_f32(a, cols, twi, rev);
  }
  free(twf); free(twi); free(rev);
}

double orc_error_db(const double *a, const double *b, long n)
{
  double refmax = 0.0, maxsum = -201.0;
  for (long i = 0; i < 2 * n; ++i)
    if (isnan(a[i]) || isnan(b[i])) return 201.0;
  for (long i = 0; i < n; ++i)
  {
    double ma = a[2 * i] * a[2 * i] + a[2 * i + 1] * a[2 * i + 1];
    double mb = b[2 * i] * b[2 * i] + b[2 * i + 1] * b[2 * i + 1];
    if (ma > refmax) refmax = ma;
    if (mb > refmax) refmax = mb;
  }
  for (long i = 0; i < n; ++i)
  {
    double dr = a[2 * i] - b[2 * i], di = a[2 * i + 1] - b[2 * i + 1];
    double d = dr * dr + di * di;
    double s = d < 1.e-20 ? -201.0 : 10.0 * log10(d / (2.0 * refmax));
    if (s > maxsum) maxsum = s;
  }
  return maxsum;
}

void orc_lfm_chirp_c64(long len, double tbp, long n_out, double *out)
{
  memset(out, 0, sizeof(double) * 2 * (size_t)n_out);
  for (long i = 0; i < len && i < n_out; ++i)
  {
    double t = (double)i / (double)len - 0.5;
    double ph = 0.5 * TWO_PI * tbp * t * t;
    out[2 * i] = cos(ph);
    out[2 * i + 1] = sin(ph);
  }
}
