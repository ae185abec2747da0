// Real-input row FFTs (real -> complex forward, complex -> real inverse) on
// top of the complex row FFT, for fftm_backend<float, complex<float>, A,
// fft_fwd> and fftm_backend<complex<float>, float, A, fft_inv>
// (src/ovxx/signal/fft/backend.hpp:600-694; FFTW r2c / c2r rows,
// src/ovxx/fftw/fftw.cpp:778-903).
//
// Even n = 2m: the n real samples of a row are read as m complex values
// z[j] = x[2j] + i x[2j+1] and transformed by a length-m complex FFT Z.  With
// E[k] = (Z[k] + conj Z[m-k]) / 2 and O[k] = (Z[k] - conj Z[m-k]) / (2i)
// (Z[m] = Z[0]), the spectra of the even and odd samples, the output is
// X[k] = E[k] + W_n^k O[k] for k = 0 .. m.  The inverse runs the same steps
// backwards: Z[k] = E'[k] + i O'[k] with E'[k] = X[k] + conj X[m-k] and
// O'[k] = (X[k] - conj X[m-k]) W_n^-k, then an unnormalised inverse length-m
// FFT gives x[2j] + i x[2j+1].  As FFTW's c2r does, the imaginary parts of
// X[0] and X[m] are ignored (the input is taken as the half spectrum of a real
// signal).
//
// Odd n: rows go through the length-n complex FFT (Bluestein) with a zero
// imaginary part (forward) or the full Hermitian spectrum (inverse).
#include "fcb200.h"
#include "fcb_internal.h"

#include <cuda_runtime.h>

namespace fcb {

namespace {

__device__ __forceinline__ float2 cmul(float2 a, float2 b)
{
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 conjf2(float2 a) { return make_float2(a.x, -a.y); }

unsigned grid_for(long long total)
{
  long long b = (total + 255) / 256;
  return (unsigned)(b > 148 * 32 ? 148 * 32 : (b < 1 ? 1 : b));
}

// w[k] = exp(-2 pi i k / n), k = 0 .. count - 1, built in FP64.
__global__ void real_tw_kernel(float2 *w, long long n, long long count)
{
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= count) return;
  double s, c;
  sincospi(-2.0 * (double)k / (double)n, &s, &c);
  w[k] = make_float2((float)c, (float)s);
}

// X[j] = E_j + W^j O_j from Z[j] and Z[m - j], for j = k and j = m - k, in place.
__global__ void r2c_post_kernel(float2 *y, long long rs, long long m, long long rows, const float2 *w, float scale)
{
  const long long half = m / 2 + 1;  // k = 0 .. m/2
  const long long total = rows * half;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x)
  {
    const long long r = i / half, k = i % half;
    float2 *row = y + r * rs;
    if (k == 0)
    {
      const float2 z = row[0];
      row[0] = make_float2(scale * (z.x + z.y), 0.f);
      row[m] = make_float2(scale * (z.x - z.y), 0.f);
      continue;
    }
    const long long j2 = m - k;
    const float2 a = row[k], b = row[j2];
    // j = k: E = (a + conj b) / 2, O = (a - conj b) / (2i)
    const float2 e1 = make_float2(0.5f * (a.x + b.x), 0.5f * (a.y - b.y));
    const float2 d1 = make_float2(a.x - b.x, a.y + b.y);
    const float2 o1 = make_float2(0.5f * d1.y, -0.5f * d1.x);
    // j = m - k: E = (b + conj a) / 2, O = (b - conj a) / (2i)
    const float2 e2 = make_float2(0.5f * (b.x + a.x), 0.5f * (b.y - a.y));
    const float2 d2 = make_float2(b.x - a.x, b.y + a.y);
    const float2 o2 = make_float2(0.5f * d2.y, -0.5f * d2.x);
    const float2 x1 = cmul(w[k], o1), x2 = cmul(w[j2], o2);
    row[k] = make_float2(scale * (e1.x + x1.x), scale * (e1.y + x1.y));
    if (j2 != k) row[j2] = make_float2(scale * (e2.x + x2.x), scale * (e2.y + x2.y));
  }
}

// Z[k] = E'[k] + i O'[k], k = 0 .. m - 1, from the half spectrum X[0 .. m].
__global__ void c2r_pre_kernel(const float2 *x, long long x_rs, float2 *z, long long z_rs, long long m,
                               long long rows, const float2 *w)
{
  const long long total = rows * m;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x)
  {
    const long long r = i / m, k = i % m;
    const float2 *row = x + r * x_rs;
    float2 a = row[k], b = row[m - k];
    if (k == 0)
    {
      a.y = 0.f;
      b.y = 0.f;
    }
    const float2 e = make_float2(a.x + b.x, a.y - b.y);               // X[k] + conj X[m-k]
    const float2 o = cmul(make_float2(a.x - b.x, a.y + b.y), conjf2(w[k]));  // (X[k] - conj X[m-k]) W^-k
    z[r * z_rs + k] = make_float2(e.x - o.y, e.y + o.x);               // E' + i O'
  }
}

__global__ void real_expand_kernel(const float *x, long long x_rs, float2 *z, long long n, long long rows)
{
  const long long total = rows * n;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x)
  {
    const long long r = i / n, k = i % n;
    z[i] = make_float2(x[r * x_rs + k], 0.f);
  }
}

// Full spectrum of a real signal of odd length n from its half X[0 .. n/2].
__global__ void herm_expand_kernel(const float2 *x, long long x_rs, float2 *z, long long n, long long rows)
{
  const long long total = rows * n, h = n / 2;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x)
  {
    const long long r = i / n, k = i % n;
    const float2 *row = x + r * x_rs;
    float2 v = k <= h ? row[k] : conjf2(row[n - k]);
    if (k == 0) v.y = 0.f;
    z[i] = v;
  }
}

__global__ void take_real_kernel(const float2 *z, long long n, float *out, long long out_rs, long long rows)
{
  const long long total = rows * n;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x)
  {
    const long long r = i / n, k = i % n;
    out[r * out_rs + k] = z[i].x;
  }
}

int launched(const char *what)
{
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? FCB_OK : cuda_error(e, what);
}

}  // namespace

int real_twiddles(long long n, long long count, float2 **out, cudaStream_t st)
{
  float2 *w = nullptr;
  cudaError_t e = cudaMalloc(&w, sizeof(float2) * (size_t)count);
  if (e != cudaSuccess) return set_error(FCB_ERR_NOMEM, "real-FFT twiddles: %s", cudaGetErrorString(e));
  real_tw_kernel<<<(unsigned)((count + 255) / 256), 256, 0, st>>>(w, n, count);
  int rc = launched("real-FFT twiddles");
  if (rc) { cudaFree(w); return rc; }
  *out = w;
  return FCB_OK;
}

int r2c_post(float2 *y, long long rs, long long m, long long rows, const float2 *w, float scale, cudaStream_t st)
{
  r2c_post_kernel<<<grid_for(rows * (m / 2 + 1)), 256, 0, st>>>(y, rs, m, rows, w, scale);
  return launched("real FFT split");
}

int c2r_pre(const float2 *x, long long x_rs, float2 *z, long long z_rs, long long m, long long rows,
            const float2 *w, cudaStream_t st)
{
  c2r_pre_kernel<<<grid_for(rows * m), 256, 0, st>>>(x, x_rs, z, z_rs, m, rows, w);
  return launched("real FFT merge");
}

int real_expand(const float *x, long long x_rs, float2 *z, long long n, long long rows, cudaStream_t st)
{
  real_expand_kernel<<<grid_for(rows * n), 256, 0, st>>>(x, x_rs, z, n, rows);
  return launched("real expand");
}

int herm_expand(const float2 *x, long long x_rs, float2 *z, long long n, long long rows, cudaStream_t st)
{
  herm_expand_kernel<<<grid_for(rows * n), 256, 0, st>>>(x, x_rs, z, n, rows);
  return launched("Hermitian expand");
}

int take_real(const float2 *z, long long n, float *out, long long out_rs, long long rows, cudaStream_t st)
{
  take_real_kernel<<<grid_for(rows * n), 256, 0, st>>>(z, n, out, out_rs, rows);
  return launched("real part");
}

}  // namespace fcb
