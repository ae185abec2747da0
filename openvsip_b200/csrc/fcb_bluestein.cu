// Row FFTs of any length N (not only powers of two) by Bluestein's chirp-z
// algorithm, built on the power-of-two fused fast convolution.
//
// The reference's FFTW3 backend plans any length (src/ovxx/fftw/fftw.cpp:39-116)
// and its own tests use such lengths (tests/fftm.cpp: 18, 68, 252;
// tests/fft_ext/data: 19, 768).  With c[n] = exp(s i pi n^2 / N) (s = -1
// forward, +1 inverse), n k = (n^2 + k^2 - (k - n)^2) / 2 gives
//     X[k] = c[k] * sum_n (x[n] c[n]) conj(c[k - n]),
// a linear convolution of a = x .* c with b[m] = conj(c[m]), |m| < N.  With
// M >= 2N - 1 a power of two it is the circular convolution IFFT_M(FFT_M(a) .*
// FFT_M(b)) -- exactly what the fused kernel computes, with FFT_M(b) as its
// "replica" spectrum (built once per plan in FP64).  A row then costs a
// pre-multiply pass, one fused length-M pass and a post-multiply pass.
#include "fcb200.h"
#include "fcb_internal.h"

#include <cuda_runtime.h>

namespace fcb {

// c[n] = exp(s i pi n^2 / N), with n^2 reduced mod 2N exactly before FP64 sincospi.
__device__ __forceinline__ double2 chirp64(long long n, long long N, int sign)
{
  const unsigned long long m = ((unsigned long long)n * (unsigned long long)n) % (2ULL * (unsigned long long)N);
  double s, c;
  sincospi((double)sign * (double)m / (double)N, &s, &c);
  return make_double2(c, s);
}

__global__ void bluestein_chirp_kernel(float2 *c, long long N, int sign)
{
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const double2 v = chirp64(i, N, sign);
  c[i] = make_float2((float)v.x, (float)v.y);
}

// b[m] = conj(c[m]) for 0 <= m < N, b[M - m] = conj(c[m]) for 1 <= m < N, 0 elsewhere.
__global__ void bluestein_filter_kernel(float2 *b, long long N, long long M, int sign)
{
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= M) return;
  const long long m = i < N ? i : (i > M - N ? M - i : -1);
  if (m < 0)
  {
    b[i] = make_float2(0.f, 0.f);
    return;
  }
  const double2 v = chirp64(m, N, sign);
  b[i] = make_float2((float)v.x, (float)-v.y);
}

// a[r][j] = x[r][j] c[j] for j < N, 0 for N <= j < M.
__global__ void bluestein_pre_kernel(const float2 *x, long long x_rs, const float2 *c, float2 *a, long long N,
                                     long long M, long long rows)
{
  const long long total = rows * M;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x)
  {
    const long long r = i / M, j = i % M;
    float2 v = make_float2(0.f, 0.f);
    if (j < N)
    {
      const float2 u = x[r * x_rs + j], w = c[j];
      v = make_float2(u.x * w.x - u.y * w.y, u.x * w.y + u.y * w.x);
    }
    a[i] = v;
  }
}

// out[r][k] = scale * c[k] * y[r][k], k < N.
__global__ void bluestein_post_kernel(const float2 *y, long long M, const float2 *c, float2 *out, long long out_rs,
                                      long long N, long long rows, float scale)
{
  const long long total = rows * N;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x)
  {
    const long long r = i / N, k = i % N;
    const float2 u = y[r * M + k], w = c[k];
    out[r * out_rs + k] = make_float2(scale * (u.x * w.x - u.y * w.y), scale * (u.x * w.y + u.y * w.x));
  }
}

// Fast convolution between the two Bluestein passes: the forward pass's
// post-multiply by c and the inverse pass's pre-multiply by conj(c) cancel
// (|c| = 1), leaving y[r][k] = R[r][k] y[r][k] for k < N and 0 beyond.
// rep holds R / N (rep_rs 0: one row for all).
__global__ void bluestein_mid_kernel(float2 *y, long long M, const float2 *rep, long long rep_rs, long long N,
                                     long long rows)
{
  const long long total = rows * M;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x)
  {
    const long long r = i / M, k = i % M;
    float2 v = make_float2(0.f, 0.f);
    if (k < N)
    {
      const float2 u = y[i], w = rep[r * rep_rs + k];
      v = make_float2(u.x * w.x - u.y * w.y, u.x * w.y + u.y * w.x);
    }
    y[i] = v;
  }
}

__global__ void scale_kernel(const float2 *in, float2 *out, long long total, float s)
{
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x)
    out[i] = make_float2(in[i].x * s, in[i].y * s);
}

static unsigned grid_for(long long total)
{
  long long b = (total + 255) / 256;
  return (unsigned)(b > 148 * 32 ? 148 * 32 : (b < 1 ? 1 : b));
}

int bluestein_tables(long long N, long long M, int sign, float2 **chirp, float2 **spectrum, cudaStream_t st)
{
  float2 *c = nullptr, *b = nullptr, *B = nullptr;
  cudaError_t e = cudaMalloc(&c, sizeof(float2) * (size_t)N);
  if (e == cudaSuccess) e = cudaMalloc(&b, sizeof(float2) * (size_t)M);
  if (e == cudaSuccess) e = cudaMalloc(&B, sizeof(float2) * (size_t)M);
  if (e != cudaSuccess)
  {
    cudaFree(c); cudaFree(b); cudaFree(B);
    return set_error(FCB_ERR_NOMEM, "Bluestein tables: %s", cudaGetErrorString(e));
  }
  bluestein_chirp_kernel<<<(unsigned)((N + 255) / 256), 256, 0, st>>>(c, N, sign);
  bluestein_filter_kernel<<<(unsigned)((M + 255) / 256), 256, 0, st>>>(b, N, M, sign);
  int rc = replica_spectrum_dev(b, M, 0, B, st);
  if (!rc && (e = cudaStreamSynchronize(st)) != cudaSuccess) rc = cuda_error(e, "Bluestein tables");
  cudaFree(b);
  if (rc) { cudaFree(c); cudaFree(B); return rc; }
  *chirp = c;
  *spectrum = B;
  return FCB_OK;
}

int bluestein_pre(const float2 *x, long long x_rs, const float2 *c, float2 *a, long long N, long long M,
                  long long rows, cudaStream_t st)
{
  bluestein_pre_kernel<<<grid_for(rows * M), 256, 0, st>>>(x, x_rs, c, a, N, M, rows);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? FCB_OK : cuda_error(e, "Bluestein pre-multiply");
}

int bluestein_post(const float2 *y, long long M, const float2 *c, float2 *out, long long out_rs, long long N,
                   long long rows, float scale, cudaStream_t st)
{
  bluestein_post_kernel<<<grid_for(rows * N), 256, 0, st>>>(y, M, c, out, out_rs, N, rows, scale);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? FCB_OK : cuda_error(e, "Bluestein post-multiply");
}

int bluestein_mid(float2 *y, long long M, const float2 *rep, long long rep_rs, long long N, long long rows,
                  cudaStream_t st)
{
  bluestein_mid_kernel<<<grid_for(rows * M), 256, 0, st>>>(y, M, rep, rep_rs, N, rows);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? FCB_OK : cuda_error(e, "Bluestein replica multiply");
}

int scale_copy(const float2 *in, float2 *out, long long total, float s, cudaStream_t st)
{
  scale_kernel<<<grid_for(total), 256, 0, st>>>(in, out, total, s);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? FCB_OK : cuda_error(e, "scale copy");
}

}  // namespace fcb
