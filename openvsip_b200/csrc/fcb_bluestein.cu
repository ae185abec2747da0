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
// "replica" spectrum (built once per plan in FP64).  The pre- and
// post-multiplies by c, the zero padding to M and the truncation to N are done
// by the fused kernel itself in its kChirpconv mode (on its row loads and
// stores), so a row costs one pass over its N samples.
#include "fcb200.h"
#include "fcb_engine.cuh"
#include "fcb_internal.h"

#include <cuda_runtime.h>

#include <mutex>

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

int scale_copy(const float2 *in, float2 *out, long long total, float s, cudaStream_t st)
{
  scale_kernel<<<grid_for(total), 256, 0, st>>>(in, out, total, s);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? FCB_OK : cuda_error(e, "scale copy");
}

// Kernel table of the kChirpconv mode: work rows of 8 .. 65536 samples, the
// same variants as the other modes ([0] 256, [1] 512, [2] 128 threads with 32
// samples each, [3] 256 threads with 64 samples for 16384-sample rows).
template <int LOGN, int T, int EPTW = 32>
static KernelInfo chirp_info()
{
  using S = Sched<LOGN, T, EPTW>;
  KernelInfo k;
  k.fn = (const void *)&rows_kernel<LOGN, kChirpconv, T, EPTW>;
  k.threads = T;
  k.cluster = S::CS;
  k.rows_per_cta = S::ROWS;
  k.smem = S::SMEM;
  k.tw_bytes = S::tw_bytes();
  k.ept = EPTW;
  return k;
}

template <int LOGN>
static void fill_chirp(KernelInfo (*tab)[kVariants])
{
  if constexpr (LOGN >= 3)
  {
    tab[LOGN][0] = chirp_info<LOGN, 256>();
    if constexpr (LOGN >= kMin512) tab[LOGN][1] = chirp_info<LOGN, 512>();
    if constexpr (LOGN >= kMin128 && LOGN <= kMax128) tab[LOGN][2] = chirp_info<LOGN, 128>();
    if constexpr (LOGN >= kWideLog && LOGN <= kWideMaxLog) tab[LOGN][3] = chirp_info<LOGN, 256, 64>();
    fill_chirp<LOGN - 1>(tab);
  }
}

static KernelInfo g_chirp[kMaxLogN + 1][kVariants];
static std::once_flag g_chirp_once;

const KernelInfo *chirp_kernel(int logn, const KernelInfo *like)
{
  std::call_once(g_chirp_once, [] { fill_chirp<kMaxLogN>(g_chirp); });
  if (logn < 3 || logn > kMaxLogN || !like) return nullptr;
  const int t = like->threads;
  const int v = (like->ept == 64 && logn >= kWideLog && logn <= kWideMaxLog) ? 3
              : (t == 512 && logn >= kMin512) ? 1
              : (t == 128 && logn >= kMin128 && logn <= kMax128) ? 2 : 0;
  const KernelInfo *k = &g_chirp[logn][v];
  return k->ept == like->ept ? k : nullptr;  // the tables it reads are built for like->ept
}

}  // namespace fcb
