// C-ABI implementation of the fcb200 backend: plans, FP64 table builders,
// kernel dispatch and host-buffer staging.  Entry points are declared in
// include/fcb200.h, which also cites the reference interface each replaces.
#include "fcb200.h"
#include "fcb_engine.cuh"
#include "fcb_internal.h"

#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <mutex>

namespace fcb {

// ---------------------------------------------------------------------------
// Error reporting: thread-local message, status code returned to the caller.
static thread_local char g_err[512] = "";

int set_error(int code, const char *fmt, ...)
{
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return code;
}

const char *error_text() { return g_err; }

int cuda_error(cudaError_t e, const char *what)
{
  return set_error(FCB_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

// ---------------------------------------------------------------------------
// Runtime view of the compile-time schedule (for table builders).
SchedRT sched_rt(int logn, int ept)
{
  SchedRT s;
  s.logn = logn;
  s.n = 1 << logn;
  s.ept = ept;
  s.rb = ept / 2;
  s.lrb = ept == 64 ? 5 : 4;
  s.ns = (logn <= s.lrb + 1) ? 1 : 1 + (logn - (s.lrb + 1) + s.lrb - 1) / s.lrb;
  s.r1 = 1 << (logn - s.lrb * (s.ns - 1));
  s.d = s.n / s.r1;
  s.half = s.n / 2;
  s.tw2_size = 0;
  for (int k = 2; k <= s.ns; ++k) s.tw2_size += s.d >> (s.lrb * (k - 2));
  return s;
}

// Twiddle tables in FP64, rounded to float (forward sign; kernels conjugate).
//   stage 1 (float4) [q'*D + n] = (W^{n 2q'}.re, W^{n(2q'+1)}.re, W^{n 2q'}.im, W^{n(2q'+1)}.im),
//                                 W = e^{-2 pi i / N}
//   stage s >= 2 (float2, after the float4 part) [tw2_off(s) + q*S_s + n] = e^{-2 pi i n q / L_s}
__global__ void build_tw_kernel(float4 *tw, SchedRT s)
{
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < s.half)
  {
    long long qp = i / s.d, n = i % s.d;
    long long m0 = (n * (2 * qp)) % s.n, m1 = (n * (2 * qp + 1)) % s.n;
    double s0, c0, s1, c1;
    sincospi(-2.0 * (double)m0 / (double)s.n, &s0, &c0);
    sincospi(-2.0 * (double)m1 / (double)s.n, &s1, &c1);
    tw[i] = make_float4((float)c0, (float)c1, (float)s0, (float)s1);
    return;
  }
  long long j = i - s.half;  // float2 index in the stage >= 2 part
  float2 *tw2 = reinterpret_cast<float2 *>(tw + s.half);
  long long off = 0;
  for (int k = 2; k <= s.ns; ++k)
  {
    long long L = s.d >> (s.lrb * (k - 2)), St = L / s.rb;
    if (j < off + L)
    {
      long long jj = j - off, q = jj / St, n = jj % St;
      long long m = (n * q) % L;
      double sn, cs;
      sincospi(-2.0 * (double)m / (double)L, &sn, &cs);
      tw2[j] = make_float2((float)cs, (float)sn);
      return;
    }
    off += L;
  }
}

// Replica pair table, (R[k]/N, R[k+1]/N) split per entry (1/N is exact).
// Slot sigma = q'*D + P holds the pair k = 2q' + R1 * digitrev_RB(P).  Rows of
// one stage keep slot order.  Multi-stage rows use the order in which the
// last stage reads: there thread tr of a row (TPR = N/EPT threads) owns slots
// RB tr .. RB tr + RB - 1 and multiplies its i-th value by slot RB tr +
// bitrev(i), so entry i * TPR + tr holds that slot and the i-th loads of a
// warp read consecutive entries (one coalesced 512-byte access).
__global__ void build_rep_kernel(const float2 *spec, long long spec_rs, float4 *rep,
                                 long long rows, SchedRT s)
{
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long total = rows * s.half;
  if (i >= total) return;
  long long r = i / s.half, e = i % s.half;
  long long sigma = e;
  if (s.ns > 1)
  {
    const long long tpr = s.n / s.ept, j = e / tpr, tr = e % tpr;
    sigma = s.rb * tr + bitrev((int)j, s.lrb);
  }
  int qp = (int)(sigma / s.d), P = (int)(sigma % s.d);
  int k = 2 * qp + s.r1 * digitrev16(P, s.ns - 1, s.lrb);
  const float inv = 1.0f / (float)s.n;
  float2 a = spec[r * spec_rs + k], b = spec[r * spec_rs + k + 1];
  rep[i] = make_float4(a.x * inv, b.x * inv, a.y * inv, b.y * inv);
}

// FP64 radix-2 Stockham FFT of one vector in global memory, one CTA.
// Used once per replica (plan time), so simplicity beats speed here.
__global__ void fft_fp64_kernel(const float2 *in, double2 *buf0, double2 *buf1, long long n,
                                int matched, float2 *out)
{
  for (long long i = threadIdx.x; i < n; i += blockDim.x)
    buf0[i] = make_double2(in[i].x, in[i].y);
  __syncthreads();
  double2 *src = buf0, *dst = buf1;
  // Stockham autosort, radix 2: for each pass with sub-length l (1, 2, 4, ...)
  for (long long l = 1; l < n; l <<= 1)
  {
    long long half = n / 2;
    for (long long j = threadIdx.x; j < half; j += blockDim.x)
    {
      long long k = j % l;                  // index within the current sub-transform
      long long base = (j / l) * 2 * l;     // output block
      double2 a = src[j], b = src[j + half];
      double sn, cs;
      sincospi(-(double)k / (double)l, &sn, &cs);  // e^{-i pi k / l}
      double2 tb = make_double2(b.x * cs - b.y * sn, b.x * sn + b.y * cs);
      dst[base + k] = make_double2(a.x + tb.x, a.y + tb.y);
      dst[base + k + l] = make_double2(a.x - tb.x, a.y - tb.y);
    }
    __syncthreads();
    double2 *tmp = src; src = dst; dst = tmp;
  }
  for (long long i = threadIdx.x; i < n; i += blockDim.x)
    out[i] = make_float2((float)src[i].x, (float)(matched ? -src[i].y : src[i].y));
}

// FP64 DFT of one vector of non-power-of-two length n <= 32768 (so j * k
// stays below 2^30), one CTA per output bin; w[m] = e^{-2 pi i m / n}.
// Plan-time only (replica spectra of Bluestein plans).
__global__ void dft_table_kernel(double2 *w, long long n)
{
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double sn, cs;
  sincospi(-2.0 * (double)i / (double)n, &sn, &cs);
  w[i] = make_double2(cs, sn);
}

__global__ void dft_fp64_kernel(const float2 *in, const double2 *w, unsigned n, int matched, float2 *out)
{
  __shared__ double part[2][32];
  const unsigned k = blockIdx.x;
  double re = 0.0, im = 0.0;
  for (unsigned j = threadIdx.x; j < n; j += blockDim.x)
  {
    const double2 t = w[(j * k) % n];
    const float2 x = in[j];
    re += (double)x.x * t.x - (double)x.y * t.y;
    im += (double)x.x * t.y + (double)x.y * t.x;
  }
  for (int o = 16; o > 0; o >>= 1)
  {
    re += __shfl_xor_sync(0xffffffffu, re, o);
    im += __shfl_xor_sync(0xffffffffu, im, o);
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) { part[0][warp] = re; part[1][warp] = im; }
  __syncthreads();
  if (threadIdx.x == 0)
  {
    re = im = 0.0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) { re += part[0][i]; im += part[1][i]; }
    out[k] = make_float2((float)re, (float)(matched ? -im : im));
  }
}

__global__ void vmmul_kernel(const float2 *v, const float2 *m, long long m_rs, float2 *out,
                             long long out_rs, long long rows, long long cols)
{
  long long total = rows * cols;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x)
  {
    long long r = i / cols, c = i % cols;
    float2 a = v[c], b = m[r * m_rs + c];
    out[r * out_rs + c] = make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
  }
}

// out[c][r] = in[r][c] for a rows x cols matrix, through 32 x 32 tiles in
// shared memory (coalesced reads and writes); one CTA of 32 x 8 threads per
// tile.  Used by 2-D FFT plans whose sizes the transposing row kernels do not
// cover.
__global__ void transpose_kernel(const float2 *in, long long in_rs, float2 *out, long long out_rs, long long rows,
                                 long long cols)
{
  __shared__ float2 tile[32][33];
  const long long c0 = (long long)blockIdx.x * 32, r0 = (long long)blockIdx.y * 32;
  for (int k = threadIdx.y; k < 32; k += 8)
  {
    const long long r = r0 + k, c = c0 + threadIdx.x;
    if (r < rows && c < cols) tile[k][threadIdx.x] = in[r * in_rs + c];
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += 8)
  {
    const long long c = c0 + k, r = r0 + threadIdx.x;
    if (r < rows && c < cols) out[c * out_rs + r] = tile[threadIdx.x][k];
  }
}

// Length-1 rows: out = in * w (w = scale, or the replica value).
__global__ void scale_rows_kernel(const float2 *in, long long in_rs, float2 *out, long long out_rs,
                                  long long rows, const float4 *rep, long long rep_rs, float scale)
{
  long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= rows) return;
  float2 x = in[r * in_rs];
  if (rep)
  {
    float4 w = rep[r * rep_rs];  // (re, -, im, -) of the single-sample spectrum / 1
    out[r * out_rs] = make_float2(x.x * w.x - x.y * w.z, x.x * w.z + x.y * w.x);
  }
  else
    out[r * out_rs] = make_float2(x.x * scale, x.y * scale);
}

// ---------------------------------------------------------------------------
// Kernel table: [logn][mode][variant], variant 0 = 256-thread CTAs, 1 = 512.
template <int LOGN, int MODE, int T, int EPTW = 32>
static KernelInfo make_info()
{
  using S = Sched<LOGN, T, EPTW>;
  KernelInfo k;
  k.fn = (const void *)&rows_kernel<LOGN, MODE, T, EPTW>;
  k.ept = EPTW;
  k.threads = T;
  k.cluster = S::CS;
  k.rows_per_cta = S::ROWS;
  k.smem = S::SMEM;
  k.tw_bytes = S::tw_bytes();
  return k;
}


template <int LOGN>
static void fill_table(KernelInfo (*tab)[3][kVariants])
{
  if constexpr (LOGN >= 1)
  {
    tab[LOGN][kFwd][0] = make_info<LOGN, kFwd, 256>();
    tab[LOGN][kInv][0] = make_info<LOGN, kInv, 256>();
    tab[LOGN][kFastconv][0] = make_info<LOGN, kFastconv, 256>();
    if constexpr (LOGN >= kMin512)
    {
      tab[LOGN][kFwd][1] = make_info<LOGN, kFwd, 512>();
      tab[LOGN][kInv][1] = make_info<LOGN, kInv, 512>();
      tab[LOGN][kFastconv][1] = make_info<LOGN, kFastconv, 512>();
    }
    if constexpr (LOGN >= kMin128 && LOGN <= kMax128)
    {
      tab[LOGN][kFwd][2] = make_info<LOGN, kFwd, 128>();
      tab[LOGN][kInv][2] = make_info<LOGN, kInv, 128>();
      tab[LOGN][kFastconv][2] = make_info<LOGN, kFastconv, 128>();
    }
    if constexpr (LOGN >= kWideLog && LOGN <= kWideMaxLog)
    {
      tab[LOGN][kFwd][3] = make_info<LOGN, kFwd, 256, 64>();
      tab[LOGN][kInv][3] = make_info<LOGN, kInv, 256, 64>();
      tab[LOGN][kFastconv][3] = make_info<LOGN, kFastconv, 256, 64>();
    }
    fill_table<LOGN - 1>(tab);
  }
}

static KernelInfo g_table[kMaxLogN + 1][3][kVariants];
static std::once_flag g_table_once;
// Variant chosen per (logn, mode); set by the autotuner through fcb_tune_set.
static int g_variant[kMaxLogN + 1][3];
static std::mutex g_variant_mu;

static void init_table()
{
  std::call_once(g_table_once, [] {
    fill_table<kMaxLogN>(g_table);
    for (int l = 0; l <= kMaxLogN; ++l)
      for (int m = 0; m < 3; ++m)
        // defaults (measured): 4 CTAs of 128 threads per SM for rows of 256 ..
        // 4096 samples, 256-thread CTAs for 8192, 512-thread CTAs from 16384
        // up (clusters of 2 and 4 of them for 32768 and 65536; clusters of
        // smaller CTAs measured slower at every length), except the wide
        // variant for the fused fast convolution of 16384-sample rows (one
        // stage, two slot exchanges fewer: 13 % faster) and for the forward and
        // inverse transforms of 32768-sample rows (clusters of two wide CTAs:
        // 2.8 % / 1.7 % faster; the fused form there measured the same)
        g_variant[l][m] = (l == kWideLog && m == kFastconv) ? 3
                        : (l == kWideMaxLog && m != kFastconv) ? 3
                        : (l >= 14) ? 1 : (l >= kMin128 && l <= 12) ? 2 : 0;
  });
}

const KernelInfo *kernel_info(int logn, int mode)
{
  init_table();
  if (logn < 1 || logn > kMaxLogN || mode < 0 || mode > 2) return nullptr;
  std::lock_guard<std::mutex> lk(g_variant_mu);
  return &g_table[logn][mode][g_variant[logn][mode]];
}

// Public tuning values: 128, 256, 512 threads (32 samples per thread), or -256
// for the wide variant (256 threads x 64 samples).
static int variant_id(int logn, int threads)
{
  if (threads == -256 && logn >= kWideLog && logn <= kWideMaxLog) return 3;
  if (threads == 512 && logn >= kMin512) return 1;
  if (threads == 128 && logn >= kMin128 && logn <= kMax128) return 2;
  return threads == 256 ? 0 : -1;
}
static const int kVariantValue[kVariants] = {256, 512, 128, -256};

const KernelInfo *kernel_variant(int logn, int mode, int threads)
{
  init_table();
  if (logn < 1 || logn > kMaxLogN || mode < 0 || mode > 2) return nullptr;
  const int v = variant_id(logn, threads);
  return &g_table[logn][mode][v < 0 ? 0 : v];
}

int set_variant(int logn, int mode, int threads)
{
  init_table();
  if (logn < 1 || logn > kMaxLogN || mode < 0 || mode > 2)
    return set_error(FCB_ERR_INVALID, "bad length or mode for tuning");
  if (threads != 128 && threads != 256 && threads != 512 && threads != -256)
    return set_error(FCB_ERR_INVALID, "threads must be 128, 256, 512 or -256 (wide)");
  const int v = variant_id(logn, threads);
  if (v < 0)
    return set_error(FCB_ERR_UNSUPPORTED, "no %d-thread variant for rows of %d samples (512: 4096 and more; "
                     "128: 256 .. 8192; -256: 16384 and 32768)", threads, 1 << logn);
  std::lock_guard<std::mutex> lk(g_variant_mu);
  g_variant[logn][mode] = v;
  return FCB_OK;
}

int get_variant(int logn, int mode)
{
  init_table();
  if (logn < 1 || logn > kMaxLogN || mode < 0 || mode > 2) return 0;
  std::lock_guard<std::mutex> lk(g_variant_mu);
  return kVariantValue[g_variant[logn][mode]];
}

int prepare_kernel(const KernelInfo *k)
{
  // Idempotent; cheap after the first call per device.
  cudaError_t e = cudaFuncSetAttribute(k->fn, cudaFuncAttributeMaxDynamicSharedMemorySize, k->smem);
  if (e != cudaSuccess) return cuda_error(e, "cudaFuncSetAttribute(smem)");
  // tiles resident at once: the L2 prefetch distance
  int dev = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k->fn, k->threads, k->smem);
  if (e != cudaSuccess) return cuda_error(e, "occupancy query");
  const_cast<KernelInfo *>(k)->resident_tiles = (long long)sms * (per_sm > 0 ? per_sm : 1) / k->cluster;
  return FCB_OK;
}

int launch_rows(const KernelInfo *k, long long rows, const RowArgs &args, cudaStream_t st)
{
  if (rows <= 0) return FCB_OK;
  long long ctas = k->cluster > 1 ? rows * k->cluster : (rows + k->rows_per_cta - 1) / k->rows_per_cta;
  if (ctas > 0x7fffffffLL) return set_error(FCB_ERR_INVALID, "too many rows in one call");
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)ctas);
  cfg.blockDim = dim3(k->threads);
  cfg.dynamicSmemBytes = k->smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  if (k->cluster > 1)
  {
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = k->cluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
  }
  RowArgs a = args;
  if (a.ahead < 0) a.ahead = (k->resident_tiles + 1) / 2;  // half a resident wave ahead (measured best)
  void *params[] = {&a};
  cudaError_t e = cudaLaunchKernelExC(&cfg, k->fn, params);
  if (e != cudaSuccess) return cuda_error(e, "row kernel launch");
  return FCB_OK;
}

int build_twiddles(int logn, int ept, float4 **out, cudaStream_t st)
{
  SchedRT s = sched_rt(logn, ept);
  float4 *tw = nullptr;
  const size_t bytes = 16 * (size_t)s.half + 8 * (size_t)s.tw2_size;
  cudaError_t e = cudaMalloc(&tw, bytes);
  if (e != cudaSuccess) return set_error(FCB_ERR_NOMEM, "twiddle table: %s", cudaGetErrorString(e));
  const long long entries = s.half + s.tw2_size;
  build_tw_kernel<<<(unsigned)((entries + 255) / 256), 256, 0, st>>>(tw, s);
  e = cudaGetLastError();
  if (e != cudaSuccess) { cudaFree(tw); return cuda_error(e, "twiddle build"); }
  *out = tw;
  return FCB_OK;
}

int build_replica_table(int logn, int ept, const float2 *spec_dev, long long spec_rs, long long rows,
                        float4 *rep_dev, cudaStream_t st)
{
  SchedRT s = sched_rt(logn, ept);
  long long total = rows * s.half;
  build_rep_kernel<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(spec_dev, spec_rs, rep_dev, rows, s);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_error(e, "replica table build");
  return FCB_OK;
}

int replica_spectrum_dev(const float2 *rep_dev, long long n, int matched, float2 *spec_dev,
                         cudaStream_t st)
{
  double2 *buf = nullptr;
  cudaError_t e = cudaMallocAsync(&buf, sizeof(double2) * 2 * (size_t)n, st);
  if (e != cudaSuccess) return set_error(FCB_ERR_NOMEM, "replica FFT buffer: %s", cudaGetErrorString(e));
  if ((n & (n - 1)) == 0)
    fft_fp64_kernel<<<1, 1024, 0, st>>>(rep_dev, buf, buf + n, n, matched, spec_dev);
  else if (n <= 32768)
  {
    dft_table_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(buf, n);
    dft_fp64_kernel<<<(unsigned)n, 256, 0, st>>>(rep_dev, buf, (unsigned)n, matched, spec_dev);
  }
  else
  {
    cudaFreeAsync(buf, st);
    return set_error(FCB_ERR_UNSUPPORTED, "replica length %lld: not a power of two and above 32768", n);
  }
  e = cudaGetLastError();
  cudaFreeAsync(buf, st);
  if (e != cudaSuccess) return cuda_error(e, "replica FFT");
  return FCB_OK;
}

int launch_vmmul(const float2 *v, const float2 *m, long long m_rs, float2 *out, long long out_rs,
                 long long rows, long long cols, cudaStream_t st)
{
  long long total = rows * cols;
  if (total <= 0) return FCB_OK;
  long long blocks = (total + 255) / 256;
  if (blocks > 148 * 64) blocks = 148 * 64;
  vmmul_kernel<<<(unsigned)blocks, 256, 0, st>>>(v, m, m_rs, out, out_rs, rows, cols);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_error(e, "vmmul launch");
  return FCB_OK;
}

int launch_transpose(const float2 *in, long long in_rs, float2 *out, long long out_rs, long long rows,
                     long long cols, cudaStream_t st)
{
  if (rows <= 0 || cols <= 0) return FCB_OK;
  const long long gx = (cols + 31) / 32, gy = (rows + 31) / 32;
  if (gy > 65535 || gx > 0x7fffffffLL) return set_error(FCB_ERR_INVALID, "matrix too large to transpose");
  transpose_kernel<<<dim3((unsigned)gx, (unsigned)gy), dim3(32, 8), 0, st>>>(in, in_rs, out, out_rs, rows, cols);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_error(e, "transpose launch");
  return FCB_OK;
}

int launch_scale_rows(const float2 *in, long long in_rs, float2 *out, long long out_rs, long long rows,
                      const float4 *rep, long long rep_rs, float scale, cudaStream_t st)
{
  if (rows <= 0) return FCB_OK;
  scale_rows_kernel<<<(unsigned)((rows + 255) / 256), 256, 0, st>>>(in, in_rs, out, out_rs, rows, rep,
                                                                    rep_rs, scale);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_error(e, "scale launch");
  return FCB_OK;
}

}  // namespace fcb

// ---------------------------------------------------------------------------
// Replica spectrum without any allocation.
//
// Some callers cannot allocate device memory once they are running: a
// real-time pulse-compression loop that must not stall in the allocator or
// fail on a fragmented heap mid-mission, a process whose device memory is
// fully reserved up front, or code that runs while another component owns
// the allocator.  fcb_replica_spectrum_noalloc computes the same FP64 replica
// spectrum as fcb_replica_spectrum, but its two FP64 ping-pong buffers live in
// the file-scope array below instead of a per-call cudaMallocAsync.
//
// The array is 2 * 65536 double2 = 2 MiB; every GPU that loads this library
// holds it until the process exits.  Calls share it and it keeps the last
// call's contents; nothing in it needs to start at zero (each call writes a
// buffer completely before reading it).  Calls that overlap on the GPU (on
// different streams, or from different threads) race on it.
namespace {
constexpr long long kNoAllocMaxN = 65536;
__device__ __align__(256) double2 g_noalloc_scratch[2 * kNoAllocMaxN];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
double2 *g_noalloc_ptr[kMaxDevices] = {};

// Device address of the scratch array on the current device.  The first call
// on each device looks it up with cudaGetSymbolAddress (host code cannot use
// the array's name as a device address).  The address is cached per device
// ordinal, i.e. for the device's primary context, which is the context the
// CUDA runtime uses; callers that switch to contexts of their own made with the
// driver API are not supported by this entry point.
int noalloc_scratch(double2 **out)
{
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fcb::cuda_error(e, "cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices) return fcb::set_error(FCB_ERR_UNSUPPORTED, "device index %d too large", dev);
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_ptr[dev])
  {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return fcb::cuda_error(e, "cudaGetSymbolAddress(scratch)");
    g_noalloc_ptr[dev] = static_cast<double2 *>(p);
  }
  *out = g_noalloc_ptr[dev];
  return FCB_OK;
}
}  // namespace

extern "C" FCB_API int fcb_replica_spectrum_noalloc(const fcb_cf32 *replica_dev, long long n, int matched,
                                                    fcb_cf32 *spectrum_dev, void *stream)
{
  // the size limit first: any n above it is FCB_ERR_INVALID, power of two or not
  if (n > kNoAllocMaxN)
    return fcb::set_error(FCB_ERR_INVALID, "length %lld exceeds the no-allocation scratch limit of %lld samples",
                          n, kNoAllocMaxN);
  if (n < 1 || (n & (n - 1)) != 0)
    return fcb::set_error(FCB_ERR_UNSUPPORTED, "length %lld is not a power of two (the no-allocation entry point "
                          "runs the radix-2 FP64 FFT only)", n);
  if (!replica_dev || !spectrum_dev) return fcb::set_error(FCB_ERR_INVALID, "NULL pointer");
  double2 *scratch = nullptr;
  int rc = noalloc_scratch(&scratch);
  if (rc) return rc;
  fcb::fft_fp64_kernel<<<1, 1024, 0, (cudaStream_t)stream>>>(reinterpret_cast<const float2 *>(replica_dev),
                                                             scratch, scratch + n, n, matched,
                                                             reinterpret_cast<float2 *>(spectrum_dev));
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fcb::cuda_error(e, "replica FFT (no allocation)");
  return FCB_OK;
}
