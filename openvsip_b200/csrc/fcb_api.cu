// fcb200 C ABI: plan objects and execution (declarations in include/fcb200.h).
#include "fcb200.h"
#include "fcb_engine.cuh"
#include "fcb_internal.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <mutex>
#include <new>
#include <vector>

using namespace fcb;

struct fcb_plan_s
{
  int device = 0;
  long long n = 0;
  int logn = 0;
  int mode = kFwd;
  long long rows_max = 0;
  float scale = 1.f;
  const KernelInfo *k = nullptr;
  float4 *tw = nullptr;
  float4 *rep = nullptr;          // fastconv: replica pair table(s), slot order
  long long rep_rows = 0;         // 1 = shared vector, else one per data row
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;  // current stream (own or caller's)
  // host calls: chunks pipelined through kMaxStage device buffers, copies in
  // on cin, kernels on the plan stream, copies out on cout
  static constexpr int kMaxStage = 8;
  cudaStream_t cin = nullptr, cout = nullptr;
  float2 *stage[kMaxStage] = {};
  long long stage_rows = 0;
  int nstage = 0;
  int stage_next = 0;  // buffer of the next call's first chunk (the rotation continues across calls)
  // host calls on pageable memory: each shared pinned staging buffer's last
  // copy for this plan ([0] to the device, [1] from it)
  cudaEvent_t ev_h[2][kMaxStage] = {};
  cudaEvent_t ev_in[kMaxStage] = {}, ev_k[kMaxStage] = {}, ev_out[kMaxStage] = {}, ev_start = nullptr;
  // 2-D FFT (rows x cols): pass 1 transforms rows into a transposed scratch
  // matrix, pass 2 transforms its rows (the columns) back transposed.
  bool is2d = false;
  long long rows2d = 0, cols2d = 0;
  const KernelInfo *kc = nullptr;  // pass 2 kernel (length rows2d)
  float4 *twc = nullptr;
  float2 *scratch = nullptr;
  float2 *stage2d_in = nullptr, *stage2d_out = nullptr;
  // 2-D FFT of other sizes (any dimensions the row plans support): a row plan
  // of length cols, a transpose, a row plan of length rows on the transposed
  // matrix, and a transpose back; scratch2 holds the transposed matrix.
  bool general2d = false;
  fcb_plan sub2d[2] = {nullptr, nullptr};
  float2 *scratch2 = nullptr;
  // Rows of non-power-of-two length n (Bluestein): the fused kernel's
  // kChirpconv mode runs on work rows of blue_m >= 2n - 1 samples, reading the
  // n samples times a chirp (zero beyond) and writing n samples times a chirp.
  // Index 0 is the forward direction, 1 the inverse.
  long long blue_m = 0;
  long long blue_chunk = 0;                    // fastconv: rows per pass through blue_buf
  float2 *chirp[2] = {nullptr, nullptr};       // c[k] = e^{-+ i pi k^2 / n}
  float2 *chirp_out = nullptr;                 // Fftm: c[k] * scale (the output multiplier)
  fcb_plan inner[2] = {nullptr, nullptr};      // length-blue_m tables: twiddles, replica FFT(conj(c))
  const KernelInfo *kchirp = nullptr;          // the kChirpconv kernel for blue_m
  float2 *blue_rep = nullptr;                  // fastconv: replica spectra / n, rows of n
  float2 *blue_buf[2] = {nullptr, nullptr};    // fastconv: rows of n between its two passes
  // Real-input rows of n = rn samples: 1 = real -> complex (n/2 + 1 outputs),
  // 2 = complex -> real.  Even n: a length-n/2 complex plan plus the split /
  // merge step; odd n: a length-n complex plan on expanded rows.
  int real = 0;
  long long rn = 0;
  fcb_plan cplx = nullptr;
  float2 *rtw = nullptr;               // W_n^k, k = 0 .. n/2 (even n)
  float2 *rbuf = nullptr;              // work rows (odd n, or unaligned rows)
  long long rbuf_rows = 0, rbuf_cols = 0;
  void *rstage[2] = {nullptr, nullptr};  // host calls: device copies of in / out
  long long rstage_rows = 0;
};

namespace {

int log2_exact(long long n)
{
  if (n < 1 || (n & (n - 1)) != 0) return -1;
  int l = 0;
  while ((1LL << l) < n) ++l;
  return l;
}

// Non-power-of-two lengths up to half the longest fused row run by Bluestein.
constexpr long long kMaxBlueN = 1LL << (kMaxLogN - 1);
constexpr long long kBlueChunkSamples = 1LL << 25;  // work buffer: 256 MiB at most

bool blue_length(long long n) { return n > 0 && n <= kMaxBlueN && (n & (n - 1)) != 0; }

#define FCB_LENGTH_RULE "any length in [1, 32768], or a power of two up to 65536"

struct DeviceGuard
{
  int prev = -1;
  explicit DeviceGuard(int dev)
  {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard()
  {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

int check_device()
{
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0) return set_error(FCB_ERR_NODEVICE, "no CUDA device: %s", cudaGetErrorString(e));
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceProp p;
  e = cudaGetDeviceProperties(&p, dev);
  if (e != cudaSuccess) return cuda_error(e, "cudaGetDeviceProperties");
  // sm_100a code runs on compute capability 10.0 only
  if (p.major != 10 || p.minor != 0)
    return set_error(FCB_ERR_NODEVICE, "device %d is sm_%d%d; this library is built for sm_100a (compute capability 10.0)",
                     dev, p.major, p.minor);
  return FCB_OK;
}

void plan_free(fcb_plan p)
{
  if (!p) return;
  DeviceGuard g(p->device);
  if (p->own_stream) cudaStreamSynchronize(p->own_stream);
  if (p->cin) cudaStreamSynchronize(p->cin);
  if (p->cout) cudaStreamSynchronize(p->cout);
  cudaFree(p->tw);
  cudaFree(p->twc);
  cudaFree(p->scratch);
  cudaFree(p->stage2d_in);
  cudaFree(p->stage2d_out);
  cudaFree(p->scratch2);
  plan_free(p->sub2d[0]);
  plan_free(p->sub2d[1]);
  cudaFree(p->rep);
  for (auto b : p->stage) cudaFree(b);
  for (auto &dir : p->ev_h)
    for (auto ev : dir)
      if (ev) cudaEventDestroy(ev);
  for (int d = 0; d < 2; ++d)
  {
    plan_free(p->inner[d]);
    cudaFree(p->chirp[d]);
    cudaFree(p->blue_buf[d]);
  }
  cudaFree(p->blue_rep);
  cudaFree(p->chirp_out);
  plan_free(p->cplx);
  cudaFree(p->rtw);
  cudaFree(p->rbuf);
  cudaFree(p->rstage[0]);
  cudaFree(p->rstage[1]);
  for (int i = 0; i < fcb_plan_s::kMaxStage; ++i)
  {
    if (p->ev_in[i]) cudaEventDestroy(p->ev_in[i]);
    if (p->ev_k[i]) cudaEventDestroy(p->ev_k[i]);
    if (p->ev_out[i]) cudaEventDestroy(p->ev_out[i]);
  }
  if (p->ev_start) cudaEventDestroy(p->ev_start);
  if (p->own_stream) cudaStreamDestroy(p->own_stream);
  if (p->cin) cudaStreamDestroy(p->cin);
  if (p->cout) cudaStreamDestroy(p->cout);
  delete p;
}

int plan_common(fcb_plan p, long long n, long long rows_max, int mode)
{
  int rc = check_device();
  if (rc) return rc;
  cudaGetDevice(&p->device);
  p->n = n;
  p->logn = log2_exact(n);
  p->mode = mode;
  p->rows_max = rows_max;
  cudaError_t e = cudaStreamCreateWithFlags(&p->own_stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) return cuda_error(e, "cudaStreamCreate");
  p->stream = p->own_stream;
  if (p->logn >= 1)
  {
    p->k = kernel_info(p->logn, mode);
    rc = prepare_kernel(p->k);
    if (rc) return rc;
    rc = build_twiddles(p->logn, p->k->ept, &p->tw, p->stream);
    if (rc) return rc;
  }
  return FCB_OK;
}

// Bluestein plan for non-power-of-two n: a chirp and an inner length-m
// fastconv plan per direction needed (fwd / inv), and one work buffer.
int blue_setup(fcb_plan p, long long n, long long rows_max, int mode, bool need_fwd, bool need_inv)
{
  int rc = check_device();
  if (rc) return rc;
  cudaGetDevice(&p->device);
  p->n = n;
  p->logn = -1;
  p->mode = mode;
  p->rows_max = rows_max;
  cudaError_t e = cudaStreamCreateWithFlags(&p->own_stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) return cuda_error(e, "cudaStreamCreate");
  p->stream = p->own_stream;
  long long m = 1;
  while (m < 2 * n - 1) m <<= 1;
  p->blue_m = m;
  p->blue_chunk = std::max<long long>(1, std::min(rows_max, kBlueChunkSamples / n));
  for (int d = 0; d < 2; ++d)
  {
    if (!(d == 0 ? need_fwd : need_inv)) continue;
    float2 *spec = nullptr;
    rc = bluestein_tables(n, m, d == 0 ? -1 : +1, &p->chirp[d], &spec, p->stream);
    if (rc) return rc;
    rc = fcb_plan_fastconv(m, 1, reinterpret_cast<const fcb_cf32 *>(spec), 1, m, FCB_REPLICA_SPECTRUM, FCB_DEVICE,
                           &p->inner[d]);
    cudaFree(spec);
    if (rc) return rc;
  }
  const fcb_plan any = p->inner[0] ? p->inner[0] : p->inner[1];
  p->kchirp = chirp_kernel(log2_exact(m), any->k);
  if (!p->kchirp) return set_error(FCB_ERR_UNSUPPORTED, "no Bluestein kernel for work rows of %lld", m);
  rc = prepare_kernel(p->kchirp);
  if (rc) return rc;
  if (mode == kFastconv)
  {
    e = cudaMalloc(&p->blue_buf[0], sizeof(float2) * (size_t)(p->blue_chunk * n));
    if (e != cudaSuccess) return set_error(FCB_ERR_NOMEM, "Bluestein rows: %s", cudaGetErrorString(e));
  }
  return FCB_OK;
}

// One kChirpconv pass over `rows` rows of n samples with the tables of `inner`:
// y = cout .* (the first n samples of IFFT_m(FFT_m(pad_m(cin .* x)) .* B) / m).
int blue_pass(fcb_plan p, fcb_plan inner, const float2 *x, long long x_rs, float2 *y, long long y_rs, long long rows,
              const float2 *cin, long long cin_rs, const float2 *cout, cudaStream_t st)
{
  RowArgs a = {};
  a.in = x;
  a.in_rs = x_rs;
  a.out = y;
  a.out_rs = y_rs;
  a.rows = rows;
  a.tw = a.twi = inner->tw;
  a.rep = inner->rep;
  a.rep_rs = 0;
  a.scale = 1.f;
  a.cin = cin;
  a.cin_rs = cin_rs;
  a.n_in = p->n;
  a.cout = cout;
  a.n_out = p->n;
  a.ahead = -1;
  return launch_rows(p->kchirp, rows, a, st);
}

int exec_device(fcb_plan p, const float2 *in, long long in_rs, float2 *out, long long out_rs,
                long long rows, long long row0, cudaStream_t st, int slot = 0);

// Bluestein execution on stream st.  Fftm: one pass, chirp in and chirp *
// scale out.  Fast convolution: a forward pass (chirp in, nothing out) into
// rows of n, then an inverse pass (replica / n in, inverse chirp out); the
// forward post-multiply and the inverse pre-multiply cancel (c_f c_i = 1).  In
// place is fine: each row is read completely before it is written.
int exec_blue(fcb_plan p, const float2 *in, long long in_rs, float2 *out, long long out_rs, long long rows,
              long long row0, cudaStream_t st, int slot)
{
  if (p->mode != kFastconv)
  {
    const int d = p->mode == kFwd ? 0 : 1;
    return blue_pass(p, p->inner[d], in, in_rs, out, out_rs, rows, p->chirp[d], 0, p->chirp_out, st);
  }
  float2 *buf = p->blue_buf[slot];
  const long long n = p->n;
  const bool per_row = p->rep_rows > 1;
  int rc = FCB_OK;
  for (long long r0 = 0; !rc && r0 < rows; r0 += p->blue_chunk)
  {
    const long long nr = std::min(p->blue_chunk, rows - r0);
    rc = blue_pass(p, p->inner[0], in + r0 * in_rs, in_rs, buf, n, nr, p->chirp[0], 0, nullptr, st);
    if (!rc)
      rc = blue_pass(p, p->inner[1], buf, n, out + r0 * out_rs, out_rs, nr,
                     p->blue_rep + (per_row ? (row0 + r0) * n : 0), per_row ? n : 0, p->chirp[1], st);
  }
  return rc;
}

bool aligned8(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 7) == 0; }

int ensure_rbuf(fcb_plan p, long long cols)
{
  if (p->rbuf) return FCB_OK;
  p->rbuf_cols = cols;
  p->rbuf_rows = std::max<long long>(1, std::min<long long>(std::max<long long>(p->rows_max, 1), (1LL << 24) / cols));
  cudaError_t e = cudaMalloc(&p->rbuf, sizeof(float2) * (size_t)(p->rbuf_rows * cols));
  if (e != cudaSuccess) return set_error(FCB_ERR_NOMEM, "real-FFT work rows: %s", cudaGetErrorString(e));
  return FCB_OK;
}

// Real-input rows on device pointers, stream st.  in / out: float rows of n
// (real side) or complex rows of n/2 + 1 (spectrum side); strides in elements.
int exec_real_device(fcb_plan p, const void *in, long long in_rs, void *out, long long out_rs, long long rows,
                     cudaStream_t st)
{
  const long long n = p->rn;
  int rc = FCB_OK;
  if (n % 2 == 0)
  {
    const long long m = n / 2;
    if (p->real == 1)
    {
      const float *x = static_cast<const float *>(in);
      float2 *y = static_cast<float2 *>(out);
      const bool direct = aligned8(x) && (in_rs % 2 == 0 || rows == 1);
      if (!direct && (rc = ensure_rbuf(p, m))) return rc;
      const long long chunk = direct ? rows : p->rbuf_rows;
      for (long long r0 = 0; !rc && r0 < rows; r0 += chunk)
      {
        const long long nr = std::min(chunk, rows - r0);
        const float2 *z = reinterpret_cast<const float2 *>(x + r0 * in_rs);
        long long z_rs = rows == 1 ? m : in_rs / 2;
        if (!direct)
        {
          cudaError_t e = cudaMemcpy2DAsync(p->rbuf, sizeof(float2) * (size_t)m, x + r0 * in_rs,
                                            sizeof(float) * (size_t)in_rs, sizeof(float) * (size_t)n, (size_t)nr,
                                            cudaMemcpyDeviceToDevice, st);
          if (e != cudaSuccess) return cuda_error(e, "real rows copy");
          z = p->rbuf;
          z_rs = m;
        }
        rc = exec_device(p->cplx, z, z_rs, y + r0 * out_rs, out_rs, nr, 0, st);
        if (!rc) rc = r2c_post(y + r0 * out_rs, out_rs, m, nr, p->rtw, p->scale, st);
      }
    }
    else
    {
      const float2 *x = static_cast<const float2 *>(in);
      float *y = static_cast<float *>(out);
      const bool direct = aligned8(y) && (out_rs % 2 == 0 || rows == 1);
      if (!direct && (rc = ensure_rbuf(p, m))) return rc;
      const long long chunk = direct ? rows : p->rbuf_rows;
      for (long long r0 = 0; !rc && r0 < rows; r0 += chunk)
      {
        const long long nr = std::min(chunk, rows - r0);
        float2 *z = direct ? reinterpret_cast<float2 *>(y + r0 * out_rs) : p->rbuf;
        const long long z_rs = direct ? (rows == 1 ? m : out_rs / 2) : m;
        rc = c2r_pre(x + r0 * in_rs, in_rs, z, z_rs, m, nr, p->rtw, st);
        if (!rc) rc = exec_device(p->cplx, z, z_rs, z, z_rs, nr, 0, st);
        if (!rc && !direct)
        {
          cudaError_t e = cudaMemcpy2DAsync(y + r0 * out_rs, sizeof(float) * (size_t)out_rs, p->rbuf,
                                            sizeof(float2) * (size_t)m, sizeof(float) * (size_t)n, (size_t)nr,
                                            cudaMemcpyDeviceToDevice, st);
          if (e != cudaSuccess) return cuda_error(e, "real rows copy");
        }
      }
    }
    return rc;
  }
  // odd n: through full-length complex rows
  if ((rc = ensure_rbuf(p, n))) return rc;
  for (long long r0 = 0; !rc && r0 < rows; r0 += p->rbuf_rows)
  {
    const long long nr = std::min(p->rbuf_rows, rows - r0);
    if (p->real == 1)
    {
      const float *x = static_cast<const float *>(in) + r0 * in_rs;
      float2 *y = static_cast<float2 *>(out) + r0 * out_rs;
      rc = real_expand(x, in_rs, p->rbuf, n, nr, st);
      if (!rc) rc = exec_device(p->cplx, p->rbuf, n, p->rbuf, n, nr, 0, st);
      if (!rc)
      {
        cudaError_t e = cudaMemcpy2DAsync(y, sizeof(float2) * (size_t)out_rs, p->rbuf, sizeof(float2) * (size_t)n,
                                          sizeof(float2) * (size_t)(n / 2 + 1), (size_t)nr,
                                          cudaMemcpyDeviceToDevice, st);
        if (e != cudaSuccess) rc = cuda_error(e, "half-spectrum copy");
      }
    }
    else
    {
      const float2 *x = static_cast<const float2 *>(in) + r0 * in_rs;
      float *y = static_cast<float *>(out) + r0 * out_rs;
      rc = herm_expand(x, in_rs, p->rbuf, n, nr, st);
      if (!rc) rc = exec_device(p->cplx, p->rbuf, n, p->rbuf, n, nr, 0, st);
      if (!rc) rc = take_real(p->rbuf, n, y, out_rs, nr, st);
    }
  }
  return rc;
}

long long stage_bytes();
int stage_depth();

// Pinned host buffers for the staged copies of pageable memory, shared by all
// plans (one set per process rather than per plan: a program may hold many
// plans), portable so that plans on any device can use them.  A call that
// stages holds `mu` from its first copy until none of its copies through
// these buffers is queued or running.
constexpr int kNoPinned = -1;  // pinned memory could not be had: copy directly instead
struct PinnedStaging
{
  std::mutex mu;
  float2 *buf[2][fcb_plan_s::kMaxStage] = {};  // [0] to the device, [1] from it
  size_t bytes[2] = {0, 0};
  int count[2] = {0, 0};
};
PinnedStaging &pinned()
{
  static PinnedStaging *s = new PinnedStaging;  // kept for the process's lifetime
  return *s;
}

// With pinned().mu held: `depth` pinned buffers of at least `bytes` bytes for
// direction d (0: to the device, 1: from it), and the plan's events that track
// each buffer's last copy.  kNoPinned if the pinned memory could not be had.
int ensure_host_staging(fcb_plan p, int d, size_t bytes, int depth)
{
  if (!p->ev_h[d][0])
    for (int i = 0; i < fcb_plan_s::kMaxStage; ++i)
    {
      const cudaError_t e = cudaEventCreateWithFlags(&p->ev_h[d][i], cudaEventDisableTiming);
      if (e != cudaSuccess) return cuda_error(e, "staging events");
    }
  PinnedStaging &ps = pinned();
  if (ps.bytes[d] >= bytes && ps.count[d] >= depth) return FCB_OK;
  for (auto &b : ps.buf[d])
  {
    cudaFreeHost(b);
    b = nullptr;
  }
  ps.bytes[d] = 0;
  ps.count[d] = 0;
  for (int i = 0; i < depth; ++i)
    if (cudaHostAlloc(reinterpret_cast<void **>(&ps.buf[d][i]), bytes, cudaHostAllocPortable) != cudaSuccess)
    {
      cudaGetLastError();
      for (auto &b : ps.buf[d])
      {
        cudaFreeHost(b);
        b = nullptr;
      }
      return kNoPinned;
    }
  ps.bytes[d] = bytes;
  ps.count[d] = depth;
  return FCB_OK;
}

// Host -> device copy of `rows` rows of `rb` bytes (pitches in bytes) on
// stream st.  Pinned host memory moves directly (queued only).  Pageable host
// memory moves through the shared pinned buffers in chunks of about the
// staging size, each copied by the copy threads while the copy engine moves
// the previous one; returns once every chunk has arrived.
int copy_h2d(fcb_plan p, void *dev, size_t dp, const void *host, size_t hp, size_t rb, size_t rows,
             cudaStream_t st)
{
  cudaError_t e;
  if (host_pageable(host, hp * (rows - 1) + rb))
  {
    std::lock_guard<std::mutex> lk(pinned().mu);
    const int depth = stage_depth();
    const size_t chunk = std::max<size_t>(1, (size_t)stage_bytes() / rb);
    int rc = ensure_host_staging(p, 0, std::min(chunk, rows) * rb, depth);
    if (rc != kNoPinned)
    {
      if (rc) return rc;
      size_t c = 0;
      for (size_t r0 = 0; r0 < rows; r0 += chunk, ++c)
      {
        const int b = (int)(c % depth);
        const size_t nr = std::min(chunk, rows - r0);
        if ((e = cudaEventSynchronize(p->ev_h[0][b])) != cudaSuccess) return cuda_error(e, "host->device copy");
        host_copy_rows(pinned().buf[0][b], rb, static_cast<const char *>(host) + r0 * hp, hp, rb, nr);
        e = cudaMemcpy2DAsync(static_cast<char *>(dev) + r0 * dp, dp, pinned().buf[0][b], rb, rb, nr,
                              cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) return cuda_error(e, "host->device copy");
        cudaEventRecord(p->ev_h[0][b], st);
      }
      // the buffers go back to the other plans only once their copies are done
      for (int b = 0; b < depth; ++b)
        if ((e = cudaEventSynchronize(p->ev_h[0][b])) != cudaSuccess) return cuda_error(e, "host->device copy");
      return FCB_OK;
    }
  }
  e = cudaMemcpy2DAsync(dev, dp, host, hp, rb, rows, cudaMemcpyHostToDevice, st);
  return e == cudaSuccess ? FCB_OK : cuda_error(e, "host->device copy");
}

// Device -> host copy of `rows` rows of `rb` bytes on stream st, after the work
// queued on it.  Pageable host memory: through the shared pinned buffers, the
// copy threads draining each chunk while the copy engine moves the next ones;
// returns once the host rows are written.  Pinned host memory: queued only.
int copy_d2h(fcb_plan p, void *host, size_t hp, const void *dev, size_t dp, size_t rb, size_t rows,
             cudaStream_t st)
{
  cudaError_t e;
  if (host_pageable(host, hp * (rows - 1) + rb))
  {
    std::lock_guard<std::mutex> lk(pinned().mu);
    const int depth = stage_depth(), lag = depth - 1;
    const size_t chunk = std::max<size_t>(1, (size_t)stage_bytes() / rb);
    int rc = ensure_host_staging(p, 1, std::min(chunk, rows) * rb, depth);
    if (rc != kNoPinned)
    {
      if (rc) return rc;
      const size_t nc = (rows + chunk - 1) / chunk;
      auto drain = [&](size_t c) -> int {
        const int b = (int)(c % depth);
        const size_t r0 = c * chunk, nr = std::min(chunk, rows - r0);
        const cudaError_t e2 = cudaEventSynchronize(p->ev_h[1][b]);
        if (e2 != cudaSuccess) return cuda_error(e2, "device->host copy");
        host_copy_rows(static_cast<char *>(host) + r0 * hp, hp, pinned().buf[1][b], rb, rb, nr);
        return FCB_OK;
      };
      for (size_t c = 0; c < nc; ++c)
      {
        const int b = (int)(c % depth);
        const size_t r0 = c * chunk, nr = std::min(chunk, rows - r0);
        // the pinned buffer's previous chunk was drained lag chunks ago
        e = cudaMemcpy2DAsync(pinned().buf[1][b], rb, static_cast<const char *>(dev) + r0 * dp, dp, rb, nr,
                              cudaMemcpyDeviceToHost, st);
        if (e != cudaSuccess) return cuda_error(e, "device->host copy");
        cudaEventRecord(p->ev_h[1][b], st);
        if (c >= (size_t)lag && (rc = drain(c - lag))) return rc;
      }
      for (size_t c = nc > (size_t)lag ? nc - lag : 0; c < nc; ++c)
        if ((rc = drain(c))) return rc;
      return FCB_OK;
    }
  }
  e = cudaMemcpy2DAsync(host, hp, dev, dp, rb, rows, cudaMemcpyDeviceToHost, st);
  return e == cudaSuccess ? FCB_OK : cuda_error(e, "device->host copy");
}

// A host-buffer call returns only once none of its copies is queued or running,
// on an error too: its caller may free or reuse the host buffers as soon as
// the call returns.  Waits for the plan's streams and keeps the first error.
int host_done(fcb_plan p, int rc, const char *what)
{
  const cudaStream_t ss[3] = {p->cin, p->cout, p->stream};
  for (int i = 0; i < 3; ++i)
  {
    if (i < 2 && !ss[i]) continue;  // copy streams not created yet (the plan stream may be NULL: default stream)
    const cudaError_t e = cudaStreamSynchronize(ss[i]);
    if (e != cudaSuccess && rc == FCB_OK) rc = cuda_error(e, what);
  }
  return rc;
}

// Real-input rows on host pointers: chunks staged through two device buffers.
int exec_real_host(fcb_plan p, const void *in, long long in_rs, void *out, long long out_rs, long long rows)
{
  const long long n = p->rn, h = n / 2 + 1;
  const size_t in_el = p->real == 1 ? sizeof(float) : sizeof(float2);
  const size_t out_el = p->real == 1 ? sizeof(float2) : sizeof(float);
  const long long in_cols = p->real == 1 ? n : h, out_cols = p->real == 1 ? h : n;
  // even column counts keep every staged row 8-byte aligned
  const long long in_pitch = in_cols + (in_cols & 1), out_pitch = out_cols + (out_cols & 1);
  const long long row_bytes = (long long)(in_el * in_pitch + out_el * out_pitch);
  const long long chunk = std::min(rows, std::max<long long>(1, (32LL << 20) / row_bytes));
  if (p->rstage_rows < chunk)
  {
    cudaFree(p->rstage[0]);
    cudaFree(p->rstage[1]);
    p->rstage[0] = p->rstage[1] = nullptr;
    p->rstage_rows = 0;
    cudaError_t e = cudaMalloc(&p->rstage[0], in_el * (size_t)(chunk * in_pitch));
    if (e == cudaSuccess) e = cudaMalloc(&p->rstage[1], out_el * (size_t)(chunk * out_pitch));
    if (e != cudaSuccess) return set_error(FCB_ERR_NOMEM, "staging buffer: %s", cudaGetErrorString(e));
    p->rstage_rows = chunk;
  }
  const char *src = static_cast<const char *>(in);
  char *dst = static_cast<char *>(out);
  for (long long r0 = 0; r0 < rows; r0 += chunk)
  {
    const long long nr = std::min(chunk, rows - r0);
    int rc = copy_h2d(p, p->rstage[0], in_el * (size_t)in_pitch, src + in_el * (size_t)(r0 * in_rs),
                      in_el * (size_t)in_rs, in_el * (size_t)in_cols, (size_t)nr, p->stream);
    if (rc) return host_done(p, rc, "real FFT (host)");
    rc = exec_real_device(p, p->rstage[0], in_pitch, p->rstage[1], out_pitch, nr, p->stream);
    if (rc) return host_done(p, rc, "real FFT (host)");
    rc = copy_d2h(p, dst + out_el * (size_t)(r0 * out_rs), out_el * (size_t)out_rs, p->rstage[1],
                  out_el * (size_t)out_pitch, out_el * (size_t)out_cols, (size_t)nr, p->stream);
    if (rc) return host_done(p, rc, "real FFT (host)");
  }
  return host_done(p, FCB_OK, "real FFT (host)");
}

int exec_real(fcb_plan p, int kind, const void *in, long long in_rs, void *out, long long out_rs, long long rows,
              int where)
{
  if (!p) return set_error(FCB_ERR_INVALID, "plan is NULL");
  if (p->real != kind)
    return set_error(FCB_ERR_INVALID, p->real ? "wrong direction for this real-FFT plan"
                                              : "not a real-FFT plan (use fcb_exec)");
  if (rows < 0 || rows > p->rows_max) return set_error(FCB_ERR_INVALID, "rows %lld outside [0, %lld]", rows, p->rows_max);
  if (rows == 0) return FCB_OK;
  if (!in || !out) return set_error(FCB_ERR_INVALID, "NULL data pointer");
  const long long h = p->rn / 2 + 1;
  const long long in_min = kind == 1 ? p->rn : h, out_min = kind == 1 ? h : p->rn;
  if (in_rs < in_min || out_rs < out_min) return set_error(FCB_ERR_INVALID, "row stride smaller than the row length");
  if (where != FCB_HOST && where != FCB_DEVICE) return set_error(FCB_ERR_INVALID, "bad location");
  DeviceGuard g(p->device);
  if (where == FCB_DEVICE) return exec_real_device(p, in, in_rs, out, out_rs, rows, p->stream);
  return exec_real_host(p, in, in_rs, out, out_rs, rows);
}

// 2-D FFT on device pointers: two transposing row passes.
int exec_2d(fcb_plan p, const float2 *in, long long in_rs, float2 *out, long long out_rs, cudaStream_t st)
{
  if (p->general2d)
  {
    const long long R = p->rows2d, C = p->cols2d;
    int rc = exec_device(p->sub2d[0], in, in_rs, p->scratch, C, R, 0, st);
    if (!rc) rc = launch_transpose(p->scratch, C, p->scratch2, R, R, C, st);        // scratch2 = scratch^T
    if (!rc) rc = exec_device(p->sub2d[1], p->scratch2, R, p->scratch2, R, C, 0, st);  // the columns, scaled
    if (!rc) rc = launch_transpose(p->scratch2, R, out, out_rs, C, R, st);
    return rc;
  }
  RowArgs a = {};
  a.in = in;
  a.in_rs = in_rs;
  a.out = p->scratch;
  a.out_rs = p->rows2d;
  a.rows = p->rows2d;
  a.tw = a.twi = p->tw;
  a.scale = 1.f;
  a.transpose_out = 1;
  a.ahead = -1;
  int rc = launch_rows(p->k, p->rows2d, a, st);
  if (rc) return rc;
  a.in = p->scratch;
  a.in_rs = p->rows2d;
  a.out = out;
  a.out_rs = out_rs;
  a.rows = p->cols2d;
  a.tw = a.twi = p->twc;
  a.scale = p->scale;
  return launch_rows(p->kc, p->cols2d, a, st);
}

// Device-pointer execution on stream st (slot: Bluestein work buffer).
int exec_device(fcb_plan p, const float2 *in, long long in_rs, float2 *out, long long out_rs,
                long long rows, long long row0, cudaStream_t st, int slot)
{
  if (p->blue_m) return exec_blue(p, in, in_rs, out, out_rs, rows, row0, st, slot);
  const float4 *rep = p->rep ? p->rep + (p->rep_rows > 1 ? row0 * (p->n > 1 ? p->n / 2 : 1) : 0) : nullptr;
  long long rep_rs = p->rep_rows > 1 ? (p->n > 1 ? p->n / 2 : 1) : 0;
  if (p->logn == 0)
    return launch_scale_rows(in, in_rs, out, out_rs, rows, p->mode == kFastconv ? rep : nullptr, rep_rs,
                             p->scale, st);
  RowArgs a = {};
  a.in = in;
  a.in_rs = in_rs;
  a.out = out;
  a.out_rs = out_rs;
  a.rows = rows;
  a.tw = p->tw;
  a.twi = p->tw;
  a.rep = rep;
  a.rep_rs = rep_rs;
  a.scale = p->scale;
  a.vec_out = (reinterpret_cast<uintptr_t>(out) % 16 == 0) && (out_rs % 2 == 0 || rows == 1);
  a.ahead = -1;  // launch_rows picks half a resident wave
  return launch_rows(p->k, rows, a, st);
}

// Host staging shape: chunk bytes and pipeline depth.  FCB200_STAGE_MB and
// FCB200_STAGES override the defaults (16 MB, 4 buffers; queued calls use
// chunks of twice the size).
long long stage_bytes()
{
  static const long long v = [] {
    const char *e = std::getenv("FCB200_STAGE_MB");
    const long long mb = e ? std::atoll(e) : 16;
    return std::max<long long>(1, mb) << 20;
  }();
  return v;
}
int stage_depth()
{
  static const int v = [] {
    const char *e = std::getenv("FCB200_STAGES");
    const int d = e ? std::atoi(e) : 4;
    return std::min(std::max(d, 2), (int)fcb_plan_s::kMaxStage);
  }();
  return v;
}

int ensure_staging(fcb_plan p, long long chunk_rows, int depth)
{
  if (p->stage_rows >= chunk_rows && p->nstage >= depth) return FCB_OK;
  for (auto &b : p->stage)
  {
    cudaFree(b);
    b = nullptr;
  }
  p->stage_rows = 0;
  p->nstage = 0;
  for (int i = 0; i < depth; ++i)
  {
    cudaError_t e = cudaMalloc(&p->stage[i], sizeof(float2) * (size_t)(chunk_rows * p->n));
    if (e != cudaSuccess) return set_error(FCB_ERR_NOMEM, "staging buffer: %s", cudaGetErrorString(e));
  }
  if (!p->cin)
  {
    cudaError_t e = cudaStreamCreateWithFlags(&p->cin, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&p->cout, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&p->ev_start, cudaEventDisableTiming);
    for (int i = 0; e == cudaSuccess && i < fcb_plan_s::kMaxStage; ++i)
    {
      e = cudaEventCreateWithFlags(&p->ev_in[i], cudaEventDisableTiming);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&p->ev_k[i], cudaEventDisableTiming);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&p->ev_out[i], cudaEventDisableTiming);
    }
    if (e != cudaSuccess) return cuda_error(e, "staging streams");
  }
  p->stage_rows = chunk_rows;
  p->nstage = depth;
  return FCB_OK;
}

// Host-pointer execution: rows move through `depth` device buffers in chunks.
// Copies in run on cin, kernels on the plan stream, copies out on cout, linked
// by events, so both copy directions and the kernels overlap and the PCIe link
// stays busy in both directions; a buffer is refilled once its copy out is done.
// sync = false (fcb_exec_async): return once everything is queued.
int exec_host_staged(fcb_plan p, const float2 *in, long long in_rs, float2 *out, long long out_rs,
                     long long rows, bool stage_in, bool stage_out);

int exec_host(fcb_plan p, const float2 *in, long long in_rs, float2 *out, long long out_rs,
              long long rows, bool sync = true)
{
  const size_t row_bytes = sizeof(float2) * (size_t)p->n;
  {
    // pageable host memory goes through the plan's pinned buffers
    const size_t in_span = sizeof(float2) * (size_t)((rows - 1) * in_rs + p->n);
    const size_t out_span = sizeof(float2) * (size_t)((rows - 1) * out_rs + p->n);
    const bool stage_in = host_pageable(in, in_span), stage_out = host_pageable(out, out_span);
    if (stage_in || stage_out)
    {
      const int rc = exec_host_staged(p, in, in_rs, out, out_rs, rows, stage_in, stage_out);
      if (rc != kNoPinned) return rc;
      // no pinned memory to be had: the CUDA runtime copies the pageable memory
    }
  }
  // A queued call (sync = false) is expected to have neighbours on the link:
  // it moves twice the chunk size per copy and skips the ramps below (fewer,
  // larger copies; the fill and drain overlap the neighbouring calls).  The
  // staging buffers always hold the larger chunk, so that switching between
  // waiting and queued calls never reallocates them (a cudaFree waits for
  // the whole device).
  const long long base = std::max<long long>(1, stage_bytes() / (long long)row_bytes);
  long long chunk = sync ? base : 2 * base;
  long long alloc = 2 * base;
  if (p->k && p->k->cluster == 1)
  {
    chunk = std::max<long long>(chunk, p->k->rows_per_cta);
    alloc = std::max<long long>(alloc, p->k->rows_per_cta);
  }
  chunk = std::min(chunk, rows);
  const int depth = stage_depth();
  int rc = ensure_staging(p, std::min(alloc, rows), depth);
  if (rc) return rc;
  // nothing starts before earlier work on the plan stream
  cudaEventRecord(p->ev_start, p->stream);
  cudaStreamWaitEvent(p->cin, p->ev_start, 0);
  cudaStreamWaitEvent(p->cout, p->ev_start, 0);
  // Chunk sizes of a call that waits for its result ramp up over the first
  // chunks and down over the last ones (1/8, 1/4, 1/2 of a full chunk), so the
  // first copy out and the last copy in overlap the other direction sooner:
  // the link idles in one direction only for a small chunk at each end.
  const long long unit = std::max<long long>(1, (p->k && p->k->cluster == 1) ? p->k->rows_per_cta : 1);
  std::vector<long long> sizes;
  {
    const long long ramp[3] = {chunk / 8, chunk / 4, chunk / 2};
    long long head = 0;
    for (long long v : ramp) head += std::max(unit, v);
    if (sync && rows >= 2 * head + chunk)
    {
      long long left = rows;
      for (long long v : ramp) { sizes.push_back(std::max(unit, v)); left -= sizes.back(); }
      left -= head;  // reserved for the tail ramp
      while (left > 0) { sizes.push_back(std::min(chunk, left)); left -= sizes.back(); }
      for (int i = 2; i >= 0; --i) sizes.push_back(std::max(unit, ramp[i]));
    }
    else
      for (long long left = rows; left > 0; left -= sizes.back()) sizes.push_back(std::min(chunk, left));
  }
  long long r0 = 0;
  // The buffer rotation continues from the previous call, so that a call
  // queued behind another one (fcb_exec_async) fills first the buffers whose
  // copies out finished earliest instead of waiting for the last ones.
  const int b0 = p->stage_next % depth;
  p->stage_next = (int)((b0 + sizes.size()) % depth);
  for (size_t c = 0; c < sizes.size(); r0 += sizes[c], ++c)
  {
    const int b = (int)((b0 + c) % depth);
    const long long nr = sizes[c];
    float2 *buf = p->stage[b];
    // buffer drained: by this call's copy out of chunk c - depth, or by the last
    // copy out from it of an earlier call still in flight (asynchronous calls);
    // an event never recorded is no wait
    cudaStreamWaitEvent(p->cin, p->ev_out[b], 0);
    // dense rows move as one linear copy, strided rows as a pitched one
    cudaError_t e = in_rs == p->n
                      ? cudaMemcpyAsync(buf, in + r0 * in_rs, row_bytes * (size_t)nr, cudaMemcpyHostToDevice, p->cin)
                      : cudaMemcpy2DAsync(buf, row_bytes, in + r0 * in_rs, sizeof(float2) * (size_t)in_rs, row_bytes,
                                          (size_t)nr, cudaMemcpyHostToDevice, p->cin);
    if (e != cudaSuccess) return host_done(p, cuda_error(e, "host->device copy"), "fcb_exec (host)");
    cudaEventRecord(p->ev_in[b], p->cin);
    cudaStreamWaitEvent(p->stream, p->ev_in[b], 0);
    rc = exec_device(p, buf, p->n, buf, p->n, nr, r0, p->stream, 0);
    if (rc) return host_done(p, rc, "fcb_exec (host)");
    cudaEventRecord(p->ev_k[b], p->stream);
    cudaStreamWaitEvent(p->cout, p->ev_k[b], 0);
    e = out_rs == p->n
          ? cudaMemcpyAsync(out + r0 * out_rs, buf, row_bytes * (size_t)nr, cudaMemcpyDeviceToHost, p->cout)
          : cudaMemcpy2DAsync(out + r0 * out_rs, sizeof(float2) * (size_t)out_rs, buf, row_bytes, row_bytes,
                              (size_t)nr, cudaMemcpyDeviceToHost, p->cout);
    if (e != cudaSuccess) return host_done(p, cuda_error(e, "device->host copy"), "fcb_exec (host)");
    cudaEventRecord(p->ev_out[b], p->cout);
  }
  if (!sync)
  {
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? FCB_OK : cuda_error(e, "fcb_exec_async (host)");
  }
  return host_done(p, FCB_OK, "fcb_exec (host)");
}

// Host call with pageable input and/or output: each chunk is copied by the
// copy threads into a shared pinned buffer, moved in, transformed, moved out
// into another pinned buffer and copied to the caller's rows, while the copy
// engines and the kernels work on the neighbouring chunks.  A pinned side
// moves directly.  Returns when the output is written, queued or not;
// kNoPinned, before any work, if the pinned buffers could not be had.
int exec_host_staged(fcb_plan p, const float2 *in, long long in_rs, float2 *out, long long out_rs,
                     long long rows, bool stage_in, bool stage_out)
{
  std::lock_guard<std::mutex> lk(pinned().mu);
  const size_t row_bytes = sizeof(float2) * (size_t)p->n;
  long long chunk = std::max<long long>(1, stage_bytes() / (long long)row_bytes);
  long long alloc = 2 * chunk;  // the device buffers as the pinned path sizes them
  if (p->k && p->k->cluster == 1)
  {
    chunk = std::max<long long>(chunk, p->k->rows_per_cta);
    alloc = std::max<long long>(alloc, p->k->rows_per_cta);
  }
  chunk = std::min(chunk, rows);
  const int depth = stage_depth();
  int rc = ensure_staging(p, std::min(alloc, rows), depth);
  if (rc) return rc;
  if (stage_in && (rc = ensure_host_staging(p, 0, row_bytes * (size_t)chunk, depth))) return rc;
  if (stage_out && (rc = ensure_host_staging(p, 1, row_bytes * (size_t)chunk, depth))) return rc;
  cudaEventRecord(p->ev_start, p->stream);
  cudaStreamWaitEvent(p->cin, p->ev_start, 0);
  cudaStreamWaitEvent(p->cout, p->ev_start, 0);
  const long long nc = (rows + chunk - 1) / chunk;
  const int b0 = p->stage_next % depth;
  p->stage_next = (int)((b0 + nc) % depth);
  const int lag = depth - 1;  // chunks between a chunk's copy in and its copy out on the host
  auto buf_of = [&](long long c) { return (int)((b0 + c) % depth); };
  // copy chunk d's result from its pinned buffer to the caller's rows
  auto drain = [&](long long d) -> int {
    const int b = buf_of(d);
    const long long r0 = d * chunk, nr = std::min(chunk, rows - r0);
    const cudaError_t e = cudaEventSynchronize(p->ev_h[1][b]);
    if (e != cudaSuccess) return cuda_error(e, "device->host copy");
    host_copy_rows(out + r0 * out_rs, sizeof(float2) * (size_t)out_rs, pinned().buf[1][b], row_bytes, row_bytes,
                   (size_t)nr);
    return FCB_OK;
  };
  for (long long c = 0; c < nc; ++c)
  {
    const int b = buf_of(c);
    const long long r0 = c * chunk, nr = std::min(chunk, rows - r0);
    const float2 *src = in + r0 * in_rs;
    long long src_rs = in_rs;
    if (stage_in)
    {
      // the pinned buffer's previous chunk has moved in
      cudaError_t e = cudaEventSynchronize(p->ev_h[0][b]);
      if (e != cudaSuccess) return host_done(p, cuda_error(e, "host->device copy"), "fcb_exec (host)");
      host_copy_rows(pinned().buf[0][b], row_bytes, src, sizeof(float2) * (size_t)in_rs, row_bytes, (size_t)nr);
      src = pinned().buf[0][b];
      src_rs = p->n;
    }
    float2 *buf = p->stage[b];
    cudaStreamWaitEvent(p->cin, p->ev_out[b], 0);
    cudaError_t e = src_rs == p->n
                      ? cudaMemcpyAsync(buf, src, row_bytes * (size_t)nr, cudaMemcpyHostToDevice, p->cin)
                      : cudaMemcpy2DAsync(buf, row_bytes, src, sizeof(float2) * (size_t)src_rs, row_bytes, (size_t)nr,
                                          cudaMemcpyHostToDevice, p->cin);
    if (e != cudaSuccess) return host_done(p, cuda_error(e, "host->device copy"), "fcb_exec (host)");
    cudaEventRecord(p->ev_in[b], p->cin);
    if (stage_in) cudaEventRecord(p->ev_h[0][b], p->cin);
    cudaStreamWaitEvent(p->stream, p->ev_in[b], 0);
    rc = exec_device(p, buf, p->n, buf, p->n, nr, r0, p->stream, 0);
    if (rc) return host_done(p, rc, "fcb_exec (host)");
    cudaEventRecord(p->ev_k[b], p->stream);
    cudaStreamWaitEvent(p->cout, p->ev_k[b], 0);
    // the output's pinned buffer was drained on the host depth chunks ago
    e = stage_out ? cudaMemcpyAsync(pinned().buf[1][b], buf, row_bytes * (size_t)nr, cudaMemcpyDeviceToHost, p->cout)
        : out_rs == p->n
          ? cudaMemcpyAsync(out + r0 * out_rs, buf, row_bytes * (size_t)nr, cudaMemcpyDeviceToHost, p->cout)
          : cudaMemcpy2DAsync(out + r0 * out_rs, sizeof(float2) * (size_t)out_rs, buf, row_bytes, row_bytes,
                              (size_t)nr, cudaMemcpyDeviceToHost, p->cout);
    if (e != cudaSuccess) return host_done(p, cuda_error(e, "device->host copy"), "fcb_exec (host)");
    cudaEventRecord(p->ev_out[b], p->cout);
    if (stage_out) cudaEventRecord(p->ev_h[1][b], p->cout);
    if (stage_out && c >= lag)
    {
      rc = drain(c - lag);
      if (rc) return host_done(p, rc, "fcb_exec (host)");
    }
  }
  if (stage_out)
    for (long long d = std::max<long long>(0, nc - lag); d < nc; ++d)
    {
      rc = drain(d);
      if (rc) return host_done(p, rc, "fcb_exec (host)");
    }
  return host_done(p, FCB_OK, "fcb_exec (host)");
}

}  // namespace

extern "C" {

const char *fcb_last_error(void)
{
  return error_text();
}

const char *fcb_version(void) { return "fcb200 0.1 (sm_100a)"; }

int fcb_init(int device)
{
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0) return set_error(FCB_ERR_NODEVICE, "no CUDA device");
  if (device < 0 || device >= count) return set_error(FCB_ERR_INVALID, "device %d out of range [0,%d)", device, count);
  e = cudaSetDevice(device);
  if (e != cudaSuccess) return cuda_error(e, "cudaSetDevice");
  return check_device();
}

int fcb_supported_length(long long n)
{
  int l = log2_exact(n);
  return (l >= 0 && l <= kMaxLogN) || blue_length(n);
}

int fcb_plan_fftm(long long n, long long rows_max, int exponent, float scale, fcb_plan *plan)
{
  if (!plan) return set_error(FCB_ERR_INVALID, "plan pointer is NULL");
  *plan = nullptr;
  if (!fcb_supported_length(n))
    return set_error(FCB_ERR_UNSUPPORTED, "row length %lld unsupported: " FCB_LENGTH_RULE, n);
  if (rows_max < 0) return set_error(FCB_ERR_INVALID, "rows_max < 0");
  if (exponent != FCB_FORWARD && exponent != FCB_INVERSE) return set_error(FCB_ERR_INVALID, "exponent must be -1 or +1");
  fcb_plan p = new (std::nothrow) fcb_plan_s;
  if (!p) return set_error(FCB_ERR_NOMEM, "plan allocation");
  p->scale = scale;
  const int mode = exponent == FCB_FORWARD ? kFwd : kInv;
  int rc = blue_length(n) ? blue_setup(p, n, rows_max, mode, mode == kFwd, mode == kInv)
                          : plan_common(p, n, rows_max, mode);
  if (!rc && blue_length(n))
  {
    // the output multiplier of a Bluestein row: the chirp times the scale
    cudaError_t e = cudaMalloc(&p->chirp_out, sizeof(float2) * (size_t)n);
    if (e != cudaSuccess) rc = set_error(FCB_ERR_NOMEM, "Bluestein chirp: %s", cudaGetErrorString(e));
    else rc = scale_copy(p->chirp[mode == kFwd ? 0 : 1], p->chirp_out, n, scale, p->stream);
  }
  if (!rc)
  {
    cudaError_t e = cudaStreamSynchronize(p->stream);
    if (e != cudaSuccess) rc = cuda_error(e, "plan tables");
  }
  if (rc) { plan_free(p); return rc; }
  *plan = p;
  return FCB_OK;
}

int fcb_plan_fastconv(long long n, long long rows_max, const fcb_cf32 *replica, long long replica_rows,
                      long long replica_rs, int replica_kind, int where, fcb_plan *plan)
{
  if (!plan) return set_error(FCB_ERR_INVALID, "plan pointer is NULL");
  *plan = nullptr;
  if (!fcb_supported_length(n))
    return set_error(FCB_ERR_UNSUPPORTED, "row length %lld unsupported: " FCB_LENGTH_RULE, n);
  if (!replica) return set_error(FCB_ERR_INVALID, "replica is NULL");
  if (replica_rows < 1) return set_error(FCB_ERR_INVALID, "replica_rows < 1");
  if (replica_rows > 1 && replica_rs < n) return set_error(FCB_ERR_INVALID, "replica row stride < n");
  if (replica_kind < FCB_REPLICA_SPECTRUM || replica_kind > FCB_REPLICA_TIME_MATCHED)
    return set_error(FCB_ERR_INVALID, "bad replica kind");
  if (where != FCB_HOST && where != FCB_DEVICE) return set_error(FCB_ERR_INVALID, "bad location");
  fcb_plan p = new (std::nothrow) fcb_plan_s;
  if (!p) return set_error(FCB_ERR_NOMEM, "plan allocation");
  const bool blue = blue_length(n);
  int rc = blue ? blue_setup(p, n, rows_max, kFastconv, true, true) : plan_common(p, n, rows_max, kFastconv);
  float2 *spec = nullptr, *tmp = nullptr;
  if (!rc)
  {
    const long long rs = replica_rows > 1 ? replica_rs : n;
    const size_t bytes = sizeof(float2) * (size_t)(replica_rows * n);
    cudaError_t e = cudaMalloc(&spec, bytes);
    if (e != cudaSuccess) rc = set_error(FCB_ERR_NOMEM, "replica buffer: %s", cudaGetErrorString(e));
    if (!rc)
    {
      e = cudaMemcpy2DAsync(spec, sizeof(float2) * (size_t)n, replica, sizeof(float2) * (size_t)rs,
                            sizeof(float2) * (size_t)n, (size_t)replica_rows,
                            where == FCB_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, p->stream);
      if (e != cudaSuccess) rc = cuda_error(e, "replica copy");
    }
    if (!rc && replica_kind != FCB_REPLICA_SPECTRUM)
    {
      e = cudaMalloc(&tmp, bytes);
      if (e != cudaSuccess) rc = set_error(FCB_ERR_NOMEM, "replica buffer: %s", cudaGetErrorString(e));
      for (long long r = 0; !rc && r < replica_rows; ++r)
        rc = replica_spectrum_dev(spec + r * n, n, replica_kind == FCB_REPLICA_TIME_MATCHED, tmp + r * n, p->stream);
      if (!rc) std::swap(spec, tmp);
    }
    if (!rc && blue)
    {
      // R / n per row; 1/n is the inverse FFT's normalisation
      p->rep_rows = replica_rows;
      e = cudaMalloc(&p->blue_rep, bytes);
      if (e != cudaSuccess) rc = set_error(FCB_ERR_NOMEM, "replica table: %s", cudaGetErrorString(e));
      if (!rc) rc = scale_copy(spec, p->blue_rep, replica_rows * n, (float)(1.0 / (double)n), p->stream);
    }
    else if (!rc)
    {
      const long long slots = n > 1 ? n / 2 : 1;
      e = cudaMalloc(&p->rep, sizeof(float4) * (size_t)(replica_rows * slots));
      if (e != cudaSuccess) rc = set_error(FCB_ERR_NOMEM, "replica table: %s", cudaGetErrorString(e));
      p->rep_rows = replica_rows;
      if (!rc)
      {
        if (p->logn >= 1)
          rc = build_replica_table(p->logn, p->k->ept, spec, n, replica_rows, p->rep, p->stream);
        else
        {
          // length 1: table entry (R.re, -, R.im, -)
          cudaMemset2DAsync(p->rep, sizeof(float4), 0, sizeof(float4), (size_t)replica_rows, p->stream);
          e = cudaMemcpy2DAsync(p->rep, sizeof(float4), spec, sizeof(float2), sizeof(float), (size_t)replica_rows,
                                cudaMemcpyDeviceToDevice, p->stream);
          if (e == cudaSuccess)
            e = cudaMemcpy2DAsync(reinterpret_cast<char *>(p->rep) + 8, sizeof(float4),
                                  reinterpret_cast<char *>(spec) + 4, sizeof(float2), sizeof(float),
                                  (size_t)replica_rows, cudaMemcpyDeviceToDevice, p->stream);
          if (e != cudaSuccess) rc = cuda_error(e, "replica table (n=1)");
        }
      }
    }
    if (!rc)
    {
      e = cudaStreamSynchronize(p->stream);
      if (e != cudaSuccess) rc = cuda_error(e, "replica preparation");
    }
  }
  cudaFree(spec);
  cudaFree(tmp);
  if (rc) { plan_free(p); return rc; }
  *plan = p;
  return FCB_OK;
}

int exec_impl(fcb_plan p, const fcb_cf32 *in, long long in_rs, fcb_cf32 *out, long long out_rs, long long rows,
              int where, bool sync);

int fcb_exec(fcb_plan p, const fcb_cf32 *in, long long in_rs, fcb_cf32 *out, long long out_rs,
             long long rows, int where)
{
  return exec_impl(p, in, in_rs, out, out_rs, rows, where, true);
}

int fcb_exec_async(fcb_plan p, const fcb_cf32 *in, long long in_rs, fcb_cf32 *out, long long out_rs,
                   long long rows, int where)
{
  return exec_impl(p, in, in_rs, out, out_rs, rows, where, false);
}

}  // extern "C"

int exec_impl(fcb_plan p, const fcb_cf32 *in, long long in_rs, fcb_cf32 *out, long long out_rs, long long rows,
              int where, bool sync)
{
  if (!p) return set_error(FCB_ERR_INVALID, "plan is NULL");
  if (p->real) return set_error(FCB_ERR_INVALID, "real-FFT plans run through fcb_exec_r2c / fcb_exec_c2r");
  if (rows < 0 || rows > p->rows_max) return set_error(FCB_ERR_INVALID, "rows %lld outside [0, %lld]", rows, p->rows_max);
  if (p->mode == kFastconv && p->rep_rows > 1 && rows > p->rep_rows)
    return set_error(FCB_ERR_INVALID, "rows %lld exceed the replica matrix rows %lld", rows, p->rep_rows);
  if (rows == 0) return FCB_OK;
  if (!in || !out) return set_error(FCB_ERR_INVALID, "NULL data pointer");
  if (in_rs < p->n || out_rs < p->n) return set_error(FCB_ERR_INVALID, "row stride smaller than the row length");
  if (where != FCB_HOST && where != FCB_DEVICE) return set_error(FCB_ERR_INVALID, "bad location");
  // in-place with different strides would overlap rows
  if ((const void *)in == (const void *)out && in_rs != out_rs)
    return set_error(FCB_ERR_INVALID, "in-place call with different row strides");
  DeviceGuard g(p->device);
  const float2 *i2 = reinterpret_cast<const float2 *>(in);
  float2 *o2 = reinterpret_cast<float2 *>(out);
  if (p->is2d)
  {
    if (rows != p->rows2d) return set_error(FCB_ERR_INVALID, "a 2-D FFT transforms the whole %lld-row matrix", p->rows2d);
    if ((const void *)in == (const void *)out && in_rs != out_rs)
      return set_error(FCB_ERR_INVALID, "in-place call with different row strides");
    if (where == FCB_DEVICE) return exec_2d(p, i2, in_rs, o2, out_rs, p->stream);
    const size_t bytes = sizeof(float2) * (size_t)(p->rows2d * p->cols2d);
    cudaError_t e = cudaSuccess;
    if (!p->stage2d_in && (e = cudaMalloc(&p->stage2d_in, bytes)) != cudaSuccess)
      return set_error(FCB_ERR_NOMEM, "staging buffer: %s", cudaGetErrorString(e));
    const size_t rb = sizeof(float2) * (size_t)p->cols2d;
    int rc = copy_h2d(p, p->stage2d_in, rb, i2, sizeof(float2) * (size_t)in_rs, rb, (size_t)p->rows2d, p->stream);
    if (rc) return host_done(p, rc, "fcb_exec (2-D, host)");
    rc = exec_2d(p, p->stage2d_in, p->cols2d, p->stage2d_in, p->cols2d, p->stream);
    if (rc) return host_done(p, rc, "fcb_exec (2-D, host)");
    rc = copy_d2h(p, o2, sizeof(float2) * (size_t)out_rs, p->stage2d_in, rb, rb, (size_t)p->rows2d, p->stream);
    return host_done(p, rc, "fcb_exec (2-D, host)");
  }
  if (where == FCB_DEVICE) return exec_device(p, i2, in_rs, o2, out_rs, rows, 0, p->stream);
  return exec_host(p, i2, in_rs, o2, out_rs, rows, sync);
}

extern "C" {

int fcb_set_stream(fcb_plan p, void *stream)
{
  if (!p) return set_error(FCB_ERR_INVALID, "plan is NULL");
  p->stream = (cudaStream_t)stream;  // NULL is the CUDA default stream, as in CUDA
  return FCB_OK;
}

int fcb_sync(fcb_plan p)
{
  if (!p) return set_error(FCB_ERR_INVALID, "plan is NULL");
  DeviceGuard g(p->device);
  return host_done(p, FCB_OK, "fcb_sync");
}

int fcb_destroy(fcb_plan p)
{
  plan_free(p);
  return FCB_OK;
}

int fcb_plan_info(fcb_plan p, long long *n, int *cluster_ctas, int *rows_per_cta, int *smem_bytes,
                  int *threads)
{
  if (!p) return set_error(FCB_ERR_INVALID, "plan is NULL");
  if (n) *n = p->n;
  // Bluestein and real-input plans report the kernel of their power-of-two work rows
  fcb_plan q = p->cplx ? p->cplx : p;
  const KernelInfo *k = q->k ? q->k : q->inner[0] ? q->inner[0]->k : q->inner[1] ? q->inner[1]->k : nullptr;
  if (threads) *threads = k ? k->threads : 0;
  if (cluster_ctas) *cluster_ctas = k ? k->cluster : 1;
  if (rows_per_cta) *rows_per_cta = k ? k->rows_per_cta : 1;
  if (smem_bytes) *smem_bytes = k ? k->smem : 0;
  return FCB_OK;
}

int fcb_supported_real_length(long long n)
{
  if (n < 1) return 0;
  return n % 2 == 0 ? fcb_supported_length(n / 2) : fcb_supported_length(n);
}

int fcb_plan_fftm_real(long long n, long long rows_max, int exponent, float scale, fcb_plan *plan)
{
  if (!plan) return set_error(FCB_ERR_INVALID, "plan pointer is NULL");
  *plan = nullptr;
  if (!fcb_supported_real_length(n))
    return set_error(FCB_ERR_UNSUPPORTED, "real row length %lld unsupported: even with n/2 " FCB_LENGTH_RULE
                     ", or odd up to 32767", n);
  if (rows_max < 0) return set_error(FCB_ERR_INVALID, "rows_max < 0");
  if (exponent != FCB_FORWARD && exponent != FCB_INVERSE) return set_error(FCB_ERR_INVALID, "exponent must be -1 or +1");
  int rc = check_device();
  if (rc) return rc;
  fcb_plan p = new (std::nothrow) fcb_plan_s;
  if (!p) return set_error(FCB_ERR_NOMEM, "plan allocation");
  cudaGetDevice(&p->device);
  p->real = exponent == FCB_FORWARD ? 1 : 2;
  p->rn = n;
  p->n = n;
  p->logn = -1;
  p->mode = exponent == FCB_FORWARD ? kFwd : kInv;
  p->rows_max = rows_max;
  p->scale = scale;
  cudaError_t e = cudaStreamCreateWithFlags(&p->own_stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) rc = cuda_error(e, "cudaStreamCreate");
  p->stream = p->own_stream;
  const bool even = n % 2 == 0;
  if (!rc)
    rc = fcb_plan_fftm(even ? n / 2 : n, std::max<long long>(rows_max, 1), exponent,
                       (even && p->real == 1) ? 1.f : scale, &p->cplx);
  if (!rc && even) rc = real_twiddles(n, n / 2 + 1, &p->rtw, p->stream);
  if (!rc && (e = cudaStreamSynchronize(p->stream)) != cudaSuccess) rc = cuda_error(e, "real-FFT tables");
  if (rc) { plan_free(p); return rc; }
  *plan = p;
  return FCB_OK;
}

int fcb_exec_r2c(fcb_plan p, const float *in, long long in_rs, fcb_cf32 *out, long long out_rs, long long rows,
                 int where)
{
  return exec_real(p, 1, in, in_rs, out, out_rs, rows, where);
}

int fcb_exec_c2r(fcb_plan p, const fcb_cf32 *in, long long in_rs, float *out, long long out_rs, long long rows,
                 int where)
{
  return exec_real(p, 2, in, in_rs, out, out_rs, rows, where);
}

int fcb_plan_fft2d(long long rows, long long cols, int exponent, float scale, fcb_plan *plan)
{
  if (!plan) return set_error(FCB_ERR_INVALID, "plan pointer is NULL");
  *plan = nullptr;
  if (exponent != FCB_FORWARD && exponent != FCB_INVERSE) return set_error(FCB_ERR_INVALID, "exponent must be -1 or +1");
  const int lr = log2_exact(rows), lc = log2_exact(cols);
  if (lr < 6 || lr > 14 || lc < 6 || lc > 14)
  {
    // other sizes: two row plans and two transposes (four passes)
    if (rows < 1 || cols < 1 || !fcb_supported_length(rows) || !fcb_supported_length(cols))
      return set_error(FCB_ERR_UNSUPPORTED, "2-D FFT dimensions %lld x %lld: each must be " FCB_LENGTH_RULE, rows,
                       cols);
    int rc = check_device();
    if (rc) return rc;
    fcb_plan p = new (std::nothrow) fcb_plan_s;
    if (!p) return set_error(FCB_ERR_NOMEM, "plan allocation");
    cudaGetDevice(&p->device);
    p->n = cols;
    p->logn = -1;
    p->mode = exponent == FCB_FORWARD ? kFwd : kInv;
    p->rows_max = rows;
    p->scale = scale;
    p->is2d = p->general2d = true;
    p->rows2d = rows;
    p->cols2d = cols;
    cudaError_t e = cudaStreamCreateWithFlags(&p->own_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) rc = cuda_error(e, "cudaStreamCreate");
    p->stream = p->own_stream;
    if (!rc) rc = fcb_plan_fftm(cols, rows, exponent, 1.f, &p->sub2d[0]);
    if (!rc) rc = fcb_plan_fftm(rows, cols, exponent, scale, &p->sub2d[1]);
    const size_t bytes = sizeof(float2) * (size_t)(rows * cols);
    if (!rc && (e = cudaMalloc(&p->scratch, bytes)) != cudaSuccess)
      rc = set_error(FCB_ERR_NOMEM, "2-D scratch: %s", cudaGetErrorString(e));
    if (!rc && (e = cudaMalloc(&p->scratch2, bytes)) != cudaSuccess)
      rc = set_error(FCB_ERR_NOMEM, "2-D scratch: %s", cudaGetErrorString(e));
    if (rc) { plan_free(p); return rc; }
    *plan = p;
    return FCB_OK;
  }
  fcb_plan p = new (std::nothrow) fcb_plan_s;
  if (!p) return set_error(FCB_ERR_NOMEM, "plan allocation");
  const int mode = exponent == FCB_FORWARD ? kFwd : kInv;
  p->scale = scale;
  p->is2d = true;
  p->rows2d = rows;
  p->cols2d = cols;
  int rc = plan_common(p, cols, rows, mode);
  if (!rc)
  {
    // 512-thread CTAs hold 4 rows of 4096 (or more of shorter rows), so each
    // transposed store writes whole 32-byte sectors
    const int built_ept = p->k->ept;
    p->k = kernel_variant(lc, mode, 512);
    p->kc = kernel_variant(lr, mode, 512);
    rc = prepare_kernel(p->k);
    if (!rc) rc = prepare_kernel(p->kc);
    if (!rc && built_ept != p->k->ept)
    {
      // pass 1 runs another variant than the tuned one the tables were built for
      cudaFree(p->tw);
      p->tw = nullptr;
      rc = build_twiddles(lc, p->k->ept, &p->tw, p->stream);
    }
    if (!rc) rc = build_twiddles(lr, p->kc->ept, &p->twc, p->stream);  // pass-2 table (length rows)
  }
  if (!rc)
  {
    cudaError_t e = cudaMalloc(&p->scratch, sizeof(float2) * (size_t)(rows * cols));
    if (e != cudaSuccess) rc = set_error(FCB_ERR_NOMEM, "2-D scratch: %s", cudaGetErrorString(e));
  }
  if (!rc)
  {
    cudaError_t e = cudaStreamSynchronize(p->stream);
    if (e != cudaSuccess) rc = cuda_error(e, "plan tables");
  }
  if (rc) { plan_free(p); return rc; }
  *plan = p;
  return FCB_OK;
}

int fcb_tune_set(long long n, int kind, int threads)
{
  int l = log2_exact(n);
  if (l < 1 || l > kMaxLogN) return set_error(FCB_ERR_UNSUPPORTED, "length %lld has no tunable kernel", n);
  return set_variant(l, kind, threads);
}

int fcb_tune_get(long long n, int kind)
{
  int l = log2_exact(n);
  if (l < 1 || l > kMaxLogN || kind < 0 || kind > 2) return 0;
  return get_variant(l, kind);
}

int fcb_vmmul_rows(const fcb_cf32 *v, const fcb_cf32 *m, long long m_rs, fcb_cf32 *out, long long out_rs,
                   long long rows, long long cols, void *stream)
{
  if (rows < 0 || cols < 0) return set_error(FCB_ERR_INVALID, "negative size");
  if (rows == 0 || cols == 0) return FCB_OK;
  if (!v || !m || !out) return set_error(FCB_ERR_INVALID, "NULL pointer");
  if (m_rs < cols || out_rs < cols) return set_error(FCB_ERR_INVALID, "row stride smaller than cols");
  return launch_vmmul(reinterpret_cast<const float2 *>(v), reinterpret_cast<const float2 *>(m), m_rs,
                      reinterpret_cast<float2 *>(out), out_rs, rows, cols, (cudaStream_t)stream);
}

int fcb_replica_spectrum(const fcb_cf32 *replica_dev, long long n, int matched, fcb_cf32 *spectrum_dev)
{
  if (!fcb_supported_length(n)) return set_error(FCB_ERR_UNSUPPORTED, "length %lld unsupported: " FCB_LENGTH_RULE, n);
  if (!replica_dev || !spectrum_dev) return set_error(FCB_ERR_INVALID, "NULL pointer");
  int rc = check_device();
  if (rc) return rc;
  rc = replica_spectrum_dev(reinterpret_cast<const float2 *>(replica_dev), n, matched,
                            reinterpret_cast<float2 *>(spectrum_dev), 0);
  if (rc) return rc;
  cudaError_t e = cudaStreamSynchronize(0);
  if (e != cudaSuccess) return cuda_error(e, "replica spectrum");
  return FCB_OK;
}

}  // extern "C"
