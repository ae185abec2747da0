/* fcb200 -- B200-native fast convolution (pulse compression) for OpenVSIP.
 *
 * C ABI of the drop-in backend.  Plain pointers and sizes only; complex data is
 * interleaved complex<float> (fcb_cf32), row-major, unit stride along a row,
 * row stride in complex elements.  Every function returns FCB_OK (0) or an
 * error code; fcb_last_error() gives the calling thread's last message.
 *
 * Which reference interface each entry point replaces:
 *
 *   fcb_plan_fftm / fcb_exec      ovxx::signal::fft::fftm_backend<complex<float>,
 *                                 complex<float>, row, D> (src/ovxx/signal/fft/
 *                                 backend.hpp:696-784): constructed once per
 *                                 vsip::Fftm object with the full (rows, N) domain
 *                                 and scale (src/ovxx/fftw/fftw.cpp:904-919), then
 *                                 out_of_place / in_place per call with fewer or
 *                                 equal rows (fftw.cpp:965-1001).  The scale is
 *                                 applied inside the kernel, i.e. supports_scale()
 *                                 is true and the workspace scale pass
 *                                 (src/ovxx/signal/fft/workspace.hpp:474-478) is
 *                                 skipped.
 *   fcb_plan_fastconv / fcb_exec  the fused fast-convolution expression
 *                                 inv_fftm(vmmul<0>(replica, fwd_fftm(data)))
 *                                 (tests/fastconv.cpp:204; benchmarks/fastconv.cpp
 *                                 :100-106 phased form) that the reference routes
 *                                 through the empty be::fc_expr slot
 *                                 (src/ovxx/dispatcher/tags.hpp:33-34) to
 *                                 be::rbo_expr (src/ovxx/assign/rbo.hpp:18-32).
 *                                 A replica MATRIX (one spectrum per row) covers
 *                                 inv_fftm(W * fwd_fftm(data))
 *                                 (tests/fastconv.cpp:213-246).
 *   fcb_vmmul_rows                vmmul<0>(v, m) (src/vsip/impl/vmmul.hpp:114-128,
 *                                 src/ovxx/expr/vmmul.hpp:53-59).
 *   fcb_replica_spectrum          the replica transform t2f(weights)
 *                                 (tests/fastconv.cpp:21-26), done in FP64 on the
 *                                 GPU.
 *   fcb_batch_*                   no single reference counterpart: many
 *                                 Fftm+vmmul+Fftm jobs of uneven shapes in one
 *                                 persistent launch.
 *
 * Lengths: Fftm, fast-convolution and replica plans take any length from 1 to
 * 32768 (lengths that are not powers of two run Bluestein's algorithm) and
 * powers of two up to 65536; the batch entry points take powers of two from
 * 256 to 32768; the 2-D plans take any supported length per dimension.
 */
#ifndef FCB200_H
#define FCB200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define FCB_API __attribute__((visibility("default")))
#else
#define FCB_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef struct { float re, im; } fcb_cf32;
typedef struct fcb_plan_s *fcb_plan;

enum fcb_status
{
  FCB_OK = 0,
  FCB_ERR_INVALID = 1,      /* bad argument (size, stride, pointer) */
  FCB_ERR_UNSUPPORTED = 2,  /* valid request this backend does not implement */
  FCB_ERR_CUDA = 3,         /* CUDA runtime or launch failure */
  FCB_ERR_NOMEM = 4,        /* device or host allocation failed */
  FCB_ERR_TIMEOUT = 5,      /* a bounded wait gave up */
  FCB_ERR_NODEVICE = 6      /* no usable sm_100 device */
};

/* Where a buffer lives. */
enum fcb_where { FCB_HOST = 0, FCB_DEVICE = 1 };

/* Transform direction: the reference's fft_fwd (-2) / fft_inv (-1) tags map to
 * exponents -1 / +1 (src/ovxx/signal/fft/util.hpp:41-51). */
enum fcb_exponent { FCB_FORWARD = -1, FCB_INVERSE = +1 };

/* How a replica is given. */
enum fcb_replica_kind
{
  FCB_REPLICA_SPECTRUM = 0,      /* already in the frequency domain (vmmul vector) */
  FCB_REPLICA_TIME = 1,          /* time domain: spectrum = FFT(replica), FP64 on GPU */
  FCB_REPLICA_TIME_MATCHED = 2   /* time domain: spectrum = conj(FFT(replica)) */
};

/* Library status. */
FCB_API const char *fcb_last_error(void);
FCB_API const char *fcb_version(void);
/* Select the CUDA device for subsequent plans of the calling thread. */
FCB_API int fcb_init(int device);
/* 1 if n is a supported row length for Fftm and fast-convolution plans: any
 * length in [1, 32768], or a power of two up to 65536.  Powers of two run as
 * one fused pass; other lengths by Bluestein's chirp-z algorithm: the fused
 * kernel runs on work rows of the next power of two >= 2n - 1 samples and
 * applies the chirps, the zero padding and the truncation to n samples on its
 * own loads and stores (one pass per transform).  The reference's FFTW
 * backend plans any length (src/ovxx/fftw/fftw.cpp:39-116). */
FCB_API int fcb_supported_length(long long n);

/* Row-wise multiple FFT plan: n samples per row, up to rows_max rows per call,
 * exponent FCB_FORWARD or FCB_INVERSE, output multiplied by scale.  Replaces
 * fftm_backend<complex<float>, complex<float>, 0, D> (src/ovxx/signal/fft/
 * backend.hpp:696-784; FFTW plan src/ovxx/fftw/fftw.cpp:904-1001). */
FCB_API int fcb_plan_fftm(long long n, long long rows_max, int exponent, float scale,
                  fcb_plan *plan);

/* Real-input row FFTs.  exponent FCB_FORWARD: real rows of n samples ->
 * complex rows of n/2 + 1 (the non-negative frequencies), run with
 * fcb_exec_r2c; FCB_INVERSE: complex rows of n/2 + 1 -> real rows of n,
 * unnormalised like FFTW's c2r (imaginary parts of bins 0 and n/2 ignored),
 * run with fcb_exec_c2r.  Output times scale.  Replaces
 * fftm_backend<float, complex<float>, A, fft_fwd> and
 * fftm_backend<complex<float>, float, A, fft_inv> (src/ovxx/signal/fft/
 * backend.hpp:600-694; FFTW rows src/ovxx/fftw/fftw.cpp:778-903).  Even n:
 * one length-n/2 complex row FFT plus a split (forward) or merge (inverse)
 * pass; odd n: the length-n complex row FFT. */
FCB_API int fcb_supported_real_length(long long n);
FCB_API int fcb_plan_fftm_real(long long n, long long rows_max, int exponent, float scale,
                               fcb_plan *plan);
/* in: rows of n floats (stride in_rs floats); out: rows of n/2 + 1 complex
 * (stride out_rs complex).  in and out must not overlap.  where as fcb_exec. */
FCB_API int fcb_exec_r2c(fcb_plan plan, const float *in, long long in_rs, fcb_cf32 *out,
                         long long out_rs, long long rows, int where);
/* in: rows of n/2 + 1 complex (stride in_rs complex); out: rows of n floats
 * (stride out_rs floats).  in and out must not overlap. */
FCB_API int fcb_exec_c2r(fcb_plan plan, const fcb_cf32 *in, long long in_rs, float *out,
                         long long out_rs, long long rows, int where);

/* 2-D FFT plan over a rows x cols matrix, output times scale; fcb_exec then
 * takes rows == the plan's rows.  Replaces fft_backend<2, complex<float>,
 * complex<float>, S> (src/ovxx/signal/fft/backend.hpp:294-375; FFTW 2-D plan
 * src/ovxx/fftw/fftw.cpp:436-511), used by vsip::Fft<const_Matrix, ...>.
 * Both dimensions powers of two in [64, 16384]: two passes, each a row
 * transform that stores its result transposed (one rows x cols scratch
 * matrix).  Other dimensions (each any length fcb_supported_length accepts):
 * a row pass, a transpose, a column pass and a transpose back (two scratch
 * matrices). */
FCB_API int fcb_plan_fft2d(long long rows, long long cols, int exponent, float scale,
                           fcb_plan *plan);

/* Fused fast-convolution plan: y = IFFT(R .* FFT(x)) / n per row.
 * replica: replica_rows rows (1 = one vector shared by all rows, or one per
 * data row) of n samples at row stride replica_rs, kind fcb_replica_kind,
 * located at `where`.  The plan keeps the spectrum resident on the device. */
FCB_API int fcb_plan_fastconv(long long n, long long rows_max, const fcb_cf32 *replica,
                      long long replica_rows, long long replica_rs,
                      int replica_kind, int where, fcb_plan *plan);

/* Execute a plan on `rows` rows (rows <= rows_max).  in and out may alias
 * (in-place).  where = FCB_DEVICE: both pointers are device pointers and the
 * call is asynchronous on the plan's stream.  where = FCB_HOST: host pointers;
 * the call copies through the device and returns when out is written.  Pinned
 * (page-locked) host buffers move directly; a pageable buffer is copied chunk
 * by chunk through pinned buffers shared by all plans of the process (at most
 * 2 x FCB200_STAGES x FCB200_STAGE_MB, 128 MB by default; one such call at a
 * time) by a pool of host threads (FCB200_COPY_THREADS, default three quarters
 * of the host's threads, at most 16), which measured 3-4x faster than handing
 * pageable memory to the CUDA runtime; if no pinned memory can be had, the
 * runtime copies it. */
FCB_API int fcb_exec(fcb_plan plan, const fcb_cf32 *in, long long in_rs, fcb_cf32 *out,
             long long out_rs, long long rows, int where);

/* fcb_exec without waiting: with where = FCB_HOST it queues the copies in,
 * the kernels and the copies out of `rows` rows (chunked through the plan's
 * device staging buffers) and returns; the caller keeps both host buffers
 * untouched until fcb_sync returns.  Calls queued back to back on one plan run
 * in order and overlap: the next call's copies in run while the previous
 * call's last copies out drain (a streaming caller keeps the PCIe link busy in
 * both directions across calls).  A queued call copies in chunks of twice the
 * size fcb_exec uses, without fcb_exec's smaller chunks at both ends of the
 * call (those shorten one call's fill and drain, which a stream of calls
 * overlaps anyway).  Host buffers should be pinned: with a pageable buffer the
 * call is fcb_exec (it returns when out is written).   2-D plans
 * run host calls synchronously.  No reference counterpart (the reference's
 * Fftm calls are synchronous).  With where = FCB_DEVICE it is fcb_exec. */
FCB_API int fcb_exec_async(fcb_plan plan, const fcb_cf32 *in, long long in_rs, fcb_cf32 *out,
                           long long out_rs, long long rows, int where);

/* Queue the plan's device work on a caller-owned cudaStream_t (NULL is the
 * CUDA default stream).  A new plan uses a private non-blocking stream. */
FCB_API int fcb_set_stream(fcb_plan plan, void *stream);
/* Wait for all work queued on the plan's stream and, after host calls, its
 * copy streams. */
FCB_API int fcb_sync(fcb_plan plan);
FCB_API int fcb_destroy(fcb_plan plan);

/* Plan introspection: the kernel configuration chosen for this plan. */
FCB_API int fcb_plan_info(fcb_plan plan, long long *n, int *cluster_ctas,
                  int *rows_per_cta, int *smem_bytes, int *threads);

/* Kernel variant for row length n and kind (FCB_KIND_*): CTAs of 128, 256 or
 * 512 threads with 32 samples per thread (128: rows of 256 .. 8192 samples;
 * 512: 4096 and more), or -256: CTAs of 256 threads with 64 samples per thread
 * (rows of 16384 samples; one stage fewer).  Set by the autotuner; applies to
 * plans created afterwards.  No reference counterpart (FFTW's planning rigor,
 * src/ovxx/fftw/fft.cpp:44-52, is the closest analogue). */
enum fcb_kind { FCB_KIND_FORWARD = 0, FCB_KIND_INVERSE = 1, FCB_KIND_FASTCONV = 2 };
FCB_API int fcb_tune_set(long long n, int kind, int threads);
/* Current variant (128, 256, 512 or -256) for n and kind, 0 if n has none. */
FCB_API int fcb_tune_get(long long n, int kind);

/* out[r][c] = v[c] * m[r][c] on the device (asynchronous on `stream`). */
FCB_API int fcb_vmmul_rows(const fcb_cf32 *v, const fcb_cf32 *m, long long m_rs,
                   fcb_cf32 *out, long long out_rs, long long rows,
                   long long cols, void *stream);

/* Replica spectrum in FP64 on the GPU, rounded to complex<float>:
 * spectrum = FFT(replica) or conj(FFT(replica)) (matched), n a supported
 * length (radix-2 FFT for powers of two, a direct DFT otherwise).
 * Device pointers; synchronous. */
FCB_API int fcb_replica_spectrum(const fcb_cf32 *replica_dev, long long n, int matched,
                         fcb_cf32 *spectrum_dev);

/* The same replica spectrum for callers that must not allocate device memory
 * while running (for example a real-time pulse-compression loop with a fixed
 * memory budget, or a process whose device memory is reserved up front).  No
 * counterpart in the reference.  Its FP64 work buffers are a 2 MiB array built
 * into the library (held on every GPU that loads it until exit) instead of a
 * per-call allocation, so n is limited to 65536; larger n is rejected with
 * FCB_ERR_INVALID.  Unlike fcb_replica_spectrum it runs the radix-2 FP64 FFT
 * only: n must be a power of two, other lengths are rejected with
 * FCB_ERR_UNSUPPORTED.  Asynchronous on `stream` (NULL: the default stream); it
 * calls no allocator.  The first call on a device looks up the array's device
 * address (cudaGetSymbolAddress), so make that first call before any stream
 * capture; the address is kept per device for its primary context (the CUDA
 * runtime's).  All calls share the array and it keeps the last call's
 * contents: calls that overlap on the GPU (different streams or threads) race,
 * so serialise them, e.g. on one stream. */
FCB_API int fcb_replica_spectrum_noalloc(const fcb_cf32 *replica_dev, long long n, int matched,
                                         fcb_cf32 *spectrum_dev, void *stream);

/* ---- Batched fast convolution ------------------------------------------
 * Many pulse-compression jobs of uneven shapes (rows x samples, each with its
 * own replica) run in ONE persistent kernel launch, replayed from a CUDA graph
 * (the graph resets the kernel's work counter and launches it).  No single
 * reference counterpart: the reference runs each job's Fftm -> vmmul -> Fftm
 * (benchmarks/fastconv.cpp:100-106) separately.  Device pointers only; row
 * lengths are powers of two from 256 to 32768. */
typedef struct fcb_batch_s *fcb_batch;
typedef struct
{
  const fcb_cf32 *in;   /* device, pulses x n, row stride in_rs */
  long long in_rs;
  fcb_cf32 *out;        /* device, may equal in (in place) */
  long long out_rs;
  long long pulses;     /* rows */
  long long n;          /* samples per row */
  int replica;          /* id from fcb_batch_add_replica (its length must be n) */
} fcb_job;

/* threads: 256 or 512 (CTAs of 32 samples per thread; clusters of 4 x 256 or
 * 2 x 512 threads share a 32768-sample row), -256 (the wide kernel: one
 * 256-thread CTA per SM; rows of 16384 and 32768 samples run 64 samples per
 * thread, 32768 on clusters of two CTAs), or 0 for the default (512). */
FCB_API int fcb_batch_create(int threads, fcb_batch *batch);
/* Keep a replica resident on the device (spectrum built in FP64 for the time
 * kinds); returns its id. */
FCB_API int fcb_batch_add_replica(fcb_batch batch, const fcb_cf32 *replica, long long n,
                                  int replica_kind, int where, int *id);
/* Define the job list (copied).  order bit 0: 0 = longest rows first (default
 * load balance), 1 = as given.  order bit 1 (value 2): launch directly instead
 * of capturing a CUDA graph -- for job sets that change with every run, as in
 * a serving loop; the job table is then copied on the batch's stream. */
FCB_API int fcb_batch_set_jobs(fcb_batch batch, const fcb_job *jobs, int njobs, int order);
/* Run all jobs once: one graph launch on the batch's stream (asynchronous). */
FCB_API int fcb_batch_run(fcb_batch batch);
FCB_API int fcb_batch_set_stream(fcb_batch batch, void *stream);
FCB_API int fcb_batch_sync(fcb_batch batch);
FCB_API int fcb_batch_info(fcb_batch batch, long long *units, long long *samples, int *grid,
                           int *threads);
FCB_API int fcb_batch_destroy(fcb_batch batch);

#ifdef __cplusplus
}
#endif
#endif
