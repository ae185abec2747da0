// Internal declarations shared by the fcb200 translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>

namespace fcb {

struct RowArgs;

// Runtime copy of the compile-time schedule (see Sched<> in fcb_engine.cuh).
struct SchedRT
{
  int logn, n, ns, r1, d, half;
  int ept, rb, lrb;    // samples per thread, later-stage radix and its log2
  long long tw2_size;  // float2 entries of the stage >= 2 twiddle tables
};
SchedRT sched_rt(int logn, int ept = 32);

struct KernelInfo
{
  const void *fn = nullptr;
  int threads = 256;     // threads per CTA
  int cluster = 1;       // CTAs per row (thread-block cluster size)
  int rows_per_cta = 1;  // rows per CTA when cluster == 1
  int smem = 0;          // dynamic shared memory per CTA, bytes
  long long tw_bytes = 0; // twiddle table size
  int ept = 32;          // samples per thread (the tables depend on it)
  long long resident_tiles = 0;  // CTAs (or clusters) resident at once, set by prepare_kernel
};

constexpr int kMin512 = 12;  // 512-thread variants exist for rows of 4096 samples and more
constexpr int kMin128 = 8, kMax128 = 13;  // 128-thread variants: rows of 256 .. 8192 samples
constexpr int kWideLog = 14;     // the wide variant (256 threads x 64 samples): rows of 16384 samples,
constexpr int kWideMaxLog = 15;  // and 32768 on clusters of two CTAs
// Variant ids: [0] 256, [1] 512, [2] 128 threads with 32 samples each, [3] the
// wide one.  Its public tuning value is -256.
constexpr int kVariants = 4;

const KernelInfo *kernel_info(int logn, int mode);
// Fused kernel with element-wise multipliers (kChirpconv, fcb_bluestein.cu)
// for work rows of 2^logn samples, in the same variant as `like` (whose
// tables it reads).
const KernelInfo *chirp_kernel(int logn, const KernelInfo *like);
int set_variant(int logn, int mode, int threads);
const KernelInfo *kernel_variant(int logn, int mode, int threads);
int get_variant(int logn, int mode);
int prepare_kernel(const KernelInfo *k);
int launch_rows(const KernelInfo *k, long long rows, const RowArgs &args, cudaStream_t st);

int build_twiddles(int logn, int ept, float4 **out, cudaStream_t st);
int build_replica_table(int logn, int ept, const float2 *spec_dev, long long spec_rs, long long rows,
                        float4 *rep_dev, cudaStream_t st);
int replica_spectrum_dev(const float2 *rep_dev, long long n, int matched, float2 *spec_dev,
                         cudaStream_t st);
int launch_vmmul(const float2 *v, const float2 *m, long long m_rs, float2 *out, long long out_rs,
                 long long rows, long long cols, cudaStream_t st);
// out[c][r] = in[r][c], rows x cols (strides in complex elements)
int launch_transpose(const float2 *in, long long in_rs, float2 *out, long long out_rs, long long rows,
                     long long cols, cudaStream_t st);
int launch_scale_rows(const float2 *in, long long in_rs, float2 *out, long long out_rs, long long rows,
                      const float4 *rep, long long rep_rs, float scale, cudaStream_t st);

// Bluestein chirp-z pieces (fcb_bluestein.cu) for rows of non-power-of-two
// length N, computed through power-of-two work rows of M >= 2N - 1 samples.
int bluestein_tables(long long N, long long M, int sign, float2 **chirp, float2 **spectrum, cudaStream_t st);
int scale_copy(const float2 *in, float2 *out, long long total, float s, cudaStream_t st);

// Real-input row FFTs (fcb_real.cu).
int real_twiddles(long long n, long long count, float2 **out, cudaStream_t st);
int r2c_post(float2 *y, long long rs, long long m, long long rows, const float2 *w, float scale, cudaStream_t st);
int c2r_pre(const float2 *x, long long x_rs, float2 *z, long long z_rs, long long m, long long rows,
            const float2 *w, cudaStream_t st);
int real_expand(const float *x, long long x_rs, float2 *z, long long n, long long rows, cudaStream_t st);
int herm_expand(const float2 *x, long long x_rs, float2 *z, long long n, long long rows, cudaStream_t st);
int take_real(const float2 *z, long long n, float *out, long long out_rs, long long rows, cudaStream_t st);

// Host-side copies (fcb_hostcopy.cu): rows x row_bytes between host buffers
// with the given pitches, split over the copy threads; and whether a host
// range is pageable (not pinned or registered with CUDA).
void host_copy_rows(void *dst, size_t dst_pitch, const void *src, size_t src_pitch, size_t row_bytes, size_t rows);
bool host_pageable(const void *ptr, size_t bytes);

int set_error(int code, const char *fmt, ...);
const char *error_text();
int cuda_error(cudaError_t e, const char *what);

}  // namespace fcb
