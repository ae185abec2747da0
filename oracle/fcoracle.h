/* CPU oracle for the fast-convolution path.  TEST INFRASTRUCTURE ONLY: the
 * product never links or calls this; tests, the smoke check and the CPU
 * baseline leg of the benchmark use it as the checker.
 *
 * Complex data is interleaved (re, im); "c64" arrays are double pairs, "c32"
 * arrays are float pairs.  Row-major matrices, row stride in complex elements.
 * exponent: -1 forward, +1 inverse (the reference's fft_fwd / fft_inv map to
 * these in src/ovxx/signal/fft/util.hpp:41-51). */
#ifndef FCORACLE_H
#define FCORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* O(N^2) DFT of one vector, accumulating in double
 * (src/ovxx/signal/fft/dft.hpp:57-66, dft<1,complex,complex>). */
void orc_dft_c64(const double *in, long in_stride, double *out,
                 long out_stride, long n, int exponent, double scale);

/* FP64 FFT of one vector: iterative radix-2 Cooley-Tukey for powers of two,
 * the O(N^2) DFT otherwise. */
void orc_fft_c64(const double *in, double *out, long n, int exponent,
                 double scale);

/* Row-wise multiple FFT (src/ovxx/signal/fft/dft.hpp:1040-1058, dftm rows).
 * method 0: O(N^2) DFT per row; method 1: FFT per row. */
void orc_fftm_rows_c64(const double *in, long in_rs, double *out, long out_rs,
                       long rows, long cols, int exponent, double scale,
                       int method);

/* out[r][c] = v[c] * m[r][c] (src/ovxx/expr/vmmul.hpp:53-59, vmmul<0>). */
void orc_vmmul_rows_c64(const double *v, const double *m, long m_rs,
                        double *out, long out_rs, long rows, long cols);

/* Fast convolution in FP64: forward row FFT, vmmul by the replica spectrum
 * (one vector, or one row per input row when rep_rs != 0), inverse row FFT
 * scaled by 1/cols.  Inputs are complex<float>, outputs complex<double>.
 * method as in orc_fftm_rows_c64. */
void orc_fastconv_c64(const float *in, long rows, long cols, const float *rep,
                      long rep_rs, double *out, int method);

/* Same arithmetic in FP32 with the radix-2 FFT (twiddles from double); used as
 * a CPU speed baseline.  Single-threaded (threads is honoured only in an OpenMP
 * build); callers parallelise over disjoint row slices. */
void orc_fastconv_c32(const float *in, long rows, long cols, const float *rep,
                      long rep_rs, float *out, int threads);

/* Reference accuracy metric (support/test/diff.hpp:41-96): max over elements of
 * 10 log10(|a-b|^2 / (2 max(|a|^2,|b|^2))), -201 for differences below 1e-20,
 * +201 if either input holds a NaN.  a and b are c64 vectors of n elements. */
double orc_error_db(const double *a, const double *b, long n);

/* LFM chirp c[n] = exp(j pi tbp (n/len - 1/2)^2), n < len, zero-padded to n_out. */
void orc_lfm_chirp_c64(long len, double tbp, long n_out, double *out);

#ifdef __cplusplus
}
#endif
#endif
