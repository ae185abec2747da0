// OpenVSIP plugin that routes the fast-convolution path to the B200 backend
// (libfcb200.so, C ABI in include/fcb200.h).  Include it (or pass it with
// -include) before any code that constructs a vsip::Fftm; link -lfcb200.
// No reference header is modified: the plugin fills dispatch slots the
// reference already reserves.
//
//  1. be::user for op::fftm<complex<float>, complex<float>, row | col, D, R, N>
//     and for the real-input forms op::fftm<float, complex<float>, A, fft_fwd>
//     and op::fftm<complex<float>, float, A, fft_inv>.  be::user is the first
//     entry of List<op::fftm> (src/ovxx/signal/fft.hpp:57-64), so every
//     complex<float> / float vsip::Fftm whose length the backend supports (any
//     length up to 32768, powers of two up to 65536; twice that for the real
//     forms) is built on the B200.  The backend objects follow the fftm_backend
//     contract (src/ovxx/signal/fft/backend.hpp:600-784): they ask the DDA
//     layer for dense, interleaved data with unit stride along the transform
//     axis (anything else, split storage included, is copied by dda::Rt_data
//     before the call) and apply the scale themselves (supports_scale() ==
//     true), so the workspace's separate scale pass (src/ovxx/signal/fft/
//     workspace.hpp:474-478) is skipped.  Lengths the backend does not support
//     fail rt_valid() and the dispatcher moves on to the next backend in the
//     list, exactly as for any other plugin.
//
//  2. be::fc_expr for op::assign<2>, the "fused fastconv" slot that the
//     reference lists (src/ovxx/assign_fwd.hpp:58, src/ovxx/dispatcher/
//     tags.hpp:33-34) but never implements.  It matches
//         out = inv_fftm(vmmul<0>(weights, fwd_fftm(in)))     (vector form)
//         out = inv_fftm(W * fwd_fftm(in)), inv_fftm(fwd_fftm(in) * W)
//                                                              (matrix form)
//     when both Fftm objects are B200 ones, and runs the whole expression as
//     one fused kernel pass (one HBM read and write per sample) instead of
//     falling through to be::rbo_expr (src/ovxx/assign/rbo.hpp:18-32), which
//     evaluates the forward FFT into a temporary, copies the vmmul element by
//     element and runs the inverse and the scale pass.
//
// Errors: construction throws (std::runtime_error, or std::bad_alloc when the
// device is out of memory) like the reference's planners
// (src/ovxx/fftw/fftw.cpp:97-102).  A failure inside a VSIP_NOTHROW call is
// raised through OVXX_DO_THROW, as the base-class backends do for
// unimplemented paths.  A missing GPU is an error at construction, not a
// silent fall back.
//
//  3. be::user for op::fft<2, complex<float>, complex<float>, S> (the 2-D
//     vsip::Fft<const_Matrix, ...>; backend contract src/ovxx/signal/fft/
//     backend.hpp:294-375), through fcb_plan_fft2d, and for op::fft<1, ...>
//     (the 1-D vsip::Fft<const_Vector, ...> that builds replica spectra;
//     backend.hpp:132-205), through a one-row fcb_plan_fftm.
//
// Environment: FCB200_DEVICE selects the CUDA device (default 0);
// FCB200_TRACE=1 prints one line per backend constructed and per fused call.
#ifndef OVXX_FCB200_HPP
#define OVXX_FCB200_HPP

#include <vsip/support.hpp>
#include <vsip/domain.hpp>
#include <vsip/vector.hpp>
#include <vsip/matrix.hpp>
#include <vsip/signal.hpp>
#include <vsip/math.hpp>
#include <vsip/dda.hpp>
#include <ovxx/signal/fft/backend.hpp>

#include <fcb200.h>

#include <algorithm>
#include <atomic>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <new>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

namespace ovxx
{
namespace fcb200
{
typedef std::complex<float> ctype;

inline bool trace()
{
  static bool const t = std::getenv("FCB200_TRACE") != 0;
  return t;
}

inline void check(int rc)
{
  if (rc == FCB_OK) return;
  std::string msg = std::string("fcb200: ") + fcb_last_error();
  if (rc == FCB_ERR_NOMEM) OVXX_DO_THROW(std::bad_alloc());
  OVXX_DO_THROW(std::runtime_error(msg));
}

// True when the rows x cols values at a (row stride a_rs) equal those at b
// (row stride b_rs).  Large matrices are compared in row ranges on several
// threads: a 1024 x 16384 weight matrix is 128 MB on each side, which one
// thread reads in about as long as the fused call takes.
template <typename T>
bool equal_rows(T const *a, stride_type a_rs, T const *b, stride_type b_rs, length_type rows, length_type cols)
{
  size_t const rb = sizeof(T) * cols;
  unsigned nt = std::min(8u, std::max(1u, std::thread::hardware_concurrency() / 2));
  if ((size_t)rows * rb < (size_t(8) << 20) || rows < nt) nt = 1;
  std::atomic<bool> differ(false);
  auto part = [&](unsigned k) {
    length_type const r0 = rows * k / nt, r1 = rows * (k + 1) / nt;
    for (length_type r = r0; r < r1 && !differ.load(std::memory_order_relaxed); ++r)
      if (std::memcmp(a + r * a_rs, b + r * b_rs, rb) != 0) differ.store(true);
  };
  std::vector<std::thread> ts;
  unsigned started = 1;
  try
  {
    for (; started < nt; ++started) ts.emplace_back(part, started);
  }
  catch (...)
  {
  }  // no thread to be had: this one takes the remaining ranges
  for (unsigned k = started; k < nt; ++k) part(k);
  part(0);
  for (auto &t : ts) t.join();
  return !differ.load();
}

// Select the device once per thread (reference library init is per thread,
// src/ovxx/library.cpp:36-48).
inline void ensure_device()
{
  static thread_local bool done = false;
  if (done) return;
  char const *env = std::getenv("FCB200_DEVICE");
  check(fcb_init(env ? std::atoi(env) : 0));
  done = true;
}

/// fftm_backend for row-wise complex<float> multiple FFTs on the B200.
template <int D>
class fftm : public signal::fft::fftm_backend<ctype, ctype, 0, D>
{
public:
  fftm(Domain<2> const &dom, float scale)
    : rows_(dom[0].size()), cols_(dom[1].size()), scale_(scale), plan_(0), fused_(0), fused_scale_(0.f)
  {
    ensure_device();
    check(fcb_plan_fftm((long long)cols_, (long long)rows_, D == fft_fwd ? FCB_FORWARD : FCB_INVERSE,
                        scale, &plan_));
    if (trace())
      std::fprintf(stderr, "[fcb200] Fftm<%s> %lu x %lu scale %g on the B200\n",
                   D == fft_fwd ? "fwd" : "inv", (unsigned long)rows_, (unsigned long)cols_, (double)scale);
  }
  ~fftm()
  {
    if (fused_) fcb_destroy(fused_);
    if (plan_) fcb_destroy(plan_);
  }
  virtual char const *name() { return "fcb200::fftm"; }
  virtual bool supports_scale() { return true; }
  virtual void query_layout(Rt_layout<2> &inout)
  {
    inout.packing = dense;
    inout.order = tuple<0, 1, 2>();
    inout.storage_format = array;
  }
  virtual void query_layout(Rt_layout<2> &in, Rt_layout<2> &out)
  {
    query_layout(in);
    out = in;
  }
  virtual bool requires_copy(Rt_layout<2> &) { return false; }
  virtual void in_place(ctype *inout, stride_type r, stride_type c, length_type rows, length_type cols)
  {
    run(inout, r, c, inout, r, c, rows, cols);
  }
  virtual void out_of_place(ctype *in, stride_type ir, stride_type ic, ctype *out, stride_type o_r,
                            stride_type oc, length_type rows, length_type cols)
  {
    run(in, ir, ic, out, o_r, oc, rows, cols);
  }

  float scale() const { return scale_; }
  length_type rows() const { return rows_; }
  length_type cols() const { return cols_; }

  /// Fused plan for inv(weights .* fwd(x)) * s, cached while the weights
  /// (already multiplied by s * N) stay the same.  weights: wrows x cols.
  fcb_plan fused(ctype const *w, stride_type w_rs, length_type wrows, float s, length_type rows_max)
  {
    size_t const n = (size_t)(wrows * cols_);
    bool const same = fused_ && fused_rows_ == wrows && fused_scale_ == s && fused_w_.size() == n &&
                      equal_rows(fused_w_.data(), (stride_type)cols_, w, w_rs, wrows, cols_);
    if (same) return fused_;
    if (fused_) fcb_destroy(fused_);
    fused_ = 0;
    fused_w_.resize(n);
    std::vector<ctype> scaled(n);
    for (length_type r = 0; r < wrows; ++r)
      for (length_type c = 0; c < cols_; ++c)
      {
        fused_w_[r * cols_ + c] = w[r * w_rs + c];
        scaled[r * cols_ + c] = w[r * w_rs + c] * (s * (float)cols_);
      }
    check(fcb_plan_fastconv((long long)cols_, (long long)rows_max,
                            reinterpret_cast<fcb_cf32 const *>(scaled.data()), (long long)wrows,
                            (long long)cols_, FCB_REPLICA_SPECTRUM, FCB_HOST, &fused_));
    fused_rows_ = wrows;
    fused_scale_ = s;
    return fused_;
  }

private:
  void run(ctype *in, stride_type ir, stride_type ic, ctype *out, stride_type o_r, stride_type oc,
           length_type rows, length_type cols)
  {
    OVXX_PRECONDITION(ic == 1 && oc == 1 && cols == cols_);
    if (rows == 0) return;
    check(fcb_exec(plan_, reinterpret_cast<fcb_cf32 const *>(in), rows > 1 ? ir : cols,
                   reinterpret_cast<fcb_cf32 *>(out), rows > 1 ? o_r : cols, (long long)rows, FCB_HOST));
  }

  length_type rows_, cols_;
  float scale_;
  fcb_plan plan_;
  fcb_plan fused_;
  std::vector<ctype> fused_w_;
  length_type fused_rows_ = 0;
  float fused_scale_;
};

/// fftm_backend for column-wise complex<float> multiple FFTs (Fftm<C, C, col,
/// D>).  query_layout asks for column-major dense data (tuple<1,0,2>), so the
/// DDA layer hands every column over as one contiguous run -- the layout the
/// reference's FFTW backend requests for this axis (src/ovxx/fftw/fftw.cpp:
/// 920-932) -- and the columns run as rows of the B200 row kernel.
template <int D>
class fftm_col : public signal::fft::fftm_backend<ctype, ctype, 1, D>
{
public:
  fftm_col(Domain<2> const &dom, float scale) : n_(dom[0].size()), plan_(0)
  {
    ensure_device();
    check(fcb_plan_fftm((long long)n_, (long long)dom[1].size(), D == fft_fwd ? FCB_FORWARD : FCB_INVERSE,
                        scale, &plan_));
    if (trace())
      std::fprintf(stderr, "[fcb200] Fftm<%s, col> %lu x %lu scale %g on the B200\n",
                   D == fft_fwd ? "fwd" : "inv", (unsigned long)n_, (unsigned long)dom[1].size(), (double)scale);
  }
  ~fftm_col() { if (plan_) fcb_destroy(plan_); }
  virtual char const *name() { return "fcb200::fftm_col"; }
  virtual bool supports_scale() { return true; }
  virtual void query_layout(Rt_layout<2> &inout)
  {
    inout.packing = dense;
    inout.order = tuple<1, 0, 2>();
    inout.storage_format = array;
  }
  virtual void query_layout(Rt_layout<2> &in, Rt_layout<2> &out)
  {
    query_layout(in);
    out = in;
  }
  virtual bool requires_copy(Rt_layout<2> &) { return false; }
  virtual void in_place(ctype *inout, stride_type r, stride_type c, length_type rows, length_type cols)
  {
    run(inout, r, c, inout, r, c, rows, cols);
  }
  virtual void out_of_place(ctype *in, stride_type ir, stride_type ic, ctype *out, stride_type o_r,
                            stride_type oc, length_type rows, length_type cols)
  {
    run(in, ir, ic, out, o_r, oc, rows, cols);
  }

private:
  void run(ctype *in, stride_type ir, stride_type ic, ctype *out, stride_type o_r, stride_type oc,
           length_type rows, length_type cols)
  {
    OVXX_PRECONDITION(ir == 1 && o_r == 1 && rows == n_);
    if (cols == 0) return;
    check(fcb_exec(plan_, reinterpret_cast<fcb_cf32 const *>(in), cols > 1 ? ic : rows,
                   reinterpret_cast<fcb_cf32 *>(out), cols > 1 ? oc : rows, (long long)cols, FCB_HOST));
  }

  length_type n_;
  fcb_plan plan_;
};

/// Layout of the real-input backends: unit stride along the transform axis
/// (rows for A == row, columns for A == col), interleaved complex.
template <int A>
inline void real_layout(Rt_layout<2> &in, Rt_layout<2> &out)
{
  in.packing = out.packing = dense;
  if (A == vsip::col) in.order = tuple<1, 0, 2>();
  else in.order = tuple<0, 1, 2>();
  out.order = in.order;
  in.storage_format = out.storage_format = array;
}

/// fftm_backend for real -> complex multiple FFTs (Fftm<float, complex<float>,
/// A, fft_fwd>): n real samples in, n/2 + 1 bins out, along rows (A == row) or
/// columns (A == col).  The reference's own backends leave the scale to the
/// workspace; this one folds it into the transform.
template <int A>
class fftm_r2c : public signal::fft::fftm_backend<float, ctype, A, fft_fwd>
{
  static int const axis = A == vsip::col ? 0 : 1;

public:
  fftm_r2c(Domain<2> const &dom, float scale) : n_(dom[axis].size()), plan_(0)
  {
    ensure_device();
    check(fcb_plan_fftm_real((long long)n_, (long long)dom[1 - axis].size(), FCB_FORWARD, scale, &plan_));
    if (trace())
      std::fprintf(stderr, "[fcb200] Fftm<real->complex, %s> n %lu x %lu scale %g on the B200\n",
                   axis == 1 ? "row" : "col", (unsigned long)n_, (unsigned long)dom[1 - axis].size(), (double)scale);
  }
  ~fftm_r2c() { if (plan_) fcb_destroy(plan_); }
  virtual char const *name() { return "fcb200::fftm_r2c"; }
  virtual bool supports_scale() { return true; }
  virtual void query_layout(Rt_layout<2> &in, Rt_layout<2> &out) { real_layout<A>(in, out); }
  virtual bool requires_copy(Rt_layout<2> &) { return false; }
  virtual void out_of_place(float *in, stride_type i0, stride_type i1, ctype *out, stride_type o0, stride_type o1,
                            length_type rows, length_type cols)
  {
    length_type const mult = axis == 1 ? rows : cols;
    stride_type const in_rs = axis == 1 ? i0 : i1, out_rs = axis == 1 ? o0 : o1;
    OVXX_PRECONDITION((axis == 1 ? i1 : i0) == 1 && (axis == 1 ? o1 : o0) == 1);
    if (mult == 0) return;
    check(fcb_exec_r2c(plan_, in, mult > 1 ? in_rs : n_, reinterpret_cast<fcb_cf32 *>(out),
                       mult > 1 ? out_rs : n_ / 2 + 1, (long long)mult, FCB_HOST));
  }

private:
  length_type n_;
  fcb_plan plan_;
};

/// fftm_backend for complex -> real multiple FFTs (Fftm<complex<float>, float,
/// A, fft_inv>): n/2 + 1 bins in, n real samples out.
template <int A>
class fftm_c2r : public signal::fft::fftm_backend<ctype, float, A, fft_inv>
{
  static int const axis = A == vsip::col ? 0 : 1;

public:
  fftm_c2r(Domain<2> const &dom, float scale) : n_(dom[axis].size()), plan_(0)
  {
    ensure_device();
    check(fcb_plan_fftm_real((long long)n_, (long long)dom[1 - axis].size(), FCB_INVERSE, scale, &plan_));
    if (trace())
      std::fprintf(stderr, "[fcb200] Fftm<complex->real, %s> n %lu x %lu scale %g on the B200\n",
                   axis == 1 ? "row" : "col", (unsigned long)n_, (unsigned long)dom[1 - axis].size(), (double)scale);
  }
  ~fftm_c2r() { if (plan_) fcb_destroy(plan_); }
  virtual char const *name() { return "fcb200::fftm_c2r"; }
  virtual bool supports_scale() { return true; }
  virtual void query_layout(Rt_layout<2> &in, Rt_layout<2> &out) { real_layout<A>(in, out); }
  virtual bool requires_copy(Rt_layout<2> &) { return false; }
  virtual void out_of_place(ctype *in, stride_type i0, stride_type i1, float *out, stride_type o0, stride_type o1,
                            length_type rows, length_type cols)
  {
    length_type const mult = axis == 1 ? rows : cols;
    stride_type const in_rs = axis == 1 ? i0 : i1, out_rs = axis == 1 ? o0 : o1;
    OVXX_PRECONDITION((axis == 1 ? i1 : i0) == 1 && (axis == 1 ? o1 : o0) == 1);
    if (mult == 0) return;
    check(fcb_exec_c2r(plan_, reinterpret_cast<fcb_cf32 const *>(in), mult > 1 ? in_rs : n_ / 2 + 1, out,
                       mult > 1 ? out_rs : n_, (long long)mult, FCB_HOST));
  }

private:
  length_type n_;
  fcb_plan plan_;
};

// Fused plan for a weights block: a vector (one replica spectrum for all rows)
// or a matrix (one per row), read through the DDA layer (direct pointer when
// the block is dense, a copy otherwise).
template <typename W, dimension_type Dim = W::dim> struct fused_plan_for;
template <typename W> struct fused_plan_for<W, 1>
{
  static fcb_plan get(fftm<fft_inv> &g, W const &w, float s, length_type rows)
  {
    vsip::dda::Data<W, vsip::dda::in, Layout<1, row1_type, dense, array> > d(w);
    return g.fused(d.ptr(), g.cols(), 1, s, rows);
  }
};
template <typename W> struct fused_plan_for<W, 2>
{
  static fcb_plan get(fftm<fft_inv> &g, W const &w, float s, length_type rows)
  {
    vsip::dda::Data<W, vsip::dda::in, Layout<2, row2_type, dense, array> > d(w);
    return g.fused(d.ptr(), d.size(0) > 1 ? d.stride(0) : g.cols(), d.size(0), s, rows);
  }
};

// Run one fused call: in -> out with weights (vector or matrix) on the plans
// of the two B200 Fftm objects.
template <typename LHS, typename IN, typename W>
void run_fused(LHS &lhs, IN const &in_block, W const &w_block, length_type wrows, fftm<fft_fwd> const &f,
               fftm<fft_inv> &g)
{
  typedef Layout<2, row2_type, dense, array> L2;
  length_type const rows = lhs.size(2, 0), cols = lhs.size(2, 1);
  vsip::dda::Data<IN, vsip::dda::in, L2> in_data(in_block);
  vsip::dda::Data<LHS, vsip::dda::out, L2> out_data(lhs);
  fcb_plan plan = fused_plan_for<W>::get(g, w_block, f.scale() * g.scale(), rows);
  if (trace())
    std::fprintf(stderr, "[fcb200] fused fastconv %lu x %lu (%s weights) on the B200\n", (unsigned long)rows,
                 (unsigned long)cols, wrows == 1 ? "vector" : "matrix");
  check(fcb_exec(plan, reinterpret_cast<fcb_cf32 const *>(in_data.ptr()), rows > 1 ? in_data.stride(0) : cols,
                 reinterpret_cast<fcb_cf32 *>(out_data.ptr()), rows > 1 ? out_data.stride(0) : cols,
                 (long long)rows, FCB_HOST));
}

template <typename F>
fftm<fft_fwd> const *as_fwd(F const &functor)
{
  return dynamic_cast<fftm<fft_fwd> const *>(&functor.backend());
}
template <typename F>
fftm<fft_inv> *as_inv(F const &functor)
{
  return const_cast<fftm<fft_inv> *>(dynamic_cast<fftm<fft_inv> const *>(&functor.backend()));
}

/// fft_backend for the 2-D complex<float> FFT (vsip::Fft<const_Matrix, C, C,
/// S>) on the B200, the contract of src/ovxx/signal/fft/backend.hpp:294-375.
/// It asks for dense row-major interleaved data (the DDA layer copies anything
/// else), applies the scale itself (supports_scale() == true, so the
/// workspace's scale pass, src/ovxx/signal/fft/workspace.hpp:474-478, is
/// skipped) and runs in place or out of place through fcb_plan_fft2d.
template <int S>
class fft2d : public signal::fft::fft_backend<2, ctype, ctype, S>
{
public:
  fft2d(Domain<2> const &dom, float scale) : rows_(dom[0].size()), cols_(dom[1].size()), plan_(0)
  {
    ensure_device();
    check(fcb_plan_fft2d((long long)rows_, (long long)cols_, S == fft_fwd ? FCB_FORWARD : FCB_INVERSE, scale,
                         &plan_));
    if (trace())
      std::fprintf(stderr, "[fcb200] Fft<2,%s> %lu x %lu scale %g on the B200\n", S == fft_fwd ? "fwd" : "inv",
                   (unsigned long)rows_, (unsigned long)cols_, (double)scale);
  }
  ~fft2d()
  {
    if (plan_) fcb_destroy(plan_);
  }
  virtual bool supports_scale() { return true; }
  virtual void query_layout(Rt_layout<2> &inout)
  {
    inout.packing = dense;
    inout.order = tuple<0, 1, 2>();
    inout.storage_format = array;
  }
  virtual void query_layout(Rt_layout<2> &in, Rt_layout<2> &out)
  {
    query_layout(in);
    out = in;
  }
  virtual bool requires_copy(Rt_layout<2> &) { return false; }
  virtual void in_place(ctype *inout, stride_type r, stride_type c, length_type rows, length_type cols)
  {
    run(inout, r, c, inout, r, c, rows, cols);
  }
  virtual void out_of_place(ctype *in, stride_type ir, stride_type ic, ctype *out, stride_type o_r,
                            stride_type oc, length_type rows, length_type cols)
  {
    run(in, ir, ic, out, o_r, oc, rows, cols);
  }

private:
  void run(ctype *in, stride_type ir, stride_type ic, ctype *out, stride_type o_r, stride_type oc,
           length_type rows, length_type cols)
  {
    OVXX_PRECONDITION(ic == 1 && oc == 1 && rows == rows_ && cols == cols_);
    check(fcb_exec(plan_, reinterpret_cast<fcb_cf32 const *>(in), rows > 1 ? ir : cols,
                   reinterpret_cast<fcb_cf32 *>(out), rows > 1 ? o_r : cols, (long long)rows, FCB_HOST));
  }

  length_type rows_, cols_;
  fcb_plan plan_;
};

/// fft_backend for the 1-D complex<float> FFT (vsip::Fft<const_Vector, C, C,
/// S>, the replica's t2f in tests/fastconv.cpp:21-26 and benchmarks/
/// fastconv.cpp:437), the contract of src/ovxx/signal/fft/backend.hpp:132-205:
/// one row of a row plan (fcb_plan_fftm with rows_max 1), dense interleaved
/// data (the DDA layer copies anything else), the scale applied in the kernel.
template <int S>
class fft1d : public signal::fft::fft_backend<1, ctype, ctype, S>
{
public:
  fft1d(Domain<1> const &dom, float scale) : n_(dom.size()), plan_(0)
  {
    ensure_device();
    check(fcb_plan_fftm((long long)n_, 1, S == fft_fwd ? FCB_FORWARD : FCB_INVERSE, scale, &plan_));
    if (trace())
      std::fprintf(stderr, "[fcb200] Fft<1,%s> %lu scale %g on the B200\n", S == fft_fwd ? "fwd" : "inv",
                   (unsigned long)n_, (double)scale);
  }
  ~fft1d()
  {
    if (plan_) fcb_destroy(plan_);
  }
  virtual bool supports_scale() { return true; }
  virtual void query_layout(Rt_layout<1> &inout)
  {
    inout.packing = dense;
    inout.order = tuple<0, 1, 2>();
    inout.storage_format = array;
  }
  virtual void query_layout(Rt_layout<1> &in, Rt_layout<1> &out)
  {
    query_layout(in);
    out = in;
  }
  virtual bool requires_copy(Rt_layout<1> &) { return false; }
  virtual void in_place(ctype *inout, stride_type stride, length_type n) { run(inout, stride, inout, stride, n); }
  virtual void out_of_place(ctype *in, stride_type is, ctype *out, stride_type os, length_type n)
  {
    run(in, is, out, os, n);
  }

private:
  void run(ctype *in, stride_type is, ctype *out, stride_type os, length_type n)
  {
    OVXX_PRECONDITION(is == 1 && os == 1 && n == n_);
    check(fcb_exec(plan_, reinterpret_cast<fcb_cf32 const *>(in), (long long)n, reinterpret_cast<fcb_cf32 *>(out),
                   (long long)n, 1, FCB_HOST));
  }

  length_type n_;
  fcb_plan plan_;
};

} // namespace ovxx::fcb200

namespace dispatcher
{

/// 1-D complex<float> Fft on the B200 (be::user slot, the first entry of
/// List<op::fft> in src/ovxx/signal/fft.hpp:41-49); lengths the row plans do
/// not support fall through to the next backend in the list.
template <int S, vsip::return_mechanism_type R, unsigned N>
struct Evaluator<op::fft<1, std::complex<float>, std::complex<float>, S, R, N>, be::user,
                 std::unique_ptr<signal::fft::fft_backend<1, std::complex<float>, std::complex<float>, S> >
                 (Domain<1> const &, float)>
{
  typedef signal::fft::fft_backend<1, std::complex<float>, std::complex<float>, S> backend_type;
  static bool const ct_valid = true;
  static char const *name() { return "fcb200 fft 1-D (B200)"; }
  static bool rt_valid(Domain<1> const &dom, float)
  {
    return dom.size() > 0 && fcb_supported_length((long long)dom.size());
  }
  static std::unique_ptr<backend_type> exec(Domain<1> const &dom, float scale)
  {
    return std::unique_ptr<backend_type>(new fcb200::fft1d<S>(dom, scale));
  }
};

/// 2-D complex<float> Fft on the B200 (be::user slot, the first entry of
/// List<op::fft> in src/ovxx/signal/fft.hpp:41-49).  Any dimensions the row
/// plans support; other sizes fail rt_valid and fall through to the next
/// backend in the list.
template <int S, vsip::return_mechanism_type R, unsigned N>
struct Evaluator<op::fft<2, std::complex<float>, std::complex<float>, S, R, N>, be::user,
                 std::unique_ptr<signal::fft::fft_backend<2, std::complex<float>, std::complex<float>, S> >
                 (Domain<2> const &, float)>
{
  typedef signal::fft::fft_backend<2, std::complex<float>, std::complex<float>, S> backend_type;
  static bool const ct_valid = true;
  static char const *name() { return "fcb200 fft 2-D (B200)"; }
  static bool rt_valid(Domain<2> const &dom, float)
  {
    return dom[0].size() > 0 && dom[1].size() > 0 && fcb_supported_length((long long)dom[0].size()) &&
           fcb_supported_length((long long)dom[1].size());
  }
  static std::unique_ptr<backend_type> exec(Domain<2> const &dom, float scale)
  {
    return std::unique_ptr<backend_type>(new fcb200::fft2d<S>(dom, scale));
  }
};

/// Row-wise complex<float> Fftm on the B200 (be::user slot).
template <int D, vsip::return_mechanism_type R, unsigned N>
struct Evaluator<op::fftm<std::complex<float>, std::complex<float>, 0, D, R, N>, be::user,
                 std::unique_ptr<signal::fft::fftm_backend<std::complex<float>, std::complex<float>, 0, D> >
                 (Domain<2> const &, float)>
{
  typedef signal::fft::fftm_backend<std::complex<float>, std::complex<float>, 0, D> backend_type;
  static bool const ct_valid = true;
  static char const *name() { return "fcb200 fftm (B200)"; }
  static bool rt_valid(Domain<2> const &dom, float)
  {
    return fcb_supported_length((long long)dom[1].size()) && dom[0].size() > 0;
  }
  static std::unique_ptr<backend_type> exec(Domain<2> const &dom, float scale)
  {
    return std::unique_ptr<backend_type>(new fcb200::fftm<D>(dom, scale));
  }
};

/// Column-wise complex<float> Fftm on the B200 (be::user slot).
template <int D, vsip::return_mechanism_type R, unsigned N>
struct Evaluator<op::fftm<std::complex<float>, std::complex<float>, 1, D, R, N>, be::user,
                 std::unique_ptr<signal::fft::fftm_backend<std::complex<float>, std::complex<float>, 1, D> >
                 (Domain<2> const &, float)>
{
  typedef signal::fft::fftm_backend<std::complex<float>, std::complex<float>, 1, D> backend_type;
  static bool const ct_valid = true;
  static char const *name() { return "fcb200 fftm, columns (B200)"; }
  static bool rt_valid(Domain<2> const &dom, float)
  {
    return fcb_supported_length((long long)dom[0].size()) && dom[1].size() > 0;
  }
  static std::unique_ptr<backend_type> exec(Domain<2> const &dom, float scale)
  {
    return std::unique_ptr<backend_type>(new fcb200::fftm_col<D>(dom, scale));
  }
};

/// Real -> complex Fftm, rows or columns (be::user slot).
template <int A, vsip::return_mechanism_type R, unsigned N>
struct Evaluator<op::fftm<float, std::complex<float>, A, fft_fwd, R, N>, be::user,
                 std::unique_ptr<signal::fft::fftm_backend<float, std::complex<float>, A, fft_fwd> >
                 (Domain<2> const &, float)>
{
  typedef signal::fft::fftm_backend<float, std::complex<float>, A, fft_fwd> backend_type;
  static bool const ct_valid = true;
  static char const *name() { return "fcb200 fftm real->complex (B200)"; }
  static bool rt_valid(Domain<2> const &dom, float)
  {
    int const axis = A == vsip::col ? 0 : 1;
    return fcb_supported_real_length((long long)dom[axis].size()) && dom[1 - axis].size() > 0;
  }
  static std::unique_ptr<backend_type> exec(Domain<2> const &dom, float scale)
  {
    return std::unique_ptr<backend_type>(new fcb200::fftm_r2c<A>(dom, scale));
  }
};

/// Complex -> real Fftm, rows or columns (be::user slot).
template <int A, vsip::return_mechanism_type R, unsigned N>
struct Evaluator<op::fftm<std::complex<float>, float, A, fft_inv, R, N>, be::user,
                 std::unique_ptr<signal::fft::fftm_backend<std::complex<float>, float, A, fft_inv> >
                 (Domain<2> const &, float)>
{
  typedef signal::fft::fftm_backend<std::complex<float>, float, A, fft_inv> backend_type;
  static bool const ct_valid = true;
  static char const *name() { return "fcb200 fftm complex->real (B200)"; }
  static bool rt_valid(Domain<2> const &dom, float)
  {
    int const axis = A == vsip::col ? 0 : 1;
    return fcb_supported_real_length((long long)dom[axis].size()) && dom[1 - axis].size() > 0;
  }
  static std::unique_ptr<backend_type> exec(Domain<2> const &dom, float scale)
  {
    return std::unique_ptr<backend_type>(new fcb200::fftm_c2r<A>(dom, scale));
  }
};

/// out = inv_fftm(vmmul<0>(weights, fwd_fftm(in))) as one fused pass (be::fc_expr slot).
template <typename LHS, template <typename> class O1, typename VB, template <typename> class O2, typename MB>
struct Evaluator<op::assign<2>, be::fc_expr,
                 void(LHS &, expr::Unary<O1, expr::Vmmul<0, VB, expr::Unary<O2, MB> const> const> const &)>
{
  typedef std::complex<float> C;
  typedef expr::Unary<O2, MB> fwd_block;
  typedef expr::Vmmul<0, VB, fwd_block const> vmmul_block;
  typedef expr::Unary<O1, vmmul_block const> RHS;
  typedef O1<vmmul_block const> inv_functor;
  typedef O2<MB> fwd_functor;
  static bool const ct_valid =
    is_same<typename inv_functor::backend_type, signal::fft::fftm_backend<C, C, 0, fft_inv> >::value &&
    is_same<typename fwd_functor::backend_type, signal::fft::fftm_backend<C, C, 0, fft_fwd> >::value &&
    is_same<typename VB::value_type, C>::value && is_same<typename LHS::value_type, C>::value &&
    is_same<typename MB::value_type, C>::value;
  static char const *name() { return "fcb200 fused fastconv, vector weights (B200)"; }
  static bool rt_valid(LHS &, RHS const &rhs)
  {
    return fcb200::as_inv(rhs.operation()) && fcb200::as_fwd(rhs.arg().get_mblk().operation());
  }
  static void exec(LHS &lhs, RHS const &rhs)
  {
    fwd_functor const &f = rhs.arg().get_mblk().operation();
    fcb200::run_fused(lhs, f.arg(), rhs.arg().get_vblk(), 1, *fcb200::as_fwd(f), *fcb200::as_inv(rhs.operation()));
  }
};

/// out = inv_fftm(W * fwd_fftm(in)) and inv_fftm(fwd_fftm(in) * W): one
/// replica spectrum per row (matrix of coefficients).
template <typename LHS, template <typename> class O1, template <typename, typename> class M, typename WB,
          template <typename> class O2, typename MB>
struct Evaluator<op::assign<2>, be::fc_expr,
                 void(LHS &, expr::Unary<O1, expr::Binary<M, WB, expr::Unary<O2, MB> const, true> const> const &)>
{
  typedef std::complex<float> C;
  typedef expr::Unary<O2, MB> fwd_block;
  typedef expr::Binary<M, WB, fwd_block const, true> mul_block;
  typedef expr::Unary<O1, mul_block const> RHS;
  typedef O1<mul_block const> inv_functor;
  typedef O2<MB> fwd_functor;
  static bool const ct_valid =
    is_same<M<C, C>, expr::op::Mult<C, C> >::value &&
    is_same<typename inv_functor::backend_type, signal::fft::fftm_backend<C, C, 0, fft_inv> >::value &&
    is_same<typename fwd_functor::backend_type, signal::fft::fftm_backend<C, C, 0, fft_fwd> >::value &&
    is_same<typename WB::value_type, C>::value && is_same<typename LHS::value_type, C>::value &&
    is_same<typename MB::value_type, C>::value && WB::dim == 2;
  static char const *name() { return "fcb200 fused fastconv, matrix weights (B200)"; }
  static bool rt_valid(LHS &lhs, RHS const &rhs)
  {
    return fcb200::as_inv(rhs.operation()) && fcb200::as_fwd(rhs.arg().arg2().operation()) &&
           rhs.arg().arg1().size(2, 0) == lhs.size(2, 0);
  }
  static void exec(LHS &lhs, RHS const &rhs)
  {
    fwd_functor const &f = rhs.arg().arg2().operation();
    fcb200::run_fused(lhs, f.arg(), rhs.arg().arg1(), lhs.size(2, 0), *fcb200::as_fwd(f),
                      *fcb200::as_inv(rhs.operation()));
  }
};

template <typename LHS, template <typename> class O1, template <typename, typename> class M, typename WB,
          template <typename> class O2, typename MB>
struct Evaluator<op::assign<2>, be::fc_expr,
                 void(LHS &, expr::Unary<O1, expr::Binary<M, expr::Unary<O2, MB> const, WB, true> const> const &)>
{
  typedef std::complex<float> C;
  typedef expr::Unary<O2, MB> fwd_block;
  typedef expr::Binary<M, fwd_block const, WB, true> mul_block;
  typedef expr::Unary<O1, mul_block const> RHS;
  typedef O1<mul_block const> inv_functor;
  typedef O2<MB> fwd_functor;
  static bool const ct_valid =
    is_same<M<C, C>, expr::op::Mult<C, C> >::value &&
    is_same<typename inv_functor::backend_type, signal::fft::fftm_backend<C, C, 0, fft_inv> >::value &&
    is_same<typename fwd_functor::backend_type, signal::fft::fftm_backend<C, C, 0, fft_fwd> >::value &&
    is_same<typename WB::value_type, C>::value && is_same<typename LHS::value_type, C>::value &&
    is_same<typename MB::value_type, C>::value && WB::dim == 2;
  static char const *name() { return "fcb200 fused fastconv, matrix weights (B200)"; }
  static bool rt_valid(LHS &lhs, RHS const &rhs)
  {
    return fcb200::as_inv(rhs.operation()) && fcb200::as_fwd(rhs.arg().arg1().operation()) &&
           rhs.arg().arg2().size(2, 0) == lhs.size(2, 0);
  }
  static void exec(LHS &lhs, RHS const &rhs)
  {
    fwd_functor const &f = rhs.arg().arg1().operation();
    fcb200::run_fused(lhs, f.arg(), rhs.arg().arg2(), lhs.size(2, 0), *fcb200::as_fwd(f),
                      *fcb200::as_inv(rhs.operation()));
  }
};

} // namespace ovxx::dispatcher
} // namespace ovxx

#endif
