// Host-side copies between pageable user memory and the plans' pinned staging
// buffers, split over a pool of worker threads.
//
// The CUDA runtime moves pageable memory through small bounce buffers of its
// own, one copy at a time and synchronously with the calling thread: a
// 128 MB in / 128 MB out call measured about 5.6 GB/s each way that way,
// against 42-46 GB/s from pinned memory.  Host calls on pageable buffers
// therefore copy each chunk into a shared pinned buffer (and out of one) with
// several threads at once, while the copy engines move the neighbouring
// chunks.
#include "fcb_internal.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <thread>
#include <unistd.h>
#if defined(__x86_64__)
#include <emmintrin.h>
#endif

namespace fcb {

namespace {

// memcpy with non-temporal stores for the 16-byte aligned body (x86-64): the
// destination lines are written without being read first, and stay out of
// the caches (the copy engine or the caller reads them next, not this thread).
// The caller fences (sfence) before another thread or a DMA reads the data.
inline void stream_copy(char *dst, const char *src, size_t n)
{
#if defined(__x86_64__)
  const size_t head = (16 - (reinterpret_cast<uintptr_t>(dst) & 15)) & 15;
  if (n < head + 256)
  {
    std::memcpy(dst, src, n);
    return;
  }
  std::memcpy(dst, src, head);
  dst += head;
  src += head;
  n -= head;
  const size_t body = n & ~size_t(63);
  for (size_t i = 0; i < body; i += 64)
  {
    const __m128i a = _mm_loadu_si128(reinterpret_cast<const __m128i *>(src + i));
    const __m128i b = _mm_loadu_si128(reinterpret_cast<const __m128i *>(src + i + 16));
    const __m128i c = _mm_loadu_si128(reinterpret_cast<const __m128i *>(src + i + 32));
    const __m128i d = _mm_loadu_si128(reinterpret_cast<const __m128i *>(src + i + 48));
    _mm_stream_si128(reinterpret_cast<__m128i *>(dst + i), a);
    _mm_stream_si128(reinterpret_cast<__m128i *>(dst + i + 16), b);
    _mm_stream_si128(reinterpret_cast<__m128i *>(dst + i + 32), c);
    _mm_stream_si128(reinterpret_cast<__m128i *>(dst + i + 48), d);
  }
  std::memcpy(dst + body, src + body, n - body);
#else
  std::memcpy(dst, src, n);
#endif
}

inline void store_fence()
{
#if defined(__x86_64__)
  _mm_sfence();
#endif
}

// One job at a time (callers serialise on job_mu_); the calling thread works
// on its own job next to the workers.  Pieces are whole rows, or for dense
// data byte ranges of at least 1 MB.
class CopyPool
{
public:
  explicit CopyPool(int workers) : pid_(getpid())
  {
    for (int i = 0; i < workers; ++i) std::thread([this] { worker(); }).detach();
  }

  void copy(void *dst, size_t dst_pitch, const void *src, size_t src_pitch, size_t row_bytes, size_t rows,
            int parts)
  {
    if (rows == 0 || row_bytes == 0) return;
    std::lock_guard<std::mutex> job(job_mu_);
    std::unique_lock<std::mutex> lk(mu_);
    // a worker that woke late for the previous job may still be in it
    done_cv_.wait(lk, [&] { return active_ == 0; });
    dst_ = static_cast<char *>(dst);
    src_ = static_cast<const char *>(src);
    dp_ = dst_pitch;
    sp_ = src_pitch;
    rb_ = row_bytes;
    rows_ = rows;
    dense_ = dst_pitch == row_bytes && src_pitch == row_bytes;
    if (dense_)
    {
      total_ = row_bytes * rows;
      const size_t want = std::max<size_t>(1, (size_t)parts * 2);
      piece_ = std::max<size_t>(1 << 20, (total_ / want + 63) & ~size_t(63));
      npieces_ = (total_ + piece_ - 1) / piece_;
    }
    else
    {
      piece_ = std::max<size_t>(1, (rows + (size_t)parts * 2 - 1) / ((size_t)parts * 2));
      npieces_ = (rows + piece_ - 1) / piece_;
    }
    next_.store(0);
    done_ = 0;
    ++gen_;  // the job's fields are published under mu_ with the generation
    lk.unlock();
    cv_.notify_all();
    run(false);
    lk.lock();
    done_cv_.wait(lk, [&] { return done_ == npieces_ && active_ == 0; });
  }

  pid_t pid() const { return pid_; }

private:
  void piece(size_t k)
  {
    if (dense_)
    {
      const size_t b0 = k * piece_, nb = std::min(piece_, total_ - b0);
      stream_copy(dst_ + b0, src_ + b0, nb);
      return;
    }
    const size_t r0 = k * piece_, r1 = std::min(rows_, r0 + piece_);
    for (size_t r = r0; r < r1; ++r) stream_copy(dst_ + r * dp_, src_ + r * sp_, rb_);
  }

  // Claim pieces until none is left.  A worker counts itself active from the
  // moment it sees a job's generation (under mu_) until it leaves here, and no
  // job is published while one is active, so its fields stay put meanwhile.
  void run(bool worker)
  {
    size_t mine = 0;
    for (size_t k; (k = next_.fetch_add(1)) < npieces_;)
    {
      piece(k);
      ++mine;
    }
    store_fence();  // this thread's streaming stores are visible before the job counts as done
    std::lock_guard<std::mutex> lk(mu_);
    done_ += mine;
    if (worker) --active_;
    if (done_ == npieces_ && active_ == 0) done_cv_.notify_all();
  }

  void worker()
  {
    unsigned seen = 0;
    for (;;)
    {
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return gen_ != seen; });
        seen = gen_;
        ++active_;
      }
      run(true);
    }
  }

  const pid_t pid_;
  std::mutex job_mu_, mu_;
  std::condition_variable cv_, done_cv_;
  unsigned gen_ = 0;
  size_t done_ = 0, npieces_ = 0;
  int active_ = 0;
  std::atomic<size_t> next_{0};
  char *dst_ = nullptr;
  const char *src_ = nullptr;
  size_t dp_ = 0, sp_ = 0, rb_ = 0, rows_ = 0, piece_ = 1, total_ = 0;
  bool dense_ = true;
};

// Threads per copy, the calling one included: FCB200_COPY_THREADS, else three
// quarters of the host's hardware threads, at most 16 (on a 16-thread host, 1024
// x 16384 pageable rows in and out: 2 threads 1.1, 4 1.6, 8 1.4-2.6, 12 2.6,
// 16 2.5-2.7 G samples/s, the copies bound by host memory bandwidth).  Returns
// the worker count (one less).
int copy_workers()
{
  static const int v = [] {
    const char *e = std::getenv("FCB200_COPY_THREADS");
    if (e) return std::max(1, std::atoi(e)) - 1;
    const unsigned hw = std::thread::hardware_concurrency();
    return std::min(16, std::max(1, (int)(hw * 3 / 4))) - 1;  // the calling thread is one of them
  }();
  return v;
}

CopyPool &pool()
{
  // Never destroyed (detached workers wait on it until the process ends).  A
  // child process made by fork() has none of the parent's workers: it gets a
  // pool of its own.
  static std::mutex mu;
  static CopyPool *p = nullptr;
  std::lock_guard<std::mutex> lk(mu);
  if (!p || p->pid() != getpid()) p = new CopyPool(copy_workers());
  return *p;
}

}  // namespace

void host_copy_rows(void *dst, size_t dst_pitch, const void *src, size_t src_pitch, size_t row_bytes, size_t rows)
{
  CopyPool &p = pool();
  p.copy(dst, dst_pitch, src, src_pitch, row_bytes, rows, copy_workers() + 1);
}

bool host_pageable(const void *ptr, size_t bytes)
{
  if (!ptr || bytes == 0) return false;
  const char *ends[2] = {static_cast<const char *>(ptr), static_cast<const char *>(ptr) + bytes - 1};
  for (const char *q : ends)
  {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, q) != cudaSuccess)
    {
      cudaGetLastError();  // clear the error the query left; stage to be safe
      return true;
    }
    if (a.type == cudaMemoryTypeUnregistered) return true;
  }
  return false;
}

}  // namespace fcb
