// Batched fast convolution: many pulse-compression jobs of uneven shapes
// (pulses x samples, each with its own replica) in ONE persistent launch,
// replayed from a CUDA graph.
//
// There is no single counterpart in the reference: there each job is its own
// Fftm -> vmmul -> Fftm sequence (benchmarks/fastconv.cpp:100-106), run one
// after another on the host.
//
// Work decomposition: a job of P rows of N samples is cut into "units".  Jobs
// whose rows span CS > 1 CTAs of a cluster come first: their unit is the work
// of one hardware cluster of CSMAX CTAs for one step (CSMAX/CS rows).  The
// other jobs' unit is one row tile of one CTA.  Each group of units forms one
// index space (jobs ordered longest rows first by default); a cluster takes
// the next cluster unit from a global ticket counter until those are gone,
// then each of its CTAs takes single-CTA units from a second counter on its
// own, so uneven jobs balance across the GPU and short rows never wait on a
// cluster barrier.  The two counters are the only scratch memory, reset by a
// memset node of the same graph.
#include "fcb200.h"
#include "fcb_engine.cuh"
#include "fcb_internal.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <new>
#include <numeric>
#include <vector>

namespace fcb {

struct BatchJob
{
  RowArgs args;
  int logn;
  int tiles_per_unit;
  long long unit_begin;
};

constexpr int kBatchMinLog = 8;   // 256 samples
constexpr int kBatchMaxLog = 15;  // 32768 samples

__device__ __forceinline__ long long ld_cluster_s64(uint32_t addr)
{
  long long v;
  asm volatile("ld.shared::cluster.s64 %0, [%1];" : "=l"(v) : "r"(addr) : "memory");
  return v;
}

// WIDE = 1: the wide kernel (T = 256, one CTA per SM): rows of 16384 and
// 32768 samples run 64 samples per thread (the wide tile; 32768 on a cluster
// of two CTAs), shorter rows 32 per thread.  Its tiles all run one CTA per SM,
// so they stagger the two halves of the CTA as the single-job one-CTA-per-SM
// kernels do (measured: rows of 4096 samples 0.392 -> 0.406 of HBM, the
// 512-job mix 0.330 -> 0.334).
template <int L, int T, int WIDE>
using BatchSched = Sched<L, T, (WIDE && L >= 14) ? 64 : 32>;

// One unit of a job of rows of 2^logn samples: `r` is the CTA's place in the
// unit (its cluster rank for units that span the cluster, 0 for units of one
// CTA).  A unit is tiles_per_unit tiles; a tile of a row that spans CS CTAs is
// run by the CS CTAs of ranks sub * CS .. sub * CS + CS - 1.
template <int T, int CSMAX, int WIDE>
__device__ __forceinline__ void run_unit(const RowArgs &A, int logn, long long lu, int tiles_per_unit, int r,
                                         bool copy)
{
  switch (logn)
  {
#define FCB_BATCH_CASE(L)                                                                    \
  case L:                                                                                    \
  {                                                                                          \
    using S = BatchSched<L, T, WIDE>;                                                        \
    constexpr int CS = S::CS;                                                                \
    static_assert(CS <= CSMAX, "row longer than the launch's cluster");                      \
    const int sub = r / CS;                                                                  \
    row_tile<L, kFastconv, T, (WIDE && L >= 14) ? 64 : 32, WIDE>(A, lu * tiles_per_unit + sub, r % CS, sub * CS, \
                                                                 copy);                      \
  }                                                                                          \
  break;
    FCB_BATCH_CASE(8)
    FCB_BATCH_CASE(9)
    FCB_BATCH_CASE(10)
    FCB_BATCH_CASE(11)
    FCB_BATCH_CASE(12)
    FCB_BATCH_CASE(13)
    FCB_BATCH_CASE(14)
    FCB_BATCH_CASE(15)
#undef FCB_BATCH_CASE
    default:
      break;
  }
}

// Persistent batch kernel.  Jobs [0, ncl) have rows that span several CTAs of
// the cluster (units of the whole cluster, counted by ticket[0]); jobs
// [ncl, njobs) have rows of one CTA (units of one CTA, ticket[1]).  A cluster
// first takes cluster units, one ticket per cluster broadcast from rank 0, in
// step; once they are gone each CTA takes single-CTA units on its own, with no
// cluster barrier, so CTAs of a cluster do not wait on each other for short
// rows.
// Jobs whose first unit index is kept in shared memory for the lookup of a
// unit's job (larger job lists are searched in global memory).
constexpr int kSmemJobs = 1024;

template <int T, int CSMAX, int WIDE = 0>
__global__ void __launch_bounds__(T, WIDE ? 1 : 512 / T)
    batch_kernel(const BatchJob *__restrict__ jobs, int ncl, int njobs, long long cl_units, long long solo_units,
                 unsigned long long *ticket)
{
  // the unit and its job, double-buffered by the parity of the iteration
  // (slot it&1 is rewritten only after the barrier of the next iteration)
  __shared__ long long s_unit[2];
  __shared__ int s_lo[2], s_logn[2], s_tpu[2];
  // the current job's arguments: read from shared memory where they are used
  // rather than held in registers across the tile (fewer spills)
  __shared__ RowArgs s_args;
  __shared__ long long s_begin[kSmemJobs];
  constexpr bool HC = CSMAX > 1;
  constexpr int W = sizeof(RowArgs) / 8;
  static_assert(sizeof(RowArgs) % 8 == 0 && W <= T, "job arguments are copied as 8-byte words");
  const int hw_rank = HC ? (int)cg::this_cluster().block_rank() : 0;
  const bool smem_jobs = njobs <= kSmemJobs;
  if (smem_jobs)
    for (int i = threadIdx.x; i < njobs; i += T) s_begin[i] = jobs[i].unit_begin;
  __syncthreads();
  auto begin = [&](int i) { return smem_jobs ? s_begin[i] : jobs[i].unit_begin; };
  // job of unit u among jobs [from, last]: a CTA's units only increase within
  // a phase, so the search starts at its current job
  auto find = [&](long long u, int from, int last) {
    int lo = from, hi = last;
    while (lo < hi)
    {
      const int mid = (lo + hi + 1) >> 1;
      if (begin(mid) <= u) lo = mid; else hi = mid - 1;
    }
    return lo;
  };
  // loop state kept in shared memory (CTA-uniform), so that it holds no
  // registers across the tile code
  __shared__ int s_state[4];  // cur_logn, cur_job, it, cluster_phase
  if (threadIdx.x == 0)
  {
    s_state[0] = -1;
    s_state[1] = -1;
    s_state[2] = 0;
    s_state[3] = (HC && cl_units > 0) ? 1 : 0;
  }
  __syncthreads();
  // Thread 0 (of rank 0 in the cluster phase) asks for the next unit while the
  // current one runs, so the ticket's round trip is off the critical path.
  long long next = 0;
  if (threadIdx.x == 0 && (s_state[3] ? hw_rank == 0 : true))
    next = (long long)atomicAdd(&ticket[s_state[3] ? 0 : 1], 1ULL);
  // one loop and one call of the tile code (two inlined copies of it would
  // not fit the wide kernel's registers)
#pragma unroll 1
  for (;;)
  {
    const int it = s_state[2];
    const int cur_logn = s_state[0], cur_job = s_state[1];
    const bool cluster_phase = s_state[3] != 0;
    const int rank = HC ? (int)cg::this_cluster().block_rank() : 0;
    const int slot = it & 1;
    long long u;
    int lo, logn, tpu, r;
    if (cluster_phase)
    {
      if (rank == 0 && threadIdx.x == 0) s_unit[slot] = next;
      cluster_sync();
      u = ld_cluster_s64(cluster_addr(smem_addr(&s_unit[slot]), 0));
      if (u >= cl_units)
      {
        cluster_sync();  // rank 0 stays until every CTA has read
        if (threadIdx.x == 0)
        {
          s_state[3] = 0;
          s_state[2] = it + 1;
          next = (long long)atomicAdd(&ticket[1], 1ULL);
        }
        __syncthreads();
        continue;
      }
      if (rank == 0 && threadIdx.x == 0) next = (long long)atomicAdd(&ticket[0], 1ULL);
      lo = find(u, cur_job >= 0 ? cur_job : 0, ncl - 1);
      logn = jobs[lo].logn;
      tpu = jobs[lo].tiles_per_unit;
      r = rank;
    }
    else
    {
      // warp 0 finds the unit's job before the barrier, while the other warps
      // finish the previous tile
      if ((threadIdx.x >> 5) == 0)
      {
        const long long uu = __shfl_sync(0xffffffffu, next, 0);
        if (uu < solo_units)
        {
          const int l = find(uu, cur_job >= ncl ? cur_job : ncl, njobs - 1);
          if (threadIdx.x == 0)
          {
            s_lo[slot] = l;
            s_logn[slot] = jobs[l].logn;
            s_tpu[slot] = jobs[l].tiles_per_unit;
            next = (long long)atomicAdd(&ticket[1], 1ULL);
          }
        }
        if (threadIdx.x == 0) s_unit[slot] = uu;
      }
      __syncthreads();
      u = s_unit[slot];
      if (u >= solo_units) break;
      lo = s_lo[slot];
      logn = s_logn[slot];
      tpu = s_tpu[slot];
      r = 0;
    }
    if (lo != cur_job)
    {
      // every thread of the CTA has left the previous tile (the barrier above)
      if (threadIdx.x < W)
        reinterpret_cast<long long *>(&s_args)[threadIdx.x] =
            reinterpret_cast<const long long *>(&jobs[lo].args)[threadIdx.x];
      __syncthreads();
    }
    const bool copy = logn != cur_logn;
    // every thread has read this iteration's state (the barriers above); the next
    // iteration reads it after the tile's own barriers
    if (threadIdx.x == 0)
    {
      s_state[0] = logn;
      s_state[1] = lo;
      s_state[2] = it + 1;
    }
    run_unit<T, CSMAX, WIDE>(s_args, logn, u - begin(lo), tpu, r, copy);
  }
}

// Largest shared-memory footprint over the lengths a batch kernel handles.
template <int T, int WIDE = 0, int L = kBatchMinLog>
constexpr int batch_smem()
{
  if constexpr (L > kBatchMaxLog)
    return 0;
  else
  {
    constexpr int a = BatchSched<L, T, WIDE>::SMEM, b = batch_smem<T, WIDE, L + 1>();
    return a > b ? a : b;
  }
}

struct BatchVariant
{
  const void *fn;
  int threads, csmax, smem;
  int wide;  // 1: 64 samples per thread at 16384 and 32768 (their tables are built for that)
};

static BatchVariant batch_variant(int threads)
{
  using SW = BatchSched<kBatchMaxLog, 256, 1>;
  if (threads == -256)
    return {(const void *)&batch_kernel<256, SW::CS, 1>, 256, SW::CS, batch_smem<256, 1>(), 1};
  if (threads == 256)
    return {(const void *)&batch_kernel<256, Sched<kBatchMaxLog, 256>::CS>, 256, Sched<kBatchMaxLog, 256>::CS,
            batch_smem<256>(), 0};
  return {(const void *)&batch_kernel<512, Sched<kBatchMaxLog, 512>::CS>, 512, Sched<kBatchMaxLog, 512>::CS,
          batch_smem<512>(), 0};
}

}  // namespace fcb

using namespace fcb;

struct fcb_batch_s
{
  int device = 0;
  BatchVariant v{};
  int grid = 0;
  int ctas_per_sm = 0;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  float4 *tw[kMaxLogN + 1] = {};
  struct Replica { float4 *table; int logn; };
  std::vector<Replica> replicas;
  BatchJob *d_jobs = nullptr;
  size_t jobs_cap = 0;            // capacity of d_jobs (grown, never shrunk)
  BatchJob *h_jobs = nullptr;     // pinned staging for the job table
  bool direct = false;            // launch without a graph (job sets that change every run)
  int njobs = 0;
  int ncl = 0;                    // jobs [0, ncl) have rows that span several CTAs
  long long cl_units = 0;         // units of the whole cluster (ticket 0)
  long long solo_units = 0;       // units of one CTA (ticket 1)
  long long total_units = 0;
  long long total_samples = 0;
  unsigned long long *d_ticket = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

namespace {

int ilog2_exact(long long n)
{
  if (n < 1 || (n & (n - 1)) != 0) return -1;
  int l = 0;
  while ((1LL << l) < n) ++l;
  return l;
}

void drop_graph(fcb_batch b)
{
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
}

void batch_free(fcb_batch b)
{
  if (!b) return;
  cudaSetDevice(b->device);
  if (b->own_stream) cudaStreamSynchronize(b->own_stream);
  if (b->stream && b->stream != b->own_stream) cudaStreamSynchronize(b->stream);
  drop_graph(b);
  for (auto &r : b->replicas) cudaFree(r.table);
  for (auto *t : b->tw) cudaFree(t);
  cudaFree(b->d_jobs);
  cudaFreeHost(b->h_jobs);
  cudaFree(b->d_ticket);
  if (b->own_stream) cudaStreamDestroy(b->own_stream);
  delete b;
}

int launch_batch(fcb_batch b, cudaStream_t st)
{
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)b->grid);
  cfg.blockDim = dim3(b->v.threads);
  cfg.dynamicSmemBytes = b->v.smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  if (b->v.csmax > 1)
  {
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = b->v.csmax;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
  }
  const BatchJob *jobs = b->d_jobs;
  int ncl = b->ncl, njobs = b->njobs;
  long long cl_units = b->cl_units, solo_units = b->solo_units;
  unsigned long long *ticket = b->d_ticket;
  void *params[] = {&jobs, &ncl, &njobs, &cl_units, &solo_units, &ticket};
  cudaError_t e = cudaLaunchKernelExC(&cfg, b->v.fn, params);
  if (e != cudaSuccess) return cuda_error(e, "batch kernel launch");
  return FCB_OK;
}

// Capture "reset the ticket, run the persistent kernel" into a CUDA graph.
int build_graph(fcb_batch b)
{
  drop_graph(b);
  cudaError_t e = cudaStreamBeginCapture(b->own_stream, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return cuda_error(e, "graph capture");
  e = cudaMemsetAsync(b->d_ticket, 0, 2 * sizeof(unsigned long long), b->own_stream);
  int rc = e == cudaSuccess ? launch_batch(b, b->own_stream) : cuda_error(e, "ticket reset");
  cudaGraph_t g = nullptr;
  cudaError_t e2 = cudaStreamEndCapture(b->own_stream, &g);
  if (rc) { if (g) cudaGraphDestroy(g); return rc; }
  if (e2 != cudaSuccess) return cuda_error(e2, "graph capture");
  b->graph = g;
  e = cudaGraphInstantiate(&b->exec, g, 0);
  if (e != cudaSuccess) { drop_graph(b); return cuda_error(e, "graph instantiate"); }
  return FCB_OK;
}

}  // namespace

extern "C" {

int fcb_batch_create(int threads, fcb_batch *out)
{
  if (!out) return set_error(FCB_ERR_INVALID, "batch pointer is NULL");
  *out = nullptr;
  // default: 512 threads (measured fastest on the uneven 512-job mix: 0.337 of HBM against
  // 0.3325 for the wide kernel)
  if (threads == 0) threads = 512;
  if (threads != 256 && threads != 512 && threads != -256)
    return set_error(FCB_ERR_INVALID, "threads must be 0, 256, 512 or -256 (wide)");
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return set_error(FCB_ERR_NODEVICE, "no CUDA device");
  fcb_batch b = new (std::nothrow) fcb_batch_s;
  if (!b) return set_error(FCB_ERR_NOMEM, "batch allocation");
  cudaGetDevice(&b->device);
  b->v = batch_variant(threads);
  cudaError_t e = cudaFuncSetAttribute(b->v.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, b->v.smem);
  int rc = e == cudaSuccess ? FCB_OK : cuda_error(e, "batch kernel attributes");
  if (!rc)
  {
    // persistent grid: as many CTAs (whole clusters) as can be resident at once
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device);
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b->ctas_per_sm, b->v.fn, b->v.threads, b->v.smem);
    if (e != cudaSuccess || b->ctas_per_sm < 1) rc = cuda_error(e, "batch occupancy");
    else if (b->v.csmax > 1)
    {
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3((unsigned)(sms * b->ctas_per_sm));
      cfg.blockDim = dim3(b->v.threads);
      cfg.dynamicSmemBytes = b->v.smem;
      cudaLaunchAttribute attr[1];
      attr[0].id = cudaLaunchAttributeClusterDimension;
      attr[0].val.clusterDim.x = b->v.csmax;
      attr[0].val.clusterDim.y = 1;
      attr[0].val.clusterDim.z = 1;
      cfg.attrs = attr;
      cfg.numAttrs = 1;
      int clusters = 0;
      e = cudaOccupancyMaxActiveClusters(&clusters, b->v.fn, &cfg);
      if (e != cudaSuccess || clusters < 1) rc = cuda_error(e, "batch cluster occupancy");
      else b->grid = clusters * b->v.csmax;
    }
    else
      b->grid = sms * b->ctas_per_sm;
  }
  if (!rc && (e = cudaStreamCreateWithFlags(&b->own_stream, cudaStreamNonBlocking)) != cudaSuccess)
    rc = cuda_error(e, "cudaStreamCreate");
  b->stream = b->own_stream;
  if (!rc && (e = cudaMalloc(&b->d_ticket, 2 * sizeof(unsigned long long))) != cudaSuccess)
    rc = set_error(FCB_ERR_NOMEM, "ticket counter: %s", cudaGetErrorString(e));
  if (rc) { batch_free(b); return rc; }
  *out = b;
  return FCB_OK;
}

int fcb_batch_add_replica(fcb_batch b, const fcb_cf32 *replica, long long n, int kind, int where, int *id)
{
  if (!b || !replica || !id) return set_error(FCB_ERR_INVALID, "NULL argument");
  const int l = ilog2_exact(n);
  if (l < kBatchMinLog || l > kBatchMaxLog)
    return set_error(FCB_ERR_UNSUPPORTED, "batch rows must be powers of two in [%d, %d], got %lld", 1 << kBatchMinLog,
                     1 << kBatchMaxLog, n);
  if (kind < FCB_REPLICA_SPECTRUM || kind > FCB_REPLICA_TIME_MATCHED) return set_error(FCB_ERR_INVALID, "bad replica kind");
  if (where != FCB_HOST && where != FCB_DEVICE) return set_error(FCB_ERR_INVALID, "bad location");
  cudaSetDevice(b->device);
  float2 *spec = nullptr, *tmp = nullptr;
  float4 *table = nullptr;
  const size_t bytes = sizeof(float2) * (size_t)n;
  cudaError_t e = cudaMalloc(&spec, bytes);
  int rc = e == cudaSuccess ? FCB_OK : set_error(FCB_ERR_NOMEM, "replica buffer");
  if (!rc && (e = cudaMemcpyAsync(spec, replica, bytes, where == FCB_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice,
                                  b->own_stream)) != cudaSuccess)
    rc = cuda_error(e, "replica copy");
  if (!rc && kind != FCB_REPLICA_SPECTRUM)
  {
    if ((e = cudaMalloc(&tmp, bytes)) != cudaSuccess) rc = set_error(FCB_ERR_NOMEM, "replica buffer");
    if (!rc) rc = replica_spectrum_dev(spec, n, kind == FCB_REPLICA_TIME_MATCHED, tmp, b->own_stream);
    if (!rc) std::swap(spec, tmp);
  }
  if (!rc && (e = cudaMalloc(&table, sizeof(float4) * (size_t)(n / 2))) != cudaSuccess)
    rc = set_error(FCB_ERR_NOMEM, "replica table");
  // the batch kernels run 32 samples per thread, the wide one 64 at 16384 and 32768
  const int ept = (b->v.wide && l >= 14) ? 64 : 32;
  if (!rc) rc = build_replica_table(l, ept, spec, n, 1, table, b->own_stream);
  if (!rc && !b->tw[l]) rc = build_twiddles(l, ept, &b->tw[l], b->own_stream);
  if (!rc && (e = cudaStreamSynchronize(b->own_stream)) != cudaSuccess) rc = cuda_error(e, "replica preparation");
  cudaFree(spec);
  cudaFree(tmp);
  if (rc) { cudaFree(table); return rc; }
  b->replicas.push_back({table, l});
  *id = (int)b->replicas.size() - 1;
  return FCB_OK;
}

int fcb_batch_set_jobs(fcb_batch b, const fcb_job *jobs, int njobs, int order)
{
  if (!b || (njobs > 0 && !jobs) || njobs < 0) return set_error(FCB_ERR_INVALID, "bad job list");
  std::vector<BatchJob> hj;
  std::vector<int> idx(njobs);
  std::iota(idx.begin(), idx.end(), 0);
  for (int i = 0; i < njobs; ++i)
  {
    const fcb_job &j = jobs[i];
    if (j.replica < 0 || j.replica >= (int)b->replicas.size()) return set_error(FCB_ERR_INVALID, "job %d: bad replica id", i);
    if ((1LL << b->replicas[j.replica].logn) != j.n) return set_error(FCB_ERR_INVALID, "job %d: replica length != row length", i);
    if (j.pulses < 0 || (j.pulses > 0 && (!j.in || !j.out))) return set_error(FCB_ERR_INVALID, "job %d: bad buffers", i);
    if (j.in_rs < j.n || j.out_rs < j.n) return set_error(FCB_ERR_INVALID, "job %d: row stride < row length", i);
  }
  const bool direct = (order & 2) != 0;
  order &= 1;
  if (order == 0)  // longest rows first, then most rows: large units start early
    std::stable_sort(idx.begin(), idx.end(), [&](int a, int c) {
      return jobs[a].n != jobs[c].n ? jobs[a].n > jobs[c].n : jobs[a].pulses > jobs[c].pulses;
    });
  // geometry of a length on the variant's CTAs (as in Sched<>): CTAs per row
  auto ctas_per_row = [&](int l) {
    const int ept = (b->v.wide && l >= 14) ? 64 : 32;
    const int half = 1 << (l - 1), spc = b->v.threads * ept / 2;
    return half > spc ? half / spc : 1;
  };
  // jobs whose rows span several CTAs first (units of the whole cluster),
  // then the others (units of one CTA), each group in the chosen order
  std::stable_partition(idx.begin(), idx.end(),
                        [&](int i) { return ctas_per_row(b->replicas[jobs[i].replica].logn) > 1; });
  long long units = 0, samples = 0, cl_units = 0;
  int ncl = 0;
  bool cluster_group = true;
  for (int i : idx)
  {
    const fcb_job &j = jobs[i];
    if (j.pulses == 0) continue;
    const int l = b->replicas[j.replica].logn;
    BatchJob bj = {};
    bj.logn = l;
    const int T = b->v.threads;
    const int ept = (b->v.wide && l >= 14) ? 64 : 32;
    const int cs = ctas_per_row(l);
    if (cluster_group && cs == 1)
    {
      // the single-CTA group starts its own unit count
      cluster_group = false;
      cl_units = units;
      units = 0;
    }
    if (cs > 1) ++ncl;
    const int rows_per_tile = cs > 1 ? 1 : (T * ept) / (int)j.n;
    bj.tiles_per_unit = cs > 1 ? b->v.csmax / cs : 1;
    const long long rows_per_unit = (long long)bj.tiles_per_unit * rows_per_tile;
    bj.unit_begin = units;
    units += (j.pulses + rows_per_unit - 1) / rows_per_unit;
    samples += j.pulses * j.n;
    RowArgs &a = bj.args;
    a.in = reinterpret_cast<const float2 *>(j.in);
    a.in_rs = j.in_rs;
    a.out = reinterpret_cast<float2 *>(j.out);
    a.out_rs = j.out_rs;
    a.rows = j.pulses;
    a.tw = b->tw[l];
    a.twi = b->tw[l];
    a.rep = b->replicas[j.replica].table;
    a.rep_rs = 0;
    a.scale = 1.f;
    // L2 prefetch of the same job's rows about a quarter of a wave of units
    // later (units are taken in order; across a job boundary nothing is
    // prefetched).  Measured on the 512-job mix: a quarter wave 0.321 of HBM,
    // half a wave 0.319, a whole wave 0.316, none 0.309.
    a.ahead = cs > 1 ? (long long)std::max(1, b->grid / b->v.csmax / 4) * bj.tiles_per_unit
                     : (long long)std::max(1, b->grid / 4);
    hj.push_back(bj);
  }
  if (cluster_group)
  {
    // every job spans the cluster (or there are none)
    cl_units = units;
    units = 0;
  }
  cudaSetDevice(b->device);
  // the previous run of this batch may still read the job table
  cudaStreamSynchronize(b->stream);
  drop_graph(b);
  b->njobs = (int)hj.size();
  b->ncl = ncl;
  b->cl_units = cl_units;
  b->solo_units = units;
  b->total_units = cl_units + units;
  b->total_samples = samples;
  b->direct = direct;
  if (hj.empty()) return FCB_OK;
  if (hj.size() > b->jobs_cap)
  {
    cudaFree(b->d_jobs);
    cudaFreeHost(b->h_jobs);
    b->d_jobs = nullptr;
    b->h_jobs = nullptr;
    b->jobs_cap = 0;
    // grown geometrically: every growth frees the old table (a device-wide
    // synchronisation), so a job count that ramps up must not regrow it each call
    const size_t cap = std::max<size_t>(hj.size(), std::max<size_t>(64, 2 * b->jobs_cap));
    cudaError_t e = cudaMalloc(&b->d_jobs, sizeof(BatchJob) * cap);
    if (e != cudaSuccess) return set_error(FCB_ERR_NOMEM, "job table");
    e = cudaMallocHost(&b->h_jobs, sizeof(BatchJob) * cap);
    if (e != cudaSuccess) return set_error(FCB_ERR_NOMEM, "job table staging");
    b->jobs_cap = cap;
  }
  std::copy(hj.begin(), hj.end(), b->h_jobs);
  cudaError_t e = cudaMemcpyAsync(b->d_jobs, b->h_jobs, sizeof(BatchJob) * hj.size(), cudaMemcpyHostToDevice,
                                  b->stream);
  if (e != cudaSuccess) return cuda_error(e, "job table copy");
  if (direct) return FCB_OK;
  e = cudaStreamSynchronize(b->stream);
  if (e != cudaSuccess) return cuda_error(e, "job table copy");
  return build_graph(b);
}

int fcb_batch_run(fcb_batch b)
{
  if (!b) return set_error(FCB_ERR_INVALID, "batch is NULL");
  if (b->njobs == 0) return FCB_OK;
  cudaSetDevice(b->device);
  if (b->direct)
  {
    cudaError_t e = cudaMemsetAsync(b->d_ticket, 0, 2 * sizeof(unsigned long long), b->stream);
    if (e != cudaSuccess) return cuda_error(e, "ticket reset");
    return launch_batch(b, b->stream);
  }
  if (!b->exec) return set_error(FCB_ERR_INVALID, "no jobs set");
  cudaError_t e = cudaGraphLaunch(b->exec, b->stream);
  if (e != cudaSuccess) return cuda_error(e, "graph launch");
  return FCB_OK;
}

int fcb_batch_set_stream(fcb_batch b, void *stream)
{
  if (!b) return set_error(FCB_ERR_INVALID, "batch is NULL");
  b->stream = (cudaStream_t)stream;
  return FCB_OK;
}

int fcb_batch_sync(fcb_batch b)
{
  if (!b) return set_error(FCB_ERR_INVALID, "batch is NULL");
  cudaSetDevice(b->device);
  cudaError_t e = cudaStreamSynchronize(b->stream);
  if (e != cudaSuccess) return cuda_error(e, "batch");
  return FCB_OK;
}

int fcb_batch_info(fcb_batch b, long long *units, long long *samples, int *grid, int *threads)
{
  if (!b) return set_error(FCB_ERR_INVALID, "batch is NULL");
  if (units) *units = b->total_units;
  if (samples) *samples = b->total_samples;
  if (grid) *grid = b->grid;
  if (threads) *threads = b->v.threads;
  return FCB_OK;
}

int fcb_batch_destroy(fcb_batch b)
{
  batch_free(b);
  return FCB_OK;
}

}  // extern "C"
