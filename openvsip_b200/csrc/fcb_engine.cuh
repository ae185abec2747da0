// Device engine for row-wise power-of-two FFTs and the fused fast convolution
// (forward row FFT -> multiply by replica spectrum -> inverse row FFT * 1/N).
//
// Reference behaviour replaced (the reference's CPU path):
//   forward / inverse Fftm      src/ovxx/fftw/fftw.cpp:965-977 (row loop of
//                               fftwf_execute_dft), scale pass in
//                               src/ovxx/signal/fft/workspace.hpp:474-478
//   vmmul<0>                    src/ovxx/expr/vmmul.hpp:53-59
//   fused fast convolution      benchmarks/fastconv.cpp:100-106 (phased) and
//                               tests/fastconv.cpp:204 (by-value expression)
//
// Algorithm (decimation in frequency, "complex pairs"):
//  * A thread owns EPT complex samples (32, or 64 in the wide variant) held as
//    RB = EPT/2 complex PAIRS in split form {re: (a.re, b.re), im: (a.im,
//    b.im)} so that every butterfly, twiddle and replica multiply runs on
//    Blackwell's packed f32x2 add/mul/fma, two complex lanes per instruction.
//  * Stage 1 is a radix-R1 DIF step over the whole row (stride N/R1).  Its first
//    radix-2 level is done in scalar and places the even-q outputs in lane 0 and
//    the odd-q outputs in lane 1, so every later operation is lane-parallel with
//    identical constants in both lanes.  Sub-problem 2q' and 2q'+1 (length
//    D = N/R1 each) then live side by side in one "slot" (16 bytes).
//  * Stages 2.. are radix-RB DIF steps (16, or 32 in the wide variant) inside
//    the sub-problem pairs, in place in a 16-byte-slot shared-memory array
//    (one pad slot per RB slots against bank conflicts).  A thread reads and
//    writes only its own group's slots inside a stage, so one barrier per
//    exchange suffices.  Their twiddles are read from a copy of the tables in
//    shared memory, made once per CTA.  The wide variant needs one stage fewer
//    at 16384 samples (3 instead of 4: 4 slot exchanges per fused row instead
//    of 6) at twice the registers per thread.
//  * Stage-1 twiddles W_N^{nq} for the thread's groups n = t + T*g factor into
//    W_N^{tq} (loaded once per thread) times W_EPT^{gq} (a compile-time
//    constant), because N = EPT T.
//  * After the last forward stage a slot sigma = q'*D + P holds X[k], X[k+1]
//    with k = 2q' + R1 * digitrev_RB(P).  The fused path multiplies by a
//    replica table stored in the order the last stage reads it (the i-th value
//    of every thread of a row side by side, so each load is coalesced; scaled
//    by 1/N, exact for powers of two) and runs the exact transpose of the
//    forward stages with conjugate twiddles, so no reordering pass is ever
//    needed and every row makes one HBM read and one HBM write.  The
//    standalone FFTs add one reorder exchange.
//  * A CTA of THREADS threads holds EPT*THREADS samples: several short rows,
//    one row, or -- for longer rows -- one part of a row, the row then being
//    spread over a thread-block cluster whose CTAs exchange through
//    distributed shared memory in the two exchanges next to stage 1 (stores
//    forward, loads inverse).  No TMA multicast is used anywhere.
#pragma once

#include <cuda_runtime.h>
#include <cooperative_groups.h>
#include <stdint.h>
#include <type_traits>

namespace fcb {

namespace cg = cooperative_groups;

constexpr int kMaxLogN = 16;

// ---------------------------------------------------------------------------
// Schedule of a length-2^LOGN row transform on CTAs of THREADS threads.
// ONE_PER_SM = 1: the caller runs one CTA per SM whatever the schedule's own
// occupancy (a persistent kernel), so the halves of the CTA are staggered.
template <int LOGN, int THREADS, int EPTW = 32, int ONE_PER_SM = 0>
struct Sched
{
  static constexpr int T = THREADS;
  static constexpr int N = 1 << LOGN;
  static constexpr int RB = EPTW / 2;               // radix of the later stages (pairs per thread)
  static constexpr int LRB = EPTW == 64 ? 5 : 4;
  static constexpr int NS = (LOGN <= LRB + 1) ? 1 : 1 + (LOGN - (LRB + 1) + LRB - 1) / LRB;  // stages
  static constexpr int LOGR1 = LOGN - LRB * (NS - 1);
  static constexpr int R1 = 1 << LOGR1;
  static constexpr int H1 = R1 / 2;                 // pairs per stage-1 group
  static constexpr int D = N / R1;                  // sub-problem length
  static constexpr int EPT = N < EPTW ? N : EPTW;   // samples per thread
  static constexpr int CPT = EPT / 2;               // pairs per thread
  static constexpr int TPR = N / EPT;               // threads per row (cluster-wide)
  static constexpr int G1 = EPT / R1;               // stage-1 groups per thread
  static constexpr int SPC = T * RB;                // slots per CTA for rows of >= EPTW samples
  static constexpr int HALF = N / 2;                // slots per row
  static constexpr int CS = HALF > SPC ? HALF / SPC : 1;  // CTAs per cluster
  static constexpr int TPRL = TPR / CS;             // threads per row per CTA
  static constexpr int ROWS = CS > 1 ? 1 : T / TPR; // rows per CTA
  static constexpr int SLOTS = CS > 1 ? SPC : ROWS * HALF;  // slots per CTA
  // stage s (2..NS): block length and stride in slots
  __host__ __device__ static constexpr int L(int s) { return D >> (LRB * (s - 2)); }
  __host__ __device__ static constexpr int S(int s) { return L(s) / RB; }
  // Twiddle tables in global memory: stage 1 as HALF float4 entries, then
  // stages 2..NS as float2 entries at tw2_off(s) (float2 units, counted after
  // the float4 part).  Stages 2..NS-1 (the ones with twiddles) are copied to
  // shared memory after the slot array.
  __host__ __device__ static constexpr int tw2_off(int s)
  {
    int off = 0;
    for (int k = 2; k < s; ++k) off += L(k);
    return off;
  }
  __host__ __device__ static constexpr int tw_bytes() { return HALF * 16 + tw2_off(NS + 1) * 8; }
  static constexpr int TWS = NS >= 3 ? tw2_off(NS) : 0;   // float2 entries kept in shared memory
  static constexpr int SMEM = (SLOTS + SLOTS / RB) * 16 + TWS * 8;  // padded slots, then twiddles
  // CTAs resident per SM (the register file holds 512 threads of 32 samples or
  // 256 of 64), the launch bound's minimum
  static constexpr int MINB = (EPTW == 32 ? 512 : 256) / THREADS;
  // With one CTA per SM its two halves run out of phase through the
  // sub-problem stages (see row_tile)
  static constexpr bool STAGGER = (MINB == 1 || ONE_PER_SM) && NS >= 3;
};


// ---------------------------------------------------------------------------
// Packed arithmetic.
struct cpair { float2 re, im; };

__device__ __forceinline__ float2 f2add(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 f2mul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 f2fma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 f2sub(float2 a, float2 b)
{
  unsigned long long d;
  unsigned long long x = *reinterpret_cast<unsigned long long *>(&a);
  unsigned long long y = *reinterpret_cast<unsigned long long *>(&b);
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(x), "l"(y));
  return *reinterpret_cast<float2 *>(&d);
}
__device__ __forceinline__ float2 f2neg(float2 a) { return make_float2(-a.x, -a.y); }
__device__ __forceinline__ float2 f2dup(float v) { return make_float2(v, v); }

__device__ __forceinline__ cpair cp_add(cpair a, cpair b) { return {f2add(a.re, b.re), f2add(a.im, b.im)}; }
__device__ __forceinline__ cpair cp_sub(cpair a, cpair b) { return {f2sub(a.re, b.re), f2sub(a.im, b.im)}; }

// x * (wr + i wi) with per-lane twiddles; CONJ multiplies by the conjugate.
template <bool CONJ>
__device__ __forceinline__ cpair cp_mul(cpair x, float2 wr, float2 wi)
{
  if (!CONJ)
    return {f2fma(x.im, f2neg(wi), f2mul(x.re, wr)), f2fma(x.re, wi, f2mul(x.im, wr))};
  else
    return {f2fma(x.im, wi, f2mul(x.re, wr)), f2fma(x.re, f2neg(wi), f2mul(x.im, wr))};
}

__device__ __forceinline__ cpair cp_from4(float4 v) { return {make_float2(v.x, v.y), make_float2(v.z, v.w)}; }
__device__ __forceinline__ float4 cp_to4(cpair c) { return make_float4(c.re.x, c.re.y, c.im.x, c.im.y); }

// cos(2 pi k / 32) for k in [0, 8], correctly rounded to float.
__host__ __device__ constexpr float cq32(int k)
{
  return k == 0 ? 1.0f : k == 1 ? 0.98078525066375732f : k == 2 ? 0.92387950420379639f
       : k == 3 ? 0.83146959543228149f : k == 4 ? 0.70710676908493042f
       : k == 5 ? 0.55557024478912354f : k == 6 ? 0.38268342614173889f
       : k == 7 ? 0.19509032368659973f : 0.0f;
}
// cos and sin of 2 pi k / 32 for k in [0, 32).
__host__ __device__ constexpr float c32h(int k) { return k <= 8 ? cq32(k) : -cq32(16 - k); }
__host__ __device__ constexpr float s32h(int k) { return k <= 8 ? cq32(8 - k) : cq32(k - 8); }
__host__ __device__ constexpr float c32(int k) { return k < 16 ? c32h(k) : -c32h(k - 16); }
__host__ __device__ constexpr float s32(int k) { return k < 16 ? s32h(k) : -s32h(k - 16); }

__host__ __device__ constexpr float cq64(int k)
{
  return k == 0 ? 1.0f : k == 1 ? 0.9951847195625305f : k == 2 ? 0.9807852506637573f : k == 3 ? 0.9569403529167175f
       : k == 4 ? 0.9238795042037964f : k == 5 ? 0.8819212913513184f : k == 6 ? 0.8314695954322815f
       : k == 7 ? 0.7730104327201843f : k == 8 ? 0.7071067690849304f : k == 9 ? 0.6343932747840881f
       : k == 10 ? 0.5555702447891235f : k == 11 ? 0.4713967442512512f : k == 12 ? 0.3826834261417389f
       : k == 13 ? 0.290284663438797f : k == 14 ? 0.19509032368659973f : k == 15 ? 0.0980171412229538f : 0.0f;
}
__host__ __device__ constexpr float c64h(int k) { return k <= 16 ? cq64(k) : -cq64(32 - k); }
__host__ __device__ constexpr float s64h(int k) { return k <= 16 ? cq64(16 - k) : cq64(k - 16); }
__host__ __device__ constexpr float c64(int k) { return k < 32 ? c64h(k) : -c64h(k - 32); }
__host__ __device__ constexpr float s64(int k) { return k < 32 ? s64h(k) : -s64h(k - 32); }

// Multiply a pair by the constant W_32^K = exp(SIGN * 2 pi i K / 32), 0 <= K < 16.
template <int K, int SIGN>
__device__ __forceinline__ cpair cp_rot32(cpair x)
{
  if (K == 0) return x;
  constexpr float c = c32(K);
  constexpr float s = SIGN * s32(K);
  if (K == 8)  // multiply by SIGN * i
  {
    if (SIGN < 0) return {x.im, f2neg(x.re)};
    else return {f2neg(x.im), x.re};
  }
  return {f2fma(x.im, f2dup(-s), f2mul(x.re, f2dup(c))), f2fma(x.re, f2dup(s), f2mul(x.im, f2dup(c)))};
}

// DIF butterfly b' = (a - b) * W_32^K, a' = a + b.  The +-i case folds the
// rotation into the subtraction.
template <int K, int SIGN>
__device__ __forceinline__ void cp_bfly(cpair &a, cpair &b)
{
  cpair s = cp_add(a, b);
  if (K == 8)
  {
    if (SIGN < 0) b = {f2sub(a.im, b.im), f2sub(b.re, a.re)};
    else b = {f2sub(b.im, a.im), f2sub(a.re, b.re)};
  }
  else
    b = cp_rot32<K, SIGN>(cp_sub(a, b));
  a = s;
}

// Radix-2 DIF network over R pairs (lane-parallel): natural-order input,
// bit-reversed-order output.  c[i] ends up holding X[bitrev_R(i)].
template <int R, int SIGN, int LEN = R>
struct DifNet
{
  template <int J, int BASE>
  __device__ __forceinline__ static void level_j(cpair *c)
  {
    if constexpr (J < LEN / 2)
    {
      cp_bfly<J * (32 / LEN), SIGN>(c[BASE + J], c[BASE + J + LEN / 2]);
      level_j<J + 1, BASE>(c);
    }
  }
  template <int BASE>
  __device__ __forceinline__ static void level(cpair *c)
  {
    if constexpr (BASE < R)
    {
      level_j<0, BASE>(c);
      level<BASE + LEN>(c);
    }
  }
  __device__ __forceinline__ static void run(cpair *c)
  {
    if constexpr (LEN >= 2)
    {
      level<0>(c);
      DifNet<R, SIGN, LEN / 2>::run(c);
    }
  }
};

__host__ __device__ constexpr int bitrev(int i, int bits)
{
  int r = 0;
  for (int b = 0; b < bits; ++b) r |= ((i >> b) & 1) << (bits - 1 - b);
  return r;
}
__host__ __device__ constexpr int ilog2(int n) { return n <= 1 ? 0 : 1 + ilog2(n / 2); }

// Reverse the lb-bit digits of p (ndig digits; lb = log2 of the later-stage radix).
__host__ __device__ __forceinline__ int digitrev16(int p, int ndig, int lb = 4)
{
  int r = 0;
  for (int d = 0; d < ndig; ++d) { r = (r << lb) | (p & ((1 << lb) - 1)); p >>= lb; }
  return r;
}

// Physical position of slot i in shared memory: one padding slot after every
// 2^lb slots (lb = log2 of the later-stage radix, 4 or 5).  Every exchange
// pattern of the kernel (consecutive slots across threads, slots 2^lb apart
// across threads for the last stage) then falls on distinct 16-byte banks,
// and for the stride patterns of a stage the physical address stays linear in
// the element index, so the compiler folds the per-element offsets into the
// load/store instructions.
__device__ __forceinline__ int swz(int i, int lb = 4) { return i + (i >> lb); }

// Loads that stay where they are written: volatile asm is not moved across
// other volatile asm or memory operations, so twiddle and replica loads are
// issued in small batches next to their use instead of all being hoisted to
// the top of the kernel (which would double the live registers).
__device__ __forceinline__ float4 ldv4(const float4 *p)
{
  float4 v;
  asm volatile("ld.global.nc.v4.f32 {%0, %1, %2, %3}, [%4];"
               : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "l"(p));
  return v;
}

__device__ __forceinline__ float2 ldv2(const float2 *p)
{
  float2 v;
  asm volatile("ld.global.nc.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "l"(p));
  return v;
}

// Shared-memory access through 32-bit addresses.  In a cluster, peer CTAs'
// slots are reached through their shared::cluster window (mapa); a CTA's own
// shared::cta address is used for its own slots.
__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ uint32_t cluster_addr(uint32_t cta_addr, int rank)
{
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(cta_addr), "r"(rank));
  return r;
}
template <bool CLUSTER>
__device__ __forceinline__ void st_slot(uint32_t addr, float4 v)
{
  if (CLUSTER)
    asm volatile("st.shared::cluster.v4.f32 [%0], {%1, %2, %3, %4};"
                 :: "r"(addr), "f"(v.x), "f"(v.y), "f"(v.z), "f"(v.w) : "memory");
  else
    asm volatile("st.shared.v4.f32 [%0], {%1, %2, %3, %4};"
                 :: "r"(addr), "f"(v.x), "f"(v.y), "f"(v.z), "f"(v.w) : "memory");
}
template <bool CLUSTER>
__device__ __forceinline__ float4 ld_slot(uint32_t addr)
{
  float4 v;
  if (CLUSTER)
    asm volatile("ld.shared::cluster.v4.f32 {%0, %1, %2, %3}, [%4];"
                 : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "r"(addr) : "memory");
  else
    asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];"
                 : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "r"(addr) : "memory");
  return v;
}
__device__ __forceinline__ float2 ld_tw(uint32_t addr)
{
  float2 v;
  asm volatile("ld.shared.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "r"(addr) : "memory");
  return v;
}

__device__ __forceinline__ cpair cp_mul4(cpair x, float4 w)  // per-lane (re0, re1, im0, im1)
{
  return cp_mul<false>(x, make_float2(w.x, w.y), make_float2(w.z, w.w));
}
__device__ __forceinline__ cpair cp_mul4c(cpair x, float4 w)
{
  return cp_mul<true>(x, make_float2(w.x, w.y), make_float2(w.z, w.w));
}
// Per-lane constant rotation by W_64^{k0}, W_64^{k1} (k in units of 2 pi / 64).
template <int SIGN>
__device__ __forceinline__ cpair cp_rot2w(cpair x, int k0, int k1)
{
  if (k0 == 0 && k1 == 0) return x;
  const float2 c = make_float2(c64(k0), c64(k1));
  const float2 s = make_float2(SIGN * s64(k0), SIGN * s64(k1));
  return {f2fma(x.im, f2neg(s), f2mul(x.re, c)), f2fma(x.re, s, f2mul(x.im, c))};
}

// Per-lane constant rotation: lane 0 by W_32^{k0}, lane 1 by W_32^{k1}, with
// W_32 = exp(SIGN 2 pi i / 32).  k0, k1 are compile-time constants after
// unrolling, so the cos/sin pairs fold to immediates.
template <int SIGN>
__device__ __forceinline__ cpair cp_rot2(cpair x, int k0, int k1)
{
  if (k0 == 0 && k1 == 0) return x;
  const float2 c = make_float2(c32(k0), c32(k1));
  const float2 s = make_float2(SIGN * s32(k0), SIGN * s32(k1));
  return {f2fma(x.im, f2neg(s), f2mul(x.re, c)), f2fma(x.re, s, f2mul(x.im, c))};
}

// Launch arguments.
struct RowArgs
{
  const float2 *in;
  long long in_rs;      // row stride, complex elements
  float2 *out;
  long long out_rs;
  long long rows;
  const float4 *tw;     // twiddle tables for this length (see Sched::tw2_off)
  const float4 *twi;    // the same tables, read by the inverse half of the fused
                        // kernel: a second pointer keeps the compiler from
                        // merging those loads with the forward ones and holding
                        // the forward twiddles in registers across the kernel
  const float4 *rep;    // fused: replica pair table (slot order, scaled 1/N)
  long long rep_rs;     // fused: replica row stride in slots (0 = one vector)
  float scale;          // standalone: output scale
  int transpose_out;    // standalone FFT: store the result transposed (2-D FFT passes)
  int vec_out;          // standalone FFT: every output row starts 16-byte aligned
  long long ahead;      // L2 prefetch distance in tiles (CTAs, or clusters) -- about
                        // half a resident wave, so that tile's rows stream from
                        // HBM into L2 while this tile computes; 0 = off
  // kChirpconv only (Bluestein rows, whose n samples sit in power-of-two work
  // rows): the row is read as in[k] * cin[row * cin_rs + k] for k < n_in and
  // 0 beyond, and written for k < n_out only, times cout[k] when cout is set.
  const float2 *cin;
  long long cin_rs;
  long long n_in;
  const float2 *cout;
  long long n_out;
};

__device__ __forceinline__ void prefetch_l2(const void *p)
{
  asm volatile("prefetch.global.L2 [%0];" :: "l"(p));
}

// Bulk prefetch into L2 of `bytes` bytes (16-byte aligned start, a multiple of 16 bytes).
__device__ __forceinline__ void prefetch_l2_bulk(const void *p, uint32_t bytes)
{
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" :: "l"(p), "r"(bytes) : "memory");
}

// kChirpconv is the fused fast convolution with element-wise multipliers and
// zero padding on the way in and truncation on the way out (Bluestein rows).
enum Mode { kFwd = 0, kInv = 1, kFastconv = 2, kChirpconv = 3 };

__device__ __forceinline__ float2 c_mul(float2 a, float2 b)
{
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// Where a slot of the row lives: owning cluster rank and CTA-local index.
template <class S>
struct SlotMap
{
  __device__ __forceinline__ static int owner(int sigma) { return S::CS > 1 ? sigma / S::SPC : 0; }
  __device__ __forceinline__ static int local(int sigma, int rho)
  {
    return S::CS > 1 ? (sigma & (S::SPC - 1)) : rho * S::HALF + sigma;
  }
};

template <int S_>
using ic = std::integral_constant<int, S_>;

// Cluster-wide barrier with release/acquire ordering of shared::cluster
// accesses; every thread of every CTA of the cluster executes it.
__device__ __forceinline__ void cluster_sync()
{
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// Cluster-wide barrier without release ordering, for the barrier that only
// keeps a CTA's shared memory alive until the other CTAs have finished reading
// it: their reads are complete before they arrive (the values were used), so
// the arrive need not wait for this thread's own global stores to complete
// (measured 4 % faster at 32768 and 65536 samples than a release arrive).
__device__ __forceinline__ void cluster_sync_relaxed()
{
  asm volatile("barrier.cluster.arrive.relaxed.aligned;\n\tbarrier.cluster.wait.aligned;" ::: "memory");
}

// Barrier over the NT consecutive threads that share one exchange (NT a power
// of two dividing THREADS): a warp barrier when they sit in one warp, a named
// barrier per group otherwise, the CTA barrier when the group is the CTA.
// Between stage s and s+1 only the St(s) = L(s)/16 threads that own one block
// of L(s) slots exchange data, so narrower barriers let the groups of a CTA
// run out of phase (one group's shared-memory traffic overlaps another's math).
template <int NT, int THREADS>
__device__ __forceinline__ void group_sync(int t)
{
  static_assert(NT <= 32 || NT >= THREADS || THREADS / NT <= 13, "named barriers 14 and 15 are the stagger barriers");
  if constexpr (NT <= 32)
    __syncwarp();
  else if constexpr (NT >= THREADS)
    __syncthreads();
  else
    asm volatile("bar.sync %0, %1;" :: "r"(1 + t / NT), "r"(NT) : "memory");
}

// Stagger barriers (IDs as immediates): the first half of a CTA arrives, the
// second half waits; THREADS threads in all.
template <int ID, int THREADS>
__device__ __forceinline__ void half_arrive()
{
  asm volatile("bar.arrive %0, %1;" :: "n"(ID), "n"(THREADS) : "memory");
}
template <int ID, int THREADS>
__device__ __forceinline__ void half_wait()
{
  asm volatile("bar.sync %0, %1;" :: "n"(ID), "n"(THREADS) : "memory");
}

// One tile of a row transform on this CTA: the ROWS rows of `tile` when a row
// fits in one CTA, or part `rank` of row `tile` when CS CTAs share a row (they
// are the cluster ranks rank_base .. rank_base + CS - 1).  copy_tw: load the
// later-stage twiddle tables into shared memory (a persistent caller skips it
// while consecutive tiles have the same length).  The caller guarantees that
// no thread of the CTA (or of the CS CTAs) still reads the slot array of a
// previous tile.
template <int LOGN, int MODE, int THREADS, int EPTW = 32, int ONE_PER_SM = 0>
__device__ __forceinline__ void row_tile(const RowArgs &a, long long tile, int rank, int rank_base, bool copy_tw)
{
  using S = Sched<LOGN, THREADS, EPTW, ONE_PER_SM>;
  constexpr int RB = S::RB, LRB = S::LRB;
  constexpr int SIGN = (MODE == kInv) ? +1 : -1;  // direction of the first pass
  constexpr bool CHIRP = MODE == kChirpconv;
  constexpr int MD = CHIRP ? kFastconv : MODE;    // the transform structure
  constexpr int LH1 = ilog2(S::H1);
  constexpr bool CL = S::CS > 1;
  // stage 2 reads its block of D slots from its own CTA only
  static_assert(!CL || S::D <= S::SPC, "a stage-2 block must lie within one CTA of the cluster");
  static_assert(!S::STAGGER || S::S(2) <= THREADS / 2, "a stage-2 block must lie within one half of the CTA");
  extern __shared__ float4 smem[];
  const float2 *tw2 = reinterpret_cast<const float2 *>(a.tw + S::HALF);

  const int t = threadIdx.x;
  const int rho = CL ? 0 : t / S::TPR;                       // row within CTA
  const int tr = CL ? rank * THREADS + t : t % S::TPR;       // thread within row
  const long long row = CL ? tile : tile * S::ROWS + rho;
  const bool active = row < a.rows;

  // 32-bit base address of every cluster rank's slot array (own array when CS == 1)
  uint32_t peer[S::CS];
  peer[0] = smem_addr(smem);
  if constexpr (CL)
  {
    const uint32_t own = peer[0];
#pragma unroll
    for (int r = 0; r < S::CS; ++r) peer[r] = cluster_addr(own, rank_base + r);
  }
  const uint32_t slot_base = smem_addr(smem);
  const uint32_t tw_base = slot_base + 16u * (S::SLOTS + S::SLOTS / RB);  // later-stage twiddles
  auto swz_ = [&](int i) { return swz(i, LRB); };
  auto slot_addr = [&](int local) { return slot_base + 16u * (uint32_t)swz_(local); };

  // copy the twiddle tables of stages 2..NS-1 to shared memory (read before
  // the first barrier below, used after it)
  // with asynchronous copies (no register round trip, nothing waits on them
  // before the barrier that ends stage 1)
  if (S::TWS > 0 && copy_tw)
  {
    const float4 *src = reinterpret_cast<const float4 *>(tw2);
#pragma unroll 4
    for (int i = t; i < S::TWS / 2; i += THREADS)
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;"
                   :: "r"(tw_base + 16u * i), "l"(src + i) : "memory");
    asm volatile("cp.async.commit_group;" ::: "memory");
  }

  cpair c[S::CPT];

  // ---------------- stage 1 (direction SIGN) ----------------
  {
    float2 x[S::EPT];
    const float2 *src = a.in + row * a.in_rs;
    if constexpr (CHIRP)
    {
      // samples and multipliers in batches of eight (both at once would double
      // the live registers); the multiplier loads stay in place (volatile)
      const float2 *mul = a.cin + (active ? row : 0) * a.cin_rs;
#pragma unroll
      for (int j0 = 0; j0 < S::EPT; j0 += 8)
      {
        float2 m[8];
#pragma unroll
        for (int j = j0; j < j0 + 8 && j < S::EPT; ++j)
        {
          const int k = tr + S::TPR * j;
          const bool in = active && k < a.n_in;
          x[j] = in ? __ldg(src + k) : make_float2(0.f, 0.f);
          m[j - j0] = in ? ldv2(mul + k) : make_float2(0.f, 0.f);
        }
#pragma unroll
        for (int j = j0; j < j0 + 8 && j < S::EPT; ++j) x[j] = c_mul(x[j], m[j - j0]);
      }
    }
    else
    {
#pragma unroll
      for (int j = 0; j < S::EPT; ++j)
        x[j] = active ? __ldg(src + tr + S::TPR * j) : make_float2(0.f, 0.f);
    }
    // With this tile's loads in flight, prefetch into L2 the input of the tile
    // `ahead` tiles later (about half a resident wave), so that it streams in
    // from HBM while this tile computes.  Straight-line code (a few lines per
    // thread) placed here measured faster than a loop at the kernel start.  A
    // CTA of a cluster of four or more prefetches its part of the row with one
    // bulk prefetch when that part is 16-byte aligned (measured 6 % faster at
    // 65536 samples; at 32768 samples and for single-CTA rows the per-line
    // prefetch measured as fast or faster).
    {
      constexpr int LPR = S::N >= 16 ? S::N / 16 : 1;          // 128-byte lines per row
      constexpr int LINES = S::ROWS * LPR / S::CS;             // lines of this CTA's part
      constexpr int PER = (LINES + THREADS - 1) / THREADS;
      const long long row0 = (tile + a.ahead) * S::ROWS;
      const char *part = reinterpret_cast<const char *>(a.in + row0 * a.in_rs) + rank * (8LL * S::N / S::CS);
      if (S::CS >= 4 && !CHIRP && (reinterpret_cast<uintptr_t>(part) & 15) == 0)
      {
        if (a.ahead > 0 && t == 0 && row0 < a.rows) prefetch_l2_bulk(part, (uint32_t)(8LL * S::N / S::CS));
      }
      else
      {
#pragma unroll
        for (int k = 0; k < PER; ++k)
        {
          const int i = t + THREADS * k;
          const int li = rank * LINES + i;
          const long long r = row0 + li / LPR;
          if (a.ahead > 0 && i < LINES && r < a.rows && (!CHIRP || (li % LPR) * 16 < a.n_in))
            prefetch_l2(a.in + r * a.in_rs + (li % LPR) * 16);
        }
      }
    }
    // W_N^{tr q} for q = 2q' + lane; groups g > 0 add the constant W_32^{g q}
    float4 tw1[S::H1];
    if constexpr (S::NS > 1)
    {
#pragma unroll
      for (int i = 0; i < S::H1; ++i) tw1[i] = ldv4(a.tw + bitrev(i, LH1) * S::D + tr);
    }
#pragma unroll
    for (int g = 0; g < S::G1; ++g)
    {
      cpair *cg1 = c + g * S::H1;
      // scalar first radix-2 level: lane 0 <- x_r + x_{r+h}, lane 1 <- (x_r - x_{r+h}) W_R1^r
#pragma unroll
      for (int r = 0; r < S::H1; ++r)
      {
        float2 p = x[g + S::G1 * r], q = x[g + S::G1 * (r + S::H1)];
        float ur = p.x + q.x, ui = p.y + q.y;
        float dr = p.x - q.x, di = p.y - q.y;
        const int k = r * (32 / S::R1);
        const float wc = c32(k), ws = SIGN * s32(k);
        float vr, vi;
        if (k == 0) { vr = dr; vi = di; }
        else if (k == 8) { vr = SIGN < 0 ? di : -di; vi = SIGN < 0 ? -dr : dr; }
        else { vr = fmaf(dr, wc, -di * ws); vi = fmaf(dr, ws, di * wc); }
        cg1[r] = {make_float2(ur, vr), make_float2(ui, vi)};
      }
      DifNet<S::H1, SIGN>::run(cg1);
      if constexpr (S::NS > 1)
      {
        // stage-1 twiddles W_N^{n q} (per lane), then pair (q', n) -> slot q'*D + n
        const int n = tr + S::TPR * g;
#pragma unroll
        for (int i = 0; i < S::H1; ++i)
        {
          const int qp = bitrev(i, LH1);
          cpair v = (SIGN < 0) ? cp_mul4(cg1[i], tw1[i]) : cp_mul4c(cg1[i], tw1[i]);
          v = (EPTW == 64) ? cp_rot2w<SIGN>(v, (g * 2 * qp) & 63, (g * (2 * qp + 1)) & 63) : cp_rot2<SIGN>(v, (g * 2 * qp) & 31, (g * (2 * qp + 1)) & 31);
          const int sigma = qp * S::D + n;
          st_slot<CL>(peer[SlotMap<S>::owner(sigma)] + 16u * swz_(SlotMap<S>::local(sigma, rho)), cp_to4(v));
        }
      }
    }
  }
  if constexpr (S::NS > 1)
  {
    if (S::TWS > 0 && copy_tw) asm volatile("cp.async.wait_all;" ::: "memory");
    if constexpr (CL) cluster_sync(); else __syncthreads();
  }

  // ---------------- stages 2..NS, direction SIGN ----------------
  // One radix-16 group per thread (CPT == 16 whenever NS > 1).  In the fused
  // mode the last stage also multiplies by the replica (four entries at a time).
  auto stage_fwd = [&](auto sc) {
    constexpr int s = decltype(sc)::value;
    constexpr int Lg = S::L(s), St = S::S(s);
    const int B = tr / St, n = tr % St;
    const int base = B * Lg + n;
    const float4 *rp = a.rep + (active ? row : 0) * a.rep_rs;  // inactive rows read row 0
    // Stagger (one CTA per SM, whose warps would otherwise all be reading or
    // writing slots at the same time and then all computing): the second half
    // of the CTA starts stage 2 once the first half has issued its slot reads.
    // A block of stage 2 or later belongs to at most half of the CTA, and the
    // halves meet again only at the barrier before the inverse stage 1, so
    // from here on one half's shared-memory traffic overlaps the other half's
    // arithmetic.
    if constexpr (s == 2 && S::STAGGER)
      if (t >= THREADS / 2) half_wait<15, THREADS>();
#pragma unroll
    for (int r = 0; r < RB; ++r)
      c[r] = cp_from4(ld_slot<false>(slot_addr(SlotMap<S>::local(base + St * r, rho))));
    if constexpr (s == 2 && S::STAGGER)
      if (t < THREADS / 2) half_arrive<15, THREADS>();
    float4 ra[4];  // replica entries, four at a time
    if constexpr (MD == kFastconv && s == S::NS)
    {
#pragma unroll
      for (int i = 0; i < 4; ++i) ra[i] = ldv4(rp + i * S::TPR + tr);
    }
    DifNet<RB, SIGN>::run(c);
    if constexpr (St > 1)
    {
      // twiddles in batches of four: fewer live registers (no spills)
#pragma unroll
      for (int b = 0; b < RB; b += 4)
      {
        float2 w[4];
#pragma unroll
        for (int j = 0; j < 4; ++j)
          if (b + j > 0) w[j] = ld_tw(tw_base + 8u * (S::tw2_off(s) + (b + j) * St + n));
#pragma unroll
        for (int j = 0; j < 4; ++j)
        {
          const int q = b + j, i = bitrev(q, LRB);
          if (q != 0)
            c[i] = (SIGN < 0) ? cp_mul<false>(c[i], f2dup(w[j].x), f2dup(w[j].y))
                              : cp_mul<true>(c[i], f2dup(w[j].x), f2dup(w[j].y));
        }
      }
    }
    if constexpr (MD == kFastconv && s == S::NS)
    {
#pragma unroll
      for (int b = 0; b < RB; b += 4)
      {
        if (b > 0)
        {
#pragma unroll
          for (int i = 0; i < 4; ++i) ra[i] = ldv4(rp + (b + i) * S::TPR + tr);
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) c[b + i] = cp_mul4(c[b + i], ra[i]);
      }
    }
    if constexpr (s < S::NS)
    {
#pragma unroll
      for (int i = 0; i < RB; ++i)
        st_slot<false>(slot_addr(SlotMap<S>::local(base + St * bitrev(i, LRB), rho)), cp_to4(c[i]));
      group_sync<St, THREADS>(t);  // stage s+1 reads only this block of Lg slots
    }
  };
  if constexpr (S::NS >= 2) stage_fwd(ic<2>{});
  if constexpr (S::NS >= 3) stage_fwd(ic<3>{});
  if constexpr (S::NS >= 4) stage_fwd(ic<4>{});

  if constexpr (MD != kFastconv)
  {
    // ---------------- reorder to natural frequency order and store ----------------
    // c[] holds the last stage's outputs (never written back).  Pair slot
    // sigma = q'*D + P holds X[k], X[k+1] with k = 2q' + R1 * digitrev_RB(P), so it
    // moves to natural pair index m = q' + (R1/2) * digitrev_RB(P).
    int dst[S::CPT];
    if constexpr (S::NS == 1)
    {
#pragma unroll
      for (int i = 0; i < S::H1; ++i) dst[i] = bitrev(i, LH1);  // D == 1: slot index is q'
    }
    else
    {
      constexpr int Lg = S::L(S::NS), St = S::S(S::NS);
      const int B = tr / St, n = tr % St;
#pragma unroll
      for (int i = 0; i < RB; ++i)
      {
        const int sigma = B * Lg + n + St * bitrev(i, LRB);
        dst[i] = sigma / S::D + S::H1 * digitrev16(sigma % S::D, S::NS - 1, LRB);
      }
    }
    if constexpr (CL) cluster_sync(); else __syncthreads();
#pragma unroll
    for (int i = 0; i < S::CPT; ++i)
    {
      const int m = dst[i];
      st_slot<CL>(peer[SlotMap<S>::owner(m)] + 16u * swz_(SlotMap<S>::local(m, rho)), cp_to4(c[i]));
    }
    if constexpr (CL) cluster_sync(); else __syncthreads();
    // natural-order read of this CTA's part of the row, scale, store.
    const int tl = t % S::TPRL;
    float2 *dstp = a.out + row * a.out_rs;
    const float2 sc = f2dup(a.scale);
    if constexpr (!CL && S::NS > 1)
    {
      if (a.transpose_out)
      {
        // Transposed store (one pass of a 2-D FFT): element (row, k) goes to
        // out[k * out_rs + row].  Consecutive threads take consecutive rows of
        // this CTA for the same frequency pair, so a warp writes ROWS
        // consecutive elements of each output row it touches.
        const long long row0 = tile * S::ROWS;
#pragma unroll
        for (int i = 0; i < S::CPT; ++i)
        {
          const int idx = t + THREADS * i;
          const int rr = idx % S::ROWS, m = idx / S::ROWS;
          cpair p = cp_from4(ld_slot<false>(slot_addr(rr * S::HALF + m)));
          p.re = f2mul(p.re, sc);
          p.im = f2mul(p.im, sc);
          if (row0 + rr < a.rows)
          {
            a.out[(2LL * m) * a.out_rs + row0 + rr] = make_float2(p.re.x, p.im.x);
            a.out[(2LL * m + 1) * a.out_rs + row0 + rr] = make_float2(p.re.y, p.im.y);
          }
        }
        return;
      }
    }
#pragma unroll
    for (int i = 0; i < S::CPT; ++i)
    {
      const int l = tl + S::TPRL * i;                       // CTA-local natural pair index
      const int m = rank * (S::HALF / S::CS) + l;           // row natural pair index
      cpair p = cp_from4(ld_slot<false>(slot_addr(CL ? l : rho * S::HALF + l)));
      p.re = f2mul(p.re, sc);
      p.im = f2mul(p.im, sc);
      if (active)
      {
        if (a.vec_out)  // one 16-byte store per pair (row start 16-byte aligned)
          reinterpret_cast<float4 *>(dstp)[m] = make_float4(p.re.x, p.im.x, p.re.y, p.im.y);
        else
        {
          dstp[2 * m] = make_float2(p.re.x, p.im.x);
          dstp[2 * m + 1] = make_float2(p.re.y, p.im.y);
        }
      }
    }
    return;
  }
  else
  {
    if constexpr (S::NS == 1)
    {
      // single stage: replica multiply on the stage-1 outputs (slot = q')
      const float4 *rp = a.rep + (active ? row : 0) * a.rep_rs;
      constexpr int NB = S::H1 < 8 ? S::H1 : 8;
#pragma unroll
      for (int b0 = 0; b0 < S::H1; b0 += NB)
      {
        float4 w[NB];
#pragma unroll
        for (int i = 0; i < NB; ++i) w[i] = ldv4(rp + bitrev(b0 + i, LH1));
#pragma unroll
        for (int i = 0; i < NB; ++i) c[b0 + i] = cp_mul4(c[b0 + i], w[i]);
      }
    }

    // ---------------- inverse stages NS..2 (transpose of the forward ones) ----------------
    auto stage_inv = [&](auto sc) {
      constexpr int s = decltype(sc)::value;
      constexpr int Lg = S::L(s), St = S::S(s);
      const int B = tr / St, n = tr % St;
      const int base = B * Lg + n;
      cpair z[RB];
      if constexpr (s < S::NS)
      {
#pragma unroll
        for (int q = 0; q < RB; ++q)
          z[q] = cp_from4(ld_slot<false>(slot_addr(SlotMap<S>::local(base + St * q, rho))));
      }
      else
      {
#pragma unroll
        for (int i = 0; i < RB; ++i) z[bitrev(i, LRB)] = c[i];
      }
      if constexpr (St > 1)
      {
#pragma unroll
        for (int b = 0; b < RB; b += 4)
        {
          float2 w[4];
#pragma unroll
          for (int j = 0; j < 4; ++j)
            if (b + j > 0) w[j] = ld_tw(tw_base + 8u * (S::tw2_off(s) + (b + j) * St + n));
#pragma unroll
          for (int j = 0; j < 4; ++j)
            if (b + j > 0) z[b + j] = cp_mul<true>(z[b + j], f2dup(w[j].x), f2dup(w[j].y));
        }
      }
      DifNet<RB, +1>::run(z);  // z[i] = y[bitrev(i)]
#pragma unroll
      for (int i = 0; i < RB; ++i)
        st_slot<false>(slot_addr(SlotMap<S>::local(base + St * bitrev(i, LRB), rho)), cp_to4(z[i]));
      if constexpr (s > 2) group_sync<S::S(s - 1), THREADS>(t);  // stage s-1 reads blocks of L(s-1)
    };
    if constexpr (S::NS >= 4) stage_inv(ic<4>{});
    if constexpr (S::NS >= 3) stage_inv(ic<3>{});
    if constexpr (S::NS >= 2) stage_inv(ic<2>{});

    // inverse stage-1 twiddles: issued before the barrier so that its wait
    // covers their latency
    float4 tw1[S::H1];
    if constexpr (S::NS > 1)
    {
#pragma unroll
      for (int qp = 0; qp < S::H1; ++qp) tw1[qp] = ldv4(a.twi + qp * S::D + tr);
      if constexpr (CL) cluster_sync(); else __syncthreads();
    }

    // ---------------- inverse stage 1 and store ----------------
    float2 *dst_t = a.out + row * a.out_rs + tr;  // outputs at constant offsets from here
    // all slot reads of this thread first (remote ones in a cluster have a long
    // round trip; issuing them together overlaps their latencies)
    float4 v[S::CPT];
    if constexpr (S::NS > 1)
    {
      // the same stagger for the inverse stage 1: the second half reads its
      // slots once the first half has issued its reads
      if constexpr (S::STAGGER)
        if (t >= THREADS / 2) half_wait<14, THREADS>();
#pragma unroll
      for (int g = 0; g < S::G1; ++g)
#pragma unroll
        for (int qp = 0; qp < S::H1; ++qp)
        {
          const int sigma = qp * S::D + tr + S::TPR * g;
          v[g * S::H1 + qp] = ld_slot<CL>(peer[SlotMap<S>::owner(sigma)] + 16u * swz_(SlotMap<S>::local(sigma, rho)));
        }
      if constexpr (S::STAGGER)
        if (t < THREADS / 2) half_arrive<14, THREADS>();
    }
#pragma unroll
    for (int g = 0; g < S::G1; ++g)
    {
      const int n = tr + S::TPR * g;
      cpair z[S::H1];
      if constexpr (S::NS > 1)
      {
#pragma unroll
        for (int qp = 0; qp < S::H1; ++qp)
          z[qp] = (EPTW == 64) ? cp_rot2w<+1>(cp_mul4c(cp_from4(v[g * S::H1 + qp]), tw1[qp]), (g * 2 * qp) & 63,
                                              (g * (2 * qp + 1)) & 63)
                               : cp_rot2<+1>(cp_mul4c(cp_from4(v[g * S::H1 + qp]), tw1[qp]), (g * 2 * qp) & 31,
                                             (g * (2 * qp + 1)) & 31);
      }
      else
      {
        // single stage: forward outputs are still in c in bit-reversed order
#pragma unroll
        for (int qp = 0; qp < S::H1; ++qp) z[qp] = c[g * S::H1 + bitrev(qp, LH1)];
      }
      DifNet<S::H1, +1>::run(z);  // z[i] = (A_r, B_r) with r = bitrev(i)
#pragma unroll
      for (int i = 0; i < S::H1; ++i)
      {
        const int r = bitrev(i, LH1);
        const int k = r * (32 / S::R1);
        const float wc = c32(k), ws = s32(k);  // conjugate direction: exp(+2 pi i r / R1)
        float ar = z[i].re.x, ai = z[i].im.x, br = z[i].re.y, bi = z[i].im.y;
        float tr_, ti_;
        if (k == 0) { tr_ = br; ti_ = bi; }
        else if (k == 8) { tr_ = -bi; ti_ = br; }
        else { tr_ = fmaf(br, wc, -bi * ws); ti_ = fmaf(br, ws, bi * wc); }
        if constexpr (CHIRP)
        {
          // only the first n_out samples of the work row are wanted
          const int c0 = tr + S::TPR * g + S::D * r, c1 = c0 + S::D * S::H1;
          const float2 v0 = make_float2(ar + tr_, ai + ti_), v1 = make_float2(ar - tr_, ai - ti_);
          // multiplier loads stay next to their use (volatile), not hoisted
          if (active && c0 < a.n_out)
            dst_t[S::TPR * g + S::D * r] = a.cout ? c_mul(v0, ldv2(a.cout + c0)) : v0;
          if (active && c1 < a.n_out)
            dst_t[S::TPR * g + S::D * (r + S::H1)] = a.cout ? c_mul(v1, ldv2(a.cout + c1)) : v1;
        }
        else if (active)
        {
          dst_t[S::TPR * g + S::D * r] = make_float2(ar + tr_, ai + ti_);
          dst_t[S::TPR * g + S::D * (r + S::H1)] = make_float2(ar - tr_, ai - ti_);
        }
      }
    }
    if constexpr (CL) cluster_sync_relaxed();
  }
}

// Standalone launch: one tile per CTA, or per cluster of CS CTAs.
template <int LOGN, int MODE, int THREADS, int EPTW = 32>
__global__ void __launch_bounds__(THREADS, (Sched<LOGN, THREADS, EPTW>::MINB)) rows_kernel(RowArgs a)
{
  using S = Sched<LOGN, THREADS, EPTW>;
  if constexpr (S::CS > 1)
    row_tile<LOGN, MODE, THREADS, EPTW>(a, blockIdx.x / S::CS, (int)cg::this_cluster().block_rank(), 0, true);
  else
    row_tile<LOGN, MODE, THREADS, EPTW>(a, blockIdx.x, 0, 0, true);
}

}  // namespace fcb
