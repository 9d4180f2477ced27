// Device building blocks of the batched tridiagonal solve (sm_100a).
//
// Every kernel in this library solves a system
//     a[i] x[i-1] + b[i] x[i] + c[i] x[i+1] = d[i],   i = 0..N-1
// with the partition ("Thomas-PCR hybrid") method, in three steps that keep
// every element of the system in registers between its one HBM read and its
// one HBM write:
//
//  1. chunk elimination: a thread owns a chunk of M consecutive rows and
//     runs a modified Thomas sweep (forward, then backward) over it, so that
//     each interior row i reads  x_i = d_i - a_i x_first - c_i x_last  and
//     the chunk's first and last rows form two rows of a "reduced" system
//     that couples neighbouring chunks only;
//  2. reduced solve: the 2T reduced rows of a system's T chunks (held two
//     per thread, T a power of two <= 32, all in one warp segment) are
//     reduced to one row per thread and solved by parallel cyclic reduction
//     over warp shuffles;
//  3. substitution: every thread recovers its interior rows.
//
// T = 1 is the plain Thomas algorithm (one thread per system); M = 1 (see
// pcr_solve) is pure PCR. The reference's hybrid (scalar/src/cuda/
// trid_thomaspcr.hpp:121-235, trid_thomaspcr_small.h:134-253) follows the same
// mathematics; the data layout, the reduction to one row per lane and the
// register-resident state here are this library's own.
//
// a[0] and c[N-1] are treated as zero: the reference never lets them change
// the result (scalar/src/cpu/trid_cpu.cpp:321-352), so neither does this code.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace trid {

template <typename R> struct Limits;
template <> struct Limits<double> {
  static constexpr double max() { return 1.7976931348623157e308; }
};
template <> struct Limits<float> {
  static constexpr float max() { return 3.40282347e38f; }
};

// Correctly rounded reciprocal (CUDA intrinsics), used where the reference
// computes 1/pivot and multiplies (trid_cpu.cpp:321-334).
__device__ __forceinline__ double rcp(double x) { return __drcp_rn(x); }
__device__ __forceinline__ float rcp(float x) { return __frcp_rn(x); }

// FP64 reciprocal by Newton-Raphson iteration for 1/x, r <- r + r (1 - x r)
// (each step squares the relative error), from the hardware estimate of
// PTX rcp.approx.ftz.f64. Two steps take the estimate to within one unit in
// the last place (checked against 1/x on the GPU), in fewer instructions
// than the correctly rounded form; the contiguous kernels, whose per-row work
// is issue-bound, use it. A zero (or subnormal) x gives an infinite estimate
// and a NaN result, which finite_rcp reports as a zero pivot. In FP32 the
// estimate rcp.approx.ftz.f32 is itself within one ulp and is used as it is
// (a zero or subnormal x gives infinity).
__device__ __forceinline__ double rcp_nr(double x) {
  double r;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
  double e = fma(-x, r, 1.0);
  r = fma(r, e, r);
  e = fma(-x, r, 1.0);
  return fma(r, e, r);
}
__device__ __forceinline__ float rcp_nr(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// rcp_nr when NR, else rcp
template <bool NR, typename R> __device__ __forceinline__ R rcp_sel(R x) {
  if constexpr (NR)
    return rcp_nr(x);
  else
    return rcp(x);
}

// True when r is neither infinite nor NaN: a zero pivot gives an infinite
// reciprocal, a NaN pivot a NaN one.
template <typename R> __device__ __forceinline__ bool finite_rcp(R r) {
  return fabs(r) <= Limits<R>::max();
}

// The same check as one FMA per pivot, for sweeps whose per-row work is
// issue-bound: r * 0 is a zero for a finite reciprocal and NaN for an
// infinite or NaN one, so `acc` (starting at 0) stays finite until a pivot
// is zero or NaN; acc != acc at the end is the verdict.
template <typename R> __device__ __forceinline__ void pivot_acc(R &acc, R r) { acc = fma(r, R(0), acc); }

constexpr unsigned FULL_MASK = 0xffffffffu;

template <typename R> __device__ __forceinline__ R shfl_up(R v, int s, int w) {
  return __shfl_up_sync(FULL_MASK, v, s, w);
}
template <typename R> __device__ __forceinline__ R shfl_down(R v, int s, int w) {
  return __shfl_down_sync(FULL_MASK, v, s, w);
}
template <typename R> __device__ __forceinline__ R shfl_idx(R v, int l, int w) {
  return __shfl_sync(FULL_MASK, v, l, w);
}

// One reduced row with a unit diagonal:  A x_left + x + C x_right = D.
template <typename R> struct Row {
  R A, C, D;
};

// Step 1, forward half. On entry a,b,c,d hold the chunk's rows (identity
// rows a=c=d=0, b=1 past the end of the system). On exit rows 0 and 1 are
// scaled to a unit diagonal and rows i >= 2 read
//     a_i x_0 + x_i + c_i x_{i+1} = d_i
// (x_0 the chunk's first unknown). b is consumed.
// NR: pivots inverted with rcp_nr instead of rcp.
template <typename R, int M, bool NR = false>
__device__ __forceinline__ void chunk_forward(R (&a)[M], const R (&b)[M], R (&c)[M],
                                              R (&d)[M], bool &bad) {
#pragma unroll
  for (int i = 0; i < (M < 2 ? M : 2); ++i) {
    R r = rcp_sel<NR>(b[i]);
    bad |= !finite_rcp(r);
    a[i] *= r;
    c[i] *= r;
    d[i] *= r;
  }
#pragma unroll
  for (int i = 2; i < M; ++i) {
    R r = rcp_sel<NR>(b[i] - a[i] * c[i - 1]);
    bad |= !finite_rcp(r);
    d[i] = r * (d[i] - a[i] * d[i - 1]);
    a[i] = -r * a[i] * a[i - 1];
    c[i] = r * c[i];
  }
}

// Step 1, backward half. On exit interior rows 1..M-2 read
//     a_i x_0 + x_i + c_i x_{M-1} = d_i,
// row 0 reads  a_0 x_{prev last} + x_0 + c_0 x_{M-1} = d_0  (the chunk's top
// reduced row) and row M-1, untouched, reads
//     a_{M-1} x_0 + x_{M-1} + c_{M-1} x_{next first} = d_{M-1}
// (its bottom reduced row). For M == 2 both rows are already in that form.
template <typename R, int M, bool NR = false>
__device__ __forceinline__ void chunk_backward(R (&a)[M], R (&c)[M], R (&d)[M], bool &bad) {
#pragma unroll
  for (int i = M - 3; i >= 1; --i) {
    d[i] = d[i] - c[i] * d[i + 1];
    a[i] = a[i] - c[i] * a[i + 1];
    c[i] = -c[i] * c[i + 1];
  }
  if (M >= 3) {
    R r = rcp_sel<NR>(R(1) - c[0] * a[1]);
    bad |= !finite_rcp(r);
    d[0] = r * (d[0] - c[0] * d[1]);
    a[0] = r * a[0];
    c[0] = -r * c[0] * c[1];
  }
}

// Step 2. Lane t (0 <= t < T) of a segment of T consecutive lanes holds the
// top row (first unknown y_t) and the bottom row (last unknown z_t) of chunk
// t of one system:
//     top:    A0 z_{t-1} + y_t + C0 z_t     = D0
//     bottom: A1 y_t     + z_t + C1 y_{t+1} = D1
// Substituting the bottom rows of lanes t-1 and t into the top row leaves a
// tridiagonal system in y alone, one row per lane, which PCR solves in
// log2(T) shuffle steps; z_t then follows from the bottom row.
// Every lane of the warp must call this with the same T (a power of two).
template <typename R>
__device__ __forceinline__ void reduced_solve(const Row<R> &top, const Row<R> &bot, int t, int T,
                                              R &y, R &z, bool &bad) {
  R pA = shfl_up(bot.A, 1, T);
  R pC = shfl_up(bot.C, 1, T);
  R pD = shfl_up(bot.D, 1, T);
  if (t == 0) {
    pA = R(0);
    pC = R(0);
    pD = R(0);
  }
  R al = -top.A * pA;
  R be = R(1) - top.A * pC - top.C * bot.A;
  R ga = -top.C * bot.C;
  R de = top.D - top.A * pD - top.C * bot.D;
  R r = rcp(be);
  bad |= !finite_rcp(r);
  al *= r;
  ga *= r;
  de *= r;
  for (int s = 1; s < T; s <<= 1) {
    R al_l = shfl_up(al, s, T), ga_l = shfl_up(ga, s, T), de_l = shfl_up(de, s, T);
    R al_r = shfl_down(al, s, T), ga_r = shfl_down(ga, s, T), de_r = shfl_down(de, s, T);
    if (t < s) {
      al_l = R(0);
      ga_l = R(0);
      de_l = R(0);
    }
    if (t + s >= T) {
      al_r = R(0);
      ga_r = R(0);
      de_r = R(0);
    }
    R b2 = R(1) - al * ga_l - ga * al_r;
    R d2 = de - al * de_l - ga * de_r;
    R a2 = -al * al_l;
    R g2 = -ga * ga_r;
    r = rcp(b2);
    bad |= !finite_rcp(r);
    al = a2 * r;
    ga = g2 * r;
    de = d2 * r;
  }
  y = de;
  R yn = shfl_down(y, 1, T);
  if (t == T - 1) yn = R(0);
  z = bot.D - bot.A * y - bot.C * yn;
}

// Step 3: x_i for the interior rows from the chunk's first (y) and last (z).
template <typename R, int M>
__device__ __forceinline__ void chunk_substitute(R (&a)[M], R (&c)[M], R (&d)[M], R y, R z) {
#pragma unroll
  for (int i = 1; i < M - 1; ++i) d[i] = d[i] - a[i] * y - c[i] * z;
  d[0] = y;
  if (M > 1) d[M - 1] = z;
}

// Pure PCR with one row per lane over a segment of T lanes (the M = 1
// family, for systems of at most 32 rows): rows past N are identity rows.
template <typename R>
__device__ __forceinline__ R pcr_solve(R a, R b, R c, R d, int t, int T, bool &bad) {
  R r = rcp(b);
  bad |= !finite_rcp(r);
  a *= r;
  c *= r;
  d *= r;
  for (int s = 1; s < T; s <<= 1) {
    R a_l = shfl_up(a, s, T), c_l = shfl_up(c, s, T), d_l = shfl_up(d, s, T);
    R a_r = shfl_down(a, s, T), c_r = shfl_down(c, s, T), d_r = shfl_down(d, s, T);
    if (t < s) {
      a_l = R(0);
      c_l = R(0);
      d_l = R(0);
    }
    if (t + s >= T) {
      a_r = R(0);
      c_r = R(0);
      d_r = R(0);
    }
    R b2 = R(1) - a * c_l - c * a_r;
    R d2 = d - a * d_l - c * d_r;
    R a2 = -a * a_l;
    R c2 = -c * c_r;
    r = rcp(b2);
    bad |= !finite_rcp(r);
    a = a2 * r;
    c = c2 * r;
    d = d2 * r;
  }
  return d;
}

// Report of a zero or non-finite pivot into a host-mapped word. A plain
// store: every writer stores the same value, and atomics on mapped host
// memory are not guaranteed across the bus.
__device__ __forceinline__ void report_bad_pivot(bool bad, unsigned *flag) {
  if (bad && flag) *reinterpret_cast<volatile unsigned *>(flag) = 1u;
}

// Asynchronous global -> shared copy of one 16-byte unit (cp.async, bypassing
// registers and L1); `bytes` < 16 reads only that many bytes and zero-fills
// the rest. Both addresses must be 16-byte aligned.
__device__ __forceinline__ void cp_async16(void *smem_dst, const void *gmem_src, int bytes) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem_src), "r"(bytes)
               : "memory");
}
// Asynchronous copy of one element (4 or 8 bytes, naturally aligned).
template <typename R> __device__ __forceinline__ void cp_async_elem(R *smem_dst, const R *gmem_src) {
  static_assert(sizeof(R) == 4 || sizeof(R) == 8, "4- or 8-byte elements");
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
  if constexpr (sizeof(R) == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem_src) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}
// Closes the calling thread's current group of cp.async copies (possibly
// empty), and waits until at most N of its groups are still in flight.
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait_groups() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// 16-byte vector types for contiguous rows.
template <typename R> struct Vec16;
template <> struct Vec16<double> {
  using T = double2;
  static constexpr int n = 2;
};
template <> struct Vec16<float> {
  using T = float4;
  static constexpr int n = 4;
};

template <typename R, int M>
__device__ __forceinline__ void load_vec(const R *__restrict__ p, R (&v)[M]) {
  using V = typename Vec16<R>::T;
  constexpr int n = Vec16<R>::n;
  const V *q = reinterpret_cast<const V *>(p);
#pragma unroll
  for (int i = 0; i < M / n; ++i) {
    V x = __ldg(q + i);
    if constexpr (n == 2) {
      v[2 * i] = x.x;
      v[2 * i + 1] = x.y;
    } else {
      v[4 * i] = x.x;
      v[4 * i + 1] = x.y;
      v[4 * i + 2] = x.z;
      v[4 * i + 3] = x.w;
    }
  }
}

template <typename R, int M>
__device__ __forceinline__ void store_vec(R *__restrict__ p, const R (&v)[M]) {
  using V = typename Vec16<R>::T;
  constexpr int n = Vec16<R>::n;
  V *q = reinterpret_cast<V *>(p);
#pragma unroll
  for (int i = 0; i < M / n; ++i) {
    V x;
    if constexpr (n == 2) {
      x.x = v[2 * i];
      x.y = v[2 * i + 1];
    } else {
      x.x = v[4 * i];
      x.y = v[4 * i + 1];
      x.z = v[4 * i + 2];
      x.w = v[4 * i + 3];
    }
    q[i] = x;
  }
}

}  // namespace trid
