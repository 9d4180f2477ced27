// FP32-solve tridiagonal batch with FP64 iterative refinement, in two forms:
//
//  * tridDmtsvStridedBatchMixed: the coefficients a, b, c are stored in FP32
//    and taken exactly, promoted to FP64, as the system to solve;
//  * tridDmtsvStridedBatchRefine: the system is specified in FP64 (a, b, c
//    are FP64 arrays); the FP32 factorisation is formed from their rounded
//    values, and the residual uses the FP64 values, so refinement converges
//    to the solution of the FP64 system itself.
//
// In both, d and x are FP64:
//
//   x = 0;  repeat:  r = d - T x       (FP64: FP32 coefficients times FP64 x)
//                    solve T dx = r    (FP32: the partition hybrid)
//                    x += dx           (FP64)
//   until max|dx| <= tol * max|x| over the system, or max_iters solves.
//
// Everything after the one read of a, b, c, d happens on chip: the
// coefficients stay in shared memory (contiguous systems) or registers
// (strided), d and x in registers, and x is written once. With FP32
// coefficients a call moves 3*4 + 8 + 8 = 28 bytes per element against 40
// for the plain FP64 solve; with FP64 coefficients it moves the same 40.
// The reference has no mixed-precision entry point; this is an extension
// (include/tridsolver_b200.h).
#include <cuda_runtime.h>

#include <cstring>

#include "trid_internal.h"
#include "tridsolver_b200.h"

namespace trid {

// CT: the coefficients' storage type (float: the FP32 values are the system;
// double: the FP64 values are, and only the factorisation is rounded).
template <typename CT> struct MixedArgsT {
  const CT *a, *b, *c;
  double *d;  // right-hand side in, x out
  int N;
  long long nsys, n0, st0, st1, stride;
  int max_iters;
  double tol;
  unsigned *flag;
};
using MixedArgs = MixedArgsT<float>;

// Per-call statistics: the largest iteration count and the largest final
// relative correction max|dx|/max|x| over all systems (as ordered bits; both
// are non-negative so their bit patterns order like the values).
struct MixedStats {
  unsigned iters;
  unsigned pad;
  unsigned long long corr_bits;
};
static __device__ MixedStats g_mixed_stats;

// Only values above the current maximum are sent as atomics, so the one
// shared word is mostly read, not contended.
__device__ __forceinline__ void mixed_report(int iters, double rel) {
  if ((unsigned)iters > *reinterpret_cast<volatile unsigned *>(&g_mixed_stats.iters))
    atomicMax(&g_mixed_stats.iters, (unsigned)iters);
  const unsigned long long bits = (unsigned long long)__double_as_longlong(rel);
  if (bits > *reinterpret_cast<volatile unsigned long long *>(&g_mixed_stats.corr_bits))
    atomicMax(&g_mixed_stats.corr_bits, bits);
}

// Estimated relative error of x after a correction of max-norm dmax, the
// previous correction having been dprev (0 before the first refinement):
// refinement contracts the error by about rho = dmax / dprev per pass, so
// the error left is about rho / (1 - rho) * dmax (the a-posteriori bound of
// a contraction). Without a usable rho the correction itself is the
// estimate, as is any rho >= 1/2.
__device__ __forceinline__ double mixed_error_estimate(float dmax, float dprev, double xmax) {
  if (!(xmax > 0.0)) return 0.0;
  double est = (double)dmax;
  if (dprev > 0.f && dmax < 0.5f * dprev) {
    const double rho = (double)dmax / (double)dprev;
    est = est * rho / (1.0 - rho);
  }
  return est / xmax;
}

template <typename CT>
__device__ __forceinline__ long long mixed_base(const MixedArgsT<CT> &p, long long s) {
  const long long i1 = s / p.n0;
  return (s - i1 * p.n0) * p.st0 + i1 * p.st1;
}

// Shared-memory chunk rows without padding: lane l's row is U = M*sizeof/16
// units of 16 bytes, and unit u is stored at position u ^ swz(l), so the
// 16-byte accesses of any 8 consecutive lanes to their own rows (the width of
// one shared-memory wavefront) fall on 8 distinct bank groups.
template <typename R, int M> struct Swz {
  static constexpr int V = 16 / (int)sizeof(R);  // elements per unit
  static constexpr int U = M / V;                 // units per row
  static_assert(U >= 1 && (U & (U - 1)) == 0 && U <= 8, "row of 1..8 units");
  __device__ static __forceinline__ int swz(int l) { return ((l * U) >> 3) & (U - 1); }
  // element offset of element e of the system (lane e / M) in the tile
  __device__ static __forceinline__ int off(int e) {
    const int l = e / M, u = (e % M) / V;
    return (l * U + (u ^ swz(l))) * V + e % V;
  }
  __device__ static __forceinline__ int unit(int l, int u) { return (l * U + (u ^ swz(l))) * V; }
};

template <typename R, int M>
__device__ __forceinline__ void lds_swz(const R *tile, int l, R (&v)[M]) {
  using S = Swz<R, M>;
  using Vt = typename Vec16<R>::T;
#pragma unroll
  for (int u = 0; u < S::U; ++u) {
    const Vt x = *reinterpret_cast<const Vt *>(tile + S::unit(l, u));
    if constexpr (S::V == 2) {
      v[2 * u] = x.x;
      v[2 * u + 1] = x.y;
    } else {
      v[4 * u] = x.x;
      v[4 * u + 1] = x.y;
      v[4 * u + 2] = x.z;
      v[4 * u + 3] = x.w;
    }
  }
}

template <typename R, int M>
__device__ __forceinline__ void sts_swz(R *tile, int l, const R (&v)[M]) {
  using S = Swz<R, M>;
  using Vt = typename Vec16<R>::T;
#pragma unroll
  for (int u = 0; u < S::U; ++u) {
    Vt x;
    if constexpr (S::V == 2) {
      x.x = v[2 * u];
      x.y = v[2 * u + 1];
    } else {
      x.x = v[4 * u];
      x.y = v[4 * u + 1];
      x.z = v[4 * u + 2];
      x.w = v[4 * u + 3];
    }
    *reinterpret_cast<Vt *>(tile + S::unit(l, u)) = x;
  }
}

// Approximate FP32 reciprocal (rcp.approx, within one ulp): the FP32
// factorisation only has to be good enough for refinement to converge.
__device__ __forceinline__ float rcp_fast(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// FP32 solve of T dx = r for one chunk of M rows given FP32 coefficients
// (identity rows past the system end are already in place): chunk
// elimination, reduced solve over a T-lane segment, substitution.
template <int M>
__device__ __forceinline__ void fp32_chunk_solve(float (&wa)[M], float (&wb)[M], float (&wc)[M],
                                                 float (&wd)[M], int t, int T, bool &bad) {
  chunk_forward<float, M>(wa, wb, wc, wd, bad);
  chunk_backward<float, M>(wa, wc, wd, bad);
  float y, z;
  reduced_solve<float>(Row<float>{wa[0], wc[0], wd[0]}, Row<float>{wa[M - 1], wc[M - 1], wd[M - 1]},
                       t, T, y, z, bad);
  chunk_substitute<float, M>(wa, wc, wd, y, z);
}

// Four rows (4q .. 4q+3) of a swizzled coefficient tile as FP64.
template <typename CT, int M>
__device__ __forceinline__ void lds4_swz(const CT *tile, int l, int q, double (&v)[4]) {
  using S = Swz<CT, M>;
  if constexpr (sizeof(CT) == 4) {
    const float4 x = *reinterpret_cast<const float4 *>(tile + S::unit(l, q));
    v[0] = x.x;
    v[1] = x.y;
    v[2] = x.z;
    v[3] = x.w;
  } else {
    const double2 x = *reinterpret_cast<const double2 *>(tile + S::unit(l, 2 * q));
    const double2 y = *reinterpret_cast<const double2 *>(tile + S::unit(l, 2 * q + 1));
    v[0] = x.x;
    v[1] = x.y;
    v[2] = y.x;
    v[3] = y.y;
  }
}

// A lane's coefficient row from its tile with the fix-ups of the first pass
// (identity rows past the end, a[0] = 0, c[N-1] = 0: kind 0 = a, 1 = b,
// 2 = c) written back when the chunk needs them, rounded to FP32.
template <typename CT, int M>
__device__ __forceinline__ void load_fixed_row(CT *tile, int lane, int row0, int N, int kind,
                                               float (&w)[M]) {
  CT v[M];
  lds_swz<CT, M>(tile, lane, v);
  if (row0 == 0 || row0 + M >= N) {
#pragma unroll
    for (int i = 0; i < M; ++i) {
      const int row = row0 + i;
      if (row >= N) v[i] = kind == 1 ? CT(1) : CT(0);
      if (kind == 0 && row == 0) v[i] = CT(0);
      if (kind == 2 && row == N - 1) v[i] = CT(0);
    }
    sts_swz<CT, M>(tile, lane, v);
  }
#pragma unroll
  for (int i = 0; i < M; ++i) w[i] = (float)v[i];
}

// ---------------------------------------------------------------------------
// Contiguous systems (stride 1), one warp per system, 16-byte aligned starts.
// The warp stages a, b, c (as stored: FP32 or FP64) and d (FP64) through
// shared memory with coalesced 16-byte cp.async copies into swizzled,
// unpadded rows (a lane's 16-byte reads of its own row are conflict-free).
//
// The FP32 solve is factored once: the first pass records, per row, the
// pivot reciprocal r and the forward-eliminated a' (shared memory, next to
// the fixed coefficients; c' = r c is recomputed), and per lane the reduced
// system's PCR coefficients (registers). Every refinement pass then only applies them to
// the FP32-rounded FP64 residual:
//   forward   d'_i = r_i (d_i - a_i d'_{i-1})
//   backward  the chunk's top reduced right-hand side (one running value)
//   reduced   de <- (de - al_l de_left - ga_l de_right) r_l per PCR level
//   back-substitution  dx_i = d'_i - a'_i dx_first - c'_i dx_{i+1}
// which is a few FP32 operations per row instead of a fresh elimination.
// The residual uses the coefficients as stored (exactly, in FP64).
template <int M, typename CT>
__global__ void __launch_bounds__(32, 14) mixed_contig_kernel(const MixedArgsT<CT> p) {
  static_assert(M % 4 == 0 && M >= 8, "rows per lane");
  using SC = Swz<CT, M>;
  using SF = Swz<float, M>;
  using SD = Swz<double, M>;
  constexpr int BF = 32 * M;    // elements per tile
  constexpr int VC = 16 / (int)sizeof(CT);  // coefficients per 16-byte unit
  // tiles: a, b, c (as stored, fixed), then FP32 r and a' (c' = r c is
  // recomputed), then FP64 d
  constexpr int PER_WARP = 3 * BF * (int)sizeof(CT) + 2 * BF * 4 + BF * 8;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  unsigned char *wbase = smem_raw + (threadIdx.x >> 5) * PER_WARP;
  CT *ta = reinterpret_cast<CT *>(wbase);
  CT *tb = ta + BF;
  CT *tc = tb + BF;
  float *tr = reinterpret_cast<float *>(tc + BF);
  float *tfa = tr + BF;
  double *td = reinterpret_cast<double *>(tfa + BF);
  const int lane = threadIdx.x & 31;
  const long long s = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (s >= p.nsys) return;  // uniform per warp
  const long long base = mixed_base(p, s);
  const int N = p.N;
  const bool full = N == 32 * M;  // every lane's chunk full: unrolled copies
  if (full) {
#pragma unroll
    for (int k = 0; k < M / VC; ++k) {
      const int e = VC * (lane + 32 * k);
      const int o = SC::off(e);
      cp_async16(ta + o, p.a + base + e, 16);
      cp_async16(tb + o, p.b + base + e, 16);
      cp_async16(tc + o, p.c + base + e, 16);
    }
#pragma unroll
    for (int k = 0; k < M / 2; ++k) {
      const int e = 2 * (lane + 32 * k);
      cp_async16(td + SD::off(e), p.d + base + e, 16);
    }
  } else {
    const int nu = (N + VC - 1) / VC;  // coefficient units
    for (int un = lane; un < nu; un += 32) {
      const int e = un * VC;
      const int left = (N - e) >= VC ? 16 : (N - e) * (int)sizeof(CT);
      const int o = SC::off(e);
      cp_async16(ta + o, p.a + base + e, left);
      cp_async16(tb + o, p.b + base + e, left);
      cp_async16(tc + o, p.c + base + e, left);
    }
    const int nud = (N + 1) / 2;  // FP64 units of 2
    for (int un = lane; un < nud; un += 32) {
      const int e = un * 2;
      cp_async16(td + SD::off(e), p.d + base + e, (N - e) >= 2 ? 16 : 8);
    }
  }
  cp_async_wait_all();
  __syncwarp();

  const int row0 = lane * M;
  bool bad = false;

  // ---- first pass: fix the coefficients (identity rows past the end, a[0]
  // and c[N-1] zero), factor, and solve T x = (float)d
  float wa[M], wb[M], wc[M], wd[M];
  load_fixed_row<CT, M>(ta, lane, row0, N, 0, wa);
  load_fixed_row<CT, M>(tb, lane, row0, N, 1, wb);
  load_fixed_row<CT, M>(tc, lane, row0, N, 2, wc);
  double dd[M];
  lds_swz<double, M>(td, lane, dd);
  if (row0 + M >= N) {  // chunks holding rows past the end
#pragma unroll
    for (int i = 0; i < M; ++i)
      if (row0 + i >= N) dd[i] = 0.0;
    sts_swz<double, M>(td, lane, dd);
  }
#pragma unroll
  for (int i = 0; i < M; ++i) wd[i] = (float)dd[i];
  float rr[M];
  float psum = 0.f;  // sum of |pivot reciprocals|: not finite iff some pivot is 0 or NaN
#pragma unroll
  for (int i = 0; i < M; ++i) {
    if (i < 2) {
      const float r = rcp_fast(wb[i]);
      psum += fabsf(r);
      rr[i] = r;
      wa[i] *= r;
      wc[i] *= r;
      wd[i] *= r;
    } else {
      const float r = rcp_fast(wb[i] - wa[i] * wc[i - 1]);
      psum += fabsf(r);
      rr[i] = r;
      wd[i] = r * (wd[i] - wa[i] * wd[i - 1]);
      wa[i] = -r * wa[i] * wa[i - 1];
      wc[i] = r * wc[i];
    }
  }
  sts_swz<float, M>(tr, lane, rr);
  sts_swz<float, M>(tfa, lane, wa);
  // backward recursion (matrix part once, right-hand side each pass)
  float A = wa[M - 2], C = wc[M - 2], Dd = wd[M - 2];
#pragma unroll
  for (int j = M - 3; j >= 1; --j) {
    Dd = wd[j] - wc[j] * Dd;
    A = wa[j] - wc[j] * A;
    C = -wc[j] * C;
  }
  const float r0 = rcp_fast(1.f - wc[0] * A);
  psum += fabsf(r0);
  const float c0 = wc[0];
  const float tA = r0 * wa[0], tC = -r0 * c0 * C;
  const float bA = wa[M - 1], bC = wc[M - 1];
  // reduced system: form it, recording the PCR coefficients of every level
  constexpr int L = 5;  // log2(32)
  float cal[L], cga[L], crl[L];
  float rbe;
  float y, z;
  {
    float pA = __shfl_up_sync(FULL_MASK, bA, 1), pC = __shfl_up_sync(FULL_MASK, bC, 1);
    if (lane == 0) pA = pC = 0.f;
    float al = -tA * pA;
    const float be = 1.f - tA * pC - tC * bA;
    float ga = -tC * bC;
    rbe = rcp_fast(be);
    psum += fabsf(rbe);
    al *= rbe;
    ga *= rbe;
#pragma unroll
    for (int l = 0; l < L; ++l) {
      const int sft = 1 << l;
      float al_l = __shfl_up_sync(FULL_MASK, al, sft), ga_l = __shfl_up_sync(FULL_MASK, ga, sft);
      float al_r = __shfl_down_sync(FULL_MASK, al, sft), ga_r = __shfl_down_sync(FULL_MASK, ga, sft);
      if (lane < sft) al_l = ga_l = 0.f;
      if (lane + sft >= 32) al_r = ga_r = 0.f;
      const float r = rcp_fast(1.f - al * ga_l - ga * al_r);
      psum += fabsf(r);
      cal[l] = al;
      cga[l] = ga;
      crl[l] = r;
      al = -al * al_l * r;
      ga = -ga * ga_r * r;
    }
  }
  // right-hand-side part of the reduced solve and the back-substitution,
  // shared by every pass; wd holds d' (forward-eliminated right-hand side)
  auto finish = [&](const float (&fa)[M], const float (&fc)[M], float topD, float (&dx)[M]) {
    const float botD = wd[M - 1];
    float pD = __shfl_up_sync(FULL_MASK, botD, 1);
    if (lane == 0) pD = 0.f;
    float de = (topD - tA * pD - tC * botD) * rbe;
#pragma unroll
    for (int l = 0; l < L; ++l) {
      const int sft = 1 << l;
      float de_l = __shfl_up_sync(FULL_MASK, de, sft);
      float de_r = __shfl_down_sync(FULL_MASK, de, sft);
      if (lane < sft) de_l = 0.f;
      if (lane + sft >= 32) de_r = 0.f;
      de = (de - cal[l] * de_l - cga[l] * de_r) * crl[l];
    }
    y = de;
    float yn = __shfl_down_sync(FULL_MASK, y, 1);
    if (lane == 31) yn = 0.f;
    z = botD - bA * y - bC * yn;
    float x = z;
    dx[M - 1] = z;
#pragma unroll
    for (int j = M - 2; j >= 1; --j) {
      x = wd[j] - fa[j] * y - fc[j] * x;
      dx[j] = x;
    }
    dx[0] = y;
  };
  bad |= !(psum <= 3.4e38f);
  double x64[M];
  {
    float dx[M];
    finish(wa, wc, r0 * (wd[0] - c0 * Dd), dx);
#pragma unroll
    for (int i = 0; i < M; ++i) x64[i] = (double)dx[i];
  }
  // max|dx| of this pass, and the estimated relative error of x after it
  float dprev = 0.f;
  auto converged = [&](const float (&dx)[M], double &est) {
    float dmax = 0.f;
    double xm64 = 0.0;
#pragma unroll
    for (int i = 0; i < M; ++i) {
      dmax = fmaxf(dmax, fabsf(dx[i]));
      xm64 = fmax(xm64, fabs(x64[i]));
    }
    float xmax = (float)fmin(xm64, 3.0e38);  // a norm for the stopping test: FP32 is plenty
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      dmax = fmaxf(dmax, __shfl_xor_sync(FULL_MASK, dmax, o));
      xmax = fmaxf(xmax, __shfl_xor_sync(FULL_MASK, xmax, o));
    }
    est = mixed_error_estimate(dmax, dprev, (double)xmax);
    dprev = dmax;
  };
  int it = 1;
  double rel = 0.0;
  {
    // the first correction is x itself
    float dx0[M];
#pragma unroll
    for (int i = 0; i < M; ++i) dx0[i] = (float)x64[i];
    converged(dx0, rel);
  }

  // ---- refinement passes
  while (rel > p.tol && it < p.max_iters) {  // uniform across the warp
    // FP64 residual r = d - T x, rounded to FP32, and the forward sweep
    double xl = __shfl_up_sync(FULL_MASK, x64[M - 1], 1);
    double xr = __shfl_down_sync(FULL_MASK, x64[0], 1);
    if (lane == 0) xl = 0.0;
    if (lane == 31) xr = 0.0;
#pragma unroll
    for (int q = 0; q < M / 4; ++q) {
      double av[4], bv[4], cv[4];
      lds4_swz<CT, M>(ta, lane, q, av);
      lds4_swz<CT, M>(tb, lane, q, bv);
      lds4_swz<CT, M>(tc, lane, q, cv);
      const float4 r4 = *reinterpret_cast<const float4 *>(tr + SF::unit(lane, q));
      const double2 d01 = *reinterpret_cast<const double2 *>(td + SD::unit(lane, 2 * q));
      const double2 d23 = *reinterpret_cast<const double2 *>(td + SD::unit(lane, 2 * q + 1));
      const float rv[4] = {r4.x, r4.y, r4.z, r4.w};
      const double dv[4] = {d01.x, d01.y, d23.x, d23.y};
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const int i = 4 * q + k;
        const double xm = i == 0 ? xl : x64[i - 1];
        const double xp = i == M - 1 ? xr : x64[i + 1];
        // FP64 residual with the coefficients as stored
        double res = dv[k] - bv[k] * x64[i];
        res = fma(-av[k], xm, res);
        res = fma(-cv[k], xp, res);
        const float rf = (float)res;
        // the factorisation's FP32 a
        const float af = (float)av[k];
        wd[i] = i < 2 ? rv[k] * rf : rv[k] * (rf - af * wd[i - 1]);
      }
    }
    float fa[M], fc[M], rr2[M];
    lds_swz<float, M>(tfa, lane, fa);
    lds_swz<float, M>(tr, lane, rr2);
    {
      CT cs[M];
      lds_swz<CT, M>(tc, lane, cs);
#pragma unroll
      for (int j = 0; j < M; ++j) fc[j] = (float)cs[j] * rr2[j];
    }
    float D2 = wd[M - 2];
#pragma unroll
    for (int j = M - 3; j >= 1; --j) D2 = wd[j] - fc[j] * D2;
    float dx[M];
    finish(fa, fc, r0 * (wd[0] - c0 * D2), dx);
#pragma unroll
    for (int i = 0; i < M; ++i) x64[i] += (double)dx[i];
    converged(dx, rel);
    ++it;
  }

  // x out through the FP64 tile (own row), then coalesced 16-byte stores
  sts_swz<double, M>(td, lane, x64);
  __syncwarp();
  if (full) {
#pragma unroll
    for (int k = 0; k < M / 2; ++k) {
      const int e = 2 * (lane + 32 * k);
      *reinterpret_cast<double2 *>(p.d + base + e) = *reinterpret_cast<const double2 *>(td + SD::off(e));
    }
  } else {
    const int nud = (N + 1) / 2;
    for (int un = lane; un < nud; un += 32) {
      const int e = un * 2;
      const double2 v = *reinterpret_cast<const double2 *>(td + SD::off(e));
      if (e + 2 <= N) {
        *reinterpret_cast<double2 *>(p.d + base + e) = v;
      } else {
        p.d[base + e] = v.x;
      }
    }
  }
  if (lane == 0) mixed_report(it, rel);
  report_bad_pivot(bad, p.flag);
}

// ---------------------------------------------------------------------------
// Strided systems: block = W neighbouring systems x T chunks, thread (s, t) =
// (tid % W, tid / W), as strided_kernel. The FP32 coefficients of the chunk
// stay in registers; neighbouring chunks trade their first and last x
// through shared memory for the residual, and every FP32 solve uses the
// block-level reduced solve. The block iterates until all its systems have
// converged (or max_iters), so the loop is uniform across the block.
template <int M, int KR, typename CT>
__global__ void __launch_bounds__(KR >= 4 ? 512 : 256)
    mixed_strided_kernel(const MixedArgsT<CT> p, int T, int W, long long ngx) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int TW = T * W;
  double *xf = reinterpret_cast<double *>(smem_raw);  // first x of chunk (t, s)
  double *xl = xf + TW;                                // last x of chunk (t, s)
  double *cd = xl + TW;                                // max |dx| of chunk (t, s)
  double *cx = cd + TW;                                // max |x| of chunk (t, s)
  double *relv = cx + TW;                              // per system
  double *dpv = relv + W;                              // previous max |dx|, per system
  int *conv = reinterpret_cast<int *>(dpv + W);
  float *red = reinterpret_cast<float *>(conv + W + (W & 1));
  const int tid = threadIdx.x;
  const int s = tid % W;
  const int t = tid / W;
  const long long gx = blockIdx.x % ngx;
  const long long i1 = blockIdx.x / ngx;
  const long long i0 = gx * W + s;
  const bool active = i0 < p.n0;
  const long long base = i0 * p.st0 + i1 * p.st1;
  const int N = p.N;
  const int row0 = t * M;
  CT ra[M], rb[M], rc[M];  // the coefficients as stored
  double d64[M], x64[M];
#pragma unroll
  for (int i = 0; i < M; ++i) {
    const int row = row0 + i;
    if (active && row < N) {
      const long long o = base + (long long)row * p.stride;
      ra[i] = row == 0 ? CT(0) : __ldg(p.a + o);
      rb[i] = __ldg(p.b + o);
      rc[i] = row == N - 1 ? CT(0) : __ldg(p.c + o);
      d64[i] = p.d[o];
    } else {
      ra[i] = CT(0);
      rb[i] = CT(1);
      rc[i] = CT(0);
      d64[i] = 0.0;
    }
    x64[i] = 0.0;
  }
  bool bad = false;
  int it = 0;
  const int k = t * W + s;
  for (;;) {
    float wa[M], wb[M], wc[M], wd[M];
#pragma unroll
    for (int i = 0; i < M; ++i) {
      wa[i] = (float)ra[i];
      wb[i] = (float)rb[i];
      wc[i] = (float)rc[i];
    }
    if (it == 0) {
#pragma unroll
      for (int i = 0; i < M; ++i) wd[i] = (float)d64[i];
    } else {
      xf[k] = x64[0];
      xl[k] = x64[M - 1];
      __syncthreads();
      const double xm0 = t > 0 ? xl[k - W] : 0.0;
      const double xpM = t < T - 1 ? xf[k + W] : 0.0;
#pragma unroll
      for (int i = 0; i < M; ++i) {
        const double xm = i == 0 ? xm0 : x64[i - 1];
        const double xp = i == M - 1 ? xpM : x64[i + 1];
        double r = d64[i] - (double)rb[i] * x64[i];
        r = fma(-(double)ra[i], xm, r);
        r = fma(-(double)rc[i], xp, r);
        wd[i] = (float)r;
      }
    }
    chunk_forward<float, M>(wa, wb, wc, wd, bad);
    chunk_backward<float, M>(wa, wc, wd, bad);
    float y, z;
    block_reduced_solve<float, KR>(red, Row<float>{wa[0], wc[0], wd[0]},
                                   Row<float>{wa[M - 1], wc[M - 1], wd[M - 1]}, s, t, T, W, y, z,
                                   bad);
    chunk_substitute<float, M>(wa, wc, wd, y, z);
    double dmax = 0.0, xmax = 0.0;
#pragma unroll
    for (int i = 0; i < M; ++i) {
      x64[i] += (double)wd[i];
      dmax = fmax(dmax, fabs((double)wd[i]));
      xmax = fmax(xmax, fabs(x64[i]));
    }
    cd[k] = dmax;
    cx[k] = xmax;
    __syncthreads();
    if (t == 0) {
      double dm = 0.0, xm = 0.0;
      for (int q = 0; q < T; ++q) {
        dm = fmax(dm, cd[q * W + s]);
        xm = fmax(xm, cx[q * W + s]);
      }
      const double rel = mixed_error_estimate((float)dm, it == 0 ? 0.f : (float)dpv[s], xm);
      dpv[s] = dm;
      relv[s] = rel;
      conv[s] = !(rel > p.tol);
    }
    __syncthreads();
    ++it;
    const int done = conv[s] || it >= p.max_iters;
    if (__syncthreads_and(done)) break;
  }
  if (active) {
#pragma unroll
    for (int i = 0; i < M; ++i) {
      const int row = row0 + i;
      if (row < N) p.d[base + (long long)row * p.stride] = x64[i];
    }
    if (t == 0) mixed_report(it, relv[s]);
  }
  report_bad_pivot(bad && active, p.flag);
}

// ---------------------------------------------------------------------------

// ---------------------------------------------------------------------------
// Direct FP64 solve of the promoted system for contiguous, 16-byte aligned
// systems (the automatic choice along x): contig_smem_kernel's staging with
// a, b, c kept as FP32 in shared memory (16-byte cp.async units of 4 values)
// and widened on the way into registers; d and x stay FP64. 28 bytes per
// element, no refinement, the FP64 solve of the promoted values.
template <int M>
__global__ void __launch_bounds__(128) contig_promoted_kernel(const MixedArgs p) {
  using LF = SmemLayout<float, M>;
  using LD = SmemLayout<double, M>;
  using Vd = typename Vec16<double>::T;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int PER_WARP = 3 * LF::BUF * 4 + LD::BUF * 8;  // bytes
  unsigned char *wbase = smem_raw + (threadIdx.x >> 5) * PER_WARP;
  float *fbuf = reinterpret_cast<float *>(wbase);                // a, b, c
  double *dbuf = reinterpret_cast<double *>(wbase + 3 * LF::BUF * 4);
  const int lane = threadIdx.x & 31;
  const long long s = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (s >= p.nsys) return;  // uniform per warp
  const long long i1 = s / p.n0;
  const long long base = (s - i1 * p.n0) * p.st0 + i1 * p.st1;
  const int N = p.N;
  const float *src[3] = {p.a + base, p.b + base, p.c + base};
  {
    const int nu = (N + LF::V - 1) / LF::V;
#pragma unroll
    for (int k = 0; k < 3; ++k)
      for (int un = lane; un < nu; un += 32) {
        const int e = un * LF::V;
        const int left = N - e;
        cp_async16(fbuf + k * LF::BUF + e + (e / M) * LF::V, src[k] + e,
                   (left >= LF::V ? LF::V : left) * 4);
      }
    const int nd = (N + LD::V - 1) / LD::V;
    for (int un = lane; un < nd; un += 32) {
      const int e = un * LD::V;
      const int left = N - e;
      cp_async16(dbuf + e + (e / M) * LD::V, p.d + base + e, (left >= LD::V ? LD::V : left) * 8);
    }
  }
  cp_async_wait_all();
  __syncwarp();
  const int row0 = lane * M;
  double ra[M], rb[M], rc[M], rd[M];
  {
    float fa[M];
    lds_row<float, M>(fbuf + 0 * LF::BUF + lane * LF::ROW, fa);
#pragma unroll
    for (int i = 0; i < M; ++i) ra[i] = fa[i];
    lds_row<float, M>(fbuf + 1 * LF::BUF + lane * LF::ROW, fa);
#pragma unroll
    for (int i = 0; i < M; ++i) rb[i] = fa[i];
    lds_row<float, M>(fbuf + 2 * LF::BUF + lane * LF::ROW, fa);
#pragma unroll
    for (int i = 0; i < M; ++i) rc[i] = fa[i];
  }
  lds_row<double, M>(dbuf + lane * LD::ROW, rd);
#pragma unroll
  for (int i = 0; i < M; ++i) {
    const int row = row0 + i;
    if (row >= N) {
      ra[i] = 0.0;
      rb[i] = 1.0;
      rc[i] = 0.0;
      rd[i] = 0.0;
    }
    if (row == N - 1) rc[i] = 0.0;
  }
  if (lane == 0) ra[0] = 0.0;
  bool bad = false;
  // the reciprocal of contig_smem_kernel, so the result is that kernel's
  chunk_forward<double, M, true>(ra, rb, rc, rd, bad);
  chunk_backward<double, M, true>(ra, rc, rd, bad);
  Row<double> top{ra[0], rc[0], rd[0]};
  Row<double> bot{ra[M - 1], rc[M - 1], rd[M - 1]};
  double y, z;
  reduced_solve<double>(top, bot, lane, 32, y, z, bad);
  chunk_substitute<double, M>(ra, rc, rd, y, z);
  __syncwarp();  // every lane has read its d row
  sts_row<double, M>(dbuf + lane * LD::ROW, rd);
  __syncwarp();
  double *dst = p.d + base;
  const int nd = (N + LD::V - 1) / LD::V;
  for (int un = lane; un < nd; un += 32) {
    const int e = un * LD::V;
    const int idx = e + (e / M) * LD::V;
    const Vd x = *reinterpret_cast<const Vd *>(dbuf + idx);
    if (e + LD::V <= N) {
      *reinterpret_cast<Vd *>(dst + e) = x;
    } else {
      dst[e] = x.x;
    }
  }
  report_bad_pivot(bad, p.flag);
}

template <int M>
static cudaError_t launch_contig_promoted(const MixedArgs &p, cudaStream_t st) {
  using LF = SmemLayout<float, M>;
  using LD = SmemLayout<double, M>;
  const int threads = 128;
  const size_t smem = (size_t)(threads / 32) * (3 * LF::BUF * 4 + LD::BUF * 8);
  auto kern = contig_promoted_kernel<M>;
  if (smem > 48 * 1024) {
    const cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  const long long blocks = (p.nsys * 32 + threads - 1) / threads;
  kern<<<(unsigned)blocks, threads, smem, st>>>(p);
  return cudaGetLastError();
}

static int pow2c(long long v) {
  int q = 1;
  while (q < v) q <<= 1;
  return q;
}

// One warp per CTA: 14 KB (FP32 coefficients) or 20 KB (FP64) of shared
// memory per system of up to 512 rows, so up to 14 or 11 warps per SM;
// larger CTAs would round the shared-memory use up.
template <int M, typename CT>
static cudaError_t launch_mixed_contig(const MixedArgsT<CT> &p, cudaStream_t st) {
  const int threads = 32;
  const size_t per_warp = (size_t)3 * 32 * M * sizeof(CT) + (size_t)2 * 32 * M * 4 + (size_t)32 * M * 8;
  const size_t smem = per_warp * (threads / 32);
  if (smem > 48 * 1024)
    cudaFuncSetAttribute(mixed_contig_kernel<M, CT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  const long long blocks = (p.nsys * 32 + threads - 1) / threads;
  mixed_contig_kernel<M, CT><<<(unsigned)blocks, threads, smem, st>>>(p);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return cudaGetLastError();
}

template <int M, int KR, typename CT>
static cudaError_t launch_mixed_strided(const MixedArgsT<CT> &p, int T, int W, cudaStream_t st) {
  const long long ngx = (p.n0 + W - 1) / W;
  const long long blocks = ngx * (p.nsys / p.n0);
  const size_t smem = (size_t)(4 * T * W + 2 * W) * 8 + (size_t)(W + (W & 1)) * 4 +
                      (size_t)6 * T * (W + 1) * 4;
  mixed_strided_kernel<M, KR, CT><<<(unsigned)blocks, W * T, smem, st>>>(p, T, W, ngx);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return cudaGetLastError();
}

// The refinement kernels for any layout: staged contiguous systems of
// 129..512 rows, the generic strided form otherwise (N <= 512).
template <typename CT>
static cudaError_t launch_refinement(const MixedArgsT<CT> &p, cudaStream_t st) {
  const int N = p.N;
  auto al = [](const void *q) { return (reinterpret_cast<uintptr_t>(q) & 15u) == 0; };
  const long long unit = 16 / (long long)sizeof(CT);
  const bool staged = p.stride == 1 && al(p.a) && al(p.b) && al(p.c) && al(p.d) &&
                      p.st0 % unit == 0 && p.st1 % unit == 0 && p.st0 % 2 == 0 &&
                      p.st1 % 2 == 0 && N > 128;
  if (staged) return N <= 256 ? launch_mixed_contig<8, CT>(p, st) : launch_mixed_contig<16, CT>(p, st);
  // generic addressing (strided, or contiguous but unaligned or short)
  const int T = pow2c((N + 7) / 8);
  int W = 512 / T > 16 ? 16 : 512 / T;
  if (T <= 32 && W * T > 256) W = 256 / T;
  if (W * T < 32) W = 32 / T;
  if (T <= 32) return launch_mixed_strided<8, 2, CT>(p, T, W, st);
  return launch_mixed_strided<8, 4, CT>(p, T, W, st);
}

// Argument checks and the batch description shared by the two entry points.
template <typename CT>
static tridStatus_t make_mixed_args(const CT *a, const CT *b, const CT *c, double *d, int ndim,
                                    int solvedim, const int *dims_p, const int *pads_p,
                                    int max_iters, double tol, MixedArgsT<CT> *out, bool *empty) {
  if (ndim < 1 || ndim > MAXDIM || solvedim < 0 || solvedim >= ndim || !dims_p || !pads_p ||
      max_iters < 1 || !(tol >= 0.0))
    return TRID_STATUS_INVALID_VALUE;
  long long dims[3] = {1, 1, 1}, pads[3] = {1, 1, 1};
  for (int i = 0; i < ndim; ++i) {
    if (dims_p[i] < 0) return TRID_STATUS_INVALID_VALUE;
    dims[i] = dims_p[i];
    pads[i] = pads_p[i];
    if (i < ndim - 1 && pads[i] < dims[i]) return TRID_STATUS_INVALID_VALUE;
  }
  *empty = dims[0] * dims[1] * dims[2] == 0;
  if (*empty) return TRID_STATUS_SUCCESS;
  if (!a || !b || !c || !d) return TRID_STATUS_INVALID_VALUE;
  MixedArgsT<CT> p{};
  p.a = a;
  p.b = b;
  p.c = c;
  p.d = d;
  p.N = (int)dims[solvedim];
  p.max_iters = max_iters;
  p.tol = tol;
  const long long s01 = pads[0] * pads[1];
  if (solvedim == 0) {
    p.n0 = dims[1];
    p.nsys = dims[1] * dims[2];
    p.st0 = pads[0];
    p.st1 = s01;
    p.stride = 1;
  } else if (solvedim == 1) {
    p.n0 = dims[0];
    p.nsys = dims[0] * dims[2];
    p.st0 = 1;
    p.st1 = s01;
    p.stride = pads[0];
  } else {
    p.n0 = dims[0];
    p.nsys = dims[0] * dims[1];
    p.st0 = 1;
    p.st1 = pads[0];
    p.stride = s01;
  }
  *out = p;
  return TRID_STATUS_SUCCESS;
}

static tridStatus_t device_ready() {
  int dev = 0, major = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev) != cudaSuccess) {
    cudaGetLastError();
    return TRID_STATUS_NOT_INITIALIZED;
  }
  return major == 10 ? TRID_STATUS_SUCCESS : TRID_STATUS_ARCH_MISMATCH;
}

// Waits for a blocking refinement call and reports its statistics.
static tridStatus_t finish_refinement(const Settings &cfg, int *iters_out, double *correction_out) {
  cudaError_t e = cudaStreamSynchronize(cfg.stream);
  if (e != cudaSuccess) return status_of(e);
  MixedStats st{};
  e = cudaMemcpyFromSymbol(&st, g_mixed_stats, sizeof(st));
  if (e != cudaSuccess) return status_of(e);
  if (iters_out) *iters_out = (int)st.iters;
  if (correction_out) {
    double v;
    memcpy(&v, &st.corr_bits, sizeof(v));
    *correction_out = v;
  }
  if (pivot_flag_take()) return TRID_STATUS_ZERO_PIVOT;
  return TRID_STATUS_SUCCESS;
}

}  // namespace trid

using namespace trid;

EXTERN_C tridStatus_t tridDmtsvStridedBatchMixed(const TridParams *ctx, const float *a,
                                                 const float *b, const float *c, double *d,
                                                 int ndim, int solvedim, const int *dims_p,
                                                 const int *pads_p, int max_iters, double tol,
                                                 int *iters_out, double *correction_out) {
  const TraceScope trace("tridDmtsvStridedBatchMixed");
  (void)ctx;
  if (iters_out) *iters_out = -1;
  if (correction_out) *correction_out = -1.0;
  MixedArgs p{};
  bool empty = false;
  tridStatus_t sts = make_mixed_args<float>(a, b, c, d, ndim, solvedim, dims_p, pads_p, max_iters,
                                            tol, &p, &empty);
  if (sts != TRID_STATUS_SUCCESS) return sts;
  if (empty) {
    if (iters_out) *iters_out = 0;
    if (correction_out) *correction_out = 0.0;
    return TRID_STATUS_SUCCESS;
  }
  sts = device_ready();
  if (sts != TRID_STATUS_SUCCESS) return sts;
  const Settings &cfg = settings();
  p.flag = pivot_flag_device();
  if (cfg.blocking) pivot_flag_take();
  MixedStats zero{};
  cudaError_t e = cudaMemcpyToSymbolAsync(g_mixed_stats, &zero, sizeof(zero), 0,
                                          cudaMemcpyHostToDevice, cfg.stream);
  const int N = p.N;
  if (N > 512) return TRID_STATUS_MATRIX_TYPE_NOT_SUPPORTED;
  // strided batches the streaming kernel covers: the promoted solve (FP64
  // arithmetic on the FP32 values) unless refinement is asked for
  const bool can_promote = p.stride != 1 && N > 64 && N <= 512;
  const bool promoted = can_promote && cfg.mixed_mode != 1;
  auto al = [](const void *q) { return (reinterpret_cast<uintptr_t>(q) & 15u) == 0; };
  const bool staged = p.stride == 1 && al(a) && al(b) && al(c) && al(d) && p.st0 % 4 == 0 &&
                      p.st1 % 4 == 0 && N > 128;
  const bool direct = promoted || (staged && cfg.mixed_mode != 1);
  if (e == cudaSuccess && promoted) {
    BatchArgs<double> q{};
    q.d_in = d;
    q.d_out = d;
    q.N = N;
    q.nsys = p.nsys;
    q.n0 = p.n0;
    q.st0 = p.st0;
    q.st1 = p.st1;
    q.stride = p.stride;
    q.flag = p.flag;
    const CoefPtrs<float> cf{a, b, c};
    // rows a plane apart (z solves) with at least half a 32-system group:
    // the wide kernel (FP32 coefficient rows of 128 bytes, d of 256), else
    // the 128-byte streaming kernel
    const bool zlike = p.stride * (long long)sizeof(double) >= (1LL << 16);
    if (zlike && 2 * p.n0 >= wide_width<double>())
      e = launch_strided_wide_promoted(q, cf, cfg.stream);
    else
      e = N <= 128   ? launch_strided_stream_promoted<4>(q, cf, cfg.stream)
          : N <= 256 ? launch_strided_stream_promoted<8>(q, cf, cfg.stream)
                     : launch_strided_stream_promoted<16>(q, cf, cfg.stream);
    g_launches.fetch_add(1, std::memory_order_relaxed);
  } else if (e == cudaSuccess && direct) {
    // direct FP64 solve of the promoted values
    e = N <= 256 ? launch_contig_promoted<8>(p, cfg.stream) : launch_contig_promoted<16>(p, cfg.stream);
    g_launches.fetch_add(1, std::memory_order_relaxed);
  } else if (e == cudaSuccess) {
    e = launch_refinement<float>(p, cfg.stream);
  }
  if (e != cudaSuccess) return status_of(e);
  if (!cfg.blocking) return TRID_STATUS_SUCCESS;
  if (direct) {
    e = cudaStreamSynchronize(cfg.stream);
    if (e != cudaSuccess) return status_of(e);
    if (iters_out) *iters_out = 0;
    if (correction_out) *correction_out = 0.0;
    return pivot_flag_take() ? TRID_STATUS_ZERO_PIVOT : TRID_STATUS_SUCCESS;
  }
  return finish_refinement(cfg, iters_out, correction_out);
}

EXTERN_C tridStatus_t tridDmtsvStridedBatchRefine(const TridParams *ctx, const double *a,
                                                  const double *b, const double *c, double *d,
                                                  int ndim, int solvedim, const int *dims_p,
                                                  const int *pads_p, int max_iters, double tol,
                                                  int *iters_out, double *correction_out) {
  const TraceScope trace("tridDmtsvStridedBatchRefine");
  (void)ctx;
  if (iters_out) *iters_out = -1;
  if (correction_out) *correction_out = -1.0;
  MixedArgsT<double> p{};
  bool empty = false;
  tridStatus_t sts = make_mixed_args<double>(a, b, c, d, ndim, solvedim, dims_p, pads_p,
                                             max_iters, tol, &p, &empty);
  if (sts != TRID_STATUS_SUCCESS) return sts;
  if (empty) {
    if (iters_out) *iters_out = 0;
    if (correction_out) *correction_out = 0.0;
    return TRID_STATUS_SUCCESS;
  }
  sts = device_ready();
  if (sts != TRID_STATUS_SUCCESS) return sts;
  if (p.N > 512) return TRID_STATUS_MATRIX_TYPE_NOT_SUPPORTED;
  const Settings &cfg = settings();
  p.flag = pivot_flag_device();
  if (cfg.blocking) pivot_flag_take();
  MixedStats zero{};
  cudaError_t e = cudaMemcpyToSymbolAsync(g_mixed_stats, &zero, sizeof(zero), 0,
                                          cudaMemcpyHostToDevice, cfg.stream);
  if (e == cudaSuccess) e = launch_refinement<double>(p, cfg.stream);
  if (e != cudaSuccess) return status_of(e);
  if (!cfg.blocking) return TRID_STATUS_SUCCESS;
  return finish_refinement(cfg, iters_out, correction_out);
}
