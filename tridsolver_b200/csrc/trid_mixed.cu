// FP32-storage / FP32-solve tridiagonal batch with FP64 iterative refinement.
//
// Solves T x = d where the coefficients a, b, c are stored in FP32 (and taken
// exactly, promoted to FP64, as the system to solve) and d, x are FP64:
//
//   x = 0;  repeat:  r = d - T x       (FP64: FP32 coefficients times FP64 x)
//                    solve T dx = r    (FP32: the partition hybrid)
//                    x += dx           (FP64)
//   until max|dx| <= tol * max|x| over the system, or max_iters solves.
//
// Everything after the one read of a, b, c, d happens on chip: the FP32
// coefficients stay in shared memory (contiguous systems) or registers
// (strided), d and x in registers, and x is written once. A pass moves
// 3*4 + 8 + 8 = 28 bytes per element against 40 for the plain FP64 solve, so
// refinement to FP64 accuracy can cost less time than the FP64 solve.
// The reference has no mixed-precision entry point; this is an extension
// (include/tridsolver_b200.h).
#include <cuda_runtime.h>

#include <cstring>

#include "trid_internal.h"
#include "tridsolver_b200.h"

namespace trid {

struct MixedArgs {
  const float *a, *b, *c;
  double *d;  // right-hand side in, x out
  int N;
  long long nsys, n0, st0, st1, stride;
  int max_iters;
  double tol;
  unsigned *flag;
};

// Per-call statistics: the largest iteration count and the largest final
// relative correction max|dx|/max|x| over all systems (as ordered bits; both
// are non-negative so their bit patterns order like the values).
struct MixedStats {
  unsigned iters;
  unsigned pad;
  unsigned long long corr_bits;
};
static __device__ MixedStats g_mixed_stats;

__device__ __forceinline__ void mixed_report(int iters, double rel) {
  atomicMax(&g_mixed_stats.iters, (unsigned)iters);
  atomicMax(&g_mixed_stats.corr_bits, (unsigned long long)__double_as_longlong(rel));
}

__device__ __forceinline__ long long mixed_base(const MixedArgs &p, long long s) {
  const long long i1 = s / p.n0;
  return (s - i1 * p.n0) * p.st0 + i1 * p.st1;
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

// ---------------------------------------------------------------------------
// Contiguous systems (stride 1), one warp per system, 16-byte aligned starts.
// The warp stages a, b, c (FP32) and d (FP64) through shared memory with
// coalesced 16-byte cp.async copies into padded rows (one spare 16-byte unit
// per chunk row), as contig_smem_kernel does.
template <int M>
__global__ void __launch_bounds__(128) mixed_contig_kernel(const MixedArgs p) {
  constexpr int RF = M + 4;          // padded FP32 chunk row
  constexpr int RD = M + 2;          // padded FP64 chunk row
  constexpr int BF = 32 * RF;        // floats per FP32 tile
  constexpr int BD = 32 * RD;        // doubles per FP64 tile
  extern __shared__ __align__(16) unsigned char smem_raw[];
  unsigned char *wbase = smem_raw + (threadIdx.x >> 5) * (3 * BF * 4 + BD * 8);
  float *ta = reinterpret_cast<float *>(wbase);
  float *tb = ta + BF;
  float *tc = tb + BF;
  double *td = reinterpret_cast<double *>(wbase + 3 * BF * 4);
  const int lane = threadIdx.x & 31;
  const long long s = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (s >= p.nsys) return;  // uniform per warp
  const long long base = mixed_base(p, s);
  const int N = p.N;
  {
    const int nu = (N + 3) / 4;  // FP32 units of 4
    for (int un = lane; un < nu; un += 32) {
      const int e = un * 4;
      const int left = (N - e) >= 4 ? 16 : (N - e) * 4;
      const int o = e + (e / M) * 4;
      cp_async16(ta + o, p.a + base + e, left);
      cp_async16(tb + o, p.b + base + e, left);
      cp_async16(tc + o, p.c + base + e, left);
    }
    const int nud = (N + 1) / 2;  // FP64 units of 2
    for (int un = lane; un < nud; un += 32) {
      const int e = un * 2;
      cp_async16(td + e + (e / M) * 2, p.d + base + e, (N - e) >= 2 ? 16 : 8);
    }
  }
  cp_async_wait_all();
  __syncwarp();

  const int row0 = lane * M;
  double d64[M], x64[M];
#pragma unroll
  for (int i = 0; i < M; ++i) {
    d64[i] = row0 + i < N ? td[lane * RD + i] : 0.0;
    x64[i] = 0.0;
  }
  // FP32 coefficients of this lane's rows (16-byte reads of its padded row,
  // conflict-free across neighbouring lanes), identity past the end, a[0]
  // and c[N-1] zero
  auto coef = [&](float (&wa)[M], float (&wb)[M], float (&wc)[M]) {
    lds_row<float, M>(ta + lane * RF, wa);
    lds_row<float, M>(tb + lane * RF, wb);
    lds_row<float, M>(tc + lane * RF, wc);
#pragma unroll
    for (int i = 0; i < M; ++i) {
      const int row = row0 + i;
      if (row >= N) {
        wa[i] = 0.f;
        wb[i] = 1.f;
        wc[i] = 0.f;
      }
      if (row == 0) wa[i] = 0.f;
      if (row == N - 1) wc[i] = 0.f;
    }
  };
  bool bad = false;
  int it = 0;
  double rel = 0.0;
  for (;;) {
    float wa[M], wb[M], wc[M], wd[M];
    coef(wa, wb, wc);
    if (it == 0) {
#pragma unroll
      for (int i = 0; i < M; ++i) wd[i] = (float)d64[i];
    } else {
      double xl = __shfl_up_sync(FULL_MASK, x64[M - 1], 1);
      double xr = __shfl_down_sync(FULL_MASK, x64[0], 1);
      if (lane == 0) xl = 0.0;
      if (lane == 31) xr = 0.0;
#pragma unroll
      for (int i = 0; i < M; ++i) {
        const double xm = i == 0 ? xl : x64[i - 1];
        const double xp = i == M - 1 ? xr : x64[i + 1];
        double r = d64[i] - (double)wb[i] * x64[i];
        r = fma(-(double)wa[i], xm, r);
        r = fma(-(double)wc[i], xp, r);
        wd[i] = (float)r;
      }
    }
    fp32_chunk_solve<M>(wa, wb, wc, wd, lane, 32, bad);
    double dmax = 0.0, xmax = 0.0;
#pragma unroll
    for (int i = 0; i < M; ++i) {
      x64[i] += (double)wd[i];
      dmax = fmax(dmax, fabs((double)wd[i]));
      xmax = fmax(xmax, fabs(x64[i]));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      dmax = fmax(dmax, __shfl_xor_sync(FULL_MASK, dmax, o));
      xmax = fmax(xmax, __shfl_xor_sync(FULL_MASK, xmax, o));
    }
    ++it;
    rel = xmax > 0.0 ? dmax / xmax : 0.0;
    if (!(rel > p.tol) || it >= p.max_iters) break;  // uniform across the warp
  }
  // x out through the FP64 tile (own row), then coalesced 16-byte stores
#pragma unroll
  for (int i = 0; i < M; ++i) td[lane * RD + i] = x64[i];
  __syncwarp();
  const int nud = (N + 1) / 2;
  for (int un = lane; un < nud; un += 32) {
    const int e = un * 2;
    const double2 v = *reinterpret_cast<const double2 *>(td + e + (e / M) * 2);
    if (e + 2 <= N) {
      *reinterpret_cast<double2 *>(p.d + base + e) = v;
    } else {
      p.d[base + e] = v.x;
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
template <int M, int KR>
__global__ void __launch_bounds__(KR >= 4 ? 512 : 256)
    mixed_strided_kernel(const MixedArgs p, int T, int W, long long ngx) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int TW = T * W;
  double *xf = reinterpret_cast<double *>(smem_raw);  // first x of chunk (t, s)
  double *xl = xf + TW;                                // last x of chunk (t, s)
  double *cd = xl + TW;                                // max |dx| of chunk (t, s)
  double *cx = cd + TW;                                // max |x| of chunk (t, s)
  double *relv = cx + TW;                              // per system
  int *conv = reinterpret_cast<int *>(relv + W);
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
  float ra[M], rb[M], rc[M];
  double d64[M], x64[M];
#pragma unroll
  for (int i = 0; i < M; ++i) {
    const int row = row0 + i;
    if (active && row < N) {
      const long long o = base + (long long)row * p.stride;
      ra[i] = row == 0 ? 0.f : __ldg(p.a + o);
      rb[i] = __ldg(p.b + o);
      rc[i] = row == N - 1 ? 0.f : __ldg(p.c + o);
      d64[i] = p.d[o];
    } else {
      ra[i] = 0.f;
      rb[i] = 1.f;
      rc[i] = 0.f;
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
      wa[i] = ra[i];
      wb[i] = rb[i];
      wc[i] = rc[i];
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
      const double rel = xm > 0.0 ? dm / xm : 0.0;
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

static int pow2c(long long v) {
  int q = 1;
  while (q < v) q <<= 1;
  return q;
}

template <int M>
static cudaError_t launch_mixed_contig(const MixedArgs &p, cudaStream_t st) {
  const int threads = 128;
  const size_t per_warp = (size_t)3 * 32 * (M + 4) * 4 + (size_t)32 * (M + 2) * 8;
  const size_t smem = per_warp * (threads / 32);
  if (smem > 48 * 1024)
    cudaFuncSetAttribute(mixed_contig_kernel<M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  const long long blocks = (p.nsys * 32 + threads - 1) / threads;
  mixed_contig_kernel<M><<<(unsigned)blocks, threads, smem, st>>>(p);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return cudaGetLastError();
}

template <int M, int KR>
static cudaError_t launch_mixed_strided(const MixedArgs &p, int T, int W, cudaStream_t st) {
  const long long ngx = (p.n0 + W - 1) / W;
  const long long blocks = ngx * (p.nsys / p.n0);
  const size_t smem = (size_t)(4 * T * W + W) * 8 + (size_t)(W + (W & 1)) * 4 +
                      (size_t)6 * T * (W + 1) * 4;
  mixed_strided_kernel<M, KR><<<(unsigned)blocks, W * T, smem, st>>>(p, T, W, ngx);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return cudaGetLastError();
}

}  // namespace trid

using namespace trid;

EXTERN_C tridStatus_t tridDmtsvStridedBatchMixed(const TridParams *ctx, const float *a,
                                                 const float *b, const float *c, double *d,
                                                 int ndim, int solvedim, const int *dims_p,
                                                 const int *pads_p, int max_iters, double tol,
                                                 int *iters_out, double *correction_out) {
  (void)ctx;
  if (iters_out) *iters_out = -1;
  if (correction_out) *correction_out = -1.0;
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
  if (dims[0] * dims[1] * dims[2] == 0) {
    if (iters_out) *iters_out = 0;
    if (correction_out) *correction_out = 0.0;
    return TRID_STATUS_SUCCESS;
  }
  if (!a || !b || !c || !d) return TRID_STATUS_INVALID_VALUE;
  MixedArgs p{};
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
  int dev = 0, major = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev) != cudaSuccess) {
    cudaGetLastError();
    return TRID_STATUS_NOT_INITIALIZED;
  }
  if (major != 10) return TRID_STATUS_ARCH_MISMATCH;
  const Settings &cfg = settings();
  p.flag = pivot_flag_device();
  if (cfg.blocking) pivot_flag_take();
  MixedStats zero{};
  cudaError_t e = cudaMemcpyToSymbolAsync(g_mixed_stats, &zero, sizeof(zero), 0,
                                          cudaMemcpyHostToDevice, cfg.stream);
  const int N = p.N;
  if (e == cudaSuccess) {
    auto al = [](const void *q) { return (reinterpret_cast<uintptr_t>(q) & 15u) == 0; };
    const bool staged = p.stride == 1 && al(a) && al(b) && al(c) && al(d) && p.st0 % 4 == 0 &&
                        p.st1 % 4 == 0 && N > 128;
    if (N > 512) return TRID_STATUS_MATRIX_TYPE_NOT_SUPPORTED;
    if (staged) {
      e = N <= 256 ? launch_mixed_contig<8>(p, cfg.stream) : launch_mixed_contig<16>(p, cfg.stream);
    } else {
      // generic addressing (strided, or contiguous but unaligned or short)
      const int T = pow2c((N + 7) / 8);
      int W = 512 / T > 16 ? 16 : 512 / T;
      if (T <= 32 && W * T > 256) W = 256 / T;
      if (W * T < 32) W = 32 / T;
      if (T <= 32)
        e = launch_mixed_strided<8, 2>(p, T, W, cfg.stream);
      else
        e = launch_mixed_strided<8, 4>(p, T, W, cfg.stream);
    }
  }
  if (e != cudaSuccess) return status_of(e);
  if (cfg.blocking) {
    e = cudaStreamSynchronize(cfg.stream);
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
  }
  return TRID_STATUS_SUCCESS;
}
