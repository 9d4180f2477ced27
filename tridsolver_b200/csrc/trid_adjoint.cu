// Adjoint of the batched tridiagonal solve.
//
// For x = T^{-1} d along one dimension and an upstream gradient w = dL/dx:
//   dbar = T^{-T} w                         (dL/dd)
//   abar_i = -dbar_i x_{i-1},  bbar_i = -dbar_i x_i,  cbar_i = -dbar_i x_{i+1}
// with abar_0 = cbar_{N-1} = 0 (a[0] and c[N-1] do not enter the forward map).
// T^T is tridiagonal with sub-diagonal c_{i-1}, diagonal b_i and
// super-diagonal a_{i+1}, so the transposed solve is the forward partition
// hybrid fed with a and c shifted by one row; the three products are fused
// into the same pass, which reads a, b, c, w, x once and writes the four
// gradients once (9 words per element; 5 when only dbar is wanted). Strided
// batches of 64 < N <= 512 use the streaming kernel's adjoint form
// (trid_strided_stream.cu); other shapes use adjoint_kernel below.
// The reference has no adjoint; this is an extension (tridsolver_b200.h).
#include <cuda_runtime.h>

#include "trid_internal.h"
#include "tridsolver_b200.h"

namespace trid {

template <typename R> struct AdjointArgs {
  const R *a, *b, *c, *x, *w;
  R *dbar, *abar, *bbar, *cbar;  // abar/bbar/cbar may be null
  int N;
  long long nsys, n0, st0, st1, stride;
  unsigned *flag;
};

// Block = W neighbouring systems x T chunks, thread (s, t) = (tid % W, tid / W),
// as strided_kernel; works for any stride (contiguous systems included).
template <typename R, int M, int KR, bool PROD>
__global__ void __launch_bounds__((KR >= 4 || M * sizeof(R) <= 64) ? 512 : 256)
    adjoint_kernel(const AdjointArgs<R> p, int T, int W, long long ngx) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R *sm = reinterpret_cast<R *>(smem_raw);
  const int tid = threadIdx.x;
  const int s = tid % W;
  const int t = tid / W;
  const long long gx = blockIdx.x % ngx;
  const long long i1 = blockIdx.x / ngx;
  const long long i0 = gx * W + s;
  const bool active = i0 < p.n0;
  const long long base = i0 * p.st0 + i1 * p.st1;
  const long long st = p.stride;
  const int N = p.N;
  const int row0 = t * M;
  R ra[M], rb[M], rc[M], rd[M];
#pragma unroll
  for (int i = 0; i < M; ++i) {
    const int row = row0 + i;
    if (active && row < N) {
      const long long o = base + (long long)row * st;
      ra[i] = row >= 1 ? __ldg(p.c + o - st) : R(0);      // T^T sub-diagonal
      rb[i] = __ldg(p.b + o);
      rc[i] = row <= N - 2 ? __ldg(p.a + o + st) : R(0);  // T^T super-diagonal
      rd[i] = __ldg(p.w + o);
    } else {
      ra[i] = R(0);
      rb[i] = R(1);
      rc[i] = R(0);
      rd[i] = R(0);
    }
  }
  bool bad = false;
  chunk_forward<R, M>(ra, rb, rc, rd, bad);
  chunk_backward<R, M>(ra, rc, rd, bad);
  R y, z;
  block_reduced_solve<R, KR>(sm, Row<R>{ra[0], rc[0], rd[0]}, Row<R>{ra[M - 1], rc[M - 1], rd[M - 1]},
                             s, t, T, W, y, z, bad);
  chunk_substitute<R, M>(ra, rc, rd, y, z);
  if (active) {
    if (PROD) {
      // x at rows row0-1 .. row0+M (the neighbours come from adjacent chunks)
      R xs[M + 2];
#pragma unroll
      for (int i = 0; i < M + 2; ++i) {
        const int row = row0 - 1 + i;
        xs[i] = (row >= 0 && row < N) ? __ldg(p.x + base + (long long)row * st) : R(0);
      }
#pragma unroll
      for (int i = 0; i < M; ++i) {
        const int row = row0 + i;
        if (row < N) {
          const long long o = base + (long long)row * st;
          const R g = rd[i];
          p.dbar[o] = g;
          if (p.abar) p.abar[o] = row >= 1 ? -g * xs[i] : R(0);
          if (p.bbar) p.bbar[o] = -g * xs[i + 1];
          if (p.cbar) p.cbar[o] = row <= N - 2 ? -g * xs[i + 2] : R(0);
        }
      }
    } else {
#pragma unroll
      for (int i = 0; i < M; ++i) {
        const int row = row0 + i;
        if (row < N) p.dbar[base + (long long)row * st] = rd[i];
      }
    }
  }
  report_bad_pivot(bad && active, p.flag);
}

static int pow2a(long long v) {
  int q = 1;
  while (q < v) q <<= 1;
  return q;
}

template <typename R, int KR, bool PROD>
static cudaError_t launch_adjoint(const AdjointArgs<R> &p, int T, int W, cudaStream_t st) {
  const long long ngx = (p.n0 + W - 1) / W;
  const long long blocks = ngx * (p.nsys / p.n0);
  const size_t smem = (size_t)6 * T * (W + 1) * sizeof(R);
  adjoint_kernel<R, 8, KR, PROD><<<(unsigned)blocks, W * T, smem, st>>>(p, T, W, ngx);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return cudaGetLastError();
}

template <typename R>
static tridStatus_t adjoint(const TridParams *ctx, const R *a, const R *b, const R *c, const R *x,
                            const R *w, R *dbar, R *abar, R *bbar, R *cbar, int ndim, int solvedim,
                            const int *dims_p, const int *pads_p) {
  (void)ctx;
  if (ndim < 1 || ndim > MAXDIM || solvedim < 0 || solvedim >= ndim || !dims_p || !pads_p)
    return TRID_STATUS_INVALID_VALUE;
  long long dims[3] = {1, 1, 1}, pads[3] = {1, 1, 1};
  for (int i = 0; i < ndim; ++i) {
    if (dims_p[i] < 0) return TRID_STATUS_INVALID_VALUE;
    dims[i] = dims_p[i];
    pads[i] = pads_p[i];
    if (i < ndim - 1 && pads[i] < dims[i]) return TRID_STATUS_INVALID_VALUE;
  }
  if (dims[0] * dims[1] * dims[2] == 0) return TRID_STATUS_SUCCESS;
  const bool prod = abar || bbar || cbar;
  if (!a || !b || !c || !w || !dbar || (prod && !x)) return TRID_STATUS_INVALID_VALUE;
  AdjointArgs<R> p{};
  p.a = a;
  p.b = b;
  p.c = c;
  p.x = x;
  p.w = w;
  p.dbar = dbar;
  p.abar = abar;
  p.bbar = bbar;
  p.cbar = cbar;
  p.N = (int)dims[solvedim];
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
  if (p.N > 1024) return TRID_STATUS_MATRIX_TYPE_NOT_SUPPORTED;
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
  // strided batches of 64 < N <= 512 with at least half a 128-byte group of
  // systems: the streaming kernel in its adjoint form (one pass, 9 words per
  // element with the products, 5 for dbar alone)
  if (p.stride > 1 && p.N > 64 && p.N <= 512 && 2 * p.n0 >= (long long)(128 / sizeof(R))) {
    BatchArgs<R> q{};
    q.a = a;
    q.b = b;
    q.c = c;
    q.d_in = w;
    q.d_out = dbar;
    q.u = prod ? const_cast<R *>(x) : nullptr;
    q.N = p.N;
    q.nsys = p.nsys;
    q.n0 = p.n0;
    q.st0 = p.st0;
    q.st1 = p.st1;
    q.stride = p.stride;
    q.flag = p.flag;
    AdjointOut<R> out;
    out.abar = abar;
    out.bbar = bbar;
    out.cbar = cbar;
    cudaError_t e = p.N <= 128   ? launch_strided_stream_adjoint<R, 4>(q, out, cfg.stream)
                    : p.N <= 256 ? launch_strided_stream_adjoint<R, 8>(q, out, cfg.stream)
                                 : launch_strided_stream_adjoint<R, 16>(q, out, cfg.stream);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    if (e != cudaSuccess) return status_of(e);
    if (cfg.blocking) {
      e = cudaStreamSynchronize(cfg.stream);
      if (e != cudaSuccess) return status_of(e);
      if (pivot_flag_take()) return TRID_STATUS_ZERO_PIVOT;
    }
    return TRID_STATUS_SUCCESS;
  }
  // otherwise M = 8 rows per thread, T chunks (<= 128), W systems: 64
  // contiguous bytes per row when strided, blocks of at most 512 threads
  const int T = pow2a((p.N + 7) / 8);
  int W = (int)(64 / sizeof(R));
  const int tmax = 512;
  if (W * T > tmax) W = tmax / T;
  if (W * T < 32) W = 32 / T;
  cudaError_t e;
  if (T <= 32)
    e = prod ? launch_adjoint<R, 2, true>(p, T, W, cfg.stream) : launch_adjoint<R, 2, false>(p, T, W, cfg.stream);
  else if (T == 64)
    e = prod ? launch_adjoint<R, 4, true>(p, T, W, cfg.stream) : launch_adjoint<R, 4, false>(p, T, W, cfg.stream);
  else
    e = prod ? launch_adjoint<R, 8, true>(p, T, W, cfg.stream) : launch_adjoint<R, 8, false>(p, T, W, cfg.stream);
  if (e != cudaSuccess) return status_of(e);
  if (cfg.blocking) {
    e = cudaStreamSynchronize(cfg.stream);
    if (e != cudaSuccess) return status_of(e);
    if (pivot_flag_take()) return TRID_STATUS_ZERO_PIVOT;
  }
  return TRID_STATUS_SUCCESS;
}

}  // namespace trid

using namespace trid;

EXTERN_C tridStatus_t tridDmtsvStridedBatchAdjoint(const TridParams *ctx, const double *a,
                                                   const double *b, const double *c,
                                                   const double *x, const double *w, double *dbar,
                                                   double *abar, double *bbar, double *cbar,
                                                   int ndim, int solvedim, const int *dims,
                                                   const int *pads) {
  const TraceScope trace("tridDmtsvStridedBatchAdjoint");
  return adjoint<double>(ctx, a, b, c, x, w, dbar, abar, bbar, cbar, ndim, solvedim, dims, pads);
}

EXTERN_C tridStatus_t tridSmtsvStridedBatchAdjoint(const TridParams *ctx, const float *a,
                                                   const float *b, const float *c, const float *x,
                                                   const float *w, float *dbar, float *abar,
                                                   float *bbar, float *cbar, int ndim,
                                                   int solvedim, const int *dims, const int *pads) {
  const TraceScope trace("tridSmtsvStridedBatchAdjoint");
  return adjoint<float>(ctx, a, b, c, x, w, dbar, abar, bbar, cbar, ndim, solvedim, dims, pads);
}
