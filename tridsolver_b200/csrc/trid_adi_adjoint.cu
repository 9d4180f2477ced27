// Adjoint of one ADI heat-diffusion timestep (the step of trid_adi.cu):
//
//   du0 = lambda L u        (L: 7-point Laplacian on interior points, 0 on
//                            the boundary)
//   x1 = Tx^-1 du0,  x2 = Ty^-1 x1,  x3 = Tz^-1 x2,  u' = u + x3
//
// with T = T(lambda) along each axis: a = c = -alpha lambda, b = 1 +
// 2 alpha lambda on interior points, identity rows on boundary points. Given
// g = dL/du', this computes
//
//   w3 = Tz^-T g,  w2 = Ty^-T w3,  w1 = Tx^-T w2
//   dL/du      = g + lambda L^T w1
//   dL/dlambda = w1 . (L u)
//              + alpha sum over axes and interior points p of
//                w_axis[p] (x_axis[p-e] - 2 x_axis[p] + x_axis[p+e])
//
// (the last term is sum(abar da/dlambda + bbar db/dlambda + cbar
// dc/dlambda) with abar_p = -w_p x_{p-e}, bbar_p = -w_p x_p, cbar_p =
// -w_p x_{p+e}, the products the adjoint solve would otherwise write out).
// The forward intermediates are recomputed from u (the array form of the
// step: coefficient arrays shared by the three axes), the transposed solves
// are the library's adjoint solves (d-bar only), and two kernels here form
// the stencil transpose and the lambda reductions (accumulated in FP64), so
// the whole backward of a step runs natively: about 51 words of memory
// traffic per point. No counterpart in the reference, which has no
// derivatives.
#include <cuda_runtime.h>

#include "trid_internal.h"
#include "tridsolver_b200.h"

namespace trid {

namespace {

constexpr int kThreads = 256;

// Block-wide sum of one double per thread into *acc (one atomic per block).
__device__ __forceinline__ void block_sum_add(double v, double *acc) {
  __shared__ double part[kThreads / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL_MASK, v, o);
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) part[w] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    v = threadIdx.x < kThreads / 32 ? part[threadIdx.x] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL_MASK, v, o);
    if (threadIdx.x == 0) atomicAdd(acc, v);
  }
}

__device__ __forceinline__ bool interior(long long i, long long j, long long k, int nx, int ny,
                                         int nz) {
  return i > 0 && i < nx - 1 && j > 0 && j < ny - 1 && k > 0 && k < nz - 1;
}

// acc += alpha * sum over interior p of w[p] (x[p-e] - 2 x[p] + x[p+e]),
// e = the solve axis' stride
template <typename R>
__global__ void __launch_bounds__(kThreads)
    adi_coef_grad_kernel(const R *__restrict__ w, const R *__restrict__ x, long long e, R alpha,
                         int nx, int ny, int nz, double *acc) {
  const long long nxy = (long long)nx * ny;
  const long long n = nxy * nz;
  double s = 0.0;
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n;
       p += (long long)gridDim.x * blockDim.x) {
    const long long k = p / nxy;
    const long long r = p - k * nxy;
    const long long j = r / nx;
    const long long i = r - j * nx;
    if (interior(i, j, k, nx, ny, nz))
      s += (double)w[p] * ((double)x[p - e] - 2.0 * (double)x[p] + (double)x[p + e]);
  }
  block_sum_add(s * (double)alpha, acc);
}

// ubar = g + lambda L^T w1, and acc += w1 . (L u) over interior points.
// (L^T w)[q] = sum over the interior neighbours p of q of w[p], minus 6 w[q]
// when q is interior.
template <typename R>
__global__ void __launch_bounds__(kThreads)
    adi_stencil_adjoint_kernel(const R *__restrict__ u, const R *__restrict__ w1,
                               const R *__restrict__ g, R *__restrict__ ubar, const R *lam, int nx,
                               int ny, int nz, double *acc) {
  const R l = lam[0];
  const long long nxy = (long long)nx * ny;
  const long long n = nxy * nz;
  double s = 0.0;
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n;
       q += (long long)gridDim.x * blockDim.x) {
    const long long k = q / nxy;
    const long long r = q - k * nxy;
    const long long j = r / nx;
    const long long i = r - j * nx;
    const bool in = interior(i, j, k, nx, ny, nz);
    R lt = in ? R(-6) * w1[q] : R(0);
    if (i > 0 && interior(i - 1, j, k, nx, ny, nz)) lt += w1[q - 1];
    if (i < nx - 1 && interior(i + 1, j, k, nx, ny, nz)) lt += w1[q + 1];
    if (j > 0 && interior(i, j - 1, k, nx, ny, nz)) lt += w1[q - nx];
    if (j < ny - 1 && interior(i, j + 1, k, nx, ny, nz)) lt += w1[q + nx];
    if (k > 0 && interior(i, j, k - 1, nx, ny, nz)) lt += w1[q - nxy];
    if (k < nz - 1 && interior(i, j, k + 1, nx, ny, nz)) lt += w1[q + nxy];
    ubar[q] = g[q] + l * lt;
    if (in) {
      const R lu = u[q - 1] + u[q + 1] + u[q - nx] + u[q + nx] + u[q - nxy] + u[q + nxy] - R(6) * u[q];
      s += (double)w1[q] * (double)lu;
    }
  }
  block_sum_add(s, acc);
}

template <typename R> __global__ void adi_lambar_kernel(const double *acc, R *lambar) {
  if (threadIdx.x == 0 && blockIdx.x == 0) lambar[0] += (R)acc[0];
}

}  // namespace

template <typename R>
static tridStatus_t adi_step_adjoint(const R *u, const R *g, R *ubar, R *lambar, const R *lam,
                                     R alpha, int nx, int ny, int nz) {
  if (!u || !g || !ubar || !lambar || !lam || nx < 1 || ny < 1 || nz < 1 || ubar == g || ubar == u)
    return TRID_STATUS_INVALID_VALUE;
  if (nx > 1024 || ny > 1024 || nz > 1024) return TRID_STATUS_MATRIX_TYPE_NOT_SUPPORTED;
  tridStatus_t sts = check_device();
  if (sts != TRID_STATUS_SUCCESS) return sts;
  Settings &cfg = settings();
  const bool blocking = cfg.blocking;
  cudaStream_t st = cfg.stream;
  unsigned *flag = pivot_flag_device();
  if (blocking) pivot_flag_take();
  const long long n = (long long)nx * ny * nz;
  const size_t bytes = (size_t)n * sizeof(R);
  // a, b, c, x1, x2, x3, w, then the FP64 accumulator, each on a 256-byte
  // boundary (packed back to back, an odd FP32 grid would leave the double
  // accumulator misaligned)
  const size_t slot = (bytes + 255) / 256 * 256;
  char *scratch = nullptr;
  cudaError_t e = scratch_alloc((void **)&scratch, 7 * slot + 256, st);
  if (e != cudaSuccess) return status_of(e);
  R *arr[7];
  for (int q = 0; q < 7; ++q) arr[q] = reinterpret_cast<R *>(scratch + q * slot);
  R *a = arr[0], *b = arr[1], *c = arr[2], *x1 = arr[3], *x2 = arr[4], *x3 = arr[5], *w = arr[6];
  double *acc = reinterpret_cast<double *>(scratch + 7 * slot);
  long long blocks = (n + kThreads - 1) / kThreads;
  if (blocks > 148LL * 16) blocks = 148LL * 16;
  const int dims[3] = {nx, ny, nz};
  const long long estride[3] = {1, nx, (long long)nx * ny};
  e = cudaMemsetAsync(acc, 0, sizeof(double), st);
  // forward intermediates: du0 and the coefficient arrays, then the three
  // solves, each kept
  if (e == cudaSuccess) e = launch_adi_preproc<R>(u, x1, a, b, c, lam, nullptr, alpha, nx, ny, nz, st);
  R *xs[3] = {x1, x2, x3};
  for (int sd = 0; sd < 3 && e == cudaSuccess; ++sd) {
    if (sd > 0) e = cudaMemcpyAsync(xs[sd], xs[sd - 1], bytes, cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) break;
    BatchArgs<R> p;
    bool empty = false;
    if (make_batch<R>(a, b, c, xs[sd], nullptr, false, 3, sd, dims, dims, &p, &empty) !=
        TRID_STATUS_SUCCESS) {
      e = cudaErrorInvalidValue;
      break;
    }
    p.flag = flag;
    const Plan plan = choose_plan<R>(p, vec_aligned<R>(p), false);
    e = launch_batch<R, false>(p, plan, st);
  }
  // transposed solves z, y, x (d-bar only, w in place) with the coefficient
  // gradients reduced against each forward solution
  cfg.blocking = false;
  tridStatus_t ast = TRID_STATUS_SUCCESS;
  for (int sd = 2; sd >= 0 && e == cudaSuccess && ast == TRID_STATUS_SUCCESS; --sd) {
    const R *rhs = sd == 2 ? g : w;
    if constexpr (sizeof(R) == 8)
      ast = tridDmtsvStridedBatchAdjoint(nullptr, a, b, c, nullptr, rhs, w, nullptr, nullptr,
                                         nullptr, 3, sd, dims, dims);
    else
      ast = tridSmtsvStridedBatchAdjoint(nullptr, a, b, c, nullptr, rhs, w, nullptr, nullptr,
                                         nullptr, 3, sd, dims, dims);
    if (ast != TRID_STATUS_SUCCESS) break;
    adi_coef_grad_kernel<R><<<(unsigned)blocks, kThreads, 0, st>>>(w, xs[sd], estride[sd], alpha, nx,
                                                                 ny, nz, acc);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    e = cudaGetLastError();
  }
  cfg.blocking = blocking;
  if (e == cudaSuccess && ast == TRID_STATUS_SUCCESS) {
    adi_stencil_adjoint_kernel<R><<<(unsigned)blocks, kThreads, 0, st>>>(u, w, g, ubar, lam, nx, ny,
                                                                       nz, acc);
    adi_lambar_kernel<R><<<1, 32, 0, st>>>(acc, lambar);
    g_launches.fetch_add(2, std::memory_order_relaxed);
    e = cudaGetLastError();
  }
  const cudaError_t ef = scratch_free(scratch, st);
  if (ast != TRID_STATUS_SUCCESS) return ast;
  if (e == cudaSuccess) e = ef;
  if (e != cudaSuccess) return status_of(e);
  if (blocking) {
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return status_of(e);
    if (pivot_flag_take()) return TRID_STATUS_ZERO_PIVOT;
  }
  return TRID_STATUS_SUCCESS;
}

}  // namespace trid

using namespace trid;

EXTERN_C tridStatus_t tridDADIStepAdjoint(const double *u, const double *g, double *ubar,
                                          double *lambar, const double *lam, double alpha, int nx,
                                          int ny, int nz) {
  const TraceScope trace("tridDADIStepAdjoint");
  return adi_step_adjoint<double>(u, g, ubar, lambar, lam, alpha, nx, ny, nz);
}

EXTERN_C tridStatus_t tridSADIStepAdjoint(const float *u, const float *g, float *ubar,
                                          float *lambar, const float *lam, float alpha, int nx,
                                          int ny, int nz) {
  const TraceScope trace("tridSADIStepAdjoint");
  return adi_step_adjoint<float>(u, g, ubar, lambar, lam, alpha, nx, ny, nz);
}
