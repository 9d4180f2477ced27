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
// The matrices have identity rows on the boundary and constant interior
// rows, so each transpose's interior block is the matrix's own: T^-T g is the
// solve of g's interior rows (its boundary rows taken as 0), with the
// boundary rows then w_0 = g_0 + alpha lambda w_1, w_{N-1} = g_{N-1} +
// alpha lambda w_{N-2} on interior lines, and w = g on boundary lines. For
// edges up to 512 the fused step's kernels do all solves: the forward
// intermediates recomputed from u (the x solve with the stencil, then y and
// z on copies), the transposed solves in place in their transposed mode;
// two kernels here add the boundary-row couplings, form the stencil
// transpose and reduce the lambda derivative (in FP64), so the backward of
// a step runs natively in about 28 words of memory traffic per point.
// Longer edges (up to 1024) take the coefficient-array form of the step and
// the library's array adjoint solves (51 words). No counterpart in the
// reference, which has no derivatives.
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

// Both kernels below walk the grid by x lines: block b takes lines (j, k)
// = (l % ny, l / ny) for l = b, b + gridDim.x, ... and its threads the
// points i of the line, so the index arithmetic is one 32-bit division per
// line and the accesses are coalesced.

// acc += alpha * sum over interior p of w[p] (x[p-e] - 2 x[p] + x[p+e]),
// e = the solve axis' stride
template <typename R>
__global__ void __launch_bounds__(kThreads)
    adi_coef_grad_kernel(const R *__restrict__ w, const R *__restrict__ x, long long e, R alpha,
                         int nx, int ny, int nz, double *acc) {
  const int lines = ny * nz;
  double s = 0.0;
  for (int l = blockIdx.x; l < lines; l += gridDim.x) {
    const int k = l / ny;
    const int j = l - k * ny;
    if (j == 0 || j == ny - 1 || k == 0 || k == nz - 1) continue;  // uniform per block
    const long long b = (long long)l * nx;
    for (int i = 1 + threadIdx.x; i < nx - 1; i += blockDim.x) {
      const long long p = b + i;
      s += (double)w[p] * ((double)x[p - e] - 2.0 * (double)x[p] + (double)x[p + e]);
    }
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
  const R l0 = lam[0];
  const long long nxy = (long long)nx * ny;
  const int lines = ny * nz;
  double s = 0.0;
  for (int l = blockIdx.x; l < lines; l += gridDim.x) {
    const int k = l / ny;
    const int j = l - k * ny;
    const bool jk_in = j > 0 && j < ny - 1 && k > 0 && k < nz - 1;
    // which neighbouring lines (j -+ 1, k -+ 1) are interior lines
    const bool jm = j - 1 > 0 && k > 0 && k < nz - 1, jp = j + 1 < ny - 1 && k > 0 && k < nz - 1;
    const bool km = k - 1 > 0 && j > 0 && j < ny - 1, kp = k + 1 < nz - 1 && j > 0 && j < ny - 1;
    const long long b = (long long)l * nx;
    for (int i = threadIdx.x; i < nx; i += blockDim.x) {
      const long long q = b + i;
      const bool iin = i > 0 && i < nx - 1;
      const bool in = jk_in && iin;
      R lt = in ? R(-6) * w1[q] : R(0);
      // x neighbours on the same line: interior when the line is
      if (jk_in && i - 1 > 0) lt += w1[q - 1];
      if (jk_in && i + 1 < nx - 1) lt += w1[q + 1];
      if (iin && jm) lt += w1[q - nx];
      if (iin && jp) lt += w1[q + nx];
      if (iin && km) lt += w1[q - nxy];
      if (iin && kp) lt += w1[q + nxy];
      ubar[q] = g[q] + l0 * lt;
      if (in) {
        const R lu = u[q - 1] + u[q + 1] + u[q - nx] + u[q + nx] + u[q - nxy] + u[q + nxy] - R(6) * u[q];
        s += (double)w1[q] * (double)lu;
      }
    }
  }
  block_sum_add(s, acc);
}

template <typename R> __global__ void adi_lambar_kernel(const double *acc, R *lambar) {
  if (threadIdx.x == 0 && blockIdx.x == 0) lambar[0] += (R)acc[0];
}

// The transposed matrix's boundary rows: on every interior line along the
// axis (stride e, N >= 3 rows), w_0 = g_0 + alpha lambda w_1 and w_{N-1} =
// g_{N-1} + alpha lambda w_{N-2}, where w_0, w_{N-1} still hold g_0, g_{N-1}
// (the transposed solves leave them) and w_1, w_{N-2} are solved.
template <typename R>
__global__ void __launch_bounds__(kThreads)
    adi_transposed_fixup_kernel(R *w, const R *lam, R alpha, int axis, int nx, int ny, int nz) {
  const R al = alpha * lam[0];
  const int dims[3] = {nx, ny, nz};
  const long long es[3] = {1, nx, (long long)nx * ny};
  const int N = dims[axis];
  const int o1 = axis == 0 ? 1 : 0, o2 = axis == 2 ? 1 : 2;  // the other two axes
  const int n1 = dims[o1], n2 = dims[o2];
  if (N < 3 || n1 < 3 || n2 < 3) return;
  const long long lines = (long long)(n1 - 2) * (n2 - 2);
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < lines;
       q += (long long)gridDim.x * blockDim.x) {
    const long long i1 = 1 + q % (n1 - 2);
    const long long i2 = 1 + q / (n1 - 2);
    const long long e = es[axis];
    const long long b = i1 * es[o1] + i2 * es[o2];
    w[b] += al * w[b + e];
    w[b + (N - 1) * e] += al * w[b + (N - 2) * e];
  }
}

}  // namespace

// BatchArgs of the step's y or z solve, in place on d (the fused kernels'
// addressing: systems along x fastest).
template <typename R> static BatchArgs<R> step_batch(R *d, int axis, int nx, int ny, int nz) {
  BatchArgs<R> p{};
  p.d_in = d;
  p.d_out = d;
  p.n0 = nx;
  p.st0 = 1;
  if (axis == 1) {
    p.N = ny;
    p.nsys = (long long)nx * nz;
    p.st1 = (long long)nx * ny;
    p.stride = nx;
  } else {
    p.N = nz;
    p.nsys = (long long)nx * ny;
    p.st1 = nx;
    p.stride = (long long)nx * ny;
  }
  return p;
}

// The adjoint with the fused constant-coefficient kernels (edges up to 512):
// the forward intermediates recomputed by the fused step's own solves (x1
// from u with the stencil, then y and z on copies), the transposed solves in
// place on w = g as the same solves of the interior rows plus the two
// boundary-row couplings. About 28 words of memory traffic per point.
template <typename R>
static cudaError_t adi_adjoint_fused(const R *u, const R *g, R *ubar, R *lambar, const R *lam,
                                     R alpha, int nx, int ny, int nz, unsigned *flag,
                                     cudaStream_t st) {
  const long long n = (long long)nx * ny * nz;
  const size_t bytes = (size_t)n * sizeof(R);
  const size_t slot = (bytes + 255) / 256 * 256;
  char *scratch = nullptr;
  cudaError_t e = scratch_alloc((void **)&scratch, 4 * slot + 256, st);
  if (e != cudaSuccess) return e;
  R *x1 = reinterpret_cast<R *>(scratch), *x2 = reinterpret_cast<R *>(scratch + slot),
    *x3 = reinterpret_cast<R *>(scratch + 2 * slot), *w = reinterpret_cast<R *>(scratch + 3 * slot);
  double *acc = reinterpret_cast<double *>(scratch + 4 * slot);
  const ConstCoef<R> k{lam, nullptr, alpha};
  // the line kernels: one block per x line, at most 16 per SM resident
  long long blocks = (long long)ny * nz;
  if (blocks > 148LL * 16) blocks = 148LL * 16;
  long long lblocks = ((long long)(nx > ny ? nx : ny) * (ny > nz ? ny : nz) + kThreads - 1) / kThreads;
  if (lblocks > 148LL * 8) lblocks = 148LL * 8;
  const long long estride[3] = {1, nx, (long long)nx * ny};
  e = cudaMemsetAsync(acc, 0, sizeof(double), st);
  if (e == cudaSuccess) e = launch_adi_x<R>(u, x1, k, flag, nx, ny, nz, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(x2, x1, bytes, cudaMemcpyDeviceToDevice, st);
  if (e == cudaSuccess) {
    BatchArgs<R> p = step_batch<R>(x2, 1, nx, ny, nz);
    p.flag = flag;
    e = launch_adi_yz<R, false>(p, k, st);
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(x3, x2, bytes, cudaMemcpyDeviceToDevice, st);
  if (e == cudaSuccess) {
    BatchArgs<R> p = step_batch<R>(x3, 2, nx, ny, nz);
    p.flag = flag;
    e = launch_adi_yz<R, false>(p, k, st);
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(w, g, bytes, cudaMemcpyDeviceToDevice, st);
  g_launches.fetch_add(3, std::memory_order_relaxed);
  R *xs[3] = {x1, x2, x3};
  for (int sd = 2; sd >= 0 && e == cudaSuccess; --sd) {
    if (sd == 0) {
      e = launch_adi_x_transposed<R>(w, k, nx, ny, nz, st);
    } else {
      BatchArgs<R> p = step_batch<R>(w, sd, nx, ny, nz);
      p.flag = flag;
      e = launch_adi_yz_transposed<R>(p, k, st);
    }
    if (e != cudaSuccess) break;
    adi_transposed_fixup_kernel<R><<<(unsigned)(lblocks < 1 ? 1 : lblocks), kThreads, 0, st>>>(
        w, lam, alpha, sd, nx, ny, nz);
    adi_coef_grad_kernel<R><<<(unsigned)blocks, kThreads, 0, st>>>(w, xs[sd], estride[sd], alpha, nx,
                                                                 ny, nz, acc);
    g_launches.fetch_add(3, std::memory_order_relaxed);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) {
    adi_stencil_adjoint_kernel<R><<<(unsigned)blocks, kThreads, 0, st>>>(u, w, g, ubar, lam, nx, ny,
                                                                       nz, acc);
    adi_lambar_kernel<R><<<1, 32, 0, st>>>(acc, lambar);
    g_launches.fetch_add(2, std::memory_order_relaxed);
    e = cudaGetLastError();
  }
  const cudaError_t ef = scratch_free(scratch, st);
  return e != cudaSuccess ? e : ef;
}

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
  if (nx <= 512 && ny <= 512 && nz <= 512) {
    const cudaError_t e = adi_adjoint_fused<R>(u, g, ubar, lambar, lam, alpha, nx, ny, nz, flag, st);
    if (e != cudaSuccess) return status_of(e);
    if (blocking) {
      const cudaError_t es = cudaStreamSynchronize(st);
      if (es != cudaSuccess) return status_of(es);
      if (pivot_flag_take()) return TRID_STATUS_ZERO_PIVOT;
    }
    return TRID_STATUS_SUCCESS;
  }
  // longer edges: the coefficient-array form
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
  long long blocks = (long long)ny * nz;
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
