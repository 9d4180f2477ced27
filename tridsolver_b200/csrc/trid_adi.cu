// One ADI heat-diffusion timestep on an nx x ny x nz grid (x fastest, no
// padding), the computation of the reference's ADI application
// (apps/adi/src/adi_cuda.cu:282-326 with preproc.cu:40-90):
//
//   du  = lambda * (sum of the 6 neighbours of u - 6 u)   interior points
//   du  = 0, a = c = 0, b = 1                             boundary points
//   a = c = -alpha*lambda, b = 1 + 2*alpha*lambda         interior points
//   du <- solve_x(du);  du <- solve_y(du);  u += solve_z(du)
//
// alpha = 1 gives the coefficients a = c = -lambda, b = 1 + 2 lambda;
// alpha = 0.5 the reference application's a = c = -lambda/2, b = 1 + lambda.
// lambda is read on the device from lam[*step] (lam[0] when step is NULL), and
// *step is advanced by one at the end of the timestep, so a captured CUDA
// graph of one timestep replays a sequence of per-step lambdas. The reference
// writes nine coefficient arrays (x, y and z copies of identical values). With
// a, b, c given, the three directions here share one set (a preprocessing
// kernel and three array solves, 21 words of traffic per point); with a, b, c
// all NULL the coefficients stay three scalars and the stencil is fused into
// the x solve (three kernels, 7 words per point).
#include <cuda_runtime.h>

#include "trid_internal.h"
#include "tridsolver_b200.h"

namespace trid {

template <typename R>
__global__ void __launch_bounds__(256) adi_preproc_kernel(const R *__restrict__ u, R *__restrict__ du,
                                                          R *__restrict__ a, R *__restrict__ b,
                                                          R *__restrict__ c, const R *lam,
                                                          const int *step, R alpha, int nx, int ny,
                                                          int nz) {
  const R l = lam[step ? *step : 0];
  const R ca = -alpha * l;
  const R cb = R(1) + R(2) * alpha * l;
  const long long nxy = (long long)nx * ny;
  const long long n = nxy * nz;
  for (long long ind = (long long)blockIdx.x * blockDim.x + threadIdx.x; ind < n;
       ind += (long long)gridDim.x * blockDim.x) {
    const long long k = ind / nxy;
    const long long r = ind - k * nxy;
    const long long j = r / nx;
    const long long i = r - j * nx;
    const bool bnd = i == 0 || i == nx - 1 || j == 0 || j == ny - 1 || k == 0 || k == nz - 1;
    if (bnd) {
      du[ind] = R(0);
      a[ind] = R(0);
      b[ind] = R(1);
      c[ind] = R(0);
    } else {
      const R s6 = u[ind - 1] + u[ind + 1] + u[ind - nx] + u[ind + nx] + u[ind - nxy] + u[ind + nxy];
      du[ind] = l * (s6 - R(6) * u[ind]);
      a[ind] = ca;
      b[ind] = cb;
      c[ind] = ca;
    }
  }
}

template <typename R>
cudaError_t launch_adi_preproc(const R *u, R *du, R *a, R *b, R *c, const R *lam, const int *step,
                               R alpha, int nx, int ny, int nz, cudaStream_t st) {
  const long long n = (long long)nx * ny * nz;
  const int threads = 256;
  long long blocks = (n + threads - 1) / threads;
  if (blocks > 148LL * 64) blocks = 148LL * 64;
  adi_preproc_kernel<R><<<(unsigned)blocks, threads, 0, st>>>(u, du, a, b, c, lam, step, alpha, nx, ny,
                                                            nz);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return cudaGetLastError();
}
template cudaError_t launch_adi_preproc<double>(const double *, double *, double *, double *,
                                                double *, const double *, const int *, double, int,
                                                int, int, cudaStream_t);
template cudaError_t launch_adi_preproc<float>(const float *, float *, float *, float *, float *,
                                               const float *, const int *, float, int, int, int,
                                               cudaStream_t);

__global__ void adi_advance_kernel(int *step) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *step += 1;
}

// The fused timestep: x solve with the stencil, y solve, z solve into u.
template <typename R>
static cudaError_t adi_fused(R *u, R *du, const ConstCoef<R> &k, unsigned *flag, int nx, int ny,
                             int nz, cudaStream_t st) {
  cudaError_t e = launch_adi_x<R>(u, du, k, flag, nx, ny, nz, st);
  if (e != cudaSuccess) return e;
  g_launches.fetch_add(1, std::memory_order_relaxed);
  BatchArgs<R> p{};
  p.d_in = du;
  p.d_out = du;
  p.flag = flag;
  p.n0 = nx;
  p.st0 = 1;
  // y: systems (x, z), rows nx apart
  p.N = ny;
  p.nsys = (long long)nx * nz;
  p.st1 = (long long)nx * ny;
  p.stride = nx;
  e = launch_adi_yz<R, false>(p, k, st);
  if (e != cudaSuccess) return e;
  g_launches.fetch_add(1, std::memory_order_relaxed);
  // z: systems (x, y), rows a plane apart, u += x
  p.u = u;
  p.N = nz;
  p.nsys = (long long)nx * ny;
  p.st1 = nx;
  p.stride = (long long)nx * ny;
  e = launch_adi_yz<R, true>(p, k, st);
  if (e == cudaSuccess) g_launches.fetch_add(1, std::memory_order_relaxed);
  return e;
}

// The array form: preprocessing kernel (RHS and one shared coefficient set)
// and three array solves; a, b, c NULL takes them from the library's pool
// (the fused form's fallback for systems longer than 512 rows).
template <typename R>
static cudaError_t adi_arrays(R *u, R *du, R *a, R *b, R *c, const R *lam, int *step, R alpha,
                              unsigned *flag, int nx, int ny, int nz, cudaStream_t st) {
  const long long n = (long long)nx * ny * nz;
  R *scratch = nullptr;
  if (!a) {
    const cudaError_t e = scratch_alloc((void **)&scratch, (size_t)3 * n * sizeof(R), st);
    if (e != cudaSuccess) return e;
    a = scratch;
    b = scratch + n;
    c = scratch + 2 * n;
  }
  cudaError_t e = launch_adi_preproc<R>(u, du, a, b, c, lam, step, alpha, nx, ny, nz, st);
  const long long dims[3] = {nx, ny, nz};
  for (int sd = 0; sd < 3 && e == cudaSuccess; ++sd) {
    BatchArgs<R> p{};
    p.a = a;
    p.b = b;
    p.c = c;
    p.d_in = du;
    p.d_out = du;
    p.u = sd == 2 ? u : nullptr;
    p.N = (int)dims[sd];
    p.flag = flag;
    if (sd == 0) {
      p.n0 = ny;
      p.nsys = (long long)ny * nz;
      p.st0 = nx;
      p.st1 = (long long)nx * ny;
      p.stride = 1;
    } else if (sd == 1) {
      p.n0 = nx;
      p.nsys = (long long)nx * nz;
      p.st0 = 1;
      p.st1 = (long long)nx * ny;
      p.stride = nx;
    } else {
      p.n0 = nx;
      p.nsys = (long long)nx * ny;
      p.st0 = 1;
      p.st1 = nx;
      p.stride = (long long)nx * ny;
    }
    const Plan plan = choose_plan<R>(p, vec_aligned<R>(p), false);
    e = sd == 2 ? launch_batch<R, true>(p, plan, st) : launch_batch<R, false>(p, plan, st);
  }
  if (scratch) {
    const cudaError_t ef = scratch_free(scratch, st);
    if (e == cudaSuccess) e = ef;
  }
  return e;
}

template <typename R>
static tridStatus_t adi_step(R *u, R *du, R *a, R *b, R *c, const R *lam, int *step, R alpha,
                             int nx, int ny, int nz) {
  const bool arrays = a || b || c;
  if (!u || !du || !lam || nx < 1 || ny < 1 || nz < 1 || (arrays && (!a || !b || !c)))
    return TRID_STATUS_INVALID_VALUE;
  int dev = 0, major = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev) != cudaSuccess) {
    cudaGetLastError();
    return TRID_STATUS_NOT_INITIALIZED;
  }
  if (major != 10) return TRID_STATUS_ARCH_MISMATCH;
  const Settings &cfg = settings();
  cudaStream_t st = cfg.stream;
  unsigned *flag = pivot_flag_device();
  if (cfg.blocking) pivot_flag_take();
  cudaError_t e;
  if (!arrays && nx <= 512 && ny <= 512 && nz <= 512)
    e = adi_fused<R>(u, du, ConstCoef<R>{lam, step, alpha}, flag, nx, ny, nz, st);
  else
    e = adi_arrays<R>(u, du, a, b, c, lam, step, alpha, flag, nx, ny, nz, st);
  if (e == cudaSuccess && step) {
    adi_advance_kernel<<<1, 32, 0, st>>>(step);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) return status_of(e);
  if (cfg.blocking) {
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return status_of(e);
    if (pivot_flag_take()) return TRID_STATUS_ZERO_PIVOT;
  }
  return TRID_STATUS_SUCCESS;
}

}  // namespace trid

using namespace trid;

EXTERN_C tridStatus_t tridDADIStep(double *u, double *du, double *a, double *b, double *c,
                                   const double *lam, int *step, double alpha, int nx, int ny,
                                   int nz) {
  const TraceScope trace("tridDADIStep");
  return adi_step<double>(u, du, a, b, c, lam, step, alpha, nx, ny, nz);
}

EXTERN_C tridStatus_t tridSADIStep(float *u, float *du, float *a, float *b, float *c,
                                   const float *lam, int *step, float alpha, int nx, int ny,
                                   int nz) {
  const TraceScope trace("tridSADIStep");
  return adi_step<float>(u, du, a, b, c, lam, step, alpha, nx, ny, nz);
}
