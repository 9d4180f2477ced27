// The C ABI of libtridsolver_b200: the reference's four strided-batch entry
// points (scalar/include/tridsolver.h:39-69) and the extensions declared in
// include/tridsolver_b200.h.
#include <cuda_runtime.h>

#include <nvtx3/nvToolsExt.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>

#include "trid_internal.h"
#include "tridsolver.h"

namespace trid {

Settings &settings() {
  static thread_local Settings s;
  return s;
}

// ---- zero-pivot record: one host-mapped word per device -------------------
namespace {
constexpr int kMaxDevices = 64;
std::mutex g_flag_mu;
unsigned *g_flag_host = nullptr;     // kMaxDevices words, mapped
unsigned *g_flag_dev[kMaxDevices] = {};
bool g_flag_tried = false;
}  // namespace

unsigned *pivot_flag_device() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return nullptr;
  std::lock_guard<std::mutex> lk(g_flag_mu);
  if (!g_flag_tried) {
    g_flag_tried = true;
    void *h = nullptr;
    if (cudaHostAlloc(&h, kMaxDevices * sizeof(unsigned), cudaHostAllocMapped | cudaHostAllocPortable) ==
        cudaSuccess) {
      memset(h, 0, kMaxDevices * sizeof(unsigned));
      g_flag_host = static_cast<unsigned *>(h);
    } else {
      cudaGetLastError();
    }
  }
  if (!g_flag_host) return nullptr;
  if (!g_flag_dev[dev]) {
    void *dp = nullptr;
    if (cudaHostGetDevicePointer(&dp, g_flag_host + dev, 0) == cudaSuccess)
      g_flag_dev[dev] = static_cast<unsigned *>(dp);
    else
      cudaGetLastError();
  }
  return g_flag_dev[dev];
}

bool pivot_flag_take() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return false;
  unsigned *host = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_flag_mu);
    host = g_flag_host;
  }
  if (!host) return false;
  volatile unsigned *w = host + dev;
  unsigned v = *w;
  if (v) *w = 0u;
  return v != 0;
}

// ---- NVTX ranges -------------------------------------------------------------
namespace {
std::atomic<int> g_trace{-1};  // -1: not decided yet (read the environment)
}  // namespace

static bool tracing_on() {
  int v = g_trace.load(std::memory_order_relaxed);
  if (v < 0) {
    const char *env = getenv("TRIDSOLVER_NVTX");
    int undecided = -1;
    g_trace.compare_exchange_strong(undecided, env && env[0] && env[0] != '0' ? 1 : 0);
    v = g_trace.load(std::memory_order_relaxed);
  }
  return v > 0;
}

TraceScope::TraceScope(const char *name) : on_(tracing_on()) {
  if (on_) nvtxRangePushA(name);
}

TraceScope::~TraceScope() {
  if (on_) nvtxRangePop();
}

// ---- device check ----------------------------------------------------------
tridStatus_t check_device() {
  static thread_local int checked_dev = -1;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return TRID_STATUS_NOT_INITIALIZED;
  }
  if (dev == checked_dev) return TRID_STATUS_SUCCESS;
  int major = 0;
  if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev) != cudaSuccess) {
    cudaGetLastError();
    return TRID_STATUS_NOT_INITIALIZED;
  }
  if (major != 10) return TRID_STATUS_ARCH_MISMATCH;  // built for sm_100a only
  checked_dev = dev;
  return TRID_STATUS_SUCCESS;
}

tridStatus_t status_of(cudaError_t e) {
  switch (e) {
    case cudaSuccess: return TRID_STATUS_SUCCESS;
    case cudaErrorMemoryAllocation: return TRID_STATUS_ALLOC_FAILED;
    case cudaErrorNoKernelImageForDevice:
    case cudaErrorInvalidDeviceFunction: return TRID_STATUS_ARCH_MISMATCH;
    default: return TRID_STATUS_EXECUTION_FAILED;
  }
}

// Validates the strided-batch arguments and fills a BatchArgs. Returns
// SUCCESS with *empty = true when there is nothing to solve.
template <typename R>
tridStatus_t make_batch(const R *a, const R *b, const R *c, R *d, R *u, bool inc, int ndim,
                        int solvedim, const int *dims_p, const int *pads_p, BatchArgs<R> *out,
                        bool *empty) {
  if (ndim < 1 || ndim > MAXDIM || solvedim < 0 || solvedim >= ndim || !dims_p || !pads_p)
    return TRID_STATUS_INVALID_VALUE;
  long long dims[3] = {1, 1, 1}, pads[3] = {1, 1, 1};
  for (int i = 0; i < ndim; ++i) {
    if (dims_p[i] < 0) return TRID_STATUS_INVALID_VALUE;
    dims[i] = dims_p[i];
    pads[i] = pads_p[i];
    // the padded extent of every dimension that enters the index arithmetic
    // must cover its size
    if (i < ndim - 1 && pads[i] < dims[i]) return TRID_STATUS_INVALID_VALUE;
  }
  *empty = dims[0] * dims[1] * dims[2] == 0;
  if (*empty) return TRID_STATUS_SUCCESS;
  if (!a || !b || !c || !d || (inc && !u)) return TRID_STATUS_INVALID_VALUE;
  if (dims[solvedim] > 0x7fffffffLL) return TRID_STATUS_INVALID_VALUE;
  BatchArgs<R> p{};
  p.a = a;
  p.b = b;
  p.c = c;
  p.d_in = d;
  p.d_out = d;
  p.u = inc ? u : nullptr;
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
  // Systems equally spaced over both enumerating dimensions (no padding
  // between them, e.g. a z solve with pads[0] == dims[0]) are one flat
  // dimension when the fastest one is narrower than a 256-byte group:
  // groups of neighbouring systems then span its rows (8 x 8 x 2^20 FP64
  // along z: 1.48 -> 1.04 ms). Wider rows keep the two dimensions (32 x 32
  // x 65536 along z measured 6% slower flat).
  if (p.st1 == p.n0 * p.st0 && p.n0 * (long long)sizeof(R) < 256) {
    p.n0 = p.nsys;
    p.st1 = p.nsys * p.st0;
  }
  *out = p;
  return TRID_STATUS_SUCCESS;
}
template tridStatus_t make_batch<double>(const double *, const double *, const double *, double *,
                                         double *, bool, int, int, const int *, const int *,
                                         BatchArgs<double> *, bool *);
template tridStatus_t make_batch<float>(const float *, const float *, const float *, float *, float *,
                                        bool, int, int, const int *, const int *, BatchArgs<float> *,
                                        bool *);

template <typename R, bool INC>
static tridStatus_t solve_strided(const TridParams *ctx, const R *a, const R *b, const R *c, R *d,
                                  R *u, int ndim, int solvedim, const int *dims, const int *pads) {
  // opts are hints (choose_plan's plan is used for every value);
  // mpi_params selects the distributed solve only when registered
  const bool dist = ctx && dist_registered(ctx->mpi_params);
  BatchArgs<R> p;
  bool empty = false;
  tridStatus_t st = make_batch<R>(a, b, c, d, u, INC, ndim, solvedim, dims, pads, &p, &empty);
  if (st != TRID_STATUS_SUCCESS || empty) return st;
  st = check_device();
  if (st != TRID_STATUS_SUCCESS) return st;
  const Settings &cfg = settings();
  p.flag = pivot_flag_device();
  if (cfg.blocking) pivot_flag_take();  // report only this call's pivots
  if (dist)
    return dist_solve<R, INC>(static_cast<const tridDistParams *>(ctx->mpi_params), p, solvedim,
                              cfg.stream, cfg.blocking);
  const Plan plan = choose_plan<R>(p, vec_aligned<R>(p));
  cudaError_t e = launch_batch<R, INC>(p, plan, cfg.stream);
  if (e != cudaSuccess) return status_of(e);
  if (cfg.blocking) {
    e = cudaStreamSynchronize(cfg.stream);
    if (e != cudaSuccess) return status_of(e);
    if (pivot_flag_take()) return TRID_STATUS_ZERO_PIVOT;
  }
  return TRID_STATUS_SUCCESS;
}

// The generic surface of the reference's solveBatchedTrid
// (scalar/src/cuda/trid_thomaspcr.hpp:794-832): system k starts at
//   stride1 == 1:  k * stride2
//   otherwise:     (k / subBatchSize) * subBatchStride + (k % subBatchSize) * stride2
// and its rows are stride1 apart; d is read, x written (x += solution for
// Inc). That is BatchArgs with n0 = subBatchSize, st0 = stride2,
// st1 = subBatchStride; a last, partial sub-batch is a second launch.
template <typename R, bool INC>
static tridStatus_t solve_batched(const TridParams *ctx, int numTrids, int length, int stride1,
                                  int stride2, int subBatchSize, int subBatchStride, const R *a,
                                  const R *b, const R *c, const R *d, R *x) {
  (void)ctx;
  if (numTrids < 0 || length < 0 || stride1 < 1 || stride2 < 0 || subBatchStride < 0)
    return TRID_STATUS_INVALID_VALUE;
  if (numTrids == 0 || length == 0) return TRID_STATUS_SUCCESS;
  if (!a || !b || !c || !d || !x || (stride1 != 1 && subBatchSize < 1)) return TRID_STATUS_INVALID_VALUE;
  tridStatus_t st = check_device();
  if (st != TRID_STATUS_SUCCESS) return st;
  const Settings &cfg = settings();
  BatchArgs<R> p{};
  p.a = a;
  p.b = b;
  p.c = c;
  p.d_in = d;
  p.d_out = INC ? nullptr : x;
  p.u = INC ? x : nullptr;
  p.N = length;
  p.stride = stride1;
  p.flag = pivot_flag_device();
  if (cfg.blocking) pivot_flag_take();
  auto run = [&](const BatchArgs<R> &q) -> cudaError_t {
    const Plan plan = choose_plan<R>(q, vec_aligned<R>(q));
    return launch_batch<R, INC>(q, plan, cfg.stream);
  };
  cudaError_t e = cudaSuccess;
  if (stride1 == 1) {
    p.n0 = numTrids;
    p.nsys = numTrids;
    p.st0 = stride2;
    p.st1 = 0;
    e = run(p);
  } else {
    const long long full = numTrids / subBatchSize, rem = numTrids % subBatchSize;
    p.n0 = subBatchSize;
    p.st0 = stride2;
    p.st1 = subBatchStride;
    if (full > 0) {
      p.nsys = full * subBatchSize;
      e = run(p);
    }
    if (e == cudaSuccess && rem > 0) {
      const long long o = full * (long long)subBatchStride;
      BatchArgs<R> q = p;
      q.a = a + o;
      q.b = b + o;
      q.c = c + o;
      q.d_in = d + o;
      q.d_out = INC ? nullptr : x + o;
      q.u = INC ? x + o : nullptr;
      q.n0 = rem;
      q.nsys = rem;
      q.st1 = 0;
      e = run(q);
    }
  }
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

EXTERN_C tridStatus_t tridDsolveBatchedTrid(const TridParams *ctx, int numTrids, int length,
                                            int stride1, int stride2, int subBatchSize,
                                            int subBatchStride, const double *a, const double *b,
                                            const double *c, const double *d, double *x) {
  const TraceScope trace("tridDsolveBatchedTrid");
  return solve_batched<double, false>(ctx, numTrids, length, stride1, stride2, subBatchSize,
                                      subBatchStride, a, b, c, d, x);
}

EXTERN_C tridStatus_t tridSsolveBatchedTrid(const TridParams *ctx, int numTrids, int length,
                                            int stride1, int stride2, int subBatchSize,
                                            int subBatchStride, const float *a, const float *b,
                                            const float *c, const float *d, float *x) {
  const TraceScope trace("tridSsolveBatchedTrid");
  return solve_batched<float, false>(ctx, numTrids, length, stride1, stride2, subBatchSize,
                                     subBatchStride, a, b, c, d, x);
}

EXTERN_C tridStatus_t tridDsolveBatchedTridInc(const TridParams *ctx, int numTrids, int length,
                                               int stride1, int stride2, int subBatchSize,
                                               int subBatchStride, const double *a,
                                               const double *b, const double *c, const double *d,
                                               double *x) {
  const TraceScope trace("tridDsolveBatchedTridInc");
  return solve_batched<double, true>(ctx, numTrids, length, stride1, stride2, subBatchSize,
                                     subBatchStride, a, b, c, d, x);
}

EXTERN_C tridStatus_t tridSsolveBatchedTridInc(const TridParams *ctx, int numTrids, int length,
                                               int stride1, int stride2, int subBatchSize,
                                               int subBatchStride, const float *a, const float *b,
                                               const float *c, const float *d, float *x) {
  const TraceScope trace("tridSsolveBatchedTridInc");
  return solve_batched<float, true>(ctx, numTrids, length, stride1, stride2, subBatchSize,
                                    subBatchStride, a, b, c, d, x);
}

EXTERN_C tridStatus_t tridDmtsvStridedBatch(const TridParams *ctx, const double *a, const double *b,
                                            const double *c, double *d, int ndim, int solvedim,
                                            const int *dims, const int *pads) {
  const TraceScope trace("tridDmtsvStridedBatch");
  return solve_strided<double, false>(ctx, a, b, c, d, nullptr, ndim, solvedim, dims, pads);
}

EXTERN_C tridStatus_t tridSmtsvStridedBatch(const TridParams *ctx, const float *a, const float *b,
                                            const float *c, float *d, int ndim, int solvedim,
                                            const int *dims, const int *pads) {
  const TraceScope trace("tridSmtsvStridedBatch");
  return solve_strided<float, false>(ctx, a, b, c, d, nullptr, ndim, solvedim, dims, pads);
}

EXTERN_C tridStatus_t tridDmtsvStridedBatchInc(const TridParams *ctx, const double *a,
                                               const double *b, const double *c, double *d,
                                               double *u, int ndim, int solvedim, const int *dims,
                                               const int *pads) {
  const TraceScope trace("tridDmtsvStridedBatchInc");
  return solve_strided<double, true>(ctx, a, b, c, d, u, ndim, solvedim, dims, pads);
}

EXTERN_C tridStatus_t tridSmtsvStridedBatchInc(const TridParams *ctx, const float *a,
                                               const float *b, const float *c, float *d, float *u,
                                               int ndim, int solvedim, const int *dims,
                                               const int *pads) {
  const TraceScope trace("tridSmtsvStridedBatchInc");
  return solve_strided<float, true>(ctx, a, b, c, d, u, ndim, solvedim, dims, pads);
}

// ---- extensions -------------------------------------------------------------

EXTERN_C tridStatus_t tridSetStream(void *cuda_stream) {
  settings().stream = static_cast<cudaStream_t>(cuda_stream);
  return TRID_STATUS_SUCCESS;
}

EXTERN_C void *tridGetStream(void) { return settings().stream; }

EXTERN_C tridStatus_t tridSetBlocking(int blocking) {
  settings().blocking = blocking != 0;
  return TRID_STATUS_SUCCESS;
}

EXTERN_C int tridGetBlocking(void) { return settings().blocking ? 1 : 0; }

EXTERN_C tridStatus_t tridGetPivotStatus(void) {
  return pivot_flag_take() ? TRID_STATUS_ZERO_PIVOT : TRID_STATUS_SUCCESS;
}

EXTERN_C unsigned long long tridGetLaunchCount(void) { return g_launches.load(); }

EXTERN_C tridStatus_t tridReleaseScratch(void) { return status_of(scratch_release()); }

EXTERN_C tridStatus_t tridSetTracing(int on) {
  g_trace.store(on ? 1 : 0, std::memory_order_relaxed);
  return TRID_STATUS_SUCCESS;
}

EXTERN_C tridStatus_t tridForcePlan(int family, int rows_per_thread) {
  Settings &s = settings();
  if (family < 0) {
    s.force_family = TRID_FAMILY_AUTO;
    s.force_m = 0;
    return TRID_STATUS_SUCCESS;
  }
  if (family > TRID_FAMILY_LONG) return TRID_STATUS_INVALID_VALUE;
  const int m = rows_per_thread;
  if (family == TRID_FAMILY_HYBRID && !(m == 0 || m == 2 || m == 4 || m == 8 || m == 16 || m == 32))
    return TRID_STATUS_INVALID_VALUE;
  if (family == TRID_FAMILY_LONG && !(m == 0 || m == 8 || m == 16)) return TRID_STATUS_INVALID_VALUE;
  s.force_family = family;
  s.force_m = m;
  return TRID_STATUS_SUCCESS;
}

EXTERN_C tridStatus_t tridForceSystemsPerBlock(int systems) {
  if (systems < 0 || systems > 256 || (systems & (systems - 1))) return TRID_STATUS_INVALID_VALUE;
  settings().force_w = systems;
  return TRID_STATUS_SUCCESS;
}

EXTERN_C tridStatus_t tridForceTma(int mode) {
  if (mode < -1 || mode > 1) return TRID_STATUS_INVALID_VALUE;
  settings().force_tma = mode;
  return TRID_STATUS_SUCCESS;
}

EXTERN_C tridStatus_t tridForceStream(int mode) {
  if (mode < -1 || mode > 2) return TRID_STATUS_INVALID_VALUE;
  settings().force_stream = mode;
  return TRID_STATUS_SUCCESS;
}

EXTERN_C tridStatus_t tridSetMixedMode(int mode) {
  if (mode < 0 || mode > 2) return TRID_STATUS_INVALID_VALUE;
  settings().mixed_mode = mode;
  return TRID_STATUS_SUCCESS;
}

EXTERN_C int tridDescribePlanInc(int dtype_bytes, int ndim, int solvedim, const int *dims,
                                 const int *pads, int inc, char *buf, int buflen) {
  std::string desc;
  bool empty = false;
  // alignment is taken as satisfied: the description is of the shape only
  if (dtype_bytes == 8) {
    BatchArgs<double> p;
    double *dummy = reinterpret_cast<double *>(256);
    if (make_batch<double>(dummy, dummy, dummy, dummy, inc ? dummy : nullptr, inc != 0, ndim, solvedim,
                           dims, pads, &p, &empty) != TRID_STATUS_SUCCESS)
      return -1;
    desc = empty ? "empty" : choose_plan<double>(p, vec_aligned<double>(p)).describe();
  } else if (dtype_bytes == 4) {
    BatchArgs<float> p;
    float *dummy = reinterpret_cast<float *>(256);
    if (make_batch<float>(dummy, dummy, dummy, dummy, inc ? dummy : nullptr, inc != 0, ndim, solvedim,
                          dims, pads, &p, &empty) != TRID_STATUS_SUCCESS)
      return -1;
    desc = empty ? "empty" : choose_plan<float>(p, vec_aligned<float>(p)).describe();
  } else {
    return -1;
  }
  if (buf && buflen > 0) {
    strncpy(buf, desc.c_str(), (size_t)buflen - 1);
    buf[buflen - 1] = '\0';
  }
  return (int)desc.size();
}

EXTERN_C int tridDescribePlan(int dtype_bytes, int ndim, int solvedim, const int *dims,
                              const int *pads, char *buf, int buflen) {
  return tridDescribePlanInc(dtype_bytes, ndim, solvedim, dims, pads, 0, buf, buflen);
}
