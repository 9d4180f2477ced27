// tridDmtsvStridedBatchNoAlloc: the FP64 strided-batch solve for callers that
// must not allocate device memory.
//
// Who needs it: the regular entry points allocate scratch for systems longer
// than one warp holds (the long path takes stream-ordered memory from the
// driver's pool), and the first call also pins a small host word for pivot
// reporting. Some callers cannot allow that: services that reserve all device
// memory up front and account for every byte, real-time loops where an
// allocation's latency or failure is not acceptable, and code running where a
// new allocation would interfere with its own memory management. This entry
// point solves the same problems with no allocation at all: the long path's
// reduced systems and the pivot word live in one fixed array in device memory,
// declared below, that every GPU which loads the library holds until the
// process exits.
//
// Limits and sharing rules:
//   * the array holds kNoAllocScratchBytes (16 MiB); a problem whose reduced
//     systems need more is rejected with TRID_STATUS_INVALID_VALUE and a
//     one-line message on stderr, before anything is launched. Systems short
//     enough for the single-warp kernels (N <= 512 along x, N <= 1024 along y
//     or z) need no scratch and have no limit;
//   * every call uses the same array and leaves its last contents in it. The
//     pivot word is cleared at the start of each call; the reduced systems are
//     written in full before they are read, so nothing else must start at
//     zero;
//   * calls whose work overlaps on the GPU (two streams, or two host threads
//     on one device) race on the array; serialise them;
//   * the first call on each device looks up the array's device address with
//     that device current (cudaGetSymbolAddress) and caches it; make that
//     first call before any stream capture. The cached address is not looked
//     up again, so a cudaDeviceReset after the first call (which unloads the
//     library's device code) is not supported;
//   * the plan is always the automatic one: tridForcePlan and the other
//     tridForce* settings of the calling thread are ignored;
//   * a ctx whose mpi_params were registered by tridDistInit (the distributed
//     solve, whose exchange allocates) is refused with
//     TRID_STATUS_INVALID_VALUE instead of solving only the local block.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "trid_internal.h"
#include "tridsolver_b200.h"

namespace trid {
namespace {

constexpr size_t kNoAllocScratchBytes = size_t(16) << 20;
constexpr size_t kFlagBytes = 256;  // the pivot word, then the reduced systems
constexpr int kMaxDev = 64;

// The fixed scratch. Host code must not use this name as an address: its
// device address comes from cudaGetSymbolAddress, per device.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_mu;
unsigned char *g_scratch_ptr[kMaxDev] = {};

// Device address of the fixed array on the current device, looked up once.
cudaError_t scratch_address(unsigned char **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDev) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_scratch_ptr[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_ptr[dev] = static_cast<unsigned char *>(p);
  }
  *out = g_scratch_ptr[dev];
  return cudaSuccess;
}

// Argument checks and the batch description, as the regular entry points do.
tridStatus_t describe_batch(const double *a, const double *b, const double *c, double *d, int ndim,
                            int solvedim, const int *dims_p, const int *pads_p, BatchArgs<double> *out,
                            bool *empty) {
  if (ndim < 1 || ndim > MAXDIM || solvedim < 0 || solvedim >= ndim || !dims_p || !pads_p)
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
  if (!a || !b || !c || !d || dims[solvedim] > 0x7fffffffLL) return TRID_STATUS_INVALID_VALUE;
  BatchArgs<double> p{};
  p.a = a;
  p.b = b;
  p.c = c;
  p.d_in = d;
  p.d_out = d;
  p.u = nullptr;
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
  *out = p;
  return TRID_STATUS_SUCCESS;
}

tridStatus_t to_status(cudaError_t e) {
  if (e == cudaSuccess) return TRID_STATUS_SUCCESS;
  if (e == cudaErrorNoKernelImageForDevice || e == cudaErrorInvalidDeviceFunction)
    return TRID_STATUS_ARCH_MISMATCH;
  return TRID_STATUS_EXECUTION_FAILED;
}

constexpr int kM = 16;          // rows per chunk on the long path
constexpr int kLevelsMax = 8;

}  // namespace
}  // namespace trid

using namespace trid;

EXTERN_C tridStatus_t tridDmtsvStridedBatchNoAlloc(const TridParams *ctx, const double *a,
                                                   const double *b, const double *c, double *d,
                                                   int ndim, int solvedim, const int *dims,
                                                   const int *pads) {
  const TraceScope trace("tridDmtsvStridedBatchNoAlloc");
  if (ctx && dist_registered(ctx->mpi_params)) {
    fprintf(stderr,
            "tridDmtsvStridedBatchNoAlloc: ctx->mpi_params selects the distributed solve, which this "
            "entry point does not provide (use tridDmtsvStridedBatch)\n");
    return TRID_STATUS_INVALID_VALUE;
  }
  BatchArgs<double> p;
  bool empty = false;
  tridStatus_t st = describe_batch(a, b, c, d, ndim, solvedim, dims, pads, &p, &empty);
  if (st != TRID_STATUS_SUCCESS || empty) return st;

  int dev = 0, major = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev) != cudaSuccess) {
    cudaGetLastError();
    return TRID_STATUS_NOT_INITIALIZED;
  }
  if (major != 10) return TRID_STATUS_ARCH_MISMATCH;
  unsigned char *base = nullptr;
  cudaError_t e = scratch_address(&base);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return TRID_STATUS_NOT_INITIALIZED;
  }
  unsigned *flag = reinterpret_cast<unsigned *>(base);
  double *work = reinterpret_cast<double *>(base + kFlagBytes);
  const size_t capacity = (kNoAllocScratchBytes - kFlagBytes) / sizeof(double);
  p.flag = flag;

  // The plan the regular entry point would take; only the long path needs
  // scratch. Its levels: the reduced batch of level l (2 rows per chunk of
  // kM rows) is solved by level l+1 until it fits one warp per system.
  const Plan plan = choose_plan<double>(p, vec_aligned<double>(p), false);
  BatchArgs<double> lv[kLevelsMax + 1];
  long long nc[kLevelsMax] = {};
  long long nred[kLevelsMax] = {};
  int levels = 0;
  if (plan.family == TRID_FAMILY_LONG) {
    size_t need = 0;
    BatchArgs<double> cur = p;
    for (;;) {
      if (levels == kLevelsMax) return TRID_STATUS_INVALID_VALUE;
      const long long ncl = ((long long)cur.N + kM - 1) / kM;
      lv[levels] = cur;
      nc[levels] = ncl;
      nred[levels] = cur.nsys * 2 * ncl;
      need += 4 * (size_t)nred[levels];
      BatchArgs<double> q{};
      q.N = (int)(2 * ncl);
      q.nsys = cur.nsys;
      q.n0 = cur.nsys;
      q.st0 = 2 * ncl;
      q.st1 = 0;
      q.stride = 1;
      q.flag = flag;
      ++levels;
      cur = q;
      if (choose_plan<double>(q, false, false).family != TRID_FAMILY_LONG) break;
    }
    lv[levels] = cur;
    if (need > capacity) {
      fprintf(stderr,
              "tridDmtsvStridedBatchNoAlloc: this problem needs %zu bytes of scratch; the fixed "
              "array holds %zu (use tridDmtsvStridedBatch, which allocates)\n",
              need * sizeof(double) + kFlagBytes, kNoAllocScratchBytes);
      return TRID_STATUS_INVALID_VALUE;
    }
    size_t off = 0;
    for (int l = 0; l < levels; ++l) {
      double *ra = work + off;
      const long long n = nred[l];
      off += 4 * (size_t)n;
      lv[l + 1].a = ra;
      lv[l + 1].b = ra + n;
      lv[l + 1].c = ra + 2 * n;
      lv[l + 1].d_in = ra + 3 * n;
      lv[l + 1].d_out = ra + 3 * n;
    }
  }

  const Settings &cfg = settings();
  cudaStream_t stream = cfg.stream;
  e = cudaMemsetAsync(flag, 0, sizeof(unsigned), stream);
  if (e == cudaSuccess && plan.family != TRID_FAMILY_LONG) {
    e = launch_batch<double, false>(p, plan, stream);
  } else if (e == cudaSuccess) {
    const int threads = 128;
    for (int l = 0; l < levels && e == cudaSuccess; ++l) {
      const BatchArgs<double> &q = lv[l + 1];
      const long long blocks = (lv[l].nsys * nc[l] + threads - 1) / threads;
      long_reduce_kernel<double, kM><<<(unsigned)blocks, threads, 0, stream>>>(
          lv[l], nc[l], const_cast<double *>(q.a), const_cast<double *>(q.b),
          const_cast<double *>(q.c), q.d_out);
      g_launches.fetch_add(1, std::memory_order_relaxed);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
      const Plan last = choose_plan<double>(lv[levels], vec_aligned<double>(lv[levels]), false);
      e = last.family == TRID_FAMILY_LONG ? cudaErrorInvalidValue
                                          : launch_batch<double, false>(lv[levels], last, stream);
    }
    for (int l = levels - 1; l >= 0 && e == cudaSuccess; --l) {
      const long long blocks = (lv[l].nsys * nc[l] + threads - 1) / threads;
      long_substitute_kernel<double, kM, false>
          <<<(unsigned)blocks, threads, 0, stream>>>(lv[l], nc[l], lv[l + 1].d_out);
      g_launches.fetch_add(1, std::memory_order_relaxed);
      e = cudaGetLastError();
    }
  }
  if (e != cudaSuccess) return to_status(e);
  if (cfg.blocking) {
    e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return to_status(e);
    unsigned h = 0;
    e = cudaMemcpy(&h, flag, sizeof(unsigned), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return to_status(e);
    if (h) return TRID_STATUS_ZERO_PIVOT;
  }
  return TRID_STATUS_SUCCESS;
}
