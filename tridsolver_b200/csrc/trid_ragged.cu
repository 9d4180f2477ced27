// Ragged batches: independent contiguous systems of uneven lengths, system k
// occupying rows [offsets[k], offsets[k+1]) of a, b, c, d, solved in one
// persistent launch.
//
//   1. ragged_hist_kernel / ragged_order_kernel bucket the systems by length
//      class (ceil(log2 N)) into `order`, longest class first, so the
//      persistent kernel hands out the longest work first (longest-processing
//      -time scheduling keeps the SMs evenly loaded at the end);
//   2. ragged_kernel: persistent CTAs of 256 threads. Phase 1 takes "block
//      items" (systems longer than one warp holds) one per CTA, from a
//      global atomic counter; phase 2 takes "warp items", one system per warp,
//      each warp on its own.
//
// Warp items run the partition hybrid over 32 lanes with M rows per lane
// chosen per length class from a table (M = 1 is pure PCR, one row per
// lane); the table is built in, or measured by tridRaggedAutotune.
// Block items (N up to 16384): 256 threads x 16 rows = one 4096-row segment
// per pass. Pass A eliminates every segment's chunks and keeps only their
// reduced rows in shared memory; the CTA solves that reduced system (each
// thread eliminates its 2*nseg consecutive reduced rows, then the block
// reduced solve); pass B reads each segment again (mostly from L2, the CTA
// read it moments before), eliminates it again and substitutes.
// The reference has no ragged entry point; its per-system solve trid_scalar
// (scalar/src/cpu/trid_cpu.cpp:312-353) is the oracle for each system.
#include <cuda_runtime.h>

#include <cstring>

#include "trid_internal.h"
#include "tridsolver_b200.h"

namespace trid {

constexpr int kClasses = 24;          // length classes 0..23: N <= 2^class
constexpr int kBlockThreads = 256;
constexpr int kBlockM = 16;           // rows per thread in block items
constexpr int kSegRows = kBlockThreads * kBlockM;  // 4096
constexpr int kMaxSeg = 4;            // block items up to 16384 rows

template <typename R> struct RaggedArgs {
  const R *a, *b, *c;
  R *d;
  const int64_t *off;
  const int *order;                 // systems, longest class first
  const unsigned *hist;             // systems per class
  unsigned long long *counters;     // [0] block items taken, [1] warp items taken
  long long nsys;
  int warp_max;                     // longest system a warp item takes
  int mtab[kClasses];               // rows per lane by class (warp items)
  unsigned *flag;
  unsigned *error;                  // set when a system exceeds the block-item limit
};

__device__ __forceinline__ int length_class(long long n) {
  int c = 0;
  while (c < kClasses - 1 && (1LL << c) < n) ++c;
  return c;
}

template <typename R>
__global__ void ragged_hist_kernel(RaggedArgs<R> p, unsigned *hist) {
  for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < p.nsys;
       s += (long long)gridDim.x * blockDim.x) {
    const long long n = p.off[s + 1] - p.off[s];
    atomicAdd(&hist[length_class(n > 0 ? n : 1)], 1u);
  }
}

template <typename R>
__global__ void ragged_order_kernel(RaggedArgs<R> p, const unsigned *hist, unsigned *fill,
                                    int *order) {
  for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < p.nsys;
       s += (long long)gridDim.x * blockDim.x) {
    const long long n = p.off[s + 1] - p.off[s];
    const int c = length_class(n > 0 ? n : 1);
    unsigned start = 0;
    for (int q = kClasses - 1; q > c; --q) start += hist[q];
    order[start + atomicAdd(&fill[c], 1u)] = (int)s;
  }
}

// Loads rows [row0, row0+M) of a contiguous system of n rows at `base`,
// identity rows past the end, a[0] and c[n-1] zero.
template <typename R, int M>
__device__ __forceinline__ void ragged_load(const RaggedArgs<R> &p, long long base, long long n,
                                            long long row0, R (&a)[M], R (&b)[M], R (&c)[M],
                                            R (&d)[M]) {
#pragma unroll
  for (int i = 0; i < M; ++i) {
    const long long row = row0 + i;
    if (row < n) {
      a[i] = row == 0 ? R(0) : __ldg(p.a + base + row);
      b[i] = __ldg(p.b + base + row);
      c[i] = row == n - 1 ? R(0) : __ldg(p.c + base + row);
      d[i] = p.d[base + row];
    } else {
      a[i] = R(0);
      b[i] = R(1);
      c[i] = R(0);
      d[i] = R(0);
    }
  }
}

template <typename R, int M>
__device__ __forceinline__ void ragged_store(const RaggedArgs<R> &p, long long base, long long n,
                                             long long row0, const R (&x)[M]) {
#pragma unroll
  for (int i = 0; i < M; ++i)
    if (row0 + i < n) p.d[base + row0 + i] = x[i];
}

// Segment staging for block items: the CTA copies rows [row0, row0+kSegRows)
// of a, b, c, d into shared memory with element-sized cp.async copies, so
// every warp instruction copies 32 consecutive elements (offsets need not be
// aligned). Thread t's chunk (rows t*kBlockM ...) sits in a row padded by one
// element, so its reads of neighbouring threads fall in different banks.
constexpr int kStageRow = kBlockM + 1;
constexpr int kStageArr = kBlockThreads * kStageRow;

__device__ __forceinline__ void cp_async_elem(void *smem_dst, const void *gmem_src, int bytes) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
  if (bytes == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem_src) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem_src) : "memory");
}

template <typename R>
__device__ __forceinline__ void stage_segment(const RaggedArgs<R> &p, long long base, long long n,
                                              long long row0, R *stg) {
  for (int e = threadIdx.x; e < kSegRows; e += kBlockThreads) {
    const long long row = row0 + e;
    const int o = e + e / kBlockM;
    if (row < n) {
      cp_async_elem(stg + 0 * kStageArr + o, p.a + base + row, (int)sizeof(R));
      cp_async_elem(stg + 1 * kStageArr + o, p.b + base + row, (int)sizeof(R));
      cp_async_elem(stg + 2 * kStageArr + o, p.c + base + row, (int)sizeof(R));
      cp_async_elem(stg + 3 * kStageArr + o, p.d + base + row, (int)sizeof(R));
    } else {
      stg[0 * kStageArr + o] = R(0);
      stg[1 * kStageArr + o] = R(1);
      stg[2 * kStageArr + o] = R(0);
      stg[3 * kStageArr + o] = R(0);
    }
  }
  cp_async_wait_all();
  __syncthreads();
}

// Thread t's kBlockM rows of a staged segment, a[0] and c[n-1] zero.
template <typename R>
__device__ __forceinline__ void staged_rows(const R *stg, long long n, long long row0, R (&a)[kBlockM],
                                            R (&b)[kBlockM], R (&c)[kBlockM], R (&d)[kBlockM]) {
  const int t = threadIdx.x;
#pragma unroll
  for (int i = 0; i < kBlockM; ++i) {
    const int o = t * kStageRow + i;
    a[i] = stg[0 * kStageArr + o];
    b[i] = stg[1 * kStageArr + o];
    c[i] = stg[2 * kStageArr + o];
    d[i] = stg[3 * kStageArr + o];
    const long long row = row0 + t * kBlockM + i;
    if (row == 0) a[i] = R(0);
    if (row == n - 1) c[i] = R(0);
  }
}

// One system per warp, M rows per lane (M = 1: pure PCR).
template <typename R, int M>
__device__ __forceinline__ void warp_item(const RaggedArgs<R> &p, long long base, long long n,
                                          int lane, bool &bad) {
  if constexpr (M == 1) {
    R a = R(0), b = R(1), c = R(0), d = R(0);
    if (lane < n) {
      a = lane == 0 ? R(0) : __ldg(p.a + base + lane);
      b = __ldg(p.b + base + lane);
      c = lane == n - 1 ? R(0) : __ldg(p.c + base + lane);
      d = p.d[base + lane];
    }
    const R x = pcr_solve<R>(a, b, c, d, lane, 32, bad);
    if (lane < n) p.d[base + lane] = x;
  } else {
    R a[M], b[M], c[M], d[M];
    ragged_load<R, M>(p, base, n, (long long)lane * M, a, b, c, d);
    chunk_forward<R, M>(a, b, c, d, bad);
    chunk_backward<R, M>(a, c, d, bad);
    R y, z;
    reduced_solve<R>(Row<R>{a[0], c[0], d[0]}, Row<R>{a[M - 1], c[M - 1], d[M - 1]}, lane, 32, y, z,
                     bad);
    chunk_substitute<R, M>(a, c, d, y, z);
    ragged_store<R, M>(p, base, n, (long long)lane * M, d);
  }
}

// One long system per CTA (kBlockThreads threads, NS padded segments).
template <typename R, int NS>
__device__ __forceinline__ void block_item_ns(const RaggedArgs<R> &p, long long base, long long n,
                                              R *sm_red, R *sm_bs, R *stg, bool &bad) {
  const int t = threadIdx.x;
  const int Q = kBlockThreads * NS;  // chunks of the system (padded)
  // pass A: per segment, chunk elimination; keep the two reduced rows
  for (int g = 0; g < NS; ++g) {
    R a[kBlockM], b[kBlockM], c[kBlockM], d[kBlockM];
    if ((long long)g * kSegRows < n) {
      stage_segment<R>(p, base, n, (long long)g * kSegRows, stg);
      staged_rows<R>(stg, n, (long long)g * kSegRows, a, b, c, d);
      __syncthreads();  // the staging buffer is free again
    } else {
#pragma unroll
      for (int i = 0; i < kBlockM; ++i) {
        a[i] = R(0);
        b[i] = R(1);
        c[i] = R(0);
        d[i] = R(0);
      }
    }
    chunk_forward<R, kBlockM>(a, b, c, d, bad);
    chunk_backward<R, kBlockM>(a, c, d, bad);
    const int q = g * kBlockThreads + t;
    sm_red[0 * Q + q] = a[0];
    sm_red[1 * Q + q] = c[0];
    sm_red[2 * Q + q] = d[0];
    sm_red[3 * Q + q] = a[kBlockM - 1];
    sm_red[4 * Q + q] = c[kBlockM - 1];
    sm_red[5 * Q + q] = d[kBlockM - 1];
  }
  __syncthreads();
  // the reduced system (2Q rows): thread t owns chunks [t*NS, (t+1)*NS)
  {
    constexpr int K = 2 * NS;
    R ra[K], rb[K], rc[K], rd[K];
#pragma unroll
    for (int j = 0; j < NS; ++j) {
      const int q = t * NS + j;
      ra[2 * j] = sm_red[0 * Q + q];
      rc[2 * j] = sm_red[1 * Q + q];
      rd[2 * j] = sm_red[2 * Q + q];
      ra[2 * j + 1] = sm_red[3 * Q + q];
      rc[2 * j + 1] = sm_red[4 * Q + q];
      rd[2 * j + 1] = sm_red[5 * Q + q];
      rb[2 * j] = R(1);
      rb[2 * j + 1] = R(1);
    }
    chunk_forward<R, K>(ra, rb, rc, rd, bad);
    chunk_backward<R, K>(ra, rc, rd, bad);
    R y, z;
    block_reduced_solve<R, 16>(sm_bs, Row<R>{ra[0], rc[0], rd[0]},
                               Row<R>{ra[K - 1], rc[K - 1], rd[K - 1]}, 0, t, kBlockThreads, 1, y,
                               z, bad);
    chunk_substitute<R, K>(ra, rc, rd, y, z);
    // the chunks' first and last unknowns; each q is this thread's alone
#pragma unroll
    for (int j = 0; j < NS; ++j) {
      const int q = t * NS + j;
      sm_red[0 * Q + q] = rd[2 * j];
      sm_red[1 * Q + q] = rd[2 * j + 1];
    }
  }
  __syncthreads();
  // pass B: eliminate every segment again and substitute
  for (int g = 0; g < NS; ++g) {
    if ((long long)g * kSegRows >= n) break;  // uniform across the CTA
    const long long row0 = (long long)g * kSegRows + t * kBlockM;
    R a[kBlockM], b[kBlockM], c[kBlockM], d[kBlockM];
    stage_segment<R>(p, base, n, (long long)g * kSegRows, stg);
    staged_rows<R>(stg, n, (long long)g * kSegRows, a, b, c, d);
    __syncthreads();
    chunk_forward<R, kBlockM>(a, b, c, d, bad);
    chunk_backward<R, kBlockM>(a, c, d, bad);
    const int q = g * kBlockThreads + t;
    chunk_substitute<R, kBlockM>(a, c, d, sm_red[0 * Q + q], sm_red[1 * Q + q]);
    ragged_store<R, kBlockM>(p, base, n, row0, d);
  }
  __syncthreads();
}

template <typename R>
__device__ __forceinline__ void block_item_one(const RaggedArgs<R> &p, long long base, long long n,
                                               R *sm_bs, R *stg, bool &bad) {
  const int t = threadIdx.x;
  R a[kBlockM], b[kBlockM], c[kBlockM], d[kBlockM];
  stage_segment<R>(p, base, n, 0, stg);
  staged_rows<R>(stg, n, 0, a, b, c, d);
  chunk_forward<R, kBlockM>(a, b, c, d, bad);
  chunk_backward<R, kBlockM>(a, c, d, bad);
  R y, z;
  block_reduced_solve<R, 16>(sm_bs, Row<R>{a[0], c[0], d[0]},
                             Row<R>{a[kBlockM - 1], c[kBlockM - 1], d[kBlockM - 1]}, 0, t,
                             kBlockThreads, 1, y, z, bad);
  chunk_substitute<R, kBlockM>(a, c, d, y, z);
  ragged_store<R, kBlockM>(p, base, n, (long long)t * kBlockM, d);
  __syncthreads();
}

template <typename R>
__global__ void __launch_bounds__(kBlockThreads, 1) ragged_kernel(const RaggedArgs<R> p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R *sm_red = reinterpret_cast<R *>(smem_raw);
  R *sm_bs = sm_red + 6 * kBlockThreads * kMaxSeg;
  R *stg = sm_bs + 6 * kBlockThreads * 2;
  __shared__ long long item;
  bool bad = false;
  long long nblock = 0;
  for (int c = 0; c < kClasses; ++c)
    if ((1LL << c) > p.warp_max) nblock += p.hist[c];
  // phase 1: long systems, one per CTA, longest first
  for (;;) {
    if (threadIdx.x == 0) item = (long long)atomicAdd(&p.counters[0], 1ULL);
    __syncthreads();
    const long long it = item;
    __syncthreads();
    if (it >= nblock) break;
    const int s = p.order[it];
    const long long base = p.off[s];
    const long long n = p.off[s + 1] - base;
    if (n > (long long)kSegRows * kMaxSeg) {
      if (threadIdx.x == 0) *p.error = 1u;
      continue;
    }
    if (n <= kSegRows)
      block_item_one<R>(p, base, n, sm_bs, stg, bad);
    else if (n <= 2LL * kSegRows)
      block_item_ns<R, 2>(p, base, n, sm_red, sm_bs, stg, bad);
    else
      block_item_ns<R, 4>(p, base, n, sm_red, sm_bs, stg, bad);
  }
  // phase 2: one system per warp, each warp on its own
  const int lane = threadIdx.x & 31;
  for (;;) {
    long long w = 0;
    if (lane == 0) w = (long long)atomicAdd(&p.counters[1], 1ULL);
    w = __shfl_sync(FULL_MASK, w, 0);
    const long long it = nblock + w;
    if (it >= p.nsys) break;
    const int s = p.order[it];
    const long long base = p.off[s];
    const long long n = p.off[s + 1] - base;
    const int m = p.mtab[length_class(n > 0 ? n : 1)];
    switch (m) {
      case 1: warp_item<R, 1>(p, base, n, lane, bad); break;
      case 2: warp_item<R, 2>(p, base, n, lane, bad); break;
      case 4: warp_item<R, 4>(p, base, n, lane, bad); break;
      case 8: warp_item<R, 8>(p, base, n, lane, bad); break;
      case 16: warp_item<R, 16>(p, base, n, lane, bad); break;
      default:
        if constexpr (sizeof(R) == 4) warp_item<R, 32>(p, base, n, lane, bad);
        break;
    }
  }
  report_bad_pivot(bad, p.flag);
}

// ---- host side ---------------------------------------------------------------

// Rows per lane by length class for warp items: built-in table, replaced per
// device and precision by tridRaggedAutotune.
static int g_mtab[2][64][kClasses];
static bool g_tuned[2][64];

template <typename R>
static void default_mtab(int *m) {
  for (int c = 0; c < kClasses; ++c) {
    const long long n = 1LL << c;
    m[c] = n <= 32 ? 1 : n <= 64 ? 2 : n <= 128 ? 4 : n <= 256 ? 8 : n <= 512 ? 16 : 32;
  }
}

template <typename R> static constexpr int ragged_warp_max() { return sizeof(R) == 8 ? 512 : 1024; }

template <typename R>
static size_t ragged_smem() {
  return (size_t)6 * kBlockThreads * kMaxSeg * sizeof(R) +
         (size_t)6 * kBlockThreads * 2 * sizeof(R) + (size_t)4 * kStageArr * sizeof(R);
}

template <typename R>
static cudaError_t launch_ragged(RaggedArgs<R> p, const int *mtab, cudaStream_t st) {
  for (int c = 0; c < kClasses; ++c) p.mtab[c] = mtab[c];
  p.warp_max = ragged_warp_max<R>();
  // scratch: hist, fill, counters, error, order
  const size_t head = 256;
  char *scratch = nullptr;
  cudaError_t e = cudaMallocAsync((void **)&scratch, head + (size_t)p.nsys * sizeof(int), st);
  if (e != cudaSuccess) return e;
  unsigned *hist = reinterpret_cast<unsigned *>(scratch);
  unsigned *fill = hist + kClasses;
  // hist [0, 96), fill [96, 192), counters [192, 208), error [208, 212)
  unsigned long long *counters = reinterpret_cast<unsigned long long *>(scratch + 192);
  unsigned *error = reinterpret_cast<unsigned *>(scratch + 208);
  int *order = reinterpret_cast<int *>(scratch + head);
  e = cudaMemsetAsync(scratch, 0, head, st);
  p.hist = hist;
  p.counters = counters;
  p.order = order;
  p.error = error;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess) {
    const long long g = (p.nsys + 255) / 256;
    const unsigned grid = (unsigned)(g < 4LL * sms ? (g > 0 ? g : 1) : 4LL * sms);
    ragged_hist_kernel<R><<<grid, 256, 0, st>>>(p, hist);
    ragged_order_kernel<R><<<grid, 256, 0, st>>>(p, hist, fill, order);
    g_launches.fetch_add(2, std::memory_order_relaxed);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) {
    const size_t smem = ragged_smem<R>();
    cudaFuncSetAttribute(ragged_kernel<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int per_sm = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ragged_kernel<R>, kBlockThreads, smem);
    if (per_sm < 1) per_sm = 1;
    ragged_kernel<R><<<(unsigned)(sms * per_sm), kBlockThreads, smem, st>>>(p);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    e = cudaGetLastError();
  }
  // a system longer than the block-item limit sets `error`; it can only be
  // read back when the call blocks
  if (e == cudaSuccess && settings().blocking) {
    unsigned h = 0;
    e = cudaMemcpyAsync(&h, error, sizeof(h), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e == cudaSuccess && h) e = cudaErrorNotSupported;
  }
  cudaError_t ef = cudaFreeAsync(scratch, st);
  return e != cudaSuccess ? e : ef;
}

template <typename R>
static tridStatus_t ragged(const R *a, const R *b, const R *c, R *d, const int64_t *offsets,
                           long long nsys) {
  if (nsys < 0) return TRID_STATUS_INVALID_VALUE;
  if (nsys == 0) return TRID_STATUS_SUCCESS;
  if (!a || !b || !c || !d || !offsets || nsys > 0x7fffffffLL) return TRID_STATUS_INVALID_VALUE;
  int dev = 0, major = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev) != cudaSuccess) {
    cudaGetLastError();
    return TRID_STATUS_NOT_INITIALIZED;
  }
  if (major != 10) return TRID_STATUS_ARCH_MISMATCH;
  if (dev < 0 || dev >= 64) return TRID_STATUS_INTERNAL_ERROR;
  const int pi = sizeof(R) == 8 ? 0 : 1;
  int mt[kClasses];
  if (g_tuned[pi][dev])
    memcpy(mt, g_mtab[pi][dev], sizeof(mt));
  else
    default_mtab<R>(mt);
  const Settings &cfg = settings();
  RaggedArgs<R> p{};
  p.a = a;
  p.b = b;
  p.c = c;
  p.d = d;
  p.off = offsets;
  p.nsys = nsys;
  p.flag = pivot_flag_device();
  if (cfg.blocking) pivot_flag_take();
  cudaError_t e = launch_ragged<R>(p, mt, cfg.stream);
  if (e == cudaErrorNotSupported) return TRID_STATUS_MATRIX_TYPE_NOT_SUPPORTED;
  if (e != cudaSuccess) return status_of(e);
  if (cfg.blocking) {
    e = cudaStreamSynchronize(cfg.stream);
    if (e != cudaSuccess) return status_of(e);
    if (pivot_flag_take()) return TRID_STATUS_ZERO_PIVOT;
  }
  return TRID_STATUS_SUCCESS;
}

// ---- autotuner ----------------------------------------------------------------

template <typename R>
__global__ void ragged_fill_kernel(R *a, R *b, R *c, R *d, int64_t *off, long long n, int len,
                                   long long nsys) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const unsigned h = (unsigned)(i * 2654435761u);
    const R r = R((h >> 8) & 0xffff) / R(65536);
    a[i] = R(0.25) * r;
    c[i] = R(0.25) * (R(1) - r);
    b[i] = R(1) + r;
    d[i] = r - R(0.5);
    if (i <= nsys) off[i] = i * (long long)len;
  }
}

// For every length class a warp item can take, times each rows-per-lane
// choice that holds the class (32*M >= 2^class) on a uniform batch of that
// class and keeps the fastest. Block items are not tuned (one shape).
template <typename R>
static tridStatus_t autotune(int dev) {
  int mt[kClasses];
  default_mtab<R>(mt);
  const long long cap = 1LL << 24;  // elements per timing batch
  R *buf = nullptr;
  int64_t *off = nullptr;
  if (cudaMalloc((void **)&buf, (size_t)cap * 4 * sizeof(R)) != cudaSuccess) {
    cudaGetLastError();
    return TRID_STATUS_ALLOC_FAILED;
  }
  if (cudaMalloc((void **)&off, (size_t)(cap / 8 + 2) * sizeof(int64_t)) != cudaSuccess) {
    cudaFree(buf);
    cudaGetLastError();
    return TRID_STATUS_ALLOC_FAILED;
  }
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaStream_t st = nullptr;
  tridStatus_t status = TRID_STATUS_SUCCESS;
  for (int cls = 3; (1 << cls) <= ragged_warp_max<R>() && status == TRID_STATUS_SUCCESS; ++cls) {
    const int len = 1 << cls;
    const long long nsys = cap / len;
    ragged_fill_kernel<R><<<1024, 256, 0, st>>>(buf, buf + cap, buf + 2 * cap, buf + 3 * cap, off,
                                                nsys * len, len, nsys);
    float best = 1e30f;
    int best_m = mt[cls];
    for (int m = 1; m <= (sizeof(R) == 4 ? 32 : 16); m *= 2) {
      if (32LL * m < len) continue;
      int trial[kClasses];
      memcpy(trial, mt, sizeof(trial));
      trial[cls] = m;
      RaggedArgs<R> p{};
      p.a = buf;
      p.b = buf + cap;
      p.c = buf + 2 * cap;
      p.d = buf + 3 * cap;
      p.off = off;
      p.nsys = nsys;
      float ms = 1e30f;
      for (int rep = 0; rep < 3; ++rep) {
        cudaEventRecord(e0, st);
        cudaError_t e = launch_ragged<R>(p, trial, st);
        cudaEventRecord(e1, st);
        if (e != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess) {
          status = TRID_STATUS_EXECUTION_FAILED;
          break;
        }
        float t = 0;
        cudaEventElapsedTime(&t, e0, e1);
        if (rep > 0 && t < ms) ms = t;
      }
      if (status != TRID_STATUS_SUCCESS) break;
      if (ms < best) {
        best = ms;
        best_m = m;
      }
    }
    mt[cls] = best_m;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(buf);
  cudaFree(off);
  if (status == TRID_STATUS_SUCCESS) {
    const int pi = sizeof(R) == 8 ? 0 : 1;
    memcpy(g_mtab[pi][dev], mt, sizeof(mt));
    g_tuned[pi][dev] = true;
  }
  return status;
}

}  // namespace trid

using namespace trid;

EXTERN_C tridStatus_t tridDmtsvRaggedBatch(const TridParams *ctx, const double *a, const double *b,
                                           const double *c, double *d, const int64_t *offsets,
                                           long long nsys) {
  (void)ctx;
  return ragged<double>(a, b, c, d, offsets, nsys);
}

EXTERN_C tridStatus_t tridSmtsvRaggedBatch(const TridParams *ctx, const float *a, const float *b,
                                           const float *c, float *d, const int64_t *offsets,
                                           long long nsys) {
  (void)ctx;
  return ragged<float>(a, b, c, d, offsets, nsys);
}

EXTERN_C tridStatus_t tridRaggedAutotune(int dtype_bytes) {
  int dev = 0, major = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev) != cudaSuccess) {
    cudaGetLastError();
    return TRID_STATUS_NOT_INITIALIZED;
  }
  if (major != 10) return TRID_STATUS_ARCH_MISMATCH;
  if (dev < 0 || dev >= 64) return TRID_STATUS_INTERNAL_ERROR;
  if (dtype_bytes == 8) return autotune<double>(dev);
  if (dtype_bytes == 4) return autotune<float>(dev);
  return TRID_STATUS_INVALID_VALUE;
}

EXTERN_C int tridRaggedTable(int dtype_bytes, int *rows_per_lane, int nclasses) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    dev = 0;
  }
  if (dev < 0 || dev >= 64 || (dtype_bytes != 8 && dtype_bytes != 4)) return -1;
  const int pi = dtype_bytes == 8 ? 0 : 1;
  int mt[kClasses];
  if (g_tuned[pi][dev])
    memcpy(mt, g_mtab[pi][dev], sizeof(mt));
  else if (pi == 0)
    default_mtab<double>(mt);
  else
    default_mtab<float>(mt);
  const int warp_max = pi == 0 ? ragged_warp_max<double>() : ragged_warp_max<float>();
  int n = 0;
  for (int cls = 0; cls < kClasses && (1 << cls) <= warp_max; ++cls) {
    if (rows_per_lane && cls < nclasses) rows_per_lane[cls] = mt[cls];
    n = cls + 1;
  }
  return n;
}
