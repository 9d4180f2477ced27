// Strided batches (solvedim >= 1) with TMA tiles.
//
// The LDG-based strided_kernel is bound by the number of global-memory
// instructions: every warp load moves 256 bytes spread over four rows, and
// for a z solve each row segment lies on a different large page. Here a
// persistent CTA loads the whole tile of a group of W neighbouring systems
// (W x N elements of each of a, b, c, d, and u for Inc) with a handful of
// cp.async.bulk.tensor instructions that complete on an mbarrier, while the
// previous group is solved out of shared memory (two stages when they fit).
// Results go back with TMA stores. Each element is still read once and
// written once.
//
// Tensor maps are 3-D with increasing strides: (x, rows, outer) for a y
// solve, (x, outer, rows) for a z solve; boxes of W x R rows (R <= 256), so
// rows past N and systems past n0 are zero-filled on load and clipped on
// store. Requires 16-byte aligned bases and 16-byte multiple strides (the
// plan checks; other batches use strided_kernel).
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <cstring>
#include <mutex>

#include "trid_internal.h"
#include "trid_tma.cuh"

namespace trid {

struct TmaMaps {
  CUtensorMap m[5];  // a, b, c, d (loads); [4]: the output, u for Inc, else d_out
};

constexpr unsigned kTmaWaitLimit = 1u << 22;

template <typename R, int M, int KR, bool INC>
__global__ void __launch_bounds__(256, 1)
    strided_tma_kernel(const __grid_constant__ TmaMaps maps, const BatchArgs<R> p, int T, int W,
                       long long ngx, long long ngroups, int rows_box, int nbox, int zorder,
                       int stages) {
  constexpr int NA = INC ? 5 : 4;
  constexpr int OUT = INC ? 4 : 3;
  extern __shared__ __align__(128) unsigned char tma_smem[];
  uint64_t *bar = reinterpret_cast<uint64_t *>(tma_smem);
  R *red = reinterpret_cast<R *>(tma_smem + 128);
  const size_t red_bytes = ((size_t)6 * T * (W + 1) * sizeof(R) + 127) / 128 * 128;
  R *buf0 = reinterpret_cast<R *>(tma_smem + 128 + red_bytes);
  const int rows_pad = nbox * rows_box;
  const int tile = rows_pad * W;
  R *buf[2] = {buf0, buf0 + (stages > 1 ? NA * tile : 0)};
  const unsigned stage_bytes = (unsigned)(NA * tile * sizeof(R));
  const int tid = threadIdx.x;
  const int s = tid % W;
  const int t = tid / W;
  const int N = p.N;

  auto coords = [&](long long g, int box, int &c0, int &c1, int &c2) {
    const long long gx = g % ngx;
    const long long i1 = g / ngx;
    c0 = (int)(gx * W);
    if (zorder) {
      c1 = (int)i1;
      c2 = box * rows_box;
    } else {
      c1 = box * rows_box;
      c2 = (int)i1;
    }
  };
  auto issue = [&](long long g, int b) {  // thread 0 only
    mbar_expect_tx(&bar[b], stage_bytes);
    for (int arr = 0; arr < NA; ++arr)
      for (int box = 0; box < nbox; ++box) {
        int c0, c1, c2;
        coords(g, box, c0, c1, c2);
        tma_load_3d(buf[b] + arr * tile + box * rows_box * W, &maps.m[arr], c0, c1, c2, &bar[b]);
      }
  };

  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_fence_init();
  }
  __syncthreads();
  bool bad = false;
  long long g = blockIdx.x;
  if (tid == 0 && g < ngroups) issue(g, 0);
  int it = 0;
  unsigned phase[2] = {0u, 0u};
  for (; g < ngroups; ++it, g += gridDim.x) {
    const int b = stages > 1 ? (it & 1) : 0;
    const long long gn = g + gridDim.x;
    if (stages > 1 && tid == 0 && gn < ngroups) {
      tma_store_wait_read();  // the other buffer's last store has read it
      issue(gn, b ^ 1);
    }
    const bool ok = mbar_wait(&bar[b], phase[b], kTmaWaitLimit);
    if (__syncthreads_or(!ok)) {
      // give up on this launch: record it, then let the copies already issued
      // land (again with a cap) before the CTA's shared memory goes away
      if (p.flag && tid == 0) *reinterpret_cast<volatile unsigned *>(p.flag) = 2u;
      mbar_wait(&bar[b], phase[b], kTmaWaitLimit);
      if (stages > 1 && gn < ngroups) mbar_wait(&bar[b ^ 1], phase[b ^ 1], kTmaWaitLimit);
      break;
    }
    phase[b] ^= 1u;
    R *tl = buf[b];
    const long long gx = g % ngx;
    const long long i0 = gx * W + s;
    const bool active = i0 < p.n0;
    const int row0 = t * M;
    R ra[M], rb[M], rc[M], rd[M];
#pragma unroll
    for (int i = 0; i < M; ++i) {
      const int row = row0 + i;
      if (active && row < N) {
        const int o = row * W + s;
        ra[i] = row == 0 ? R(0) : tl[0 * tile + o];
        rb[i] = tl[1 * tile + o];
        rc[i] = row == N - 1 ? R(0) : tl[2 * tile + o];
        rd[i] = tl[3 * tile + o];
      } else {
        ra[i] = R(0);
        rb[i] = R(1);
        rc[i] = R(0);
        rd[i] = R(0);
      }
    }
    chunk_forward<R, M>(ra, rb, rc, rd, bad);
    chunk_backward<R, M>(ra, rc, rd, bad);
    R y, z;
    block_reduced_solve<R, KR>(red, Row<R>{ra[0], rc[0], rd[0]},
                               Row<R>{ra[M - 1], rc[M - 1], rd[M - 1]}, s, t, T, W, y, z, bad);
    chunk_substitute<R, M>(ra, rc, rd, y, z);
#pragma unroll
    for (int i = 0; i < M; ++i) {
      const int row = row0 + i;
      if (row < rows_pad) {
        const int o = OUT * tile + row * W + s;
        if (INC)
          tl[o] += rd[i];
        else
          tl[o] = rd[i];
      }
    }
    fence_async_shared();
    __syncthreads();
    if (tid == 0) {
      for (int box = 0; box < nbox; ++box) {
        int c0, c1, c2;
        coords(g, box, c0, c1, c2);
        tma_store_3d(&maps.m[4], c0, c1, c2, tl + OUT * tile + box * rows_box * W);
      }
      tma_store_commit();
      if (stages == 1) {
        tma_store_wait_read();
        if (gn < ngroups) issue(gn, 0);
      }
    }
  }
  if (tid == 0) tma_store_wait_all();
  report_bad_pivot(bad, p.flag);
}

// ---- host side -------------------------------------------------------------------

static PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static std::once_flag once;
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  std::call_once(once, [] {
    void *ptr = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(ptr);
    else
      cudaGetLastError();
  });
  return fn;
}

// Tile geometry of a strided batch for W systems per group: rows per box,
// boxes, stages and shared-memory size; false if TMA does not apply.
template <typename R>
bool tma_geometry(const BatchArgs<R> &p, bool inc, int W, int &rows_box, int &nbox, int &stages,
                  size_t &smem, int T) {
  if (p.stride == 1 || p.N > 1024 || p.N < 1 || W < 1) return false;
  auto al = [](const void *q) { return (reinterpret_cast<uintptr_t>(q) & 15u) == 0; };
  if (!al(p.a) || !al(p.b) || !al(p.c) || !al(p.d_in) || !al(inc ? p.u : p.d_out)) return false;
  const long long es = sizeof(R);
  if ((p.stride * es) % 16 || (p.st1 * es) % 16 || p.st0 != 1) return false;
  if ((W * es) % 16) return false;
  if (p.n0 > 0x7fffffffLL || p.nsys / p.n0 > 0x7fffffffLL) return false;
  // box heights keep every box's shared-memory destination 128-byte aligned
  const int unit = (int)(128 / (W * es)) > 0 ? (int)(128 / (W * es)) : 1;
  rows_box = p.N < 256 ? (p.N + unit - 1) / unit * unit : 256;
  if (rows_box > 256) rows_box = 256;
  nbox = (p.N + rows_box - 1) / rows_box;
  const int NA = inc ? 5 : 4;
  const size_t stage = (size_t)NA * nbox * rows_box * W * es;
  const size_t red = ((size_t)6 * T * (W + 1) * es + 127) / 128 * 128;
  const size_t limit = 220 * 1024;
  if (128 + red + 2 * stage <= limit) {
    stages = 2;
  } else if (128 + red + stage <= limit) {
    stages = 1;
  } else {
    return false;
  }
  smem = 128 + red + (size_t)stages * stage;
  return true;
}

template <typename R, int M, int KR, bool INC>
cudaError_t launch_strided_tma(const BatchArgs<R> &p, const Plan &plan, cudaStream_t st) {
  int rows_box = 0, nbox = 0, stages = 0;
  size_t smem = 0;
  if (!tma_geometry<R>(p, INC, plan.W, rows_box, nbox, stages, smem, plan.T))
    return cudaErrorInvalidValue;
  auto enc = encode_fn();
  if (!enc) return cudaErrorNotSupported;
  // dims (x, rows, outer) for y-like layouts; (x, outer, rows) when the rows
  // are the outermost stride (z solves), so strides always increase
  const long long n1 = p.nsys / p.n0;
  const int zorder = p.stride > p.st1 ? 1 : 0;
  const long long es = sizeof(R);
  cuuint64_t gdim[3];
  cuuint64_t gstr[2];
  cuuint32_t box[3];
  gdim[0] = (cuuint64_t)p.n0;
  box[0] = (cuuint32_t)plan.W;
  if (zorder) {
    gdim[1] = (cuuint64_t)n1;
    gdim[2] = (cuuint64_t)p.N;
    gstr[0] = (cuuint64_t)(p.st1 * es);
    gstr[1] = (cuuint64_t)(p.stride * es);
    box[1] = 1;
    box[2] = (cuuint32_t)rows_box;
  } else {
    gdim[1] = (cuuint64_t)p.N;
    gdim[2] = (cuuint64_t)n1;
    gstr[0] = (cuuint64_t)(p.stride * es);
    gstr[1] = (cuuint64_t)(p.st1 * es);
    box[1] = (cuuint32_t)rows_box;
    box[2] = 1;
  }
  const cuuint32_t estr[3] = {1, 1, 1};
  TmaMaps maps;
  memset(&maps, 0, sizeof(maps));
  const void *ptrs[5] = {p.a, p.b, p.c, p.d_in, INC ? p.u : p.d_out};
  const CUtensorMapDataType dt =
      sizeof(R) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  for (int k = 0; k < 5; ++k) {
    CUresult r = enc(&maps.m[k], dt, 3, const_cast<void *>(ptrs[k]), gdim, gstr, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return cudaErrorInvalidValue;
  }
  const long long ngx = (p.n0 + plan.W - 1) / plan.W;
  const long long ngroups = ngx * n1;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaFuncSetAttribute(strided_tma_kernel<R, M, KR, INC>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  const long long grid = ngroups < sms ? ngroups : sms;
  strided_tma_kernel<R, M, KR, INC><<<(unsigned)grid, plan.W * plan.T, smem, st>>>(
      maps, p, plan.T, plan.W, ngx, ngroups, rows_box, nbox, zorder, stages);
  return cudaGetLastError();
}

#define INST_TMA(R, M, KR)                                                                     \
  template cudaError_t launch_strided_tma<R, M, KR, false>(const BatchArgs<R> &, const Plan &,   \
                                                           cudaStream_t);                     \
  template cudaError_t launch_strided_tma<R, M, KR, true>(const BatchArgs<R> &, const Plan &,    \
                                                          cudaStream_t);
INST_TMA(double, 8, 2)
INST_TMA(double, 8, 4)
INST_TMA(double, 8, 8)
INST_TMA(float, 8, 2)
INST_TMA(float, 8, 4)
INST_TMA(float, 8, 8)
INST_TMA(float, 16, 2)
INST_TMA(float, 16, 4)
template bool tma_geometry<double>(const BatchArgs<double> &, bool, int, int &, int &, int &,
                                   size_t &, int);
template bool tma_geometry<float>(const BatchArgs<float> &, bool, int, int &, int &, int &,
                                  size_t &, int);

}  // namespace trid
