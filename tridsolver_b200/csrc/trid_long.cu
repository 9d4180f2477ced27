// Long contiguous systems (more rows than one warp holds): two passes over
// warp tiles of tile_rows rows (512 FP64, 1024 FP32; trid_tile.cuh).
//
//   1. long_tile_kernel<R, false>: each warp stages one tile of one system
//      with coalesced 16-byte copies, eliminates its chunks, runs the warp's
//      reduced solve for the three right-hand sides and writes the tile's
//      two rows of the second-level system (unit diagonal) to scratch;
//   2. the second-level batch (2 rows per tile, K tiles: 2K rows per system)
//      is solved by the library's own batched solve, recursively;
//   3. long_tile_kernel<R, true>: each warp stages its tile again, repeats
//      the elimination, takes x_prev and x_next (the neighbouring tiles'
//      last and first unknowns) from the second-level solution, substitutes
//      and stores, coalesced through the same buffer.
// a, b, c, d are read twice and x written once: 9 words per element, the
// floor of any method that does not keep a whole system on chip. Against the
// register-chunk long path (long_reduce/long_substitute_kernel, still used
// for strided long systems) every access is coalesced and the second-level
// system is 32 times smaller (2 rows per 512 instead of per 16).
#include <cuda_runtime.h>

#include "trid_internal.h"
#include "trid_tile.cuh"

namespace trid {

namespace {

constexpr int kLongThreads = 128;  // 4 warps, one tile each

}  // namespace

// SUBST false: pass 1 (second-level rows to r*); true: pass 3 (x from the
// second-level solution xr). INC: u += x instead of d = x.
template <typename R, bool SUBST, bool INC>
__global__ void __launch_bounds__(kLongThreads)
    long_tile_kernel(const BatchArgs<R> p, long long K, bool vec16, R *__restrict__ ra,
                     R *__restrict__ rb, R *__restrict__ rc, R *__restrict__ rd,
                     const R *__restrict__ xr) {
  using L = SmemLayout<R, tile_m<R>()>;
  constexpr int kTM = tile_m<R>();
  extern __shared__ __align__(16) unsigned char long_smem[];
  R *buf = reinterpret_cast<R *>(long_smem) + (threadIdx.x >> 5) * TileBuf<R>::ELEMS;
  const int lane = threadIdx.x & 31;
  const long long item = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (item >= p.nsys * K) return;  // uniform per warp
  const long long s = item / K;
  const long long j = item - s * K;
  const long long base0 = sys_base(p, s);
  const long long r0 = j * tile_rows<R>();
  const int n = p.N;
  const int nt = (int)(n - r0 < tile_rows<R>() ? n - r0 : tile_rows<R>());
  stage_tile_rows<R>(p.a, p.b, p.c, p.d_in, vec16, base0 + r0, nt, buf, lane);

  R a[kTM], b[kTM], c[kTM], d[kTM];
  lds_row<R, kTM>(buf + 0 * L::BUF + lane * L::ROW, a);
  lds_row<R, kTM>(buf + 1 * L::BUF + lane * L::ROW, b);
  lds_row<R, kTM>(buf + 2 * L::BUF + lane * L::ROW, c);
  lds_row<R, kTM>(buf + 3 * L::BUF + lane * L::ROW, d);
  const long long row0 = r0 + (long long)lane * kTM;
  if (row0 == 0) a[0] = R(0);
#pragma unroll
  for (int i = 0; i < kTM; ++i)
    if (row0 + i == n - 1) c[i] = R(0);
  bool bad = false;
  chunk_forward<R, kTM, true>(a, b, c, d, bad);
  chunk_backward<R, kTM, true>(a, c, d, bad);
  const Row<R> top{a[0], c[0], d[0]}, bot{a[kTM - 1], c[kTM - 1], d[kTM - 1]};
  R y[3], z[3];
  reduced_solve3<R>(top, bot, lane == 0 ? -top.A : R(0), lane == 31 ? -bot.C : R(0), lane, y, z,
                    bad);
  const long long o = s * 2 * K + 2 * j;  // the tile's rows in the second-level batch
  if constexpr (!SUBST) {
    const R pf = shfl_idx(y[0], 0, 32), af = shfl_idx(y[1], 0, 32), bf = shfl_idx(y[2], 0, 32);
    const R pl = shfl_idx(z[0], 31, 32), al = shfl_idx(z[1], 31, 32), bl = shfl_idx(z[2], 31, 32);
    if (lane == 0) {
      Row<R> t2, b2;
      second_level_rows<R>(pf, af, bf, pl, al, bl, j == 0, j == K - 1, t2, b2);
      ra[o] = t2.A;
      rb[o] = R(1);
      rc[o] = t2.C;
      rd[o] = t2.D;
      ra[o + 1] = b2.A;
      rb[o + 1] = R(1);
      rc[o + 1] = b2.C;
      rd[o + 1] = b2.D;
    }
  } else {
    const R xp = j > 0 ? xr[o - 1] : R(0);
    const R xn = j < K - 1 ? xr[o + 2] : R(0);
    const R yy = y[0] + y[1] * xp + y[2] * xn;
    const R zz = z[0] + z[1] * xp + z[2] * xn;
    chunk_substitute<R, kTM>(a, c, d, yy, zz);
    // x out through the warp's d rows, then coalesced element stores
    sts_row<R, kTM>(buf + 3 * L::BUF + lane * L::ROW, d);
    __syncwarp();
    const long long bo = base0 + r0;
#pragma unroll 4
    for (int e = lane; e < nt; e += 32) {
      const R x = buf[3 * L::BUF + TileBuf<R>::slot(e)];
      if constexpr (INC)
        p.u[bo + e] += x;
      else
        p.d_out[bo + e] = x;
    }
  }
  report_bad_pivot(bad, p.flag);
}

template <typename R, bool INC>
cudaError_t launch_long_tiles(const BatchArgs<R> &p, cudaStream_t st) {
  if (p.stride != 1) return cudaErrorInvalidValue;
  const long long K = ((long long)p.N + tile_rows<R>() - 1) / tile_rows<R>();
  if (2 * K >= p.N) return cudaErrorInvalidValue;  // would not shrink
  const long long nred = p.nsys * 2 * K;
  R *scratch = nullptr;
  cudaError_t e = scratch_alloc((void **)&scratch, (size_t)nred * 4 * sizeof(R), st);
  if (e != cudaSuccess) return e;
  R *ra = scratch, *rb = ra + nred, *rc = rb + nred, *rd = rc + nred;
  auto al = [](const void *q) { return (reinterpret_cast<uintptr_t>(q) & 15u) == 0; };
  const bool vec16 = al(p.a) && al(p.b) && al(p.c) && al(p.d_in) && al(p.d_out) &&
                     (!p.u || al(p.u)) &&
                     (p.st0 * (long long)sizeof(R)) % 16 == 0 && (p.st1 * (long long)sizeof(R)) % 16 == 0;
  const size_t smem = (size_t)(kLongThreads / 32) * TileBuf<R>::ELEMS * sizeof(R);
  const long long warps = p.nsys * K;
  const long long blocks = (warps * 32 + kLongThreads - 1) / kLongThreads;
  auto k1 = long_tile_kernel<R, false, false>;
  auto k3 = long_tile_kernel<R, true, INC>;
  e = cudaFuncSetAttribute(k1, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k3, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess) {
    k1<<<(unsigned)blocks, kLongThreads, smem, st>>>(p, K, vec16, ra, rb, rc, rd, nullptr);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) {
    BatchArgs<R> q{};
    q.a = ra;
    q.b = rb;
    q.c = rc;
    q.d_in = rd;
    q.d_out = rd;
    q.u = nullptr;
    q.N = (int)(2 * K);
    q.nsys = p.nsys;
    q.n0 = p.nsys;
    q.st0 = 2 * K;
    q.st1 = 0;
    q.stride = 1;
    q.flag = p.flag;
    // the second-level batch always takes the automatic plan
    const Plan qp = choose_plan<R>(q, vec_aligned<R>(q), false);
    e = launch_batch<R, false>(q, qp, st);
  }
  if (e == cudaSuccess) {
    k3<<<(unsigned)blocks, kLongThreads, smem, st>>>(p, K, vec16, nullptr, nullptr, nullptr, nullptr,
                                                     rd);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    e = cudaGetLastError();
  }
  cudaError_t ef = scratch_free(scratch, st);
  return e != cudaSuccess ? e : ef;
}

template cudaError_t launch_long_tiles<double, false>(const BatchArgs<double> &, cudaStream_t);
template cudaError_t launch_long_tiles<double, true>(const BatchArgs<double> &, cudaStream_t);
template cudaError_t launch_long_tiles<float, false>(const BatchArgs<float> &, cudaStream_t);
template cudaError_t launch_long_tiles<float, true>(const BatchArgs<float> &, cudaStream_t);

}  // namespace trid
