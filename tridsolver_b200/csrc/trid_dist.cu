// Distributed solve: every system is split along the solve dimension over P
// ranks (each rank holds rows [0, n) of its segment of every system), the
// partition method of the reference's MPI/NCCL build
// (scalar/src/cuda/trid_cuda_mpi.cu:609-755 with the ALLGATHER strategy,
// :218-330; forward pass scalar/src/cuda/trid_linear_mpi.hpp:49-100):
//
//  1. reduce: one thread per system sweeps its segment once (or, for
//     contiguous segments of 32 M rows, a warp reduces the segment as one
//     tile of the tiled long path) and leaves two rows with unit diagonals
//     that couple the segment's first and last unknowns to the neighbouring
//     ranks' boundary unknowns,
//         top:    A0 x_prev + x_0     + C0 x_{n-1} = D0
//         bottom: A1 x_0    + x_{n-1} + C1 x_next  = D1;
//     the bottom row is the last row of the forward (Thomas) elimination;
//     the top row needs the backward elimination of rows n-2 .. 1, a chain
//         (A, C, D) <- (a'_j - c'_j A, -c'_j C, d'_j - c'_j D)
//     whose result is accumulated here in forward order (as sums of the
//     rows' a', d' weighted by running products of -c'), so nothing but
//     these six values per system is written;
//  2. the six values of every system are gathered from all ranks (a
//     callback: NCCL all-gather from torch.distributed, or any host code);
//  3. finish: one thread per system solves the 2P-row reduced system of all
//     ranks' rows (unknowns x_0 and x_{n-1} of every rank, tridiagonal in
//     that order; the global first a and last c are ignored, as in the
//     reference), takes the neighbours' boundary values and moves the
//     couplings into the right-hand side,
//         d_0 -= a_0 x_prev,   d_{n-1} -= c_{n-1} x_next;
//  4. the local segments are then independent systems: the ordinary batched
//     solve (which treats a_0 and c_{n-1} as zero) finishes them, so the
//     bulk of the work runs in the library's fastest kernels.
// For Inc, d's two corrected rows are restored afterwards.
//
// HBM traffic: 4 words per element for the reduction and the local solve's
// 5, against the reference's 11 (forward writes aa, cc, dd; backward reads
// them again).
#include <cuda_runtime.h>

#include <stdint.h>

#include <mutex>
#include <set>

#include "trid_internal.h"
#include "trid_tile.cuh"

namespace trid {

namespace {

// Segment reduction of system s (thread per system).
template <typename R>
__global__ void __launch_bounds__(128) dist_reduce_kernel(const BatchArgs<R> p, R *__restrict__ out) {
  const long long nsys = p.nsys;
  bool bad = false;
  for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < nsys;
       s += (long long)gridDim.x * blockDim.x) {
    const long long base = sys_base(p, s);
    const long long st = p.stride;
    const int n = p.N;
    // rows 0 and 1: scaled to a unit diagonal
    R r = rcp(__ldg(p.b + base));
    bad |= !finite_rcp(r);
    const R a0 = __ldg(p.a + base) * r, c0 = __ldg(p.c + base) * r, d0 = __ldg(p.d_in + base) * r;
    R ap, cp, dp;  // the last forward row
    // The backward chain over rows n-2 .. 1,
    //   A_{n-2} = a'_{n-2}, A_j = a'_j - c'_j A_{j+1}  (D likewise, C_j = -c'_j C_{j+1}),
    // unrolled: with q_1 = 1 and q_{j+1} = -c'_j q_j,
    //   A_1 = sum_{j=1}^{n-2} q_j a'_j,  D_1 = sum_{j=1}^{n-2} q_j d'_j,
    //   C_1 = q_{n-2} c'_{n-2} = -q_{n-1},
    // so row j joins the sums when the sweep moves past it.
    R q = R(1), SA = R(0), SD = R(0);
    {
      const long long o = base + st;
      r = rcp(__ldg(p.b + o));
      bad |= !finite_rcp(r);
      ap = __ldg(p.a + o) * r;
      cp = __ldg(p.c + o) * r;
      dp = __ldg(p.d_in + o) * r;
    }
    // rows 2 .. n-1 in blocks of U, the next block's loads in flight while
    // the current one is eliminated (the sweep itself is a dependent chain)
    constexpr int U = 4;
    R ca[U], cb[U], cc[U], cd[U];
    auto load_block = [&](int j0) {
#pragma unroll
      for (int k = 0; k < U; ++k) {
        const bool v = j0 + k < n;
        const long long o = base + (long long)(j0 + k) * st;
        ca[k] = v ? __ldg(p.a + o) : R(0);
        cb[k] = v ? __ldg(p.b + o) : R(1);
        cc[k] = v ? __ldg(p.c + o) : R(0);
        cd[k] = v ? __ldg(p.d_in + o) : R(0);
      }
    };
    load_block(2);
    for (int j0 = 2; j0 < n; j0 += U) {
      R xa[U], xb[U], xc[U], xd[U];
#pragma unroll
      for (int k = 0; k < U; ++k) {
        xa[k] = ca[k];
        xb[k] = cb[k];
        xc[k] = cc[k];
        xd[k] = cd[k];
      }
      if (j0 + U < n) load_block(j0 + U);
#pragma unroll
      for (int k = 0; k < U; ++k) {
        if (j0 + k < n) {
          SA += q * ap;  // row j - 1 (its forward values) joins the chain
          SD += q * dp;
          q = -cp * q;
          r = rcp(xb[k] - xa[k] * cp);
          bad |= !finite_rcp(r);
          dp = r * (xd[k] - xa[k] * dp);
          ap = -r * xa[k] * ap;
          cp = r * xc[k];
        }
      }
    }
    if (n >= 3) {
      // top row: row 0 with the chain folded in (chunk_backward's last step)
      const R C1 = -q;
      const R rr = rcp(R(1) - c0 * SA);
      bad |= !finite_rcp(rr);
      out[0 * nsys + s] = rr * a0;
      out[1 * nsys + s] = -rr * c0 * C1;
      out[2 * nsys + s] = rr * (d0 - c0 * SD);
    } else {
      // n == 2: row 0 already couples x_prev, x_0 and x_1 = x_{n-1}
      out[0 * nsys + s] = a0;
      out[1 * nsys + s] = c0;
      out[2 * nsys + s] = d0;
    }
    out[3 * nsys + s] = ap;
    out[4 * nsys + s] = cp;
    out[5 * nsys + s] = dp;
  }
  report_bad_pivot(bad, p.flag);
}

// Segment reduction for contiguous rows (solvedim 0): a warp reduces 32
// systems, one per lane, with the sweep of dist_reduce_kernel; rows arrive
// in blocks of RB through shared memory, loaded so that each load
// instruction reads RB consecutive rows of 32 / RB systems (full 64-byte
// runs) instead of one row of 32 systems a line apart each.
template <typename R>
__global__ void __launch_bounds__(128) dist_reduce_contig_kernel(const BatchArgs<R> p,
                                                                 R *__restrict__ out) {
  constexpr int RB = 8;
  constexpr int LD = RB + 1;  // odd row pitch: conflict-free per-lane reads
  __shared__ R tile[4][4][32 * LD];  // [warp][array][system * LD + row]
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const long long nsys = p.nsys;
  const int n = p.N;
  const R *arr[4] = {p.a, p.b, p.c, p.d_in};
  bool bad = false;
  for (long long g0 = ((long long)blockIdx.x * 4 + warp) * 32; g0 < nsys;
       g0 += (long long)gridDim.x * 4 * 32) {
    const long long s = g0 + lane;
    R a0 = R(0), c0 = R(0), d0 = R(0), ap = R(0), cp = R(0), dp = R(0);
    R q = R(1), SA = R(0), SD = R(0);
    // load k of a block: row lrow of system g0 + 4k + lane / RB (32 / RB = 4
    // systems per load); their first elements, -1 past the batch
    const int lrow = lane % RB;
    long long lb[RB];
#pragma unroll
    for (int k = 0; k < RB; ++k) {
      const long long ss = g0 + k * (32 / RB) + lane / RB;
      lb[k] = ss < nsys ? sys_base(p, ss) : -1;
    }
    for (int rb = 0; rb < n; rb += RB) {
      __syncwarp();  // the previous block's rows are consumed
#pragma unroll
      for (int k = 0; k < RB; ++k) {
        const int sl = k * (32 / RB) + lane / RB;
        const bool v = lb[k] >= 0 && rb + lrow < n;
        const long long o = v ? lb[k] + rb + lrow : 0;
#pragma unroll
        for (int a = 0; a < 4; ++a) tile[warp][a][sl * LD + lrow] = v ? __ldg(arr[a] + o) : R(1);
      }
      __syncwarp();
      const int rows = n - rb < RB ? n - rb : RB;
      for (int i = 0; i < rows; ++i) {
        const int j = rb + i;
        const R a = tile[warp][0][lane * LD + i], b = tile[warp][1][lane * LD + i],
                c = tile[warp][2][lane * LD + i], d = tile[warp][3][lane * LD + i];
        if (j < 2) {
          const R r = rcp(b);
          bad |= !finite_rcp(r) && s < nsys;
          if (j == 0) {
            a0 = a * r;
            c0 = c * r;
            d0 = d * r;
          } else {
            ap = a * r;
            cp = c * r;
            dp = d * r;
          }
        } else {
          SA += q * ap;  // row j - 1 joins the backward chain
          SD += q * dp;
          q = -cp * q;
          const R r = rcp(b - a * cp);
          bad |= !finite_rcp(r) && s < nsys;
          dp = r * (d - a * dp);
          ap = -r * a * ap;
          cp = r * c;
        }
      }
    }
    if (s < nsys) {
      if (n >= 3) {
        const R C1 = -q;
        const R rr = rcp(R(1) - c0 * SA);
        bad |= !finite_rcp(rr);
        out[0 * nsys + s] = rr * a0;
        out[1 * nsys + s] = -rr * c0 * C1;
        out[2 * nsys + s] = rr * (d0 - c0 * SD);
      } else {
        out[0 * nsys + s] = a0;
        out[1 * nsys + s] = c0;
        out[2 * nsys + s] = d0;
      }
      out[3 * nsys + s] = ap;
      out[4 * nsys + s] = cp;
      out[5 * nsys + s] = dp;
    }
  }
  report_bad_pivot(bad, p.flag);
}

// Segment reduction for contiguous segments of exactly 32 TM rows: a warp
// per system, the warp-tile reduction of the tiled long path (coalesced
// staging, chunk elimination, the warp's reduced solve for the segment's own
// right-hand side and the unit couplings to x_prev and x_next); the
// segment's first and last unknowns, f = pf + af x_prev + bf x_next and
// l = pl + al x_prev + bl x_next, give the two rows above
// (second_level_rows with neither end a system end). Unlike the tiles of one
// system, a segment keeps its a_0 and c_{n-1}: they are its couplings.
template <typename R, int TM>
__global__ void __launch_bounds__(128) dist_reduce_tile_kernel(const BatchArgs<R> p, R *__restrict__ out) {
  using L = SmemLayout<R, TM>;
  using TB = TileBuf<R, TM>;
  extern __shared__ __align__(16) unsigned char dist_smem[];
  R *buf = reinterpret_cast<R *>(dist_smem) + (threadIdx.x >> 5) * TB::ELEMS;
  const int lane = threadIdx.x & 31;
  const long long nsys = p.nsys;
  auto al = [](const void *q) { return (reinterpret_cast<uintptr_t>(q) & 15u) == 0; };
  const bool vec16 = al(p.a) && al(p.b) && al(p.c) && al(p.d_in);
  bool bad = false;
  for (long long s = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; s < nsys;
       s += ((long long)gridDim.x * blockDim.x) >> 5) {
    stage_tile_rows<R, TM>(p.a, p.b, p.c, p.d_in, vec16, sys_base(p, s), 32 * TM, buf, lane);
    R a[TM], c[TM], d[TM];
    lds_row<R, TM>(buf + 0 * L::BUF + lane * L::ROW, a);
    lds_row<R, TM>(buf + 2 * L::BUF + lane * L::ROW, c);
    lds_row<R, TM>(buf + 3 * L::BUF + lane * L::ROW, d);
    chunk_forward_staged<R, TM>(a, buf + 1 * L::BUF + lane * L::ROW, c, d, bad);
    chunk_backward<R, TM, true>(a, c, d, bad);
    const Row<R> top{a[0], c[0], d[0]}, bot{a[TM - 1], c[TM - 1], d[TM - 1]};
    R y[3], z[3];
    reduced_solve3<R>(top, bot, lane == 0 ? -top.A : R(0), lane == 31 ? -bot.C : R(0), lane, y, z, bad);
    const R pf = shfl_idx(y[0], 0, 32), af = shfl_idx(y[1], 0, 32), bf = shfl_idx(y[2], 0, 32);
    const R pl = shfl_idx(z[0], 31, 32), al2 = shfl_idx(z[1], 31, 32), bl = shfl_idx(z[2], 31, 32);
    if (lane == 0) {
      Row<R> t2, b2;
      second_level_rows<R>(pf, af, bf, pl, al2, bl, false, false, t2, b2);
      out[0 * nsys + s] = t2.A;
      out[1 * nsys + s] = t2.C;
      out[2 * nsys + s] = t2.D;
      out[3 * nsys + s] = b2.A;
      out[4 * nsys + s] = b2.C;
      out[5 * nsys + s] = b2.D;
    }
    __syncwarp();  // the buffer is free for the next system
  }
  report_bad_pivot(bad, p.flag);
}

template <typename R, int TM>
static cudaError_t launch_dist_reduce_tile(const BatchArgs<R> &p, R *out, cudaStream_t st) {
  const size_t smem = (size_t)4 * TileBuf<R, TM>::ELEMS * sizeof(R);  // 4 warps
  auto kern = dist_reduce_tile_kernel<R, TM>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int dev = 0, sms = 148, per_sm = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 128, smem) != cudaSuccess || per_sm < 1)
    per_sm = 1;
  const long long need = (p.nsys + 3) / 4;
  const long long cap = (long long)sms * per_sm;
  kern<<<(unsigned)(need < cap ? need : cap), 128, smem, st>>>(p, out);
  return cudaGetLastError();
}

// The warp-tile reduction where a contiguous segment fills a tile exactly
// (32 TM rows, TM = 4 .. 16 FP64, 4 .. 32 FP32); cudaErrorNotSupported
// otherwise.
template <typename R>
static cudaError_t launch_dist_reduce_tiles(const BatchArgs<R> &p, R *out, cudaStream_t st) {
  if (p.stride != 1) return cudaErrorNotSupported;
  switch (p.N) {
    case 128: return launch_dist_reduce_tile<R, 4>(p, out, st);
    case 256: return launch_dist_reduce_tile<R, 8>(p, out, st);
    case 512: return launch_dist_reduce_tile<R, 16>(p, out, st);
    case 1024:
      if constexpr (sizeof(R) == 4) return launch_dist_reduce_tile<R, 32>(p, out, st);
      return cudaErrorNotSupported;
    default: return cudaErrorNotSupported;
  }
}

// Reduced solve of system s over all ranks' rows and the right-hand-side
// correction of this rank's segment. g: P blocks of 6 * nsys values (the
// gathered outputs of dist_reduce_kernel, rank-major); row i of the reduced
// system is rank i/2's top (i even) or bottom (i odd) row, over the unknowns
// x_0^0, x_{n-1}^0, x_0^1, ... Only the neighbours' boundary values are
// needed (x_{2r-1} and x_{2r+2} for rank r), so the system is eliminated
// from both ends towards them (a twisted factorisation: top-down Thomas
// through row 2r+1, bottom-up through row 2r) with O(1) state per thread.
// save (Inc): the two original right-hand-side values.
constexpr int kMaxRanks = 4096;

template <typename R, bool INC>
__global__ void __launch_bounds__(128)
    dist_finish_kernel(const BatchArgs<R> p, const R *__restrict__ g, int P, int rank,
                       R *__restrict__ save) {
  const long long nsys = p.nsys;
  const int m = 2 * P;
  bool bad = false;
  for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < nsys;
       s += (long long)gridDim.x * blockDim.x) {
    auto row = [&](int i, R &a, R &c, R &d) {
      const R *blk = g + (long long)(i >> 1) * 6 * nsys + ((i & 1) ? 3 : 0) * nsys + s;
      a = i == 0 ? R(0) : blk[0];  // the global first a and last c are ignored
      c = i == m - 1 ? R(0) : blk[nsys];
      d = blk[2 * nsys];
    };
    // top-down: x_i = d'_i - c'_i x_{i+1}
    R cp = R(0), dp = R(0), cm1 = R(0), dm1 = R(0), cp1 = R(0), dp1 = R(0);
    const int hi = 2 * rank + 1;
    for (int i = 0; i <= hi; ++i) {
      R a, c, d;
      row(i, a, c, d);
      const R r = rcp(R(1) - a * cp);
      bad |= !finite_rcp(r);
      cp = c * r;
      dp = (d - a * dp) * r;
      if (i == 2 * rank - 1) {
        cm1 = cp;
        dm1 = dp;
      }
      if (i == hi) {
        cp1 = cp;
        dp1 = dp;
      }
    }
    // bottom-up: x_i = f'_i - e'_i x_{i-1}
    R ep = R(0), fp = R(0), e0 = R(0), f0 = R(0), e2 = R(0), f2 = R(0);
    for (int i = m - 1; i >= 2 * rank; --i) {
      R a, c, d;
      row(i, a, c, d);
      const R r = rcp(R(1) - c * ep);
      bad |= !finite_rcp(r);
      ep = a * r;
      fp = (d - c * fp) * r;
      if (i == 2 * rank + 2) {
        e2 = ep;
        f2 = fp;
      }
      if (i == 2 * rank) {
        e0 = ep;
        f0 = fp;
      }
    }
    R xprev = R(0), xnext = R(0);
    if (rank > 0) {
      const R r = rcp(R(1) - cm1 * e0);
      bad |= !finite_rcp(r);
      xprev = (dm1 - cm1 * f0) * r;
    }
    if (rank < P - 1) {
      const R r = rcp(R(1) - cp1 * e2);
      bad |= !finite_rcp(r);
      const R x1 = (dp1 - cp1 * f2) * r;  // x_{2r+1}
      xnext = f2 - e2 * x1;
    }
    const long long base = sys_base(p, s);
    const long long last = base + (long long)(p.N - 1) * p.stride;
    R *d = p.d_out;  // the caller's d (d_in == d_out for both Inc and not)
    const R d0 = d[base];
    if constexpr (INC) save[s] = d0;
    if (rank > 0) d[base] = d0 - __ldg(p.a + base) * xprev;
    const R dl = d[last];
    if constexpr (INC) save[nsys + s] = dl;
    if (rank < P - 1) d[last] = dl - __ldg(p.c + last) * xnext;
  }
  report_bad_pivot(bad, p.flag);
}

template <typename R>
__global__ void __launch_bounds__(128) dist_restore_kernel(const BatchArgs<R> p, const R *__restrict__ save) {
  const long long nsys = p.nsys;
  R *d = p.d_out;  // the caller's d (d_in == d_out for both Inc and not)
  for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < nsys;
       s += (long long)gridDim.x * blockDim.x) {
    const long long base = sys_base(p, s);
    d[base] = save[s];
    d[base + (long long)(p.N - 1) * p.stride] = save[nsys + s];
  }
}

std::mutex g_dist_mu;
std::set<const void *> g_dist_registered;

unsigned grid_for(long long n) {
  long long b = (n + 127) / 128;
  if (b > 148LL * 32) b = 148LL * 32;
  return (unsigned)(b < 1 ? 1 : b);
}

}  // namespace

bool dist_registered(const void *params) {
  if (!params) return false;
  std::lock_guard<std::mutex> lk(g_dist_mu);
  return g_dist_registered.count(params) != 0;
}

template <typename R, bool INC>
tridStatus_t dist_solve(const tridDistParams *dp, const BatchArgs<R> &p0, int solvedim,
                        cudaStream_t st, bool blocking) {
  if (dp->solvedim != solvedim || dp->nranks < 1 || dp->nranks > kMaxRanks || dp->rank < 0 ||
      dp->rank >= dp->nranks || !dp->allgather)
    return TRID_STATUS_INVALID_VALUE;
  if (p0.N < 2) return TRID_STATUS_INVALID_VALUE;  // every rank needs two rows
  BatchArgs<R> p = p0;
  const int P = dp->nranks;
  const size_t per_rank = (size_t)6 * p.nsys * sizeof(R);
  R *scratch = nullptr;
  const size_t save_bytes = INC ? (size_t)2 * p.nsys * sizeof(R) : 0;
  cudaError_t e = scratch_alloc((void **)&scratch, per_rank * (1 + P) + save_bytes, st);
  if (e != cudaSuccess) return status_of(e);
  R *send = scratch;
  R *recv = scratch + 6 * p.nsys;
  R *save = recv + (size_t)6 * p.nsys * P;
  e = launch_dist_reduce_tiles<R>(p, send, st);
  if (e == cudaErrorNotSupported) {
    if (p.stride == 1) {
      long long blocks = (p.nsys + 127) / 128;
      if (blocks > 148LL * 16) blocks = 148LL * 16;
      dist_reduce_contig_kernel<R><<<(unsigned)(blocks < 1 ? 1 : blocks), 128, 0, st>>>(p, send);
    } else {
      dist_reduce_kernel<R><<<grid_for(p.nsys), 128, 0, st>>>(p, send);
    }
    e = cudaGetLastError();
  }
  g_launches.fetch_add(1, std::memory_order_relaxed);
  tridStatus_t status = TRID_STATUS_SUCCESS;
  if (e == cudaSuccess) {
    const int rc = dp->allgather(send, recv, per_rank, dp->user, st);
    if (rc != 0) status = TRID_STATUS_EXECUTION_FAILED;
  }
  if (e == cudaSuccess && status == TRID_STATUS_SUCCESS) {
    dist_finish_kernel<R, INC><<<grid_for(p.nsys), 128, 0, st>>>(p, recv, P, dp->rank, save);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess && status == TRID_STATUS_SUCCESS) {
    const Plan plan = choose_plan<R>(p, vec_aligned<R>(p));
    e = launch_batch<R, INC>(p, plan, st);
  }
  if (INC && e == cudaSuccess && status == TRID_STATUS_SUCCESS) {
    dist_restore_kernel<R><<<grid_for(p.nsys), 128, 0, st>>>(p, save);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    e = cudaGetLastError();
  }
  const cudaError_t ef = scratch_free(scratch, st);
  if (e == cudaSuccess) e = ef;
  if (e != cudaSuccess) return status_of(e);
  if (status != TRID_STATUS_SUCCESS) return status;
  if (blocking) {
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return status_of(e);
    if (pivot_flag_take()) return TRID_STATUS_ZERO_PIVOT;
  }
  return TRID_STATUS_SUCCESS;
}

template tridStatus_t dist_solve<double, false>(const tridDistParams *, const BatchArgs<double> &, int,
                                                cudaStream_t, bool);
template tridStatus_t dist_solve<double, true>(const tridDistParams *, const BatchArgs<double> &, int,
                                               cudaStream_t, bool);
template tridStatus_t dist_solve<float, false>(const tridDistParams *, const BatchArgs<float> &, int,
                                               cudaStream_t, bool);
template tridStatus_t dist_solve<float, true>(const tridDistParams *, const BatchArgs<float> &, int,
                                              cudaStream_t, bool);

}  // namespace trid

using namespace trid;

EXTERN_C tridStatus_t tridDistInit(tridDistParams *params, int solvedim, int rank, int nranks,
                                   tridAllgatherFn allgather, void *user) {
  if (!params || !allgather || nranks < 1 || nranks > kMaxRanks || rank < 0 || rank >= nranks ||
      solvedim < 0 || solvedim >= MAXDIM)
    return TRID_STATUS_INVALID_VALUE;
  params->solvedim = solvedim;
  params->rank = rank;
  params->nranks = nranks;
  params->allgather = allgather;
  params->user = user;
  std::lock_guard<std::mutex> lk(g_dist_mu);
  g_dist_registered.insert(params);
  return TRID_STATUS_SUCCESS;
}

EXTERN_C tridStatus_t tridDistFinalize(tridDistParams *params) {
  std::lock_guard<std::mutex> lk(g_dist_mu);
  return g_dist_registered.erase(params) ? TRID_STATUS_SUCCESS : TRID_STATUS_INVALID_VALUE;
}

EXTERN_C long long tridDistExchangeBytes(int dtype_bytes, int ndim, int solvedim, const int *dims) {
  if ((dtype_bytes != 4 && dtype_bytes != 8) || ndim < 1 || ndim > MAXDIM || solvedim < 0 ||
      solvedim >= ndim || !dims)
    return -1;
  long long nsys = 1;
  for (int i = 0; i < ndim; ++i)
    if (i != solvedim) nsys *= dims[i];
  return 6 * nsys * dtype_bytes;
}
