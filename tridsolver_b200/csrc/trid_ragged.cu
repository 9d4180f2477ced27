// Ragged batches: independent contiguous systems of uneven lengths, system k
// occupying rows [offsets[k], offsets[k+1]) of a, b, c, d, solved in one
// persistent launch.
//
//   1. ragged_hist_kernel / ragged_order_kernel bucket the systems by length
//      class (ceil(log2 N)), longest class first (longest-processing-time
//      order keeps the SMs evenly loaded at the end). A system of a "tile"
//      class is cut into K tiles of 512 rows and each tile becomes one work
//      item; a system of a "warp" class (short systems,
//      rows-per-lane M from the class table) is one warp item;
//   2. ragged_kernel: persistent warps take tile items (longest systems
//      first), then warp items, from one global counter.
//
// Tile item (one warp, 16 rows per lane): the warp stages the tile's rows of
// a, b, c, d in shared memory with coalesced cp.async copies, each lane runs
// the chunk elimination on its 16 rows, and the warp's reduced solve is run
// for three right-hand sides at once: the tile's own, and the unit
// couplings to the unknown just before the tile (x_prev, the previous
// tile's last) and just after it (x_next, the next tile's first). Every
// reduced unknown of the tile is then p + alpha x_prev + beta x_next. From
// the tile's first and last unknowns the warp forms the tile's two rows of
// a second-level tridiagonal system (2 rows per tile, at most 64 rows), and
// the warp that finishes the last tile of a system solves it (two tiles a
// lane, then one warp PCR) and publishes every tile's first and last
// unknown. The other warps of
// the system park their tile's eliminated rows in tensor memory (96 32-bit
// columns FP64, 48 FP32, of the warp's lane quarter), take their next item,
// and only after
// publishing that one (or after a warp item) wait (bounded, on a flag) for
// the parked tile's system, then substitute and store. So every element is
// read once and written once, with 8 values of scratch per tile, and a wait
// has a whole item of slack (the earlier form held the tile in registers and
// waited at once: 17 us a wait on average, a third of the warps' time).
// A warp holds at most one parked tile, in its TMEM slot; each
// claimed tile is published before its warp waits on anything, and claims
// are in system order, so the tiles a warp waits for are held by running
// warps: the wait always ends.
//
// The reference has no ragged entry point; its per-system solve trid_scalar
// (scalar/src/cpu/trid_cpu.cpp:312-353) is the oracle for each system.
#include <cuda_runtime.h>

#include <atomic>
#include <cstring>
#include <mutex>

#include "trid_internal.h"
#include "trid_tile.cuh"
#include "trid_tmem.cuh"
#include "tridsolver_b200.h"

namespace trid {

constexpr int kClasses = 24;        // length classes 0..23: N <= 2^class
// Tile items (tile_m / tile_rows, trid_tile.cuh): tiles per system, N <=
// 16384 either way, so the second-level system has at most 64 rows.
// Ragged tiles: 16 rows per lane, 512 rows, in both precisions (measured on
// the 200k-system batch against 8 FP64 / 32 FP32 rows a lane: FP64 4.69 vs
// 5.20 ms, FP32 2.85 vs 2.98 ms). An FP32 lane's eliminated rows then take
// half the registers and a tile half the TMEM columns of an FP64 one, so
// four FP32 CTAs of 4 warps fit an SM against three FP64 ones; at most 32
// tiles a system of 16384 rows.
template <typename R> constexpr int rtile_m() { return 16; }
template <typename R> constexpr int ragged_ctas() { return sizeof(R) == 8 ? 3 : 4; }
template <typename R> constexpr int rtile_rows() { return 32 * rtile_m<R>(); }
template <typename R> using RTileBuf = TileBuf<R, rtile_m<R>()>;
template <typename R> constexpr int max_tiles() { return 16384 / rtile_rows<R>(); }
constexpr int kRaggedThreads = 128; // 4 warps per CTA
constexpr unsigned kWaitLimit = 1u << 22;  // polls of the ready flag (each with a short sleep)

template <typename R> struct RaggedArgs {
  const R *a, *b, *c;
  R *d;
  const int64_t *off;
  const int *order;                 // warp-item systems, longest class first
  const unsigned *hist;             // systems per class
  const unsigned long long *tiles;  // tiles per class (tile classes)
  const int4 *tile_meta;            // per tile item: system, tile index j, tiles K, rows n
  const long long *tile_base;       // per tile item: the system's first element
  R *tile_rows;                     // 6 per tile: top A, C, D; bottom A, C, D
  R *tile_fl;                       // 2 per tile: first and last unknown
  unsigned *sys_done;               // tiles of the system past the reduction
  unsigned *sys_ready;              // second-level solution published
  unsigned long long *counter;      // work items taken
  long long nsys;
  int mtab[kClasses];               // rows per lane by class; 0 = tile class
  unsigned *flag;
  unsigned *error;                  // 1: a system longer than 16384 rows; 2: a wait gave up;
                                    // 3: the tile table was too small
  long long max_tiles;              // entries of tile_meta / tile_base / tile_rows / tile_fl
  long long nelems;                 // element count the caller gave (-1: read back)
  bool vec16;                       // a, b, c, d all 16-byte aligned
  unsigned wait_limit;              // polls before a wait gives up (kWaitLimit by default)
  bool withhold;                    // failure-detection tests: never publish (waits run out)
};

// Release/acquire operations at device scope: a tile's second-level rows are
// published by the count that follows them, and read after the count
// (acquire) by the warp that completes the system.
__device__ __forceinline__ unsigned atomic_add_acq_rel(unsigned *p, unsigned v) {
  unsigned old;
  asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
  return old;
}
__device__ __forceinline__ unsigned load_acquire(const unsigned *p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ int length_class(long long n) {
  int c = 0;
  while (c < kClasses - 1 && (1LL << c) < n) ++c;
  return c;
}

template <typename R>
__global__ void ragged_hist_kernel(RaggedArgs<R> p, unsigned *hist, unsigned long long *tiles) {
  // a caller's count below the batch's: refused before anything is written
  if (p.nelems >= 0 && blockIdx.x == 0 && threadIdx.x == 0 && p.off[p.nsys] - p.off[0] > p.nelems)
    atomicExch(p.error, 3u);
  for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < p.nsys;
       s += (long long)gridDim.x * blockDim.x) {
    const long long n = p.off[s + 1] - p.off[s];
    const int c = length_class(n > 0 ? n : 1);
    atomicAdd(&hist[c], 1u);
    if (p.mtab[c] == 0) atomicAdd(&tiles[c], (unsigned long long)((n + rtile_rows<R>() - 1) / rtile_rows<R>()));
  }
}

template <typename R>
__global__ void ragged_order_kernel(RaggedArgs<R> p, const unsigned *hist,
                                    const unsigned long long *tiles, unsigned *fill,
                                    unsigned long long *tfill, int *order, int4 *tile_meta,
                                    long long *tile_base) {
  for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < p.nsys;
       s += (long long)gridDim.x * blockDim.x) {
    const long long n = p.off[s + 1] - p.off[s];
    const int c = length_class(n > 0 ? n : 1);
    if (p.mtab[c] == 0) {
      unsigned long long t0 = 0;
      for (int q = kClasses - 1; q > c; --q)
        if (p.mtab[q] == 0) t0 += tiles[q];
      const long long K = (n + rtile_rows<R>() - 1) / rtile_rows<R>();
      const long long ts = (long long)(t0 + atomicAdd(&tfill[c], (unsigned long long)K));
      if (ts + K > p.max_tiles) {  // offsets not ascending: refuse rather than overrun
        atomicExch(p.error, 3u);
        continue;
      }
      const long long base = p.off[s];
      for (long long j = 0; j < K; ++j) {
        tile_meta[ts + j] = make_int4((int)s, (int)j, (int)(K < 0x7fffffff ? K : 0x7fffffff),
                                      (int)(n < 0x7fffffff ? n : 0x7fffffff));
        tile_base[ts + j] = base;
      }
    } else {
      unsigned start = 0;
      for (int q = kClasses - 1; q > c; --q)
        if (p.mtab[q] != 0) start += hist[q];
      order[start + atomicAdd(&fill[c], 1u)] = (int)s;
    }
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

// One short system per warp, M rows per lane (M = 1: pure PCR).
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
    chunk_forward<R, M, true>(a, b, c, d, bad);
    chunk_backward<R, M, true>(a, c, d, bad);
    R y, z;
    reduced_solve<R>(Row<R>{a[0], c[0], d[0]}, Row<R>{a[M - 1], c[M - 1], d[M - 1]}, lane, 32, y, z,
                     bad);
    chunk_substitute<R, M>(a, c, d, y, z);
#pragma unroll
    for (int i = 0; i < M; ++i)
      if ((long long)lane * M + i < n) p.d[base + (long long)lane * M + i] = d[i];
  }
}


// TMEM per CTA: one parking slot in each warp's lane quarter: a', c', d' of
// the lane's interior rows 1 .. M-2 and the reduced solve's y[3], z[3], as
// 32-bit words (96 columns FP64, 48 FP32, of the CTA's 128 or 64).
template <typename R> constexpr int park_words() { return (sizeof(R) / 4) * (3 * (rtile_m<R>() - 2) + 6); }
template <typename R> constexpr int ragged_tmem_cols() { return park_words<R>() <= 64 ? 64 : 128; }
static_assert(park_words<double>() % 16 == 0 && park_words<float>() % 16 == 0, "16-column transfers");

// The values of a parked tile, one 32-bit word array per 16 columns.
template <typename R> struct ParkWords {
  static constexpr int NB = park_words<R>() / 16;
  uint32_t w[NB][16];
  __device__ __forceinline__ void put(int k, R v) {
    if constexpr (sizeof(R) == 8) {
      w[(2 * k) / 16][(2 * k) % 16] = (uint32_t)__double2loint(v);
      w[(2 * k + 1) / 16][(2 * k + 1) % 16] = (uint32_t)__double2hiint(v);
    } else {
      w[k / 16][k % 16] = __float_as_uint(v);
    }
  }
  __device__ __forceinline__ R get(int k) const {
    if constexpr (sizeof(R) == 8)
      return __hiloint2double((int)w[(2 * k + 1) / 16][(2 * k + 1) % 16], (int)w[(2 * k) / 16][(2 * k) % 16]);
    else
      return __uint_as_float(w[k / 16][k % 16]);
  }
};

// x of the tile from its rows after elimination (a, c, d: rows 0 .. M-1,
// rows 1 .. M-2 interior) and the tile's first and last unknowns, out through
// the warp's d rows with coalesced element stores.
template <typename R>
__device__ __forceinline__ void tile_store(const RaggedArgs<R> &p, long long base, int nt,
                                           R (&a)[rtile_m<R>()], R (&c)[rtile_m<R>()],
                                           R (&d)[rtile_m<R>()], R yy, R zz, R *buf, int lane) {
  using L = SmemLayout<R, rtile_m<R>()>;
  chunk_substitute<R, rtile_m<R>()>(a, c, d, yy, zz);
  sts_row<R, rtile_m<R>()>(buf + 3 * L::BUF + lane * L::ROW, d);
  __syncwarp();
#pragma unroll 4
  for (int e = lane; e < nt; e += 32) p.d[base + e] = buf[3 * L::BUF + RTileBuf<R>::slot(e)];
  __syncwarp();  // the buffer is free for the next item
}

// Tile item, first part: stage, eliminate, reduce, publish the tile's two
// second-level rows. A system of one tile, or the warp whose tile completes
// its system (which then solves the second level and publishes its
// solution), finishes the tile at once (false). Otherwise the tile's state
// is left in `pw` for parking (true): the warp
// finishes it after its next item's first part, so the wait for the rest of
// the system overlaps useful work. No wait happens here, so every claimed
// tile is published without depending on any other.
template <typename R>
__device__ __forceinline__ bool tile_publish(const RaggedArgs<R> &p, long long item, R *buf, int lane,
                                             ParkWords<R> &pw, bool &bad) {
  using L = SmemLayout<R, rtile_m<R>()>;
  const int4 meta = p.tile_meta[item];
  const int s = meta.x;
  const int j = meta.y;
  const int K = meta.z;
  const long long n = meta.w;
  const long long ts = item - j;
  const long long base0 = p.tile_base[item];
  const long long r0 = (long long)j * rtile_rows<R>();
  const int nt = (int)(n - r0 < rtile_rows<R>() ? n - r0 : rtile_rows<R>());
  stage_tile_rows<R, rtile_m<R>()>(p.a, p.b, p.c, p.d, p.vec16, base0 + r0, nt, buf, lane);

  constexpr int kTM = rtile_m<R>();
  R a[kTM], c[kTM], d[kTM];
  lds_row<R, kTM>(buf + 0 * L::BUF + lane * L::ROW, a);
  lds_row<R, kTM>(buf + 2 * L::BUF + lane * L::ROW, c);
  lds_row<R, kTM>(buf + 3 * L::BUF + lane * L::ROW, d);
  const long long row0 = r0 + (long long)lane * kTM;
  if (row0 == 0) a[0] = R(0);
#pragma unroll
  for (int i = 0; i < kTM; ++i)
    if (row0 + i == n - 1) c[i] = R(0);
  chunk_forward_staged<R, kTM>(a, buf + 1 * L::BUF + lane * L::ROW, c, d, bad);
  chunk_backward<R, kTM, true>(a, c, d, bad);
  const Row<R> top{a[0], c[0], d[0]}, bot{a[kTM - 1], c[kTM - 1], d[kTM - 1]};
  R y[3], z[3];
  reduced_solve3<R>(top, bot, lane == 0 ? -top.A : R(0), lane == 31 ? -bot.C : R(0), lane, y, z,
                    bad);
  if (K == 1) {
    tile_store<R>(p, base0 + r0, nt, a, c, d, y[0], z[0], buf, lane);
    return false;
  }
  // the tile's first unknown f = y(lane 0) and last l = z(lane 31), each
  // as p + alpha x_prev + beta x_next
  const R pf = shfl_idx(y[0], 0, 32), af = shfl_idx(y[1], 0, 32), bf = shfl_idx(y[2], 0, 32);
  const R pl = shfl_idx(z[0], 31, 32), al = shfl_idx(z[1], 31, 32), bl = shfl_idx(z[2], 31, 32);
  bool last = false;
  if (lane == 0) {
    Row<R> t2, b2;
    second_level_rows<R>(pf, af, bf, pl, al, bl, j == 0, j == K - 1, t2, b2);
    R *tr = p.tile_rows + 6 * (ts + j);
    tr[0] = t2.A;
    tr[1] = t2.C;
    tr[2] = t2.D;
    tr[3] = b2.A;
    tr[4] = b2.C;
    tr[5] = b2.D;
    // release: the rows before the count; acquire: the other tiles' rows
    // for the warp that completes the count
    last = atomic_add_acq_rel(&p.sys_done[s], 1u) == (unsigned)(K - 1);
  }
  last = __shfl_sync(FULL_MASK, last, 0);
  if (last) {
    __syncwarp();
    // the second-level system, rows f_0, l_0, f_1, l_1, ... (2 a tile, up
    // to 128): two tiles (4 rows, unit diagonal) a lane, identity rows past
    // the last tile
    R qa[4], qb[4], qc[4], qd[4];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int t = 2 * lane + h;
      qb[2 * h] = qb[2 * h + 1] = R(1);
      qa[2 * h] = qc[2 * h] = qd[2 * h] = qa[2 * h + 1] = qc[2 * h + 1] = qd[2 * h + 1] = R(0);
      if (t < K) {
        const R *tr = p.tile_rows + 6 * (ts + t);  // read from L2, not a stale L1 line
        qa[2 * h] = __ldcg(tr + 0);
        qc[2 * h] = __ldcg(tr + 1);
        qd[2 * h] = __ldcg(tr + 2);
        qa[2 * h + 1] = __ldcg(tr + 3);
        qc[2 * h + 1] = __ldcg(tr + 4);
        qd[2 * h + 1] = __ldcg(tr + 5);
      }
    }
    chunk_forward<R, 4>(qa, qb, qc, qd, bad);
    chunk_backward<R, 4>(qa, qc, qd, bad);
    R f, l;
    reduced_solve<R>(Row<R>{qa[0], qc[0], qd[0]}, Row<R>{qa[3], qc[3], qd[3]}, lane, 32, f, l, bad);
    chunk_substitute<R, 4>(qa, qc, qd, f, l);
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int t = 2 * lane + h;
      if (t < K) {
        p.tile_fl[2 * (ts + t)] = qd[2 * h];
        p.tile_fl[2 * (ts + t) + 1] = qd[2 * h + 1];
      }
    }
    __threadfence();
    __syncwarp();
    if (lane == 0 && !p.withhold) atomicExch(&p.sys_ready[s], 1u);
    const R xp = j > 0 ? __ldcg(p.tile_fl + 2 * (ts + j - 1) + 1) : R(0);
    const R xn = j < K - 1 ? __ldcg(p.tile_fl + 2 * (ts + j + 1)) : R(0);
    tile_store<R>(p, base0 + r0, nt, a, c, d, y[0] + y[1] * xp + y[2] * xn, z[0] + z[1] * xp + z[2] * xn,
                  buf, lane);
    return false;
  }
  // to park: interior rows' a', c', d', then y, z
#pragma unroll
  for (int i = 1; i < kTM - 1; ++i) {
    pw.put(i - 1, a[i]);
    pw.put(kTM - 2 + i - 1, c[i]);
    pw.put(2 * (kTM - 2) + i - 1, d[i]);
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    pw.put(3 * (kTM - 2) + k, y[k]);
    pw.put(3 * (kTM - 2) + 3 + k, z[k]);
  }
  return true;
}

// Parking slot transfers (16-column blocks). park_swap stores the new
// tile's words block by block in place of the parked tile's, which it
// returns in the same array, so at most one block of extra registers is live.
template <typename R> __device__ __forceinline__ void park_put(uint32_t slot, const ParkWords<R> &pw) {
#pragma unroll
  for (int k = 0; k < ParkWords<R>::NB; ++k) tmem_put(slot + 16 * k, pw.w[k]);
  tmem_wait_st();
}
template <typename R> __device__ __forceinline__ void park_get(uint32_t slot, ParkWords<R> &pw) {
#pragma unroll
  for (int k = 0; k < ParkWords<R>::NB; ++k) tmem_get(slot + 16 * k, pw.w[k]);
#pragma unroll
  for (int k = 0; k < ParkWords<R>::NB; ++k) tmem_wait_ld(pw.w[k]);
}
template <typename R> __device__ __forceinline__ void park_swap(uint32_t slot, ParkWords<R> &pw) {
#pragma unroll
  for (int k = 0; k < ParkWords<R>::NB; ++k) {
    uint32_t v[16];
    tmem_get(slot + 16 * k, v);
    tmem_wait_ld(v);
    tmem_put(slot + 16 * k, pw.w[k]);
    tmem_wait_st();
#pragma unroll
    for (int i = 0; i < 16; ++i) pw.w[k][i] = v[i];
  }
}

// Tile item, second part: waits (bounded) for the parked tile's system to
// publish its second-level solution, then substitutes (the tile's words in
// pw) and stores.
template <typename R>
__device__ __forceinline__ void tile_finish(const RaggedArgs<R> &p, long long item,
                                            const ParkWords<R> &pw, R *buf, int lane) {
  // the parked tile's place, read again (L2) rather than held in registers
  const int4 meta = p.tile_meta[item];
  const int s = meta.x;
  const int j = meta.y;
  const int K = meta.z;
  const long long ts = item - j;
  const long long r0 = (long long)j * rtile_rows<R>();
  const long long base = p.tile_base[item] + r0;
  const int nt = (int)(meta.w - r0 < rtile_rows<R>() ? meta.w - r0 : rtile_rows<R>());
  unsigned ok = 1;
  if (lane == 0) {
    // bounded: p.wait_limit polls (kWaitLimit unless a test lowered it), and
    // none at all once any wait of this launch has given up (error != 0)
    const volatile unsigned *err = p.error;
    unsigned it = 0;
    unsigned r = load_acquire(p.sys_ready + s);
    while (r == 0u && *err == 0u && it < p.wait_limit) {
      __nanosleep(128);
      ++it;
      r = load_acquire(p.sys_ready + s);
    }
    ok = r != 0u;
    if (!ok) atomicExch(p.error, 2u);
  }
  ok = __shfl_sync(FULL_MASK, ok, 0);
  if (!ok) return;  // reported; this tile is left unsolved
  __syncwarp();
  using L = SmemLayout<R, rtile_m<R>()>;
  constexpr int kTM = rtile_m<R>();
  constexpr int I0 = 3 * (kTM - 2);  // y[3], z[3] follow the rows
  const R xp = j > 0 ? __ldcg(p.tile_fl + 2 * (ts + j - 1) + 1) : R(0);
  const R xn = j < K - 1 ? __ldcg(p.tile_fl + 2 * (ts + j + 1)) : R(0);
  const R yy = pw.get(I0 + 0) + pw.get(I0 + 1) * xp + pw.get(I0 + 2) * xn;
  const R zz = pw.get(I0 + 3) + pw.get(I0 + 4) * xp + pw.get(I0 + 5) * xn;
  // x_i = d'_i - a'_i x_first - c'_i x_last (x_first = yy, x_last = zz),
  // straight from the parked words into the lane's staged row, 16 bytes at
  // a time
  using Vt = typename Vec16<R>::T;
  constexpr int n = Vec16<R>::n;
  Vt *row = reinterpret_cast<Vt *>(buf + 3 * L::BUF + lane * L::ROW);
#pragma unroll
  for (int g = 0; g < kTM / n; ++g) {
    R x[n];
#pragma unroll
    for (int k = 0; k < n; ++k) {
      const int i = g * n + k;
      if (i == 0)
        x[k] = yy;
      else if (i == kTM - 1)
        x[k] = zz;
      else
        x[k] = pw.get(2 * (kTM - 2) + i - 1) - pw.get(i - 1) * yy - pw.get(kTM - 2 + i - 1) * zz;
    }
    Vt v;
    if constexpr (n == 2) {
      v.x = x[0];
      v.y = x[1];
    } else {
      v.x = x[0];
      v.y = x[1];
      v.z = x[2];
      v.w = x[3];
    }
    row[g] = v;
  }
  __syncwarp();
#pragma unroll 4
  for (int e = lane; e < nt; e += 32) p.d[base + e] = buf[3 * L::BUF + RTileBuf<R>::slot(e)];
  __syncwarp();  // the buffer is free for the next item
}

// Persistent warps take tile items (longest systems first), then warp items,
// from one global counter. A warp holds at most one parked tile, in its TMEM
// slot: after the first part of each new tile it swaps the new tile in and
// finishes the one parked before (after a warp item, or a tile finished at
// once, it takes the parked one out and finishes it), so each wait has had
// a whole item of slack.
template <typename R>
__global__ void __launch_bounds__(kRaggedThreads, ragged_ctas<R>()) ragged_kernel(const RaggedArgs<R> p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ uint32_t tmem_slot;
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  R *buf = reinterpret_cast<R *>(smem_raw) + warp * RTileBuf<R>::ELEMS;
  if (*reinterpret_cast<volatile unsigned *>(p.error) == 3u) return;  // tile table refused (uniform)
  if (warp == 0) tmem_alloc_cols<ragged_tmem_cols<R>()>(&tmem_slot);
  tmem_fence_before_sync();
  __syncthreads();
  tmem_fence_after_sync();
  const uint32_t tbase = tmem_slot;
  const uint32_t slot = tbase + ((uint32_t)(32 * (warp & 3)) << 16);  // this warp's lane quarter
  long long ntiles = 0, nwarp = 0;
  for (int c = 0; c < kClasses; ++c) {
    if (p.mtab[c] == 0)
      ntiles += (long long)p.tiles[c];
    else
      nwarp += p.hist[c];
  }
  bool bad = false;
  bool parked = false;
  long long pk = 0;  // the parked tile's item
  for (;;) {
    long long it = 0;
    if (lane == 0) it = (long long)atomicAdd(p.counter, 1ULL);
    it = __shfl_sync(FULL_MASK, it, 0);
    if (it < ntiles) {
      const int4 meta = p.tile_meta[it];
      if (meta.z > max_tiles<R>()) {  // longer than 16384 rows: reported once per system
        if (lane == 0 && meta.y == 0) atomicExch(p.error, 1u);
        continue;
      }
      ParkWords<R> pw;
      if (tile_publish<R>(p, it, buf, lane, pw, bad)) {
        if (parked) {
          park_swap<R>(slot, pw);  // the new tile in, the parked one out (into pw)
          tile_finish<R>(p, pk, pw, buf, lane);
        } else {
          park_put<R>(slot, pw);
        }
        pk = it;
        parked = true;
      } else if (parked) {
        park_get<R>(slot, pw);
        tile_finish<R>(p, pk, pw, buf, lane);
        parked = false;
      }
      continue;
    }
    it -= ntiles;
    if (it < nwarp) {
      const int s = p.order[it];
      const long long base = p.off[s];
      const long long n = p.off[s + 1] - base;
      switch (p.mtab[length_class(n > 0 ? n : 1)]) {
        case 1: warp_item<R, 1>(p, base, n, lane, bad); break;
        case 2: warp_item<R, 2>(p, base, n, lane, bad); break;
        case 4: warp_item<R, 4>(p, base, n, lane, bad); break;
        default: warp_item<R, 8>(p, base, n, lane, bad); break;
      }
    }
    if (parked) {
      ParkWords<R> pw;
      park_get<R>(slot, pw);
      tile_finish<R>(p, pk, pw, buf, lane);
      parked = false;
    }
    if (it >= nwarp) break;
  }
  report_bad_pivot(bad, p.flag);
  tmem_fence_before_sync();
  __syncthreads();
  tmem_fence_after_sync();
  if (warp == 0) tmem_dealloc_cols<ragged_tmem_cols<R>()>(tbase);
}

// ---- host side ---------------------------------------------------------------

// Resident CTAs per SM of the ragged kernel (at least 1): the smallest of
// the shared-memory, register and TMEM-column limits. (Were fewer resident,
// the extra CTAs would start as others exit and find the items taken: every
// claimed tile is published before its warp waits on anything.)
template <typename K>
static int ragged_ctas_per_sm(int dev, K kernel, size_t smem, int tmem_cols) {
  int smem_sm = 0, reserved = 0, regs_sm = 0;
  cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
  cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev);
  cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev);
  cudaFuncAttributes fa{};
  if (cudaFuncGetAttributes(&fa, kernel) != cudaSuccess) {
    cudaGetLastError();
    return 1;
  }
  const long long per_cta_smem = (long long)smem + (long long)fa.sharedSizeBytes + reserved;
  const long long warp_regs = ((long long)fa.numRegs * 32 + 255) / 256 * 256;  // allocated per warp
  const long long per_cta_regs = warp_regs * (kRaggedThreads / 32);
  long long n = 512 / tmem_cols;
  if (per_cta_smem > 0 && smem_sm / per_cta_smem < n) n = smem_sm / per_cta_smem;
  if (per_cta_regs > 0 && regs_sm / per_cta_regs < n) n = regs_sm / per_cta_regs;
  return n < 1 ? 1 : (int)n;
}

// Rows per lane by length class: M > 0 for warp items, 0 for tile classes.
// Built-in table, replaced per device and precision by tridRaggedAutotune.
// g_tab_mu guards both: a call on one host thread may read the table while
// tridRaggedAutotune on another replaces it.
static int g_mtab[2][64][kClasses];
static bool g_tuned[2][64];
static std::mutex g_tab_mu;

// The table in use for precision index pi on device dev, copied into mt;
// false (mt untouched) when the device has no tuned table.
static bool tuned_table(int pi, int dev, int *mt) {
  std::lock_guard<std::mutex> lk(g_tab_mu);
  if (!g_tuned[pi][dev]) return false;
  memcpy(mt, g_mtab[pi][dev], sizeof(g_mtab[pi][dev]));
  return true;
}

static void set_tuned_table(int pi, int dev, const int *mt) {
  std::lock_guard<std::mutex> lk(g_tab_mu);
  memcpy(g_mtab[pi][dev], mt, sizeof(g_mtab[pi][dev]));
  g_tuned[pi][dev] = true;
}

// Longest class a warp per system may take (M <= 8); longer systems take tiles.
template <typename R> static constexpr int ragged_warp_max() { return 256; }

template <typename R>
static void default_mtab(int *m) {
  for (int c = 0; c < kClasses; ++c) {
    const long long n = 1LL << c;
    m[c] = n <= 32 ? 1 : n <= 64 ? 2 : 0;
  }
}

// Failure-detection hooks (tridRaggedSetWaitBound): the wait bound in polls
// (0: kWaitLimit) and whether second-level solutions are withheld.
static std::atomic<unsigned long long> g_wait_polls{0};
static std::atomic<int> g_withhold{0};

template <typename R>
static cudaError_t launch_ragged(RaggedArgs<R> p, const int *mtab, long long elems,
                                 cudaStream_t st) {
  for (int c = 0; c < kClasses; ++c) p.mtab[c] = mtab[c];
  // classes beyond one warp are always tile classes
  for (int c = 0; c < kClasses; ++c)
    if ((1LL << c) > ragged_warp_max<R>()) p.mtab[c] = 0;
  // The tile scratch is sized by the batch's element count. Without a
  // count from the caller (elems < 0) two offsets are read back, a short
  // synchronisation on `st`; with one, nothing is read back and the call
  // can be captured. The order kernel refuses a tile table the count
  // undersizes (error 3) and the solve then writes nothing.
  cudaError_t e = cudaSuccess;
  const long long given = elems;
  if (elems < 0) {
    int64_t ends[2] = {0, 0};
    e = cudaMemcpyAsync(&ends[0], p.off, sizeof(int64_t), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(&ends[1], p.off + p.nsys, sizeof(int64_t), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return e;
    elems = ends[1] - ends[0];
    if (elems < 0) return cudaErrorInvalidValue;
  }
  const long long max_tiles = elems / rtile_rows<R>() + p.nsys + 1;
  // scratch: header | order (int, nsys) | done, ready (u32, nsys each) |
  // tile_meta (int4, max_tiles) | tile_base (i64) | tile_rows (6 R) | tile_fl (2 R)
  // header: hist u32[24] @0, fill u32[24] @128, tiles u64[24] @256,
  //         tfill u64[24] @512, counter u64 @768, error u32 @776
  const size_t head = 1024;
  auto up = [](size_t v) { return (v + 255) / 256 * 256; };
  const size_t o_order = head;
  const size_t o_done = o_order + up((size_t)p.nsys * sizeof(int));
  const size_t o_ready = o_done + up((size_t)p.nsys * sizeof(unsigned));
  const size_t o_tmeta = o_ready + up((size_t)p.nsys * sizeof(unsigned));
  const size_t o_tbase = o_tmeta + up((size_t)max_tiles * sizeof(int4));
  const size_t o_trows = o_tbase + up((size_t)max_tiles * sizeof(long long));
  const size_t o_tfl = o_trows + up((size_t)max_tiles * 6 * sizeof(R));
  const size_t total = o_tfl + up((size_t)max_tiles * 2 * sizeof(R));
  char *scratch = nullptr;
  e = scratch_alloc((void **)&scratch, total, st);
  if (e != cudaSuccess) return e;
  unsigned *hist = reinterpret_cast<unsigned *>(scratch);
  unsigned *fill = reinterpret_cast<unsigned *>(scratch + 128);
  unsigned long long *tiles = reinterpret_cast<unsigned long long *>(scratch + 256);
  unsigned long long *tfill = reinterpret_cast<unsigned long long *>(scratch + 512);
  unsigned long long *counter = reinterpret_cast<unsigned long long *>(scratch + 768);
  unsigned *error = reinterpret_cast<unsigned *>(scratch + 776);
  int *order = reinterpret_cast<int *>(scratch + o_order);
  unsigned *done = reinterpret_cast<unsigned *>(scratch + o_done);
  unsigned *ready = reinterpret_cast<unsigned *>(scratch + o_ready);
  int4 *tile_meta = reinterpret_cast<int4 *>(scratch + o_tmeta);
  long long *tile_base = reinterpret_cast<long long *>(scratch + o_tbase);
  e = cudaMemsetAsync(scratch, 0, head, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(scratch + o_done, 0, o_tmeta - o_done, st);
  p.hist = hist;
  p.tiles = tiles;
  p.order = order;
  p.tile_meta = tile_meta;
  p.tile_base = tile_base;
  {
    auto al = [](const void *q) { return (reinterpret_cast<uintptr_t>(q) & 15u) == 0; };
    p.vec16 = al(p.a) && al(p.b) && al(p.c) && al(p.d);
  }
  p.tile_rows = reinterpret_cast<R *>(scratch + o_trows);
  p.tile_fl = reinterpret_cast<R *>(scratch + o_tfl);
  p.sys_done = done;
  p.sys_ready = ready;
  p.max_tiles = max_tiles;
  p.nelems = given;
  p.counter = counter;
  p.error = error;
  {
    const unsigned long long lim = g_wait_polls.load(std::memory_order_relaxed);
    p.wait_limit = lim == 0 ? kWaitLimit : (unsigned)(lim > 0xffffffffULL ? 0xffffffffULL : lim);
    p.withhold = g_withhold.load(std::memory_order_relaxed) != 0;
  }
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess) {
    const long long g = (p.nsys + 255) / 256;
    const unsigned grid = (unsigned)(g < 4LL * sms ? (g > 0 ? g : 1) : 4LL * sms);
    ragged_hist_kernel<R><<<grid, 256, 0, st>>>(p, hist, tiles);
    ragged_order_kernel<R><<<grid, 256, 0, st>>>(p, hist, tiles, fill, tfill, order, tile_meta,
                                                 tile_base);
    g_launches.fetch_add(2, std::memory_order_relaxed);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) {
    // (73.7 KB: three CTAs per SM, 3 x 128 TMEM columns)
    const size_t smem = (size_t)(kRaggedThreads / 32) * RTileBuf<R>::ELEMS * sizeof(R);
    e = cudaFuncSetAttribute(ragged_kernel<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    // CTAs per SM from the shared memory, registers and TMEM columns a CTA
    // takes (the runtime's occupancy query answers one CTA per SM for this
    // kernel, counting it as if it held all 512 TMEM columns)
    int per_sm = ragged_ctas_per_sm(dev, ragged_kernel<R>, smem, ragged_tmem_cols<R>());
    // every CTA resident at once (the waits rely on running warps only)
    if (e == cudaSuccess) ragged_kernel<R><<<(unsigned)(sms * per_sm), kRaggedThreads, smem, st>>>(p);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    e = cudaGetLastError();
  }
  // errors recorded by the kernel can only be read back when the call blocks
  if (e == cudaSuccess && settings().blocking) {
    unsigned h = 0;
    e = cudaMemcpyAsync(&h, error, sizeof(h), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e == cudaSuccess && h == 1u) e = cudaErrorNotSupported;
    if (e == cudaSuccess && h == 3u) e = cudaErrorInvalidValue;
    if (e == cudaSuccess && h >= 2u) e = cudaErrorLaunchFailure;
  }
  cudaError_t ef = scratch_free(scratch, st);
  return e != cudaSuccess ? e : ef;
}

template <typename R>
static tridStatus_t ragged(const R *a, const R *b, const R *c, R *d, const int64_t *offsets,
                           long long nsys, long long nelems) {
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
  if (!tuned_table(pi, dev, mt)) default_mtab<R>(mt);
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
  cudaError_t e = launch_ragged<R>(p, mt, nelems, cfg.stream);
  if (e == cudaErrorNotSupported) return TRID_STATUS_MATRIX_TYPE_NOT_SUPPORTED;
  if (e == cudaErrorInvalidValue) return TRID_STATUS_INVALID_VALUE;
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
// choice that holds the class (32*M >= 2^class) and the staged 512-row tile
// (table entry 0) on a uniform batch of that class, and keeps the fastest.
// Longer classes always take tiles.
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
    for (int m = 0; m <= 8; m = m ? 2 * m : 1) {
      if (m > 0 && 32LL * m < len) continue;
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
        cudaError_t e = launch_ragged<R>(p, trial, nsys * len, st);
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
    set_tuned_table(sizeof(R) == 8 ? 0 : 1, dev, mt);
  }
  return status;
}

}  // namespace trid

using namespace trid;

EXTERN_C tridStatus_t tridDmtsvRaggedBatch(const TridParams *ctx, const double *a, const double *b,
                                           const double *c, double *d, const int64_t *offsets,
                                           long long nsys) {
  const TraceScope trace("tridDmtsvRaggedBatch");
  (void)ctx;
  return ragged<double>(a, b, c, d, offsets, nsys, -1);
}

EXTERN_C tridStatus_t tridSmtsvRaggedBatch(const TridParams *ctx, const float *a, const float *b,
                                           const float *c, float *d, const int64_t *offsets,
                                           long long nsys) {
  const TraceScope trace("tridSmtsvRaggedBatch");
  (void)ctx;
  return ragged<float>(a, b, c, d, offsets, nsys, -1);
}

EXTERN_C tridStatus_t tridDmtsvRaggedBatchSized(const TridParams *ctx, const double *a,
                                                const double *b, const double *c, double *d,
                                                const int64_t *offsets, long long nsys,
                                                long long nelems) {
  const TraceScope trace("tridDmtsvRaggedBatchSized");
  (void)ctx;
  if (nelems < 0) return TRID_STATUS_INVALID_VALUE;
  return ragged<double>(a, b, c, d, offsets, nsys, nelems);
}

EXTERN_C tridStatus_t tridSmtsvRaggedBatchSized(const TridParams *ctx, const float *a,
                                                const float *b, const float *c, float *d,
                                                const int64_t *offsets, long long nsys,
                                                long long nelems) {
  const TraceScope trace("tridSmtsvRaggedBatchSized");
  (void)ctx;
  if (nelems < 0) return TRID_STATUS_INVALID_VALUE;
  return ragged<float>(a, b, c, d, offsets, nsys, nelems);
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
  if (!tuned_table(pi, dev, mt)) {
    if (pi == 0)
      default_mtab<double>(mt);
    else
      default_mtab<float>(mt);
  }
  const int warp_max = pi == 0 ? ragged_warp_max<double>() : ragged_warp_max<float>();
  int n = 0;
  for (int cls = 0; cls < kClasses && (1 << cls) <= warp_max; ++cls) {
    if (rows_per_lane && cls < nclasses) rows_per_lane[cls] = mt[cls];
    n = cls + 1;
  }
  return n;
}

EXTERN_C tridStatus_t tridRaggedSetWaitBound(unsigned long long polls, int withhold_publish) {
  g_wait_polls.store(polls, std::memory_order_relaxed);
  g_withhold.store(withhold_publish != 0, std::memory_order_relaxed);
  return TRID_STATUS_SUCCESS;
}
