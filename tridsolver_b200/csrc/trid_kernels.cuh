// Kernel templates of the batched tridiagonal solve.
//
// A batch is described by BatchArgs: system s = i0 + n0*i1 starts at element
// i0*st0 + i1*st1 and its rows are `stride` elements apart. The strided-batch
// API maps onto it as (p = pads):
//   solvedim 0:  i0 = y, i1 = z,  st0 = p0, st1 = p0*p1, stride = 1
//   solvedim 1:  i0 = x, i1 = z,  st0 = 1,  st1 = p0*p1, stride = p0
//   solvedim 2:  i0 = x, i1 = y,  st0 = 1,  st1 = p0,    stride = p0*p1
// (the reference's index arithmetic, scalar/src/cpu/trid_cpu.cpp:369-454).
//
// Families (all keep each element in registers between one read and one
// write of HBM; see trid_device.cuh for the algorithm):
//   contig_kernel   stride == 1: T consecutive lanes own the T chunks of one
//                   system, so the reduced solve is all warp shuffles and the
//                   M rows of a lane are contiguous (16-byte vector loads when
//                   aligned).
//   strided_kernel  stride > 1: a block is W neighbouring systems x T chunks
//                   with the system index fastest, so every warp load reads
//                   W contiguous elements of one row; the reduced rows are
//                   re-dealt through shared memory so each system's T chunks
//                   land in one warp segment for the shuffle solve.
//   pcr_kernel      M = 1: one row per lane, pure PCR (systems <= 32 rows).
//   long_*_kernel   systems longer than one warp can hold: chunk
//                   elimination writes two reduced rows per chunk to scratch,
//                   the reduced batch is solved recursively as a contiguous
//                   batch, then every chunk is eliminated again from its inputs
//                   and substituted.
#pragma once

#include "trid_device.cuh"

namespace trid {

template <typename R> struct BatchArgs {
  const R *a, *b, *c;
  const R *d_in;  // right-hand side (== d_out unless INC)
  R *d_out;       // x is written here when !INC
  R *u;           // u += x when INC
  int N;          // rows per system
  long long nsys;
  long long n0;   // systems along the fastest enumerating dimension
  long long st0, st1, stride;
  unsigned *flag;  // host-mapped zero-pivot word (may be null)
};

// Coefficient arrays in a storage type of their own (FP32 coefficients of an
// FP64 solve).
template <typename CR> struct CoefPtrs {
  const CR *a, *b, *c;
};

// Constant coefficients of one ADI heat timestep, read on the device:
// lambda = lam[*step] (lam[0] when step is null) and, on interior rows of
// systems through the grid's interior,
//     a = c = -alpha * lambda,  b = 1 + 2 * alpha * lambda;
// identity rows (a = c = 0, b = 1) everywhere else (the coefficient arrays
// of apps/adi/src/preproc.cu:40-90, as three scalars and a boundary test).
template <typename R> struct ConstCoef {
  const R *lam;
  const int *step;
  R alpha;
};

template <typename R>
__device__ __forceinline__ void const_coef(const ConstCoef<R> &k, R &l, R &ca, R &cb) {
  l = k.lam[k.step ? *k.step : 0];
  ca = -k.alpha * l;
  cb = R(1) + R(2) * k.alpha * l;
}

template <typename R>
__device__ __forceinline__ long long sys_base(const BatchArgs<R> &p, long long s) {
  long long i1 = s / p.n0;
  long long i0 = s - i1 * p.n0;
  return i0 * p.st0 + i1 * p.st1;
}

// Loads chunk rows [row0, row0+M) of a system starting at `base` into
// registers, identity rows past N, a[0] and c[N-1] forced to zero.
template <typename R, int M, bool VEC>
__device__ __forceinline__ void load_chunk(const BatchArgs<R> &p, long long base, int row0,
                                           bool active, R (&ra)[M], R (&rb)[M], R (&rc)[M],
                                           R (&rd)[M]) {
  const int N = p.N;
  if (VEC && active && row0 + M <= N) {
    const long long o = base + row0;  // stride == 1 for VEC
    load_vec<R, M>(p.a + o, ra);
    load_vec<R, M>(p.b + o, rb);
    load_vec<R, M>(p.c + o, rc);
    load_vec<R, M>(p.d_in + o, rd);
  } else {
#pragma unroll
    for (int i = 0; i < M; ++i) {
      const int row = row0 + i;
      if (active && row < N) {
        const long long o = base + (long long)row * p.stride;
        ra[i] = __ldg(p.a + o);
        rb[i] = __ldg(p.b + o);
        rc[i] = __ldg(p.c + o);
        rd[i] = __ldg(p.d_in + o);
      } else {
        ra[i] = R(0);
        rb[i] = R(1);
        rc[i] = R(0);
        rd[i] = R(0);
      }
    }
  }
  if (row0 == 0) ra[0] = R(0);
#pragma unroll
  for (int i = 0; i < M; ++i)
    if (row0 + i == N - 1) rc[i] = R(0);
}

// Loads u at rows [row0, row0+M) for the Inc variants, with the inputs, so
// its latency overlaps the solve (zero past the system end).
template <typename R, int M, bool VEC>
__device__ __forceinline__ void load_u(const BatchArgs<R> &p, long long base, int row0, bool active,
                                       R (&uu)[M]) {
  const int N = p.N;
  if (VEC && active && row0 + M <= N) {
    load_vec<R, M>(p.u + base + row0, uu);
  } else {
#pragma unroll
    for (int i = 0; i < M; ++i) {
      const int row = row0 + i;
      uu[i] = (active && row < N) ? p.u[base + (long long)row * p.stride] : R(0);
    }
  }
}

// Writes u + x for rows [row0, row0+M) inside the system (Inc variants,
// u loaded beforehand by load_u).
template <typename R, int M, bool VEC>
__device__ __forceinline__ void store_inc(const BatchArgs<R> &p, long long base, int row0,
                                          bool active, const R (&uu)[M], const R (&x)[M]) {
  if (!active) return;
  const int N = p.N;
  R v[M];
#pragma unroll
  for (int i = 0; i < M; ++i) v[i] = uu[i] + x[i];
  if (VEC && row0 + M <= N) {
    store_vec<R, M>(p.u + base + row0, v);
  } else {
#pragma unroll
    for (int i = 0; i < M; ++i) {
      const int row = row0 + i;
      if (row < N) p.u[base + (long long)row * p.stride] = v[i];
    }
  }
}

// Writes x (in rd) for rows [row0, row0+M) that lie inside the system.
template <typename R, int M, bool INC, bool VEC>
__device__ __forceinline__ void store_chunk(const BatchArgs<R> &p, long long base, int row0,
                                            bool active, const R (&x)[M]) {
  if (!active) return;
  const int N = p.N;
  if (VEC && row0 + M <= N) {
    const long long o = base + row0;
    if (INC) {
      R uu[M];
      load_vec<R, M>(p.u + o, uu);
#pragma unroll
      for (int i = 0; i < M; ++i) uu[i] += x[i];
      store_vec<R, M>(p.u + o, uu);
    } else {
      store_vec<R, M>(p.d_out + o, x);
    }
  } else {
#pragma unroll
    for (int i = 0; i < M; ++i) {
      const int row = row0 + i;
      if (row < N) {
        const long long o = base + (long long)row * p.stride;
        if (INC)
          p.u[o] += x[i];
        else
          p.d_out[o] = x[i];
      }
    }
  }
}

// ---------------------------------------------------------------------------
// contig_kernel: stride == 1, T lanes per system (T | 32), 32/T systems per
// warp. Block size is a multiple of 32.
template <typename R, int M, bool INC, bool VEC>
__global__ void __launch_bounds__(128) contig_kernel(const BatchArgs<R> p, int T) {
  const int t = threadIdx.x & (T - 1);
  const long long gtid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long s = gtid / T;
  const bool active = s < p.nsys;
  const long long base = active ? sys_base(p, s) : 0;
  const int row0 = t * M;
  R ra[M], rb[M], rc[M], rd[M];
  load_chunk<R, M, VEC>(p, base, row0, active, ra, rb, rc, rd);
  R uu[INC ? M : 1];
  if constexpr (INC) load_u<R, M, VEC>(p, base, row0, active, uu);
  bool bad = false;
  chunk_forward<R, M>(ra, rb, rc, rd, bad);
  chunk_backward<R, M>(ra, rc, rd, bad);
  Row<R> top{ra[0], rc[0], rd[0]};
  Row<R> bot{ra[M - 1], rc[M - 1], rd[M - 1]};
  R y, z;
  reduced_solve<R>(top, bot, t, T, y, z, bad);
  chunk_substitute<R, M>(ra, rc, rd, y, z);
  if constexpr (INC)
    store_inc<R, M, VEC>(p, base, row0, active, uu, rd);
  else
    store_chunk<R, M, false, VEC>(p, base, row0, active, rd);
  report_bad_pivot(bad && active, p.flag);
}

// ---------------------------------------------------------------------------
// contig_smem_kernel: stride == 1, one warp per system (T = 32), 16-byte
// aligned systems. The warp stages its system through shared memory: the
// copies are coalesced 16-byte cp.async units (512 contiguous bytes per warp
// instruction), and each lane then reads its own chunk row from a padded
// layout (one spare 16-byte unit per chunk row, so the 16-byte reads of eight
// neighbouring lanes hit eight different bank groups). The result goes back
// the same way. Direct per-lane chunk loads instead make every warp load
// touch 32 separate lines and saturate L1.
template <typename R, int M> struct SmemLayout {
  static constexpr int V = 16 / (int)sizeof(R);  // elements per 16-byte unit
  static constexpr int ROW = M + V;              // padded chunk row, elements
  static constexpr int BUF = 32 * ROW;           // one array of one system
};

// Stores M elements of a padded shared-memory chunk row as 16-byte units.
template <typename R, int M>
__device__ __forceinline__ void sts_row(R *row, const R (&v)[M]) {
  using Vt = typename Vec16<R>::T;
  constexpr int n = Vec16<R>::n;
  Vt *q = reinterpret_cast<Vt *>(row);
#pragma unroll
  for (int i = 0; i < M / n; ++i) {
    Vt x;
    if constexpr (n == 2) {
      x.x = v[2 * i];
      x.y = v[2 * i + 1];
    } else {
      x.x = v[4 * i];
      x.y = v[4 * i + 1];
      x.z = v[4 * i + 2];
      x.w = v[4 * i + 3];
    }
    q[i] = x;
  }
}

template <typename R, int M>
__device__ __forceinline__ void lds_row(const R *row, R (&v)[M]) {
  using Vt = typename Vec16<R>::T;
  constexpr int n = Vec16<R>::n;
  const Vt *q = reinterpret_cast<const Vt *>(row);
#pragma unroll
  for (int i = 0; i < M / n; ++i) {
    Vt x = q[i];
    if constexpr (n == 2) {
      v[2 * i] = x.x;
      v[2 * i + 1] = x.y;
    } else {
      v[4 * i] = x.x;
      v[4 * i + 1] = x.y;
      v[4 * i + 2] = x.z;
      v[4 * i + 3] = x.w;
    }
  }
}

template <typename R, int M, bool INC>
__global__ void __launch_bounds__(128) contig_smem_kernel(const BatchArgs<R> p) {
  using L = SmemLayout<R, M>;
  using Vt = typename Vec16<R>::T;
  constexpr int V = L::V;
  constexpr int NA = INC ? 5 : 4;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R *buf = reinterpret_cast<R *>(smem_raw) + (threadIdx.x >> 5) * (NA * L::BUF);
  const int lane = threadIdx.x & 31;
  const long long s = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (s >= p.nsys) return;  // uniform per warp
  const long long base = sys_base(p, s);
  const int N = p.N;
  const int nunits = (N + V - 1) / V;
  const R *src[5] = {p.a + base, p.b + base, p.c + base, p.d_in + base,
                     INC ? p.u + base : p.d_in + base};
#pragma unroll
  for (int k = 0; k < NA; ++k) {
    for (int un = lane; un < nunits; un += 32) {
      const int e = un * V;
      const int left = N - e;
      cp_async16(buf + k * L::BUF + e + (e / M) * V, src[k] + e,
                 (left >= V ? V : left) * (int)sizeof(R));
    }
  }
  cp_async_wait_all();
  __syncwarp();

  const int row0 = lane * M;
  R ra[M], rb[M], rc[M], rd[M];
  lds_row<R, M>(buf + 0 * L::BUF + lane * L::ROW, ra);
  lds_row<R, M>(buf + 1 * L::BUF + lane * L::ROW, rb);
  lds_row<R, M>(buf + 2 * L::BUF + lane * L::ROW, rc);
  lds_row<R, M>(buf + 3 * L::BUF + lane * L::ROW, rd);
#pragma unroll
  for (int i = 0; i < M; ++i) {
    const int row = row0 + i;
    if (row >= N) {
      ra[i] = R(0);
      rb[i] = R(1);
      rc[i] = R(0);
      rd[i] = R(0);
    }
    if (row == N - 1) rc[i] = R(0);
  }
  if (lane == 0) ra[0] = R(0);
  bool bad = false;
  chunk_forward<R, M, true>(ra, rb, rc, rd, bad);
  chunk_backward<R, M, true>(ra, rc, rd, bad);
  Row<R> top{ra[0], rc[0], rd[0]};
  Row<R> bot{ra[M - 1], rc[M - 1], rd[M - 1]};
  R y, z;
  reduced_solve<R>(top, bot, lane, 32, y, z, bad);
  chunk_substitute<R, M>(ra, rc, rd, y, z);
  // each lane overwrites only its own row of the `a` buffer
  {
    Vt *q = reinterpret_cast<Vt *>(buf + lane * L::ROW);
#pragma unroll
    for (int i = 0; i < M / V; ++i) {
      Vt x;
      if constexpr (V == 2) {
        x.x = rd[2 * i];
        x.y = rd[2 * i + 1];
      } else {
        x.x = rd[4 * i];
        x.y = rd[4 * i + 1];
        x.z = rd[4 * i + 2];
        x.w = rd[4 * i + 3];
      }
      q[i] = x;
    }
  }
  __syncwarp();
  R *dst = INC ? p.u + base : p.d_out + base;
  for (int un = lane; un < nunits; un += 32) {
    const int e = un * V;
    const int idx = e + (e / M) * V;
    Vt x = *reinterpret_cast<const Vt *>(buf + idx);
    if (INC) {
      const Vt uo = *reinterpret_cast<const Vt *>(buf + 4 * L::BUF + idx);
      if constexpr (V == 2) {
        x.x += uo.x;
        x.y += uo.y;
      } else {
        x.x += uo.x;
        x.y += uo.y;
        x.z += uo.z;
        x.w += uo.w;
      }
    }
    if (e + V <= N) {
      *reinterpret_cast<Vt *>(dst + e) = x;
    } else {
      const R *xs = reinterpret_cast<const R *>(&x);
      for (int i = 0; i < N - e; ++i) dst[e + i] = xs[i];
    }
  }
  report_bad_pivot(bad, p.flag);
}

// ---------------------------------------------------------------------------
// Block-level reduced solve for W systems x T chunks, thread (s, t) =
// (tid % W, tid / W). The reduced rows go to shared memory, slot (t, s) at
// t*(W+1)+s, and are dealt again so that one system's 2T reduced rows sit in
// one warp:
//   KR == 2 (T <= 32): T consecutive lanes, two rows (top, bottom) each, solved
//                      by reduced_solve over a T-lane segment;
//   KR >= 4 (T = 16*KR): one warp per system, KR consecutive reduced rows per
//                      lane, eliminated locally as a chunk of KR rows before
//                      the 32-lane reduced_solve.
// Returns the first (y) and last (z) unknown of the thread's chunk. `sm` holds
// 6*T*(W+1) values; every thread of the block must call this.
template <typename R, int KR>
__device__ __forceinline__ void block_reduced_solve(R *sm, const Row<R> &top, const Row<R> &bot,
                                                    int s, int t, int T, int W, R &y, R &z,
                                                    bool &bad) {
  const int tid = threadIdx.x;
  const int ld = W + 1;
  const int nslot = T * ld;
  __syncthreads();  // the previous use of sm is over
  {
    const int k = t * ld + s;
    sm[0 * nslot + k] = top.A;
    sm[1 * nslot + k] = top.C;
    sm[2 * nslot + k] = top.D;
    sm[3 * nslot + k] = bot.A;
    sm[4 * nslot + k] = bot.C;
    sm[5 * nslot + k] = bot.D;
  }
  __syncthreads();
  if constexpr (KR == 2) {
    const int s2 = tid / T;
    const int t2 = tid & (T - 1);
    const int k = t2 * ld + s2;
    Row<R> tp{sm[0 * nslot + k], sm[1 * nslot + k], sm[2 * nslot + k]};
    Row<R> bt{sm[3 * nslot + k], sm[4 * nslot + k], sm[5 * nslot + k]};
    R yy, zz;
    reduced_solve<R>(tp, bt, t2, T, yy, zz, bad);
    // slot k is read and rewritten by this thread only
    sm[0 * nslot + k] = yy;
    sm[1 * nslot + k] = zz;
  } else {
    const int w = tid >> 5;
    const int l = tid & 31;
    if (w < W) {  // warp w solves the reduced system of system w
      R qa[KR], qb[KR], qc[KR], qd[KR];
#pragma unroll
      for (int j = 0; j < KR / 2; ++j) {
        const int k = (l * (KR / 2) + j) * ld + w;
        qa[2 * j] = sm[0 * nslot + k];
        qc[2 * j] = sm[1 * nslot + k];
        qd[2 * j] = sm[2 * nslot + k];
        qa[2 * j + 1] = sm[3 * nslot + k];
        qc[2 * j + 1] = sm[4 * nslot + k];
        qd[2 * j + 1] = sm[5 * nslot + k];
        qb[2 * j] = R(1);
        qb[2 * j + 1] = R(1);
      }
      chunk_forward<R, KR>(qa, qb, qc, qd, bad);
      chunk_backward<R, KR>(qa, qc, qd, bad);
      Row<R> tp{qa[0], qc[0], qd[0]};
      Row<R> bt{qa[KR - 1], qc[KR - 1], qd[KR - 1]};
      R yy, zz;
      reduced_solve<R>(tp, bt, l, 32, yy, zz, bad);
      chunk_substitute<R, KR>(qa, qc, qd, yy, zz);
#pragma unroll
      for (int j = 0; j < KR / 2; ++j) {
        const int k = (l * (KR / 2) + j) * ld + w;
        sm[0 * nslot + k] = qd[2 * j];
        sm[1 * nslot + k] = qd[2 * j + 1];
      }
    }
  }
  __syncthreads();
  const int k = t * ld + s;
  y = sm[0 * nslot + k];
  z = sm[1 * nslot + k];
}

// ---------------------------------------------------------------------------
// strided_kernel: block = W systems (neighbouring i0) x T chunks, thread
// (s, t) = (tid % W, tid / W). W*T is a multiple of 32.
template <typename R, int M, int KR, bool INC>
__global__ void __launch_bounds__((KR >= 4 || M * sizeof(R) <= 64) ? 512 : 256)
    strided_kernel(const BatchArgs<R> p, int T, int W, long long ngx) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R *sm = reinterpret_cast<R *>(smem_raw);
  const int tid = threadIdx.x;
  const int s = tid % W;
  const int t = tid / W;
  const long long gx = blockIdx.x % ngx;
  const long long i1 = blockIdx.x / ngx;
  const long long i0 = gx * W + s;
  const bool active = i0 < p.n0;
  const long long base = i0 * p.st0 + i1 * p.st1;
  const int row0 = t * M;
  R ra[M], rb[M], rc[M], rd[M];
  load_chunk<R, M, false>(p, base, row0, active, ra, rb, rc, rd);
  R uu[INC ? M : 1];
  if constexpr (INC) load_u<R, M, false>(p, base, row0, active, uu);
  bool bad = false;
  chunk_forward<R, M>(ra, rb, rc, rd, bad);
  chunk_backward<R, M>(ra, rc, rd, bad);
  R y, z;
  block_reduced_solve<R, KR>(sm, Row<R>{ra[0], rc[0], rd[0]}, Row<R>{ra[M - 1], rc[M - 1], rd[M - 1]},
                             s, t, T, W, y, z, bad);
  chunk_substitute<R, M>(ra, rc, rd, y, z);
  if constexpr (INC)
    store_inc<R, M, false>(p, base, row0, active, uu, rd);
  else
    store_chunk<R, M, false, false>(p, base, row0, active, rd);
  report_bad_pivot(bad && active, p.flag);
}

// ---------------------------------------------------------------------------
// pcr_kernel: one row per lane, T lanes per system (N <= T <= 32). For
// stride == 1 the lanes of a system read consecutive elements; for strided
// batches the lane order is still row-major inside the system, which is the
// right trade only for short systems.
template <typename R, bool INC>
__global__ void __launch_bounds__(128) pcr_kernel(const BatchArgs<R> p, int T) {
  const int t = threadIdx.x & (T - 1);
  const long long gtid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long s = gtid / T;
  const bool active = s < p.nsys && t < p.N;
  const long long o = (s < p.nsys ? sys_base(p, s) : 0) + (long long)t * p.stride;
  R a = R(0), b = R(1), c = R(0), d = R(0);
  if (active) {
    a = t == 0 ? R(0) : __ldg(p.a + o);
    b = __ldg(p.b + o);
    c = t == p.N - 1 ? R(0) : __ldg(p.c + o);
    d = __ldg(p.d_in + o);
  }
  bool bad = false;
  R x = pcr_solve<R>(a, b, c, d, t, T, bad);
  if (active) {
    if (INC)
      p.u[o] += x;
    else
      p.d_out[o] = x;
  }
  report_bad_pivot(bad && active, p.flag);
}

// ---------------------------------------------------------------------------
// Long systems. Work item = (system, chunk); for stride == 1 the chunk index
// is fastest (neighbouring lanes read neighbouring chunks), otherwise i0 is
// fastest (neighbouring lanes read neighbouring systems, coalesced).
// Reduced system of system s: rows [s*2nc, s*2nc + 2nc) of ra/rb/rc/rd.
template <typename R>
__device__ __forceinline__ void long_item(const BatchArgs<R> &p, long long item, long long nc,
                                          long long &s, long long &chunk) {
  if (p.stride == 1) {
    s = item / nc;
    chunk = item - s * nc;
  } else {
    const long long i0 = item % p.n0;
    const long long rem = item / p.n0;
    chunk = rem % nc;
    s = i0 + p.n0 * (rem / nc);
  }
}

template <typename R, int M>
__global__ void __launch_bounds__(128) long_reduce_kernel(const BatchArgs<R> p, long long nc,
                                                          R *__restrict__ ra, R *__restrict__ rb,
                                                          R *__restrict__ rc,
                                                          R *__restrict__ rd) {
  const long long item = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (item >= p.nsys * nc) return;
  long long s, chunk;
  long_item(p, item, nc, s, chunk);
  const long long base = sys_base(p, s);
  const int row0 = (int)(chunk * M);
  R a[M], b[M], c[M], d[M];
  load_chunk<R, M, false>(p, base, row0, true, a, b, c, d);
  bool bad = false;
  chunk_forward<R, M>(a, b, c, d, bad);
  chunk_backward<R, M>(a, c, d, bad);
  const long long o = s * 2 * nc + 2 * chunk;
  ra[o] = a[0];
  rb[o] = R(1);
  rc[o] = c[0];
  rd[o] = d[0];
  ra[o + 1] = a[M - 1];
  rb[o + 1] = R(1);
  rc[o + 1] = c[M - 1];
  rd[o + 1] = d[M - 1];
  report_bad_pivot(bad, p.flag);
}

template <typename R, int M, bool INC>
__global__ void __launch_bounds__(128) long_substitute_kernel(const BatchArgs<R> p, long long nc,
                                                              const R *__restrict__ xr) {
  const long long item = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (item >= p.nsys * nc) return;
  long long s, chunk;
  long_item(p, item, nc, s, chunk);
  const long long base = sys_base(p, s);
  const int row0 = (int)(chunk * M);
  R a[M], b[M], c[M], d[M];
  load_chunk<R, M, false>(p, base, row0, true, a, b, c, d);
  bool bad = false;
  chunk_forward<R, M>(a, b, c, d, bad);
  chunk_backward<R, M>(a, c, d, bad);
  const long long o = s * 2 * nc + 2 * chunk;
  chunk_substitute<R, M>(a, c, d, xr[o], xr[o + 1]);
  store_chunk<R, M, INC, false>(p, base, row0, true, d);
}

}  // namespace trid
