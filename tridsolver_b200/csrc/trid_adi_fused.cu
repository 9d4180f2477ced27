// Solves of the fused ADI timestep: constant coefficients, factored once.
//
// In an ADI heat timestep (apps/adi/src/adi_cuda.cu:282-326) every system
// through the grid's interior has the same matrix: a = c = -alpha lambda and
// b = 1 + 2 alpha lambda on its interior rows, identity rows at both ends.
// Systems off the interior are identity systems with a zero right-hand side.
// So the elimination coefficients of the partition method (the reciprocal
// pivots and the scaled off-diagonals of every chunk, and those of the
// reduced system's cyclic reduction) depend only on the position of a chunk
// in its system, not on the system. Each CTA computes them once at the start
// (one warp, one lane per chunk position, the same arithmetic as the
// coefficient-array kernels) into shared-memory tables, and every system
// after that only sweeps its right-hand side: a multiply-add and a multiply
// per row forward, one multiply-add per row backward, two in the
// substitution, no reciprocals. Identity systems off the interior are
// neither read nor written (their solution is their zero right-hand side).
//
// Because the right-hand-side arithmetic is the array kernels' operation for
// operation, the results equal the coefficient-array timestep's where both
// use the same chunking:
//   adi_x_kernel      mirrors contig_smem_kernel (chunk_forward,
//                     chunk_backward, reduced_solve, chunk_substitute), with
//                     the 7-point stencil formed while the line is staged;
//   adi_stream_kernel mirrors strided_stream_kernel (forward sweep, one-row
//                     backward recursion, block-wide reduced solve,
//                     back-substitution from the forward rows).
#include <cuda_runtime.h>

#include "trid_internal.h"

namespace trid {

namespace {

constexpr int kT = 32;      // chunks per system (one warp of reduced rows)
constexpr int kSteps = 5;   // cyclic-reduction steps over 32 reduced rows

// Coefficients of the reduced system's solve (reduced_solve) by lane = chunk.
template <typename R> struct PcrTab {
  R tA[kT], tC[kT], bA[kT], bC[kT], ri[kT];
  R al[kSteps][kT], ga[kSteps][kT], rs[kSteps][kT];
};

// The coefficient half of reduced_solve for the chunk rows of lane t:
// top row A x_prev + x + C x_last, bottom row A x_first + x + C x_next.
// Every lane of the warp calls this.
template <typename R>
__device__ void pcr_factor(PcrTab<R> &q, R tA, R tC, R bA, R bC, int t, bool &bad) {
  q.tA[t] = tA;
  q.tC[t] = tC;
  q.bA[t] = bA;
  q.bC[t] = bC;
  R pA = shfl_up(bA, 1, kT);
  R pC = shfl_up(bC, 1, kT);
  if (t == 0) {
    pA = R(0);
    pC = R(0);
  }
  R al = -tA * pA;
  R be = R(1) - tA * pC - tC * bA;
  R ga = -tC * bC;
  R r = rcp(be);
  bad |= !finite_rcp(r);
  q.ri[t] = r;
  al *= r;
  ga *= r;
  int k = 0;
#pragma unroll
  for (int s = 1; s < kT; s <<= 1, ++k) {
    R al_l = shfl_up(al, s, kT), ga_l = shfl_up(ga, s, kT);
    R al_r = shfl_down(al, s, kT), ga_r = shfl_down(ga, s, kT);
    if (t < s) {
      al_l = R(0);
      ga_l = R(0);
    }
    if (t + s >= kT) {
      al_r = R(0);
      ga_r = R(0);
    }
    q.al[k][t] = al;
    q.ga[k][t] = ga;
    R b2 = R(1) - al * ga_l - ga * al_r;
    R a2 = -al * al_l;
    R g2 = -ga * ga_r;
    r = rcp(b2);
    bad |= !finite_rcp(r);
    q.rs[k][t] = r;
    al = a2 * r;
    ga = g2 * r;
  }
}

// The right-hand-side half of reduced_solve: lane t holds the D parts of
// its chunk's top and bottom reduced rows and gets the chunk's first (y) and
// last (z) unknowns. Every lane of the warp calls this.
template <typename R>
__device__ __forceinline__ void pcr_solve_d(const PcrTab<R> &q, R tD, R bD, int t, R &y, R &z) {
  R pD = shfl_up(bD, 1, kT);
  if (t == 0) pD = R(0);
  R de = tD - q.tA[t] * pD - q.tC[t] * bD;
  de *= q.ri[t];
  int k = 0;
#pragma unroll
  for (int s = 1; s < kT; s <<= 1, ++k) {
    R de_l = shfl_up(de, s, kT), de_r = shfl_down(de, s, kT);
    if (t < s) de_l = R(0);
    if (t + s >= kT) de_r = R(0);
    R d2 = de - q.al[k][t] * de_l - q.ga[k][t] * de_r;
    de = d2 * q.rs[k][t];
  }
  y = de;
  R yn = shfl_down(y, 1, kT);
  if (t == kT - 1) yn = R(0);
  z = bD - q.bA[t] * y - q.bC[t] * yn;
}

// Row `row` of a system of N rows: interior rows carry the constant
// coefficients, the first and last rows and rows past N are identity rows.
template <typename R>
__device__ __forceinline__ void cc_row(int row, int N, R ca, R cb, R &a, R &b) {
  const bool in = row >= 1 && row <= N - 2;
  a = in ? ca : R(0);
  b = in ? cb : R(1);
}

// ---- contiguous form (chunk_forward / chunk_backward / chunk_substitute) ----

template <typename R, int M> struct ContigTab {
  R r[M][kT];   // forward reciprocal pivots
  R ao[M][kT];  // unscaled sub-diagonal
  R cF[M][kT];  // super-diagonal after the forward half
  R aB[M][kT];  // after the backward half
  R cB[M][kT];
  R rb[kT];     // reciprocal of the backward half's top-row pivot
  PcrTab<R> pcr;
};

template <typename R, int M>
__device__ void contig_factor(ContigTab<R, M> &f, R ca, R cb, int N, int t, bool &bad) {
  R a[M], b[M], c[M];
#pragma unroll
  for (int i = 0; i < M; ++i) {
    cc_row<R>(t * M + i, N, ca, cb, a[i], b[i]);
    c[i] = a[i];
    f.ao[i][t] = a[i];
  }
#pragma unroll
  for (int i = 0; i < (M < 2 ? M : 2); ++i) {
    R r = rcp(b[i]);
    bad |= !finite_rcp(r);
    f.r[i][t] = r;
    a[i] *= r;
    c[i] *= r;
  }
#pragma unroll
  for (int i = 2; i < M; ++i) {
    R r = rcp(b[i] - a[i] * c[i - 1]);
    bad |= !finite_rcp(r);
    f.r[i][t] = r;
    a[i] = -r * a[i] * a[i - 1];
    c[i] = r * c[i];
  }
#pragma unroll
  for (int i = 0; i < M; ++i) f.cF[i][t] = c[i];
#pragma unroll
  for (int i = M - 3; i >= 1; --i) {
    a[i] = a[i] - c[i] * a[i + 1];
    c[i] = -c[i] * c[i + 1];
  }
  R rb = R(1);
  if (M >= 3) {
    rb = rcp(R(1) - c[0] * a[1]);
    bad |= !finite_rcp(rb);
    a[0] = rb * a[0];
    c[0] = -rb * c[0] * c[1];
  }
  f.rb[t] = rb;
#pragma unroll
  for (int i = 0; i < M; ++i) {
    f.aB[i][t] = a[i];
    f.cB[i][t] = c[i];
  }
  pcr_factor<R>(f.pcr, a[0], c[0], a[M - 1], c[M - 1], t, bad);
}

// x solve of one line held by a warp (lane t = chunk t), in place in d.
template <typename R, int M>
__device__ __forceinline__ void contig_solve_d(const ContigTab<R, M> &f, R (&d)[M], int t) {
#pragma unroll
  for (int i = 0; i < (M < 2 ? M : 2); ++i) d[i] *= f.r[i][t];
#pragma unroll
  for (int i = 2; i < M; ++i) d[i] = f.r[i][t] * (d[i] - f.ao[i][t] * d[i - 1]);
#pragma unroll
  for (int i = M - 3; i >= 1; --i) d[i] = d[i] - f.cF[i][t] * d[i + 1];
  if (M >= 3) d[0] = f.rb[t] * (d[0] - f.cF[0][t] * d[1]);
  R y, z;
  pcr_solve_d<R>(f.pcr, d[0], d[M - 1], t, y, z);
#pragma unroll
  for (int i = 1; i < M - 1; ++i) d[i] = d[i] - f.aB[i][t] * y - f.cB[i][t] * z;
  d[0] = y;
  if (M > 1) d[M - 1] = z;
}

// ---- streaming form (strided_stream_kernel) --------------------------------

template <typename R, int M> struct StreamTab {
  R r[M][kT];   // forward reciprocal pivots
  R ao[M][kT];  // unscaled sub-diagonal
  R af[M][kT];  // forward a'
  R cf[M][kT];  // forward c'
  R r0[kT];     // reciprocal of the top reduced row's pivot
  PcrTab<R> pcr;
};

template <typename R, int M>
__device__ void stream_factor(StreamTab<R, M> &f, R ca, R cb, int N, int t, bool &bad) {
  R afv[M], cfv[M];
  R ap = R(0), cp = R(0);
#pragma unroll
  for (int j = 0; j < M; ++j) {
    R a, b;
    cc_row<R>(t * M + j, N, ca, cb, a, b);
    const R c = a;
    R r, af, cf;
    if (j < 2) {
      r = rcp(b);
      af = a * r;
      cf = c * r;
    } else {
      r = rcp(b - a * cp);
      af = -r * a * ap;
      cf = r * c;
    }
    bad |= !finite_rcp(r);
    f.r[j][t] = r;
    f.ao[j][t] = a;
    f.af[j][t] = af;
    f.cf[j][t] = cf;
    afv[j] = af;
    cfv[j] = cf;
    ap = af;
    cp = cf;
  }
  R A = afv[M - 2], C = cfv[M - 2];
#pragma unroll
  for (int j = M - 3; j >= 1; --j) {
    const R cj = cfv[j];
    A = afv[j] - cj * A;
    C = -cj * C;
  }
  const R a0 = afv[0], c0 = cfv[0];
  const R r0 = rcp(R(1) - c0 * A);
  bad |= !finite_rcp(r0);
  f.r0[t] = r0;
  pcr_factor<R>(f.pcr, r0 * a0, -r0 * c0 * C, ap, cp, t, bad);
}

template <typename R> constexpr int adi_w() { return 128 / (int)sizeof(R); }
template <typename R> constexpr int adi_bs() { return kT * adi_w<R>(); }

}  // namespace

// ---------------------------------------------------------------------------
// x solve with the stencil. A persistent CTA of NW warps; each warp takes x
// lines (j, k) in turn. The right-hand side of a line is formed while it is
// staged: each lane takes V-element units (16 bytes when the lines are
// 16-byte aligned) of the line and of its neighbour lines j +- 1, k +- 1
// (which the warps of those lines read too, so mostly from L2), sums the
// 7-point stencil in the order of adi_preproc_kernel and parks du in the
// warp's padded shared-memory line; lane t then reads its chunk row.
template <typename R, int M, bool VEC, int NW>
__global__ void __launch_bounds__(NW * 32) adi_x_kernel(const R *__restrict__ u, R *__restrict__ du,
                                                        const ConstCoef<R> k, unsigned *flag,
                                                        int nx, int ny, int nz) {
  using L = SmemLayout<R, M>;
  constexpr int V = VEC ? L::V : 1;
  constexpr int UPL = M / V;  // units per lane (nx <= 32 M)
  using Vt = typename Vec16<R>::T;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  ContigTab<R, M> &f = *reinterpret_cast<ContigTab<R, M> *>(smem_raw);
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  R *buf = reinterpret_cast<R *>(smem_raw + (sizeof(ContigTab<R, M>) + 15) / 16 * 16) + warp * L::BUF;
  R l, ca, cb;
  const_coef<R>(k, l, ca, cb);
  bool bad = false;
  if (warp == 0) contig_factor<R, M>(f, ca, cb, nx, lane, bad);
  __syncthreads();
  const long long nlines = (long long)ny * nz;
  const long long nxy = (long long)nx * ny;
  const int nunits = (nx + V - 1) / V;
  for (long long line = (long long)blockIdx.x * NW + warp; line < nlines;
       line += (long long)gridDim.x * NW) {
    const long long kz = line / ny;
    const long long jy = line - kz * ny;
    R *dst = du + line * nx;
    if (jy == 0 || jy == ny - 1 || kz == 0 || kz == nz - 1) {
#pragma unroll
      for (int q = 0; q < UPL; ++q) {
        const int un = lane + 32 * q;
        const int e = un * V;
        if (un >= nunits) break;
        if (VEC && e + V <= nx) {
          Vt zv;
          R *zs = reinterpret_cast<R *>(&zv);
#pragma unroll
          for (int i = 0; i < L::V; ++i) zs[i] = R(0);
          *reinterpret_cast<Vt *>(dst + e) = zv;
        } else {
          for (int i = 0; i < V && e + i < nx; ++i) dst[e + i] = R(0);
        }
      }
      continue;
    }
    const R *c0 = u + line * nx;
    const R *nb[4] = {c0 - nx, c0 + nx, c0 - nxy, c0 + nxy};
#pragma unroll
    for (int q = 0; q < UPL; ++q) {
      const int un = lane + 32 * q;
      const int e = un * V;
      if (un < nunits) {
        R cv[V], s6[V];
        if (VEC && e + V <= nx) {
          const Vt x = __ldg(reinterpret_cast<const Vt *>(c0 + e));
#pragma unroll
          for (int i = 0; i < V; ++i) cv[i] = reinterpret_cast<const R *>(&x)[i];
        } else {
#pragma unroll
          for (int i = 0; i < V; ++i) cv[i] = e + i < nx ? __ldg(c0 + e + i) : R(0);
        }
        const R left = e > 0 ? __ldg(c0 + e - 1) : R(0);
        const R right = e + V < nx ? __ldg(c0 + e + V) : R(0);
#pragma unroll
        for (int i = 0; i < V; ++i)
          s6[i] = (i == 0 ? left : cv[i - 1]) + (i == V - 1 ? right : cv[i + 1]);
#pragma unroll
        for (int n = 0; n < 4; ++n) {
          if (VEC && e + V <= nx) {
            const Vt x = __ldg(reinterpret_cast<const Vt *>(nb[n] + e));
#pragma unroll
            for (int i = 0; i < V; ++i) s6[i] = s6[i] + reinterpret_cast<const R *>(&x)[i];
          } else {
#pragma unroll
            for (int i = 0; i < V; ++i)
              if (e + i < nx) s6[i] = s6[i] + __ldg(nb[n] + e + i);
          }
        }
#pragma unroll
        for (int i = 0; i < V; ++i) {
          const int x = e + i;
          if (x < nx) buf[x + (x / M) * L::V] = (x >= 1 && x <= nx - 2) ? l * (s6[i] - R(6) * cv[i]) : R(0);
        }
      }
    }
    __syncwarp();
    R rd[M];
    lds_row<R, M>(buf + lane * L::ROW, rd);
#pragma unroll
    for (int i = 0; i < M; ++i)
      if (lane * M + i >= nx) rd[i] = R(0);
    contig_solve_d<R, M>(f, rd, lane);
    __syncwarp();  // every lane has read its row before any row is rewritten
    sts_row<R, M>(buf + lane * L::ROW, rd);
    __syncwarp();
#pragma unroll
    for (int q = 0; q < UPL; ++q) {
      const int un = lane + 32 * q;
      const int e = un * V;
      if (un >= nunits) break;
      const int idx = e + (e / M) * L::V;
      if (VEC && e + V <= nx) {
        *reinterpret_cast<Vt *>(dst + e) = *reinterpret_cast<const Vt *>(buf + idx);
      } else {
        for (int i = 0; i < V && e + i < nx; ++i) dst[e + i] = buf[idx + i];
      }
    }
    __syncwarp();  // the line buffer is free for the next line
  }
  if (warp == 0) report_bad_pivot(__any_sync(FULL_MASK, bad), flag);
}

// ---------------------------------------------------------------------------
// y and z solves: the persistent streaming layout of strided_stream_kernel
// (groups of W systems with W * sizeof(R) = 128 bytes, T = 32 chunks of M
// rows, a D-row window of loads that runs on into the next group, L2
// prefetch PF rows ahead for rows less than 64 KiB apart), sweeping only the
// right-hand side. Inc: u is carried through the window and parked in
// private shared-memory slots until the store.
template <typename R, int M, int D, int PF, bool INC>
__global__ void __launch_bounds__(adi_bs<R>(), 1)
    adi_stream_kernel(const BatchArgs<R> p, const ConstCoef<R> k, long long ngx, long long ngroups) {
  static_assert(M >= 4 && D >= 1 && D <= M && M % D == 0, "window must tile the chunk");
  static_assert(PF == 0 || (PF > D && PF <= M), "L2 prefetch runs ahead of the window");
  constexpr int W = adi_w<R>();
  constexpr int BS = W * kT;
  constexpr int RED = (2 * kT * (W + 1) * (int)sizeof(R) + 15) / 16 * 16;
  extern __shared__ __align__(16) unsigned char stream_smem[];
  R *red = reinterpret_cast<R *>(stream_smem);
  StreamTab<R, M> &f = *reinterpret_cast<StreamTab<R, M> *>(stream_smem + RED);
  R *suf = reinterpret_cast<R *>(stream_smem + RED + (sizeof(StreamTab<R, M>) + 15) / 16 * 16) +
           threadIdx.x;  // u of row j at [j * BS] (Inc)
  const int tid = threadIdx.x;
  const int s = tid % W;
  const int t = tid / W;
  const int lane = tid & 31;
  const int N = p.N;
  const int row0 = t * M;
  const long long stride = p.stride;
  const long long n1 = p.nsys / p.n0;
  bool bad = false;
  {
    R l, ca, cb;
    const_coef<R>(k, l, ca, cb);
    if (tid < 32) stream_factor<R, M>(f, ca, cb, N, lane, bad);
  }
  __syncthreads();

  // element offset of this thread's first chunk row in group g; act: an
  // interior system (others are identity systems with zero right-hand side)
  auto group_first = [&](long long g, bool &act) -> long long {
    const long long gx = g % ngx;
    const long long i1 = g / ngx;
    const long long i0 = gx * W + s;
    act = g < ngroups && i0 >= 1 && i0 <= p.n0 - 2 && i1 >= 1 && i1 <= n1 - 2;
    return act ? i0 * p.st0 + i1 * p.st1 + (long long)row0 * stride : 0;
  };

  constexpr int NA = INC ? 2 : 1;
  const bool pf_lane = PF > 0 && lane < 2 * NA * (32 / W);
  const int pq = (lane >> 1) % NA;
  const int pt = (tid >> 5) * (32 / W) + (lane >> 1) / NA;
  const R *pbase = pq == 0 ? p.d_in : p.u;
  auto pf_first = [&](long long g, bool &ok) -> long long {
    const long long gx = g % ngx;
    const long long i1 = g / ngx;
    const long long left = p.n0 - gx * W;
    const long long i0 = gx * W + ((lane & 1) ? (left < W ? left : W) - 1 : 0);
    ok = pf_lane && g < ngroups;
    return ok ? i0 * p.st0 + i1 * p.st1 + (long long)pt * M * stride : 0;
  };

  R pd[D], pu[INC ? D : 1];
  long long g = blockIdx.x;
  bool act;
  long long first = group_first(g, act);
  long long lo = first;
#pragma unroll
  for (int j = 0; j < D; ++j) {
    const bool v = act && row0 + j < N;
    pd[j] = v ? __ldg(p.d_in + lo) : R(0);
    if constexpr (INC) pu[j] = v ? __ldg(p.u + lo) : R(0);
    lo += stride;
  }
  bool pok = false;
  long long po = 0;
  if constexpr (PF > 0) po = pf_first(g, pok) + (long long)PF * stride;

  for (; g < ngroups; g += gridDim.x) {
    bool actn;
    const long long firstn = group_first(g + gridDim.x, actn);
    long long ln = firstn;
    bool pokn = false;
    long long pon = 0;
    if constexpr (PF > 0) pon = pf_first(g + gridDim.x, pokn);

    // forward sweep of the right-hand side
    R rd[M];
    R dp = R(0);
#pragma unroll
    for (int j = 0; j < M; ++j) {
      const int kk = j % D;
      const R d = pd[kk];
      if constexpr (INC) suf[j * BS] = pu[kk];
      {
        const bool nxt = j + D >= M;
        const int row = nxt ? row0 + j + D - M : row0 + j + D;
        const bool v = (nxt ? actn : act) && row < N;
        const long long o = nxt ? ln : lo;
        pd[kk] = v ? __ldg(p.d_in + o) : R(0);
        if constexpr (INC) pu[kk] = v ? __ldg(p.u + o) : R(0);
        if (nxt)
          ln += stride;
        else
          lo += stride;
      }
      if constexpr (PF > 0) {
        if (j + PF < M) {
          if (pok && pt * M + j + PF < N) asm volatile("prefetch.global.L2 [%0];\n" ::"l"(pbase + po));
          po += stride;
        } else {
          if (pokn && pt * M + j + PF - M < N) asm volatile("prefetch.global.L2 [%0];\n" ::"l"(pbase + pon));
          pon += stride;
        }
      }
      const R df = j < 2 ? d * f.r[j][t] : f.r[j][t] * (d - f.ao[j][t] * dp);
      rd[j] = df;
      dp = df;
    }
    // top reduced row: one running row from row M-2 up to row 1
    R Dd = rd[M - 2];
#pragma unroll
    for (int j = M - 3; j >= 1; --j) Dd = rd[j] - f.cf[j][t] * Dd;
    const R topD = f.r0[t] * (rd[0] - f.cf[0][t] * Dd);

    // block-wide reduced solve: re-deal the D parts so that warp w holds the
    // 32 chunks of system w, one per lane
    constexpr int ld = W + 1;
    constexpr int nslot = kT * ld;
    __syncthreads();  // the previous group's reads of red are over
    red[0 * nslot + t * ld + s] = topD;
    red[1 * nslot + t * ld + s] = dp;
    __syncthreads();
    {
      const int s2 = tid >> 5;
      const int kk = lane * ld + s2;
      R yy, zz;
      pcr_solve_d<R>(f.pcr, red[0 * nslot + kk], red[1 * nslot + kk], lane, yy, zz);
      red[0 * nslot + kk] = yy;  // slot kk is read and rewritten by this thread only
      red[1 * nslot + kk] = zz;
    }
    __syncthreads();
    const R y = red[0 * nslot + t * ld + s];
    const R z = red[1 * nslot + t * ld + s];

    // back-substitution with the forward rows, stored as it goes
    long long o = first + (long long)(M - 1) * stride;
    R x = z;
#pragma unroll
    for (int j = M - 1; j >= 0; --j) {
      if (j < M - 1) x = j == 0 ? y : rd[j] - f.af[j][t] * y - f.cf[j][t] * x;
      if (act && row0 + j < N) {
        if constexpr (INC)
          p.u[o] = suf[j * BS] + x;
        else
          p.d_out[o] = x;
      }
      o -= stride;
    }
    first = firstn;
    act = actn;
    lo = ln;
    if constexpr (PF > 0) {
      po = pon;
      pok = pokn;
    }
  }
  if (tid < 32) report_bad_pivot(__any_sync(FULL_MASK, bad), p.flag);
}

// ---------------------------------------------------------------------------
// Launchers.

template <typename R, int M, bool VEC>
static cudaError_t launch_adi_x_mv(const R *u, R *du, const ConstCoef<R> &k, unsigned *flag, int nx,
                                   int ny, int nz, cudaStream_t st) {
  constexpr int NW = 8;
  using L = SmemLayout<R, M>;
  const size_t smem = (sizeof(ContigTab<R, M>) + 15) / 16 * 16 + (size_t)NW * L::BUF * sizeof(R);
  auto kern = adi_x_kernel<R, M, VEC, NW>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int dev = 0, sms = 148, per_sm = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, NW * 32, smem) != cudaSuccess ||
      per_sm < 1)
    per_sm = 1;
  const long long lines = (long long)ny * nz;
  const long long want = (lines + NW - 1) / NW;
  const long long cap = (long long)sms * per_sm;
  const long long grid = want < cap ? want : cap;
  kern<<<(unsigned)grid, NW * 32, smem, st>>>(u, du, k, flag, nx, ny, nz);
  return cudaGetLastError();
}

template <typename R>
cudaError_t launch_adi_x(const R *u, R *du, const ConstCoef<R> &k, unsigned *flag, int nx, int ny,
                         int nz, cudaStream_t st) {
  if (nx < 1 || nx > 512 || ny < 1 || nz < 1) return cudaErrorInvalidValue;
  auto al = [](const void *q) { return (reinterpret_cast<uintptr_t>(q) & 15u) == 0; };
  const bool vec = al(u) && al(du) && (nx * (int)sizeof(R)) % 16 == 0;
  if (nx <= 256)
    return vec ? launch_adi_x_mv<R, 8, true>(u, du, k, flag, nx, ny, nz, st)
               : launch_adi_x_mv<R, 8, false>(u, du, k, flag, nx, ny, nz, st);
  return vec ? launch_adi_x_mv<R, 16, true>(u, du, k, flag, nx, ny, nz, st)
             : launch_adi_x_mv<R, 16, false>(u, du, k, flag, nx, ny, nz, st);
}

template <typename R, int M> constexpr int adi_window() { return M < 8 ? M : 8; }
template <typename R, int M> constexpr int adi_prefetch() { return adi_window<R, M>() >= M ? 0 : 12; }

template <typename R, int M, int PF, bool INC>
static cudaError_t launch_adi_stream_pf(const BatchArgs<R> &p, const ConstCoef<R> &k, cudaStream_t st) {
  constexpr int W = adi_w<R>();
  constexpr int BS = adi_bs<R>();
  constexpr int D = adi_window<R, M>();
  const size_t red = ((size_t)2 * kT * (W + 1) * sizeof(R) + 15) / 16 * 16;
  const size_t smem = red + (sizeof(StreamTab<R, M>) + 15) / 16 * 16 +
                      (INC ? (size_t)M * BS * sizeof(R) : 0);
  auto kern = adi_stream_kernel<R, M, D, PF, INC>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const long long ngx = (p.n0 + W - 1) / W;
  const long long ngroups = ngx * (p.nsys / p.n0);
  int dev = 0, sms = 148, per_sm = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, BS, smem) != cudaSuccess || per_sm < 1)
    per_sm = 1;
  const long long cap = (long long)sms * per_sm;
  const long long grid = ngroups < cap ? ngroups : cap;
  kern<<<(unsigned)grid, BS, smem, st>>>(p, k, ngx, ngroups);
  return cudaGetLastError();
}

template <typename R, int M, bool INC>
static cudaError_t launch_adi_stream_m(const BatchArgs<R> &p, const ConstCoef<R> &k, cudaStream_t st) {
  constexpr int PF = adi_prefetch<R, M>();
  if (PF > 0 && p.stride * (long long)sizeof(R) < (1LL << 16))
    return launch_adi_stream_pf<R, M, PF, INC>(p, k, st);
  return launch_adi_stream_pf<R, M, 0, INC>(p, k, st);
}

// y or z solve of the timestep: p.d_in == p.d_out == du, p.u = u for the z
// solve (INC); any 1 <= N <= 512.
template <typename R, bool INC>
cudaError_t launch_adi_yz(const BatchArgs<R> &p, const ConstCoef<R> &k, cudaStream_t st) {
  if (p.N < 1 || p.N > 512 || p.n0 < 1 || p.nsys % p.n0) return cudaErrorInvalidValue;
  if (p.nsys == 0) return cudaSuccess;
  if (p.N <= 128) return launch_adi_stream_m<R, 4, INC>(p, k, st);
  if (p.N <= 256) return launch_adi_stream_m<R, 8, INC>(p, k, st);
  return launch_adi_stream_m<R, 16, INC>(p, k, st);
}

template cudaError_t launch_adi_x<double>(const double *, double *, const ConstCoef<double> &,
                                          unsigned *, int, int, int, cudaStream_t);
template cudaError_t launch_adi_x<float>(const float *, float *, const ConstCoef<float> &, unsigned *,
                                         int, int, int, cudaStream_t);
template cudaError_t launch_adi_yz<double, false>(const BatchArgs<double> &, const ConstCoef<double> &,
                                                  cudaStream_t);
template cudaError_t launch_adi_yz<double, true>(const BatchArgs<double> &, const ConstCoef<double> &,
                                                 cudaStream_t);
template cudaError_t launch_adi_yz<float, false>(const BatchArgs<float> &, const ConstCoef<float> &,
                                                 cudaStream_t);
template cudaError_t launch_adi_yz<float, true>(const BatchArgs<float> &, const ConstCoef<float> &,
                                                cudaStream_t);

}  // namespace trid
