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
// The right-hand-side arithmetic is the array kernels' operation for
// operation, so where both use the same chunking the results agree with the
// coefficient-array timestep's to rounding (the kernels' instruction
// selection, i.e. which products fuse into multiply-adds, may differ):
//   adi_x_kernel      mirrors contig_smem_kernel (chunk_forward,
//                     chunk_backward, reduced_solve, chunk_substitute), with
//                     the 7-point stencil formed from planes of u staged in
//                     shared memory;
//   adi_stream_kernel mirrors strided_stream_kernel (forward sweep, one-row
//                     backward recursion, block-wide reduced solve,
//                     back-substitution from the forward rows).
#include <cuda_runtime.h>

#include <type_traits>

#include "trid_internal.h"

namespace trid {

namespace {

constexpr int kT = 32;  // chunks per system of the x solve (one warp of reduced rows)
// cyclic-reduction steps over T reduced rows
constexpr int pcr_steps(int T) { return T <= 1 ? 0 : 1 + pcr_steps(T / 2); }

// Two table entries read with one vector load.
template <typename R> struct alignas(2 * sizeof(R)) Pair {
  R x, y;
};

// Coefficients of the reduced system's solve (reduced_solve over T lanes)
// by lane = chunk.
template <typename R, int T = kT> struct PcrTab {
  static constexpr int kSteps = pcr_steps(T);
  Pair<R> tAC[T], bAC[T];  // (A, C) of the top and bottom reduced rows
  R ri[T];
  Pair<R> alga[kSteps][T];  // (alpha, gamma) before each step
  R rs[kSteps][T];
};

// The coefficient half of reduced_solve for the chunk rows of lane t:
// top row A x_prev + x + C x_last, bottom row A x_first + x + C x_next.
// Every lane of the warp calls this.
template <typename R, int T>
__device__ void pcr_factor(PcrTab<R, T> &q, R tA, R tC, R bA, R bC, int t, bool &bad) {
  q.tAC[t] = Pair<R>{tA, tC};
  q.bAC[t] = Pair<R>{bA, bC};
  R pA = shfl_up(bA, 1, T);
  R pC = shfl_up(bC, 1, T);
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
  for (int s = 1; s < T; s <<= 1, ++k) {
    R al_l = shfl_up(al, s, T), ga_l = shfl_up(ga, s, T);
    R al_r = shfl_down(al, s, T), ga_r = shfl_down(ga, s, T);
    if (t < s) {
      al_l = R(0);
      ga_l = R(0);
    }
    if (t + s >= T) {
      al_r = R(0);
      ga_r = R(0);
    }
    q.alga[k][t] = Pair<R>{al, ga};
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
template <typename R, int T>
__device__ __forceinline__ void pcr_solve_d(const PcrTab<R, T> &q, R tD, R bD, int t, R &y, R &z) {
  R pD = shfl_up(bD, 1, T);
  if (t == 0) pD = R(0);
  const Pair<R> tp = q.tAC[t];
  R de = tD - tp.x * pD - tp.y * bD;
  de *= q.ri[t];
  int k = 0;
#pragma unroll
  for (int s = 1; s < T; s <<= 1, ++k) {
    R de_l = shfl_up(de, s, T), de_r = shfl_down(de, s, T);
    if (t < s) de_l = R(0);
    if (t + s >= T) de_r = R(0);
    const Pair<R> ag = q.alga[k][t];
    R d2 = de - ag.x * de_l - ag.y * de_r;
    de = d2 * q.rs[k][t];
  }
  y = de;
  R yn = shfl_down(y, 1, T);
  if (t == T - 1) yn = R(0);
  const Pair<R> bp = q.bAC[t];
  z = bD - bp.x * y - bp.y * yn;
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
//
// A chunk's elimination depends only on its own rows, so the 32 chunks of a
// line fall into four classes with equal factors: the first (row 0 is an
// identity row), the interior ones, the one holding row N-1, and those past
// N (identity rows only). The chunk tables are kept per class, so the lanes
// of a warp read them mostly from one address (a broadcast); the reduced
// solve's tables stay per lane.

__device__ __forceinline__ int chunk_class(int t, int N, int M) {
  const int tl = (N - 1) / M;  // chunk holding row N-1
  return t == 0 ? 0 : t < tl ? 1 : t == tl ? 2 : 3;
}

template <typename R, int M> struct ContigTab {
  Pair<R> rao[4][M];  // (forward reciprocal pivot, unscaled sub-diagonal)
  R cF[4][M];         // super-diagonal after the forward half
  Pair<R> acB[4][M];  // (a, c) after the backward half
  R rb[4];            // reciprocal of the backward half's top-row pivot
  PcrTab<R> pcr;
};

// Lane t factors chunk t; the lanes of one class store equal values.
template <typename R, int M>
__device__ void contig_factor(ContigTab<R, M> &f, R ca, R cb, int N, int t, bool &bad) {
  const int cl = chunk_class(t, N, M);
  R a[M], b[M], c[M];
#pragma unroll
  for (int i = 0; i < M; ++i) {
    cc_row<R>(t * M + i, N, ca, cb, a[i], b[i]);
    c[i] = a[i];
  }
#pragma unroll
  for (int i = 0; i < (M < 2 ? M : 2); ++i) {
    R r = rcp(b[i]);
    bad |= !finite_rcp(r);
    f.rao[cl][i] = Pair<R>{r, a[i]};
    a[i] *= r;
    c[i] *= r;
  }
#pragma unroll
  for (int i = 2; i < M; ++i) {
    R r = rcp(b[i] - a[i] * c[i - 1]);
    bad |= !finite_rcp(r);
    f.rao[cl][i] = Pair<R>{r, a[i]};
    a[i] = -r * a[i] * a[i - 1];
    c[i] = r * c[i];
  }
#pragma unroll
  for (int i = 0; i < M; ++i) f.cF[cl][i] = c[i];
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
  f.rb[cl] = rb;
#pragma unroll
  for (int i = 0; i < M; ++i) f.acB[cl][i] = Pair<R>{a[i], c[i]};
  pcr_factor<R, kT>(f.pcr, a[0], c[0], a[M - 1], c[M - 1], t, bad);
}

// x solves of two lines held by a warp (lane t = chunk t of class cl), in
// place in d0 and d1; every table value is read once for both.
template <typename R, int M>
__device__ __forceinline__ void contig_solve_d2(const ContigTab<R, M> &f, R (&d0)[M], R (&d1)[M],
                                                int t, int cl) {
#pragma unroll
  for (int i = 0; i < (M < 2 ? M : 2); ++i) {
    const R r = f.rao[cl][i].x;
    d0[i] *= r;
    d1[i] *= r;
  }
#pragma unroll
  for (int i = 2; i < M; ++i) {
    const Pair<R> ra = f.rao[cl][i];
    d0[i] = ra.x * (d0[i] - ra.y * d0[i - 1]);
    d1[i] = ra.x * (d1[i] - ra.y * d1[i - 1]);
  }
#pragma unroll
  for (int i = M - 3; i >= 1; --i) {
    const R cfw = f.cF[cl][i];
    d0[i] = d0[i] - cfw * d0[i + 1];
    d1[i] = d1[i] - cfw * d1[i + 1];
  }
  if (M >= 3) {
    const R rb = f.rb[cl], c0 = f.cF[cl][0];
    d0[0] = rb * (d0[0] - c0 * d0[1]);
    d1[0] = rb * (d1[0] - c0 * d1[1]);
  }
  // reduced solves of both lines, step by step
  const PcrTab<R> &q = f.pcr;
  R p0 = shfl_up(d0[M - 1], 1, kT), p1 = shfl_up(d1[M - 1], 1, kT);
  if (t == 0) {
    p0 = R(0);
    p1 = R(0);
  }
  const Pair<R> tp = q.tAC[t];
  const R ri = q.ri[t];
  R e0 = d0[0] - tp.x * p0 - tp.y * d0[M - 1];
  R e1 = d1[0] - tp.x * p1 - tp.y * d1[M - 1];
  e0 *= ri;
  e1 *= ri;
  int k = 0;
#pragma unroll
  for (int s = 1; s < kT; s <<= 1, ++k) {
    R l0 = shfl_up(e0, s, kT), r0 = shfl_down(e0, s, kT);
    R l1 = shfl_up(e1, s, kT), r1 = shfl_down(e1, s, kT);
    if (t < s) {
      l0 = R(0);
      l1 = R(0);
    }
    if (t + s >= kT) {
      r0 = R(0);
      r1 = R(0);
    }
    const Pair<R> ag = q.alga[k][t];
    const R rs = q.rs[k][t];
    R g0 = e0 - ag.x * l0 - ag.y * r0;
    R g1 = e1 - ag.x * l1 - ag.y * r1;
    e0 = g0 * rs;
    e1 = g1 * rs;
  }
  R n0 = shfl_down(e0, 1, kT), n1 = shfl_down(e1, 1, kT);
  if (t == kT - 1) {
    n0 = R(0);
    n1 = R(0);
  }
  const Pair<R> bp = q.bAC[t];
  const R z0 = d0[M - 1] - bp.x * e0 - bp.y * n0;
  const R z1 = d1[M - 1] - bp.x * e1 - bp.y * n1;
#pragma unroll
  for (int i = 1; i < M - 1; ++i) {
    const Pair<R> ac = f.acB[cl][i];
    d0[i] = d0[i] - ac.x * e0 - ac.y * z0;
    d1[i] = d1[i] - ac.x * e1 - ac.y * z1;
  }
  d0[0] = e0;
  d1[0] = e1;
  if (M > 1) {
    d0[M - 1] = z0;
    d1[M - 1] = z1;
  }
}

// ---- streaming form (strided_stream_kernel) --------------------------------

template <typename R, int M, int T> struct StreamTab {
  Pair<R> rao[M][T];  // (forward reciprocal pivot, unscaled sub-diagonal)
  Pair<R> acf[M][T];  // forward (a', c')
  R r0[T];            // reciprocal of the top reduced row's pivot
  PcrTab<R, T> pcr;
};

template <typename R, int M, int T>
__device__ void stream_factor(StreamTab<R, M, T> &f, R ca, R cb, int N, int t, bool &bad) {
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
    f.rao[j][t] = Pair<R>{r, a};
    f.acf[j][t] = Pair<R>{af, cf};
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
  pcr_factor<R, T>(f.pcr, r0 * a0, -r0 * c0 * C, ap, cp, t, bad);
}

// A line of 32 chunk rows of M elements in shared memory without padding:
// its 16-byte units are permuted within each chunk row (unit u is stored at
// u ^ ((u >> 3) & (UPR - 1)), UPR units per chunk row) so that the eight
// lanes of a quarter warp, reading unit q of their own chunk rows, hit eight
// different 16-byte bank groups.
template <typename R, int M> struct SwzLine {
  static constexpr int VN = 16 / (int)sizeof(R);  // elements per unit
  static constexpr int UPR = M / VN;               // units per chunk row
  static constexpr int LEN = 32 * M;               // elements per line
  static_assert(UPR == 2 || UPR == 4 || UPR == 8, "2, 4 or 8 units per chunk row");
  __device__ static __forceinline__ int unit(int u) { return u ^ ((u >> 3) & (UPR - 1)); }
  __device__ static __forceinline__ int idx(int e) { return unit(e / VN) * VN + e % VN; }
};

// Chunk row `lane` of a swizzled line into registers, and back.
template <typename R, int M>
__device__ __forceinline__ void lds_swz(const R *line, int lane, R (&v)[M]) {
  using S = SwzLine<R, M>;
  using Vt = typename Vec16<R>::T;
#pragma unroll
  for (int q = 0; q < S::UPR; ++q) {
    const Vt x = *reinterpret_cast<const Vt *>(line + S::unit(S::UPR * lane + q) * S::VN);
#pragma unroll
    for (int i = 0; i < S::VN; ++i) v[q * S::VN + i] = reinterpret_cast<const R *>(&x)[i];
  }
}
template <typename R, int M>
__device__ __forceinline__ void sts_swz(R *line, int lane, const R (&v)[M]) {
  using S = SwzLine<R, M>;
  using Vt = typename Vec16<R>::T;
#pragma unroll
  for (int q = 0; q < S::UPR; ++q) {
    Vt x;
#pragma unroll
    for (int i = 0; i < S::VN; ++i) reinterpret_cast<R *>(&x)[i] = v[q * S::VN + i];
    *reinterpret_cast<Vt *>(line + S::unit(S::UPR * lane + q) * S::VN) = x;
  }
}

template <typename R> constexpr int adi_w() { return 128 / (int)sizeof(R); }
// Streaming CTAs of 512 threads run two per SM (64 registers a thread:
// FP64 with up to 8 rows per thread, FP32 with 16 chunks per system): the
// second CTA's loads and sweeps fill the barrier waits of the first.
template <typename R, int M, int T> constexpr int adi_ctas_per_sm() {
  return (sizeof(R) == 8 && M <= 8) || (sizeof(R) == 4 && T <= 16) ? 2 : 1;
}
template <typename R, int T> constexpr int adi_bs() { return T * adi_w<R>(); }

}  // namespace

// ---------------------------------------------------------------------------
// x solve with the stencil, marching along z. A CTA of J / 2 warps owns a
// tile of J consecutive x lines (j0 .. j0+J-1) and walks it through a range
// of planes k. The planes' slabs of J + 2 lines (the tile and its j +- 1
// halo) stream through a ring of LA + 3 slabs in shared memory with
// cp.async, LA planes ahead of the one being solved, so u crosses L2 about
// once per element instead of five times. Warp w forms the 7-point
// right-hand sides of lines j0 + 2w and j0 + 2w + 1 of plane k (in the
// order of adi_preproc_kernel; each line is the other's j neighbour; its
// own planes k - 1 and k are carried in registers from the previous step,
// so each step reads two j-neighbour lines and plane k + 1 from the slabs),
// solves both with the factored coefficients (lane t = chunk t), and stores
// them through its own line buffers, so the global stores are coalesced. Lines in shared memory use
// the swizzled layout of SwzLine (no padding; the lanes' 16-byte chunk reads
// are free of bank conflicts).
//
// Work: the (tile, plane) steps, tile-major, are split evenly over the grid
// (the CTAs resident at once); a CTA whose range crosses into the next tile restarts
// its ring there.
// TRANS: the transposed solve of the step's x matrix in place (u == du):
// the right-hand side is the line itself with rows 0 and nx - 1 taken as 0,
// boundary lines and rows 0, nx - 1 are not stored (see launch_adi_x_transposed).
template <typename R, int M, bool VEC, int J, int LA, bool TRANS = false>
__global__ void __launch_bounds__(J * 16, 1)
    adi_x_kernel(const R *u, R *du, const ConstCoef<R> k, unsigned *flag, int nx, int ny, int nz,
                 int jtiles) {
  static_assert(!(TRANS && VEC), "the transposed form stores element by element");
  static_assert(J % 2 == 0, "two lines per warp");
  using S = SwzLine<R, M>;
  constexpr int LB = S::LEN;           // elements per line buffer
  constexpr int V = VEC ? S::VN : 1;  // elements per copy unit
  constexpr int NS = LA + 3;           // slabs in the ring
  constexpr int SL = J + 2;            // lines per slab
  constexpr int NT = J * 16;           // threads
  using Vt = typename Vec16<R>::T;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  ContigTab<R, M> &f = *reinterpret_cast<ContigTab<R, M> *>(smem_raw);
  R *ring = reinterpret_cast<R *>(smem_raw + (sizeof(ContigTab<R, M>) + 15) / 16 * 16);
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  R *outb = ring + NS * SL * LB + 2 * warp * LB;  // two line buffers per warp
  R l, ca, cb;
  const_coef<R>(k, l, ca, cb);
  bool bad = false;
  if (warp == 0) contig_factor<R, M>(f, ca, cb, nx, lane, bad);
  const int cl = chunk_class(lane, nx, M);
  const int nunits = (nx + V - 1) / V;
  const long long plane = (long long)nx * ny;
  const long long total = (long long)jtiles * nz;
  const long long s0 = total * blockIdx.x / gridDim.x;
  const long long s1 = total * (blockIdx.x + 1) / gridDim.x;

  // this thread's copy units of a slab (the same for every plane of a tile):
  // element offset in the plane and in the slab, -1 where there is none
  constexpr int UQ = ((J + 2) * 32 * (M / V) + NT - 1) / NT;
  int goff[UQ], soff[UQ];
  auto set_tile = [&](int jt) {
    const int jlo = jt * J - 1;
#pragma unroll
    for (int q = 0; q < UQ; ++q) {
      const int idx = threadIdx.x + q * NT;
      const int ll = idx / nunits;
      const int un = idx - ll * nunits;
      const int jj = jlo + ll;
      const int e = un * V;
      const bool ok = ll < SL && jj >= 0 && jj < ny;
      goff[q] = ok ? jj * nx + e : -1;
      soff[q] = ok ? ll * LB + S::idx(e) : -1;
    }
  };
  // slab of plane kp into its ring slot (planes kb - 1 .. ke of the segment
  // [kb, ke) only); always closes a copy group
  auto load_plane = [&](int kp, int kb, int ke) {
    if (kp >= 0 && kp < nz && kp <= ke) {
      R *slab = ring + ((kp - kb + 1) % NS) * SL * LB;
      const R *src = u + (long long)kp * plane;
#pragma unroll
      for (int q = 0; q < UQ; ++q) {
        if (soff[q] >= 0) {
          if constexpr (VEC)
            cp_async16(slab + soff[q], src + goff[q], 16);
          else
            cp_async_elem<R>(slab + soff[q], src + goff[q]);
        }
      }
    }
    cp_async_commit();
  };
  // stores line buffer ob to global line dst (zeros when `zero`)
  auto store_line = [&](R *dst, const R *ob, bool zero) {
    for (int un = lane; un < nunits; un += 32) {
      const int e = un * V;
      if constexpr (VEC) {
        Vt x;
        if (zero) {
#pragma unroll
          for (int i = 0; i < S::VN; ++i) reinterpret_cast<R *>(&x)[i] = R(0);
        } else {
          x = *reinterpret_cast<const Vt *>(ob + S::idx(e));
        }
        *reinterpret_cast<Vt *>(dst + e) = x;
      } else {
        dst[e] = zero ? R(0) : ob[S::idx(e)];
      }
    }
  };

  for (long long s = s0; s < s1;) {
    const int jt = (int)(s / nz);
    const int kb = (int)(s - (long long)jt * nz);
    const int ke = (int)((long long)nz < kb + (s1 - s) ? (long long)nz : kb + (s1 - s));
    s += ke - kb;
    __syncthreads();  // the ring is free (and the factor tables are published)
    set_tile(jt);
#pragma unroll
    for (int q = 0; q < LA + 2; ++q) load_plane(kb - 1 + q, kb, ke);
    const int j = jt * J + 2 * warp;  // this warp's lines j and j + 1
    // planes k - 1 and k of the warp's two lines, carried from the previous
    // step (valid while `have`): each step reads only the j-neighbour lines
    // and plane k + 1 from the slabs
    R pm0[M], pm1[M], pc0[M], pc1[M];
    bool have = false;
    for (int kz = kb; kz < ke; ++kz) {
      load_plane(kz + 1 + LA, kb, ke);
      cp_async_wait_groups<LA>();  // planes <= kz + 1 have landed
      __syncthreads();
      if (j < ny) {
        R *dst = du + (long long)kz * plane + (long long)j * nx;
        const bool kbnd = kz == 0 || kz == nz - 1;
        const bool z0 = kbnd || j == 0 || j == ny - 1;
        const bool z1 = kbnd || j + 1 == ny - 1;
        const bool has1 = j + 1 < ny;
        if (z0 && (z1 || !has1)) {
          if constexpr (!TRANS) {
            store_line(dst, outb, true);
            if (has1) store_line(dst + nx, outb, true);
          }
          have = false;
        } else if constexpr (TRANS) {
          // the lines themselves as right-hand sides, rows 0 and nx - 1 as 0
          const R *sc = ring + ((kz - kb + 1) % NS) * SL * LB;
          R d0[M], d1[M];
          lds_swz<R, M>(sc + (2 * warp + 1) * LB, lane, d0);
          lds_swz<R, M>(sc + (2 * warp + 2) * LB, lane, d1);
#pragma unroll
          for (int i = 0; i < M; ++i) {
            const int row = lane * M + i;
            const bool in = row >= 1 && row <= nx - 2;
            d0[i] = in ? d0[i] : R(0);
            d1[i] = in ? d1[i] : R(0);
          }
          contig_solve_d2<R, M>(f, d0, d1, lane, cl);
          sts_swz<R, M>(outb, lane, d0);
          sts_swz<R, M>(outb + LB, lane, d1);
          __syncwarp();
          // interior rows of interior lines only
          for (int e = 1 + lane; e < nx - 1; e += 32) {
            if (!z0) dst[e] = outb[S::idx(e)];
            if (has1 && !z1) dst[nx + e] = outb[LB + S::idx(e)];
          }
        } else {
          // slab line w2 + 1 holds line j (line 0 of the slab is j0 - 1)
          const int w2 = 2 * warp;
          const R *sc = ring + ((kz - kb + 1) % NS) * SL * LB;
          const R *sp = ring + ((kz - kb + 2) % NS) * SL * LB;
          if (!have) {
            const R *sm = ring + ((kz - kb) % NS) * SL * LB;
            lds_swz<R, M>(sm + (w2 + 1) * LB, lane, pm0);
            lds_swz<R, M>(sm + (w2 + 2) * LB, lane, pm1);
            lds_swz<R, M>(sc + (w2 + 1) * LB, lane, pc0);
            lds_swz<R, M>(sc + (w2 + 2) * LB, lane, pc1);
          }
          R d0[M], d1[M], tmp[M];
          {
            const R lf0 = shfl_up(pc0[M - 1], 1, 32), rg0 = shfl_down(pc0[0], 1, 32);
            const R lf1 = shfl_up(pc1[M - 1], 1, 32), rg1 = shfl_down(pc1[0], 1, 32);
#pragma unroll
            for (int i = 0; i < M; ++i) {
              d0[i] = (i == 0 ? lf0 : pc0[i - 1]) + (i == M - 1 ? rg0 : pc0[i + 1]);
              d1[i] = (i == 0 ? lf1 : pc1[i - 1]) + (i == M - 1 ? rg1 : pc1[i + 1]);
            }
          }
          lds_swz<R, M>(sc + w2 * LB, lane, tmp);  // j - 1 of line j
#pragma unroll
          for (int i = 0; i < M; ++i) {
            d0[i] = d0[i] + tmp[i];
            d1[i] = d1[i] + pc0[i];  // j - 1 of line j + 1
          }
          lds_swz<R, M>(sc + (w2 + 3) * LB, lane, tmp);  // j + 1 of line j + 1
#pragma unroll
          for (int i = 0; i < M; ++i) {
            d0[i] = d0[i] + pc1[i];  // j + 1 of line j
            d1[i] = d1[i] + tmp[i];
            d0[i] = d0[i] + pm0[i];  // k - 1
            d1[i] = d1[i] + pm1[i];
          }
          // k + 1: read into the k - 1 registers, which then carry plane k + 1
          lds_swz<R, M>(sp + (w2 + 1) * LB, lane, pm0);
          lds_swz<R, M>(sp + (w2 + 2) * LB, lane, pm1);
#pragma unroll
          for (int i = 0; i < M; ++i) {
            const int row = lane * M + i;
            const bool in = row >= 1 && row <= nx - 2;
            const R s0 = d0[i] + pm0[i];
            const R s1 = d1[i] + pm1[i];
            d0[i] = in ? l * (s0 - R(6) * pc0[i]) : R(0);
            d1[i] = in ? l * (s1 - R(6) * pc1[i]) : R(0);
          }
          // rotate: plane k becomes k - 1, plane k + 1 (in pm) becomes k
#pragma unroll
          for (int i = 0; i < M; ++i) {
            const R t0 = pc0[i], t1 = pc1[i];
            pc0[i] = pm0[i];
            pc1[i] = pm1[i];
            pm0[i] = t0;
            pm1[i] = t1;
          }
          have = true;
          contig_solve_d2<R, M>(f, d0, d1, lane, cl);
          sts_swz<R, M>(outb, lane, d0);
          sts_swz<R, M>(outb + LB, lane, d1);
          __syncwarp();
          store_line(dst, outb, z0);
          if (has1) store_line(dst + nx, outb + LB, z1);
        }
      }
      __syncthreads();  // every warp is done with the slab of plane kz - 1
    }
  }
  cp_async_wait_groups<0>();
  if (warp == 0) report_bad_pivot(__any_sync(FULL_MASK, bad), flag);
}

// ---------------------------------------------------------------------------
// y and z solves: the persistent streaming layout of strided_stream_kernel
// (groups of W systems with W * sizeof(R) = 128 bytes, T chunks of M rows
// (T = 32; 16 for FP32 systems up to 256 rows), a D-row window of loads
// that runs on into the next group, L2 prefetch PF rows ahead for rows less
// than 64 KiB apart), sweeping only the right-hand side. Inc: u is carried
// through the window and parked in private shared-memory slots until the
// store.
// O32: element offsets in 32 bits (the launcher's choice when they fit).
// TRANS: the transposed solve in place (p.d_in == p.d_out): rows 0 and N - 1
// of the interior systems enter as 0 and are not stored (see
// launch_adi_yz_transposed).
template <typename R, int M, int D, int PF, bool INC, int T, bool O32 = false, bool TRANS = false>
__global__ void __launch_bounds__(adi_bs<R, T>(), adi_ctas_per_sm<R, M, T>())
    adi_stream_kernel(const BatchArgs<R> p, const ConstCoef<R> k, long long ngx, long long ngroups) {
  static_assert(!(TRANS && INC), "the transposed form overwrites");
  static_assert(M >= 4 && D >= 1 && D <= M && M % D == 0, "window must tile the chunk");
  static_assert(PF == 0 || (PF > D && PF <= M), "L2 prefetch runs ahead of the window");
  constexpr int W = adi_w<R>();
  constexpr int BS = W * T;
  constexpr int RED = (2 * T * (W + 1) * (int)sizeof(R) + 15) / 16 * 16;
  extern __shared__ __align__(16) unsigned char stream_smem[];
  R *red = reinterpret_cast<R *>(stream_smem);
  StreamTab<R, M, T> &f = *reinterpret_cast<StreamTab<R, M, T> *>(stream_smem + RED);
  R *suf = reinterpret_cast<R *>(stream_smem + RED + (sizeof(StreamTab<R, M, T>) + 15) / 16 * 16) +
           threadIdx.x;  // u of row j at [j * BS] (Inc)
  const int tid = threadIdx.x;
  const int s = tid % W;
  const int t = tid / W;
  const int lane = tid & 31;
  const int N = p.N;
  const int row0 = t * M;
  using IX = typename std::conditional<O32, int, long long>::type;  // element offsets
  const IX stride = (IX)p.stride;
  const long long n1 = p.nsys / p.n0;
  bool bad = false;
  {
    R l, ca, cb;
    const_coef<R>(k, l, ca, cb);
    // lanes t and t + T (T < 32) compute the same values for chunk t
    if (tid < 32) stream_factor<R, M, T>(f, ca, cb, N, lane & (T - 1), bad);
  }
  __syncthreads();

  // Group g = gx + ngx * i1 (the launcher keeps ngx and n1 below 2^31).
  // FP64 CTAs step a cursor (gx, i1) by the grid size without dividing, in
  // 32-bit arithmetic; FP32 CTAs (1024 threads at the 64-register limit)
  // divide g instead, which measured faster there (fewer live registers).
  constexpr bool kStep = sizeof(R) == 8;
  struct Cursor {
    int gx, i1;
  };
  const int ngx32 = (int)ngx;
  const int n132 = (int)n1;
  auto advance = [&](Cursor c) -> Cursor {
    if constexpr (kStep) {
      c.gx += (int)(gridDim.x % ngx32);
      c.i1 += (int)(gridDim.x / ngx32);
      if (c.gx >= ngx32) {
        c.gx -= ngx32;
        ++c.i1;
      }
    }
    return c;
  };
  // element offset of this thread's first chunk row in group g (cursor c);
  // act: an interior system (others are identity systems with zero
  // right-hand side)
  auto group_first = [&](long long g, const Cursor &c, bool &act) -> IX {
    if constexpr (kStep) {
      const int i0 = c.gx * W + s;
      act = c.i1 < n132 && i0 >= 1 && i0 <= p.n0 - 2 && c.i1 >= 1 && c.i1 <= n132 - 2;
      return act ? (IX)(i0 * p.st0 + (long long)c.i1 * p.st1 + (long long)row0 * stride) : IX(0);
    } else {
      const long long gx = g % ngx;
      const long long i1 = g / ngx;
      const long long i0 = gx * W + s;
      act = g < ngroups && i0 >= 1 && i0 <= p.n0 - 2 && i1 >= 1 && i1 <= n1 - 2;
      return act ? (IX)(i0 * p.st0 + i1 * p.st1 + (long long)row0 * stride) : IX(0);
    }
  };

  constexpr int NA = INC ? 2 : 1;
  const bool pf_lane = PF > 0 && lane < 2 * NA * (32 / W);
  const int pq = (lane >> 1) % NA;
  const int pt = (tid >> 5) * (32 / W) + (lane >> 1) / NA;
  const R *pbase = pq == 0 ? p.d_in : p.u;
  auto pf_first = [&](long long g, const Cursor &c, bool &ok) -> IX {
    if constexpr (kStep) {
      const int left = (int)p.n0 - c.gx * W;
      const int i0 = c.gx * W + ((lane & 1) ? (left < W ? left : W) - 1 : 0);
      ok = pf_lane && c.i1 < n132;
      return ok ? (IX)(i0 * p.st0 + (long long)c.i1 * p.st1 + (long long)pt * M * stride) : IX(0);
    } else {
      const long long gx = g % ngx;
      const long long i1 = g / ngx;
      const long long left = p.n0 - gx * W;
      const long long i0 = gx * W + ((lane & 1) ? (left < W ? left : W) - 1 : 0);
      ok = pf_lane && g < ngroups;
      return ok ? (IX)(i0 * p.st0 + i1 * p.st1 + (long long)pt * M * stride) : IX(0);
    }
  };

  R pd[D], pu[INC ? D : 1];
  long long g = blockIdx.x;
  Cursor cur{0, 0};
  if constexpr (kStep) cur = Cursor{(int)(blockIdx.x % ngx32), (int)(blockIdx.x / ngx32)};
  bool act;
  IX first = group_first(g, cur, act);
  IX lo = first;
#pragma unroll
  for (int j = 0; j < D; ++j) {
    const bool v = act && row0 + j < N && !(TRANS && (row0 + j == 0 || row0 + j == N - 1));
    pd[j] = v ? __ldg(p.d_in + lo) : R(0);
    if constexpr (INC) pu[j] = v ? __ldg(p.u + lo) : R(0);
    lo += stride;
  }
  bool pok = false;
  IX po = 0;
  if constexpr (PF > 0) po = pf_first(g, cur, pok) + (IX)PF * stride;

  for (; kStep ? cur.i1 < n132 : g < ngroups; g += gridDim.x) {
    const Cursor nxt = advance(cur);
    bool actn;
    const IX firstn = group_first(g + gridDim.x, nxt, actn);
    IX ln = firstn;
    bool pokn = false;
    IX pon = 0;
    if constexpr (PF > 0) pon = pf_first(g + gridDim.x, nxt, pokn);

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
        const bool v = (nxt ? actn : act) && row < N && !(TRANS && (row == 0 || row == N - 1));
        const IX o = nxt ? ln : lo;
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
      const Pair<R> ra = f.rao[j][t];
      const R df = j < 2 ? d * ra.x : ra.x * (d - ra.y * dp);
      rd[j] = df;
      dp = df;
    }
    // top reduced row: one running row from row M-2 up to row 1
    R Dd = rd[M - 2];
#pragma unroll
    for (int j = M - 3; j >= 1; --j) Dd = rd[j] - f.acf[j][t].y * Dd;
    const R topD = f.r0[t] * (rd[0] - f.acf[0][t].y * Dd);

    // block-wide reduced solve: re-deal the D parts so that each run of T
    // lanes holds the T chunks of one system, one per lane
    constexpr int ld = W + 1;
    constexpr int nslot = T * ld;
    __syncthreads();  // the previous group's reads of red are over
    red[0 * nslot + t * ld + s] = topD;
    red[1 * nslot + t * ld + s] = dp;
    __syncthreads();
    {
      const int s2 = tid / T;
      const int t2 = tid & (T - 1);
      const int kk = t2 * ld + s2;
      R yy, zz;
      pcr_solve_d<R, T>(f.pcr, red[0 * nslot + kk], red[1 * nslot + kk], t2, yy, zz);
      red[0 * nslot + kk] = yy;  // slot kk is read and rewritten by this thread only
      red[1 * nslot + kk] = zz;
    }
    __syncthreads();
    const R y = red[0 * nslot + t * ld + s];
    const R z = red[1 * nslot + t * ld + s];

    // back-substitution with the forward rows, stored as it goes
    IX o = first + (IX)(M - 1) * stride;
    R x = z;
#pragma unroll
    for (int j = M - 1; j >= 0; --j) {
      if (j < M - 1) {
        const Pair<R> ac = f.acf[j][t];
        x = j == 0 ? y : rd[j] - ac.x * y - ac.y * x;
      }
      if (act && row0 + j < N && !(TRANS && (row0 + j == 0 || row0 + j == N - 1))) {
        if constexpr (INC)
          p.u[o] = suf[j * BS] + x;
        else
          p.d_out[o] = x;
      }
      o -= stride;
    }
    cur = nxt;
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

template <typename R, int M, bool VEC, int J, int LA>
static constexpr size_t adi_x_smem() {
  return (sizeof(ContigTab<R, M>) + 15) / 16 * 16 +
         (size_t)((LA + 3) * (J + 2) + J) * SwzLine<R, M>::LEN * sizeof(R);
}

template <typename R, int M, bool VEC, int J, int LA, bool TRANS = false>
static cudaError_t launch_adi_x_j(const R *u, R *du, const ConstCoef<R> &k, unsigned *flag, int nx,
                                  int ny, int nz, cudaStream_t st) {
  const size_t smem = adi_x_smem<R, M, VEC, J, LA>();
  auto kern = adi_x_kernel<R, M, VEC, J, LA, TRANS>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int dev = 0, sms = 148, per_sm = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, J * 16, smem) != cudaSuccess ||
      per_sm < 1)
    per_sm = 1;
  const int jtiles = (ny + J - 1) / J;
  const long long total = (long long)jtiles * nz;
  const long long cap = (long long)sms * per_sm;
  const long long grid = total < cap ? total : cap;
  kern<<<(unsigned)grid, J * 16, smem, st>>>(u, du, k, flag, nx, ny, nz, jtiles);
  return cudaGetLastError();
}

// Tiles of 8 lines with slabs one plane ahead: two 4-warp CTAs share an SM
// (ms per step, 256^3 FP64 / 512x512x128 FP32: 0.191 / 0.224 against 0.196
// / 0.228 with 16 lines at one CTA per SM; 16 lines two planes ahead 0.197,
// 8 lines two planes ahead 0.228 / 0.257, 4 lines 0.208 FP64).
template <typename R, int M, bool VEC, bool TRANS = false>
static cudaError_t launch_adi_x_mv(const R *u, R *du, const ConstCoef<R> &k, unsigned *flag, int nx,
                                   int ny, int nz, cudaStream_t st) {
  return launch_adi_x_j<R, M, VEC, 8, 1, TRANS>(u, du, k, flag, nx, ny, nz, st);
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

// The transposed solve of the step's x matrix, in place on w (1 <= nx <=
// 512). The matrix has identity rows on the boundary and constant interior
// rows, so its transpose's interior block is its own: the interior of every
// interior line is the solve of that line's interior (rows 0 and nx - 1 as
// 0), and boundary lines and rows are left as they are (adi_transposed_fixup
// then adds the one coupling of rows 0 and nx - 1).
template <typename R>
cudaError_t launch_adi_x_transposed(R *w, const ConstCoef<R> &k, int nx, int ny, int nz,
                                    cudaStream_t st) {
  if (nx < 1 || nx > 512 || ny < 1 || nz < 1) return cudaErrorInvalidValue;
  if (nx <= 256) return launch_adi_x_mv<R, 8, false, true>(w, w, k, nullptr, nx, ny, nz, st);
  return launch_adi_x_mv<R, 16, false, true>(w, w, k, nullptr, nx, ny, nz, st);
}

template <typename R, int M> constexpr int adi_window() { return M < 8 ? M : 8; }
template <typename R, int M> constexpr int adi_prefetch() { return adi_window<R, M>() >= M ? 0 : 12; }

template <typename R, int M, int T, int PF, bool INC, bool TRANS = false>
static cudaError_t launch_adi_stream_pf(const BatchArgs<R> &p, const ConstCoef<R> &k, cudaStream_t st) {
  constexpr int W = adi_w<R>();
  constexpr int BS = adi_bs<R, T>();
  // (the FP64 Inc window of 8 rows spills at two CTAs per SM)
  constexpr int D = (INC && sizeof(R) == 8 && M == 8) ? 4 : adi_window<R, M>();
  const size_t red = ((size_t)2 * T * (W + 1) * sizeof(R) + 15) / 16 * 16;
  const size_t smem = red + (sizeof(StreamTab<R, M, T>) + 15) / 16 * 16 +
                      (INC ? (size_t)M * BS * sizeof(R) : 0);
  // 32-bit element offsets where every offset fits (FP64 only: measured
  // 2% faster per timestep there, no gain in FP32)
  const long long maxoff = (p.n0 - 1) * p.st0 + (p.nsys / p.n0 - 1) * p.st1 + (long long)(p.N - 1) * p.stride;
  const bool o32 = maxoff < (1LL << 31) - 1 - 64LL * p.stride;
  auto kern = adi_stream_kernel<R, M, D, PF, INC, T, false, TRANS>;
  if constexpr (sizeof(R) == 8) {
    if (o32) kern = adi_stream_kernel<R, M, D, PF, INC, T, true, TRANS>;
  }
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

template <typename R, int M, int T, bool INC, bool TRANS = false>
static cudaError_t launch_adi_stream_m(const BatchArgs<R> &p, const ConstCoef<R> &k, cudaStream_t st) {
  constexpr int PF = adi_prefetch<R, M>();
  if (PF > 0 && p.stride * (long long)sizeof(R) < (1LL << 16))
    return launch_adi_stream_pf<R, M, T, PF, INC, TRANS>(p, k, st);
  return launch_adi_stream_pf<R, M, T, 0, INC, TRANS>(p, k, st);
}

// y or z solve of the timestep: p.d_in == p.d_out == du, p.u = u for the z
// solve (INC); any 1 <= N <= 512.
template <typename R, bool INC>
cudaError_t launch_adi_yz(const BatchArgs<R> &p, const ConstCoef<R> &k, cudaStream_t st) {
  if (p.N < 1 || p.N > 512 || p.n0 < 1 || p.nsys % p.n0) return cudaErrorInvalidValue;
  if (p.n0 >= (1LL << 31) || p.nsys / p.n0 >= (1LL << 31)) return cudaErrorInvalidValue;
  if (p.nsys == 0) return cudaSuccess;
  if constexpr (sizeof(R) == 4) {
    // FP32 systems up to 256 rows: 16 chunks of up to 16 rows (a 512-thread
    // CTA, two per SM; the reduced solve costs half that of 32 chunks)
    if (p.N <= 128) return launch_adi_stream_m<R, 8, 16, INC>(p, k, st);
    if (p.N <= 256) return launch_adi_stream_m<R, 16, 16, INC>(p, k, st);
    return launch_adi_stream_m<R, 16, 32, INC>(p, k, st);
  } else {
    if (p.N <= 128) return launch_adi_stream_m<R, 4, 32, INC>(p, k, st);
    if (p.N <= 256) return launch_adi_stream_m<R, 8, 32, INC>(p, k, st);
    return launch_adi_stream_m<R, 16, 32, INC>(p, k, st);
  }
}

// The transposed y or z solve of the step, in place on p.d_in == p.d_out
// (1 <= N <= 512): interior systems get the solve of their interior rows
// (rows 0 and N - 1 as 0, not stored), boundary systems are left as they
// are (see launch_adi_x_transposed).
template <typename R>
cudaError_t launch_adi_yz_transposed(const BatchArgs<R> &p, const ConstCoef<R> &k, cudaStream_t st) {
  if (p.N < 1 || p.N > 512 || p.n0 < 1 || p.nsys % p.n0 || p.d_in != p.d_out) return cudaErrorInvalidValue;
  if (p.n0 >= (1LL << 31) || p.nsys / p.n0 >= (1LL << 31)) return cudaErrorInvalidValue;
  if (p.nsys == 0) return cudaSuccess;
  if constexpr (sizeof(R) == 4) {
    if (p.N <= 128) return launch_adi_stream_m<R, 8, 16, false, true>(p, k, st);
    if (p.N <= 256) return launch_adi_stream_m<R, 16, 16, false, true>(p, k, st);
    return launch_adi_stream_m<R, 16, 32, false, true>(p, k, st);
  } else {
    if (p.N <= 128) return launch_adi_stream_m<R, 4, 32, false, true>(p, k, st);
    if (p.N <= 256) return launch_adi_stream_m<R, 8, 32, false, true>(p, k, st);
    return launch_adi_stream_m<R, 16, 32, false, true>(p, k, st);
  }
}

template cudaError_t launch_adi_x_transposed<double>(double *, const ConstCoef<double> &, int, int, int,
                                                     cudaStream_t);
template cudaError_t launch_adi_x_transposed<float>(float *, const ConstCoef<float> &, int, int, int,
                                                    cudaStream_t);
template cudaError_t launch_adi_yz_transposed<double>(const BatchArgs<double> &,
                                                      const ConstCoef<double> &, cudaStream_t);
template cudaError_t launch_adi_yz_transposed<float>(const BatchArgs<float> &, const ConstCoef<float> &,
                                                     cudaStream_t);
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
