// Strided batches (solvedim >= 1), streaming form of the hybrid solve.
//
// Why a second strided kernel: strided_kernel holds a whole chunk (M rows of
// a, b, c, d) in registers, so a 512-row FP64 group of 8 systems already
// takes a 512-thread CTA with ~100 registers, i.e. one CTA per SM with no
// other CTA to hide its load latency (measured: the same access pattern with
// no arithmetic reaches 61% of the copy bandwidth at one CTA per SM, 104%
// with many). Rows a whole plane apart (z solves) are in addition limited
// per 64-byte row segment (about 50 G segments/s); 128-byte segments reach
// 97% of the copy bandwidth.
//
// Here a persistent CTA walks over groups of W systems with W * sizeof(R) =
// 128 bytes (16 FP64 / 32 FP32 systems) and T = 32 chunks of M rows each
// (one warp per system for the reduced solve). Each thread
//   1. streams its chunk's rows through a D-deep register window that runs
//      on into the next group's first rows, so loads stay in flight across
//      the reduced solve and the stores. When the rows of a system are less
//      than 64 KiB apart (y solves), some lanes of each warp also ask L2 for
//      the rows PF steps ahead (no registers). For rows a plane apart (z)
//      that costs more in address translation than it saves, so it is off;
//   2. runs the forward half of the chunk elimination row by row, keeping
//      a', c' (and d' when SD, to make room for a deeper window) in its own
//      shared-memory slots [j * BS + tid] (no other thread reads them, so the
//      sweep needs no barrier; BS is a compile-time constant, so every slot
//      has an immediate address);
//   3. recovers the chunk's top reduced row with a backward recursion that
//      only carries one running row;
//   4. after the block-wide reduced solve, back-substitutes
//          x_i = d'_i - a'_i x_first - c'_i x_{i+1}
//      from the chunk's last row up, and stores.
// Inc variants carry u through the same window and park it in a third set
// of private slots until the store. The adjoint variant solves T^T the same
// way (c one row up and a one row down as its off-diagonals, w as the right-
// hand side), parks the forward x in those slots and writes
// dbar, abar = -dbar x_{i-1}, bbar = -dbar x_i, cbar = -dbar x_{i+1} in the
// same pass (9 words per element). Every element is read once and written
// once.
//
// The per-row work of the FP32 forms is issue-bound (a profile of 256^3 y
// and z solves: integer pipe at 43-54% of its peak, DRAM at 54%), so the
// sweep keeps it short: FP32 pivots are inverted with the hardware estimate
// (within one ulp of 1/x; measured 256^3 y 0.69 -> 0.73, Inc 0.66 -> 0.75 of
// the copy bandwidth) and the zero-pivot check of every precision is one FMA
// per row (pivot_acc) instead of a compare and an or.
#include <cuda_runtime.h>

#include <type_traits>

#include "trid_internal.h"

namespace trid {

namespace {

template <typename R> constexpr int stream_w() { return 128 / (int)sizeof(R); }
template <typename R> constexpr int stream_bs() { return 32 * stream_w<R>(); }

// Row `row` at element offset o: identity rows outside the system, a[0] and
// c[N-1] forced to zero; u too for Inc. The adjoint (ADJ) solves T^T: its
// sub-diagonal is c one row up and its super-diagonal a one row down, and
// the fifth value is the forward solution x (in p.u).
//
// CR: the coefficients' storage type. With CR = float and R = double (the
// promoted solve of tridDmtsvStridedBatchMixed) a, b, c are read from cf as
// FP32 and the solve runs in FP64 on their exact promoted values.
template <typename R, bool FIFTH, int ADJ, typename CR>
__device__ __forceinline__ void stream_load_row(const BatchArgs<R> &p, const CoefPtrs<CR> &cf,
                                                long long o, bool valid, int row, R &a, R &b, R &c,
                                                R &d, R &u) {
  if (valid) {
    if constexpr (!std::is_same<CR, R>::value) {
      a = row == 0 ? R(0) : R(__ldg(cf.a + o));
      c = row == p.N - 1 ? R(0) : R(__ldg(cf.c + o));
      b = R(__ldg(cf.b + o));
    } else if constexpr (ADJ) {
      a = row == 0 ? R(0) : __ldg(p.c + o - p.stride);
      c = row == p.N - 1 ? R(0) : __ldg(p.a + o + p.stride);
      b = __ldg(p.b + o);
    } else {
      // forward solve: loads cached in L2 only (ld.global.cg). Nothing is
      // read twice, and keeping the rows out of L1 measured faster with a
      // fifth stream (Inc along z at 512^3 FP64: 1.54 -> 1.47 ms), the same
      // elsewhere
      a = row == 0 ? R(0) : __ldcg(p.a + o);
      c = row == p.N - 1 ? R(0) : __ldcg(p.c + o);
      b = __ldcg(p.b + o);
    }
    if constexpr (ADJ == 0 && std::is_same<CR, R>::value) {
      d = __ldcg(p.d_in + o);
      if constexpr (FIFTH) u = __ldcg(p.u + o);
    } else {
      d = __ldg(p.d_in + o);
      if constexpr (FIFTH) u = __ldg(p.u + o);
    }
  } else {
    a = R(0);
    b = R(1);
    c = R(0);
    d = R(0);
    if constexpr (FIFTH) u = R(0);
  }
}

}  // namespace

// ADJ: 0 the forward solve, 1 the adjoint (dbar only), 2 the adjoint with
// the products abar, bbar, cbar (the forward x is read too).
template <typename R, int M, int D, bool SD, int PF, bool INC, int ADJ, typename CR = R, int TC = 32>
__global__ void __launch_bounds__(stream_w<R>() * TC, TC <= 16 ? 2 : 1)
    strided_stream_kernel(const BatchArgs<R> p, const AdjointOut<R> q, const CoefPtrs<CR> cf,
                          long long ngx, long long ngroups) {
  static_assert(std::is_same<CR, R>::value || (ADJ == 0 && PF == 0),
                "the promoted form has neither the adjoint nor the L2 prefetch");
  static_assert(!(INC && ADJ), "Inc or adjoint");
  constexpr bool FIFTH = INC || ADJ == 2;  // a fifth value per row: u (Inc) or x (adjoint)
  static_assert(M >= 4 && D >= 1 && D <= M && M % D == 0, "window must tile the chunk");
  static_assert(PF == 0 || (PF > D && PF <= M), "L2 prefetch runs ahead of the window");
  constexpr int W = stream_w<R>();
  constexpr int T = TC;
  constexpr int BS = W * T;
  constexpr int RED = (6 * T * (W + 1) * (int)sizeof(R) + 15) / 16 * 16 / (int)sizeof(R);
  extern __shared__ __align__(16) unsigned char stream_smem[];
  R *red = reinterpret_cast<R *>(stream_smem);
  const int tid = threadIdx.x;
  R *saf = red + RED + tid;             // a' of row j at [j * BS]
  R *scf = red + RED + M * BS + tid;    // c'
  R *sdf = red + RED + 2 * M * BS + tid;  // d' (SD)
  R *suf = red + RED + (SD ? 3 : 2) * M * BS + tid;  // u (Inc) or x (adjoint)
  const int s = tid % W;
  const int t = tid / W;
  const int N = p.N;
  const int row0 = t * M;
  const long long stride = p.stride;

  // element offset of this thread's first chunk row in group g (0 if none)
  auto group_first = [&](long long g, bool &act) -> long long {
    const long long gx = g % ngx;
    const long long i1 = g / ngx;
    const long long i0 = gx * W + s;
    act = g < ngroups && i0 < p.n0;
    return act ? i0 * p.st0 + i1 * p.st1 + (long long)row0 * stride : 0;
  };

  // L2 prefetch lanes (PF > 0): lane l < 2 * NA * (32 / W) covers one end
  // (first or last system) of the row segment of one of the NA arrays for
  // one of the warp's chunks
  constexpr int NA = FIFTH ? 5 : 4;
  const int lane = tid & 31;
  const bool pf_lane = PF > 0 && lane < 2 * NA * (32 / W);
  const int pq = (lane >> 1) % NA;
  const int pt = (tid >> 5) * (32 / W) + (lane >> 1) / NA;
  const R *pbase = pq == 0 ? (ADJ ? p.c : p.a) : pq == 1 ? p.b : pq == 2 ? (ADJ ? p.a : p.c)
                 : pq == 3 ? p.d_in : p.u;
  auto pf_first = [&](long long g, bool &ok) -> long long {
    const long long gx = g % ngx;
    const long long i1 = g / ngx;
    const long long left = p.n0 - gx * W;
    const long long i0 = gx * W + ((lane & 1) ? (left < W ? left : W) - 1 : 0);
    ok = pf_lane && g < ngroups;
    return ok ? i0 * p.st0 + i1 * p.st1 + (long long)pt * M * stride : 0;
  };

  R pa[D], pb[D], pc[D], pd[D], pu[FIFTH ? D : 1];
  long long g = blockIdx.x;
  bool act;
  long long first = group_first(g, act);
  long long lo = first;
#pragma unroll
  for (int j = 0; j < D; ++j) {
    stream_load_row<R, FIFTH, ADJ, CR>(p, cf, lo, act && row0 + j < N, row0 + j, pa[j], pb[j],
                                       pc[j], pd[j], pu[FIFTH ? j : 0]);
    lo += stride;
  }
  bool pok = false;
  long long po = 0;
  if constexpr (PF > 0) po = pf_first(g, pok) + (long long)PF * stride;

  bool bad = false;
  R racc = R(0);  // pivot_acc of the sweep's pivots
  for (; g < ngroups; g += gridDim.x) {
    bool actn;
    const long long firstn = group_first(g + gridDim.x, actn);
    long long ln = firstn;
    bool pokn = false;
    long long pon = 0;
    if constexpr (PF > 0) pon = pf_first(g + gridDim.x, pokn);
    // adjoint products: the forward x just outside this thread's chunk
    R xm = R(0), xp = R(0);
    if constexpr (ADJ == 2) {
      if (act && row0 >= 1 && row0 - 1 < N) xm = __ldg(p.u + first - stride);
      if (act && row0 + M <= N - 1) xp = __ldg(p.u + first + (long long)M * stride);
    }

    // forward half of the chunk elimination, streamed row by row
    R rd[SD ? 1 : M];
    R ap = R(0), cp = R(0), dp = R(0);
#pragma unroll
    for (int j = 0; j < M; ++j) {
      const int k = j % D;
      const R a = pa[k], b = pb[k], c = pc[k], d = pd[k];
      if constexpr (FIFTH) suf[j * BS] = pu[k];
      if (j + D < M) {
        const int row = row0 + j + D;
        stream_load_row<R, FIFTH, ADJ, CR>(p, cf, lo, act && row < N, row, pa[k], pb[k], pc[k],
                                           pd[k], pu[FIFTH ? k : 0]);
        lo += stride;
      } else {
        const int row = row0 + j + D - M;
        stream_load_row<R, FIFTH, ADJ, CR>(p, cf, ln, actn && row < N, row, pa[k], pb[k], pc[k],
                                           pd[k], pu[FIFTH ? k : 0]);
        ln += stride;
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
      R af, cf, df;
      if (j < 2) {
        const R r = rcp_sel<sizeof(R) == 4>(b);
        pivot_acc(racc, r);
        af = a * r;
        cf = c * r;
        df = d * r;
      } else {
        const R r = rcp_sel<sizeof(R) == 4>(b - a * cp);
        pivot_acc(racc, r);
        df = r * (d - a * dp);
        af = -r * a * ap;
        cf = r * c;
      }
      saf[j * BS] = af;
      scf[j * BS] = cf;
      if constexpr (SD)
        sdf[j * BS] = df;
      else
        rd[j] = df;
      ap = af;
      cp = cf;
      dp = df;
    }
    auto dval = [&](int j) -> R {
      if constexpr (SD)
        return sdf[j * BS];
      else
        return rd[j];
    };

    // backward half: carry one running row from row M-2 up to row 1, then
    // fold it into row 0 to get the chunk's top reduced row
    R A = saf[(M - 2) * BS], C = scf[(M - 2) * BS], Dd = dval(M - 2);
#pragma unroll
    for (int j = M - 3; j >= 1; --j) {
      const R cj = scf[j * BS];
      Dd = dval(j) - cj * Dd;
      A = saf[j * BS] - cj * A;
      C = -cj * C;
    }
    const R a0 = saf[0], c0 = scf[0];
    const R r0 = rcp(R(1) - c0 * A);
    bad |= !finite_rcp(r0);
    const Row<R> top{r0 * a0, -r0 * c0 * C, r0 * (dval(0) - c0 * Dd)};
    const Row<R> bot{ap, cp, dp};
    R y, z;
    block_reduced_solve<R, 2>(red, top, bot, s, t, T, W, y, z, bad);

    // back-substitution with the forward rows, stored as it goes (last row
    // first)
    long long o = first + (long long)(M - 1) * stride;
    R x = z;
#pragma unroll
    for (int j = M - 1; j >= 0; --j) {
      if (j < M - 1) x = j == 0 ? y : dval(j) - saf[j * BS] * y - scf[j * BS] * x;
      if (act && row0 + j < N) {
        if constexpr (INC) {
          p.u[o] = suf[j * BS] + x;
        } else {
          p.d_out[o] = x;
          if constexpr (ADJ == 2) {
            // abar_i = -dbar_i x_{i-1}, bbar_i = -dbar_i x_i, cbar_i = -dbar_i x_{i+1}
            const int row = row0 + j;
            const R xl = j > 0 ? suf[(j - 1) * BS] : xm;
            const R xr = j < M - 1 ? suf[(j + 1) * BS] : xp;
            if (q.abar) q.abar[o] = row >= 1 ? -x * xl : R(0);
            if (q.bbar) q.bbar[o] = -x * suf[j * BS];
            if (q.cbar) q.cbar[o] = row <= N - 2 ? -x * xr : R(0);
          }
        }
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
  bad |= racc != racc;
  report_bad_pivot(bad, p.flag);
}

// Group width of the streaming kernel (128 bytes of neighbouring systems).
template <typename R> int stream_width(long long n0) {
  (void)n0;
  return stream_w<R>();
}

// Window depth, d' placement and L2 prefetch distance by element type and
// chunk size, from measurements on 256^3 and 512^3 grids (fraction of the
// copy bandwidth, y / z):
//   FP64 M=16: D=4, prefetch 8 rows ahead: 0.99 / 0.77 (D=8 with d' in
//              shared memory spills registers: 0.82 / 0.58);
//   FP64 M=8:  D=8: 0.91 / 0.82 (D=4: 0.77 / 0.71);
//   FP32 M=16: D=4, prefetch 12 rows ahead: 0.87 / 0.71 (D=8 spills);
//   FP32 up to 256 rows: 16 chunks (two 512-thread CTAs per SM): 256^3
//              0.71 / 0.73 against 0.63 / 0.67 with 32 chunks of 8 rows.
// The prefetch is used only for y-like layouts (see launch_strided_stream).
template <typename R, int M> constexpr int stream_window() { return (sizeof(R) == 8 && M == 8) ? 8 : 4; }
template <typename R, int M> constexpr bool stream_sd() { return false; }
template <typename R, int M> constexpr int stream_prefetch() {
  return stream_window<R, M>() >= M ? 0 : sizeof(R) == 8 ? 8 : (M >= 16 ? 12 : M);
}

// Window of the promoted form (FP64 solve, FP32 coefficients: 5 registers
// a row in the window instead of 8).
template <int M> constexpr int promoted_window() { return M <= 8 ? M : 4; }
template <int M> constexpr bool promoted_sd() { return false; }

template <typename R, int M, bool INC, int ADJ, int PF, typename CR = R, int TC = 32>
static cudaError_t launch_stream_pf(const BatchArgs<R> &p, const AdjointOut<R> &q, cudaStream_t st,
                                    const CoefPtrs<CR> &cf = CoefPtrs<CR>{}) {
  constexpr int W = stream_w<R>();
  constexpr int BS = W * TC;
  // the adjoint's window holds 4 rows (an 8-row one spills with the
  // products); the promoted form has its own choice
  constexpr bool PROM = !std::is_same<CR, R>::value;
  constexpr int D = PROM ? promoted_window<M>()
                  : ADJ && stream_window<R, M>() > 4 ? 4 : stream_window<R, M>();
  constexpr bool SD = PROM ? promoted_sd<M>() : stream_sd<R, M>();
  const size_t red = ((size_t)6 * TC * (W + 1) * sizeof(R) + 15) / 16 * 16;
  const size_t smem = red + (size_t)(2 + (SD ? 1 : 0) + (INC || ADJ == 2 ? 1 : 0)) * M * BS * sizeof(R);
  auto kern = strided_stream_kernel<R, M, D, SD, PF, INC, ADJ, CR, TC>;
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
  kern<<<(unsigned)grid, BS, smem, st>>>(p, q, cf, ngx, ngroups);
  return cudaGetLastError();
}

template <typename R, int M, bool INC>
cudaError_t launch_strided_stream(const BatchArgs<R> &p, const Plan &plan, cudaStream_t st) {
  if ((plan.T != 32 && plan.T != 16) || plan.W != stream_w<R>() || p.N > plan.T * M)
    return cudaErrorInvalidValue;
  constexpr int PF = stream_prefetch<R, M>();
  // L2 prefetch only where the rows of a system are less than 64 KiB apart
  const AdjointOut<R> none{};
  if (plan.T == 16) {
    // 16 chunks: FP32 forward solves of up to 256 rows (choose_plan)
    if constexpr (sizeof(R) == 4 && !INC && (M == 8 || M == 16)) {
      if (PF > 0 && p.stride * (long long)sizeof(R) < (1LL << 16))
        return launch_stream_pf<R, M, INC, 0, PF, R, 16>(p, none, st);
      return launch_stream_pf<R, M, INC, 0, 0, R, 16>(p, none, st);
    }
    return cudaErrorInvalidValue;
  }
  if (PF > 0 && p.stride * (long long)sizeof(R) < (1LL << 16))
    return launch_stream_pf<R, M, INC, 0, PF>(p, none, st);
  return launch_stream_pf<R, M, INC, 0, 0>(p, none, st);
}

// Promoted solve: FP64 arithmetic on FP32-stored coefficients (cf), p.a,
// p.b, p.c unused; 64 < N <= 32 M.
template <int M>
cudaError_t launch_strided_stream_promoted(const BatchArgs<double> &p, const CoefPtrs<float> &cf,
                                           cudaStream_t st) {
  if (p.N > 32 * M) return cudaErrorInvalidValue;
  const AdjointOut<double> none{};
  return launch_stream_pf<double, M, false, 0, 0, float>(p, none, st, cf);
}

// Adjoint: p.a, p.b, p.c the forward coefficients, p.d_in = w, p.d_out =
// dbar, p.u = the forward solution x; q the other gradients (any may be
// null). Same plan rules as the forward solve.
template <typename R, int M>
cudaError_t launch_strided_stream_adjoint(const BatchArgs<R> &p, const AdjointOut<R> &q,
                                          cudaStream_t st) {
  if (p.N > 32 * M) return cudaErrorInvalidValue;
  constexpr int PF = stream_prefetch<R, M>();
  const bool yl = PF > 0 && p.stride * (long long)sizeof(R) < (1LL << 16);
  if (q.abar || q.bbar || q.cbar) {
    if (yl) return launch_stream_pf<R, M, false, 2, PF>(p, q, st);
    return launch_stream_pf<R, M, false, 2, 0>(p, q, st);
  }
  if (yl) return launch_stream_pf<R, M, false, 1, PF>(p, q, st);
  return launch_stream_pf<R, M, false, 1, 0>(p, q, st);
}

#define INST_STREAM(R, M)                                                                       \
  template cudaError_t launch_strided_stream<R, M, false>(const BatchArgs<R> &, const Plan &,    \
                                                           cudaStream_t);                      \
  template cudaError_t launch_strided_stream<R, M, true>(const BatchArgs<R> &, const Plan &,     \
                                                          cudaStream_t);
#define INST_STREAM_ADJ(R, M)                                                                   \
  template cudaError_t launch_strided_stream_adjoint<R, M>(const BatchArgs<R> &,                  \
                                                           const AdjointOut<R> &, cudaStream_t);
INST_STREAM_ADJ(double, 4)
INST_STREAM_ADJ(double, 8)
INST_STREAM_ADJ(double, 16)
INST_STREAM_ADJ(float, 4)
INST_STREAM_ADJ(float, 8)
INST_STREAM_ADJ(float, 16)
INST_STREAM(double, 4)
INST_STREAM(double, 8)
INST_STREAM(double, 16)
INST_STREAM(float, 4)
INST_STREAM(float, 8)
INST_STREAM(float, 16)
template cudaError_t launch_strided_stream_promoted<4>(const BatchArgs<double> &,
                                                       const CoefPtrs<float> &, cudaStream_t);
template cudaError_t launch_strided_stream_promoted<8>(const BatchArgs<double> &,
                                                       const CoefPtrs<float> &, cudaStream_t);
template cudaError_t launch_strided_stream_promoted<16>(const BatchArgs<double> &,
                                                        const CoefPtrs<float> &, cudaStream_t);
template int stream_width<double>(long long);
template int stream_width<float>(long long);

}  // namespace trid
