// Strided batches (solvedim >= 1) of 64 < N <= 512 rows: the wide streaming
// kernel, groups of 256 bytes of neighbouring systems.
//
// Why wider groups: when the rows of a system are a whole plane apart (z
// solves), every row of a group is a separate memory segment on its own
// page, and the rate of such segments, not the bytes, limits the solve. An
// access probe with the solve's pattern (4 arrays read, 1 written, 512^3
// FP64, rows 2 MiB apart) measured 4.6-5.3 TB/s with 128-byte segments at
// any window depth and 6.5-6.8 TB/s with 256-byte ones.
//
// A 256-byte group of 512-row systems carries 384 KiB of elimination state
// (a', c', d' of every row), more than shared memory holds. So:
//   - a' and c' of every row go to tensor memory (TMEM, 128 lanes x 512
//     columns of 32 bits per SM): the CTA allocates all 512 columns once,
//     and each warp keeps its rows in its lane quarter (warp w: lanes
//     32 (w % 4) .. + 31, columns (w / 4) * 128 .. + 127, i.e. 128 32-bit
//     words per thread: 32 rows of a' and c' of one FP64 system or of two
//     FP32 systems);
//   - d' goes to the thread's private shared-memory slots;
//   - the chunk's top reduced row is accumulated in forward order during the
//     forward sweep (x_1 = P + Q x_0 + S x_{k+1} as rows k are eliminated), so
//     the parked state is read back once, by the back-substitution.
// A CTA (T warps, warp t = chunk t of every system of the group; lane l
// holds system l, and in FP32 a second system: l + 32, or in the paired form
// the adjacent systems 2l and 2l + 1, which share one address and one 8-byte
// access per array; so a 64-system FP32 group keeps the same bytes in flight
// as a 32-system FP64 one, with two independent recurrences per thread) is
// persistent and walks over groups; each thread streams its chunk's rows
// through a D-deep register window that runs on into the next group, so
// loads stay in flight across the reduced solve and the stores. The reduced
// systems are solved 32 at a time (once per system of a thread).
// A CTA of 16 chunks (512 threads) takes all 512 TMEM columns and runs alone
// on its SM (a dynamic shared memory request of at least 120 KiB); a CTA of
// 8 chunks (256 threads) takes 256 columns and runs two per SM (80-112 KiB
// each), so one CTA's reduced solve and back-substitution overlap the
// other's streaming. Either way the shared-memory request caps the CTAs per
// SM, so an allocation never waits for another CTA of this kernel. Every
// path through the kernel reaches the deallocation at its end.
//
// Inc variants load u block by block during the back-substitution (one
// block ahead, the first block before the reduced solve).
//
// Pivots are inverted with the hardware reciprocal estimate (FP64: refined
// by two Newton-Raphson steps), within one ulp of the correctly rounded
// reciprocal, as in the contiguous kernels: measured equal in FP64 and a
// little faster in FP32 (512^3 z Inc 0.658 -> 0.628 ms).
#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

#include "trid_internal.h"
#include "trid_tmem.cuh"

namespace trid {

namespace {

template <typename R> constexpr int wide_w() { return 256 / (int)sizeof(R); }
// systems per thread: 1 FP64, 2 FP32 (systems l and l + 32 of a 64-system
// group, or 2l and 2l + 1 in the paired form: two independent recurrences
// and the same bytes in flight)
template <typename R> constexpr int wide_s() { return wide_w<R>() / 32; }
// 32-bit TMEM columns per row: a' and c' of the thread's systems
template <typename R> constexpr int wide_cpr() { return 2 * wide_s<R>() * (int)sizeof(R) / 4; }
// rows per back-substitution block (one TMEM load of 32 columns; 16 for Inc)
template <typename R, bool INC> constexpr int wide_blk() { return (INC ? 16 : 32) / wide_cpr<R>(); }
constexpr int WIDE_SMEM_MIN = 120 * 1024;  // one CTA per SM
// two CTAs per SM: more than a third and at most half of the SM's 228 KiB
// (each CTA also holds 1 KiB of the system's)
constexpr int WIDE2_SMEM_MIN = 80 * 1024;
constexpr int WIDE2_SMEM_MAX = 112 * 1024;

// one row's a', c' (of the thread's S systems) into its lane at column taddr
template <typename R, int S>
__device__ __forceinline__ void tmem_put_row(uint32_t taddr, const R (&af)[S], const R (&cf)[S]) {
  if constexpr (sizeof(R) == 8) {
    static_assert(S == 1, "one FP64 system per thread");
    asm volatile("tcgen05.st.sync.aligned.32x32b.x4.b32 [%0], {%1, %2, %3, %4};\n" ::"r"(taddr),
                 "r"(__double2loint(af[0])), "r"(__double2hiint(af[0])), "r"(__double2loint(cf[0])),
                 "r"(__double2hiint(cf[0]))
                 : "memory");
  } else {
    static_assert(S == 2, "two FP32 systems per thread");
    asm volatile("tcgen05.st.sync.aligned.32x32b.x4.b32 [%0], {%1, %2, %3, %4};\n" ::"r"(taddr),
                 "r"(__float_as_uint(af[0])), "r"(__float_as_uint(cf[0])), "r"(__float_as_uint(af[1])),
                 "r"(__float_as_uint(cf[1]))
                 : "memory");
  }
}

// a', c' of row i, system q of a block loaded by tmem_get (4 columns a row)
template <typename R, int S, int NW>
__device__ __forceinline__ void tmem_row(const uint32_t (&v)[NW], int i, int q, R &af, R &cf) {
  if constexpr (sizeof(R) == 8) {
    af = __hiloint2double((int)v[4 * i + 1], (int)v[4 * i]);
    cf = __hiloint2double((int)v[4 * i + 3], (int)v[4 * i + 2]);
  } else {
    af = __uint_as_float(v[4 * i + 2 * q]);
    cf = __uint_as_float(v[4 * i + 2 * q + 1]);
  }
}

// Row `row` at element offset o: identity rows outside the system, a[0] and
// c[N-1] forced to zero. Loads are cached in L2 only: nothing is read twice.
// CR: the coefficients' storage type; with CR = float and R = double (the
// promoted solve of tridDmtsvStridedBatchMixed) a, b, c are read from cf as
// FP32 and the solve runs in FP64 on their exact promoted values.
template <typename R, typename CR>
__device__ __forceinline__ void wide_load_row(const BatchArgs<R> &p, const CoefPtrs<CR> &cf, long long o,
                                              bool valid, int row, R &a, R &b, R &c, R &d) {
  if (valid) {
    if constexpr (std::is_same<CR, R>::value) {
      a = row == 0 ? R(0) : __ldcg(p.a + o);
      c = row == p.N - 1 ? R(0) : __ldcg(p.c + o);
      b = __ldcg(p.b + o);
    } else {
      a = row == 0 ? R(0) : R(__ldcg(cf.a + o));
      c = row == p.N - 1 ? R(0) : R(__ldcg(cf.c + o));
      b = R(__ldcg(cf.b + o));
    }
    d = __ldcg(p.d_in + o);
  } else {
    a = R(0);
    b = R(1);
    c = R(0);
    d = R(0);
  }
}

// The rows of two adjacent FP32 systems (PAIR: o even, pointers 8-byte
// aligned) in one 8-byte load per array; same rules as wide_load_row.
__device__ __forceinline__ void wide_load_pair(const BatchArgs<float> &p, long long o, bool valid, int row,
                                               float &a0, float &a1, float &b0, float &b1, float &c0,
                                               float &c1, float &d0, float &d1) {
  if (valid) {
    float2 v;
    if (row == 0) {
      a0 = a1 = 0.f;
    } else {
      v = __ldcg(reinterpret_cast<const float2 *>(p.a + o));
      a0 = v.x;
      a1 = v.y;
    }
    if (row == p.N - 1) {
      c0 = c1 = 0.f;
    } else {
      v = __ldcg(reinterpret_cast<const float2 *>(p.c + o));
      c0 = v.x;
      c1 = v.y;
    }
    v = __ldcg(reinterpret_cast<const float2 *>(p.b + o));
    b0 = v.x;
    b1 = v.y;
    v = __ldcg(reinterpret_cast<const float2 *>(p.d_in + o));
    d0 = v.x;
    d1 = v.y;
  } else {
    a0 = a1 = c0 = c1 = d0 = d1 = 0.f;
    b0 = b1 = 1.f;
  }
}

}  // namespace

// PAIR (FP32): thread l of a warp holds systems 2l and 2l + 1 of the group,
// adjacent in memory, so one address and one 8-byte access serve both rows
// (the launcher's choice when systems are contiguous along the fastest
// dimension, whole groups, and every offset even).
template <typename R, int M, int T, int D, bool INC, typename CR = R, int CTAS = 1, bool PAIR = false>
__global__ void __launch_bounds__(32 * T, CTAS)
    strided_wide_kernel(const BatchArgs<R> p, const CoefPtrs<CR> coef, long long ngx, long long ngroups) {
  static_assert(std::is_same<CR, R>::value || !INC, "the promoted form has no Inc");
  static_assert(!PAIR || (sizeof(R) == 4 && std::is_same<CR, R>::value), "pairs of FP32 systems");
  constexpr int S = wide_s<R>();  // systems per thread: lanes l and l + 32 of the group (2l, 2l + 1 PAIR)
  constexpr int W = wide_w<R>();  // = 32 * S
  constexpr int BS = 32 * T;
  constexpr int NWARP = BS / 32;
  constexpr int NCOL = 512 / CTAS;       // TMEM columns of the CTA
  constexpr int CW = NCOL / (NWARP / 4);  // TMEM columns per warp
  constexpr int CPR = wide_cpr<R>();     // columns per row (a', c' of S systems)
  // back-substitution blocks of 16 columns under a deep window
  constexpr int BK = D >= 8 ? 16 / CPR : wide_blk<R, INC>();
  constexpr int B = BK < M ? BK : M;
  constexpr int NV = B * CPR;
  static_assert(NV == 16 || NV == 32, "one TMEM load per block");
  static_assert(NWARP % 4 == 0, "whole lane quarters");
  static_assert(M * CPR <= CW, "a' and c' of a chunk fit the warp's TMEM columns");
  static_assert(M % B == 0 && M % D == 0 && D <= M && M >= 4, "blocks and window tile the chunk");
  // reduced rows of one half-group (32 systems) at a time
  constexpr int RED = (6 * T * 33 * (int)sizeof(R) + 15) / 16 * 16 / (int)sizeof(R);
  extern __shared__ __align__(16) unsigned char wide_smem[];
  __shared__ uint32_t tmem_slot;
  R *red = reinterpret_cast<R *>(wide_smem);
  const int tid = threadIdx.x;
  // d' of row j, system q at [(j * S + q) * BS]; PAIR: both systems' d' as
  // one 8-byte slot [j * BS] of sdf2
  R *sdf = red + RED + tid;
  float2 *sdf2 = reinterpret_cast<float2 *>(red + RED) + tid;
  const int lane = tid & 31;
  const int t = tid >> 5;    // chunk = warp
  const int warp = t;
  const int N = p.N;
  const int row0 = t * M;
  const long long stride = p.stride;

  if (warp == 0) tmem_alloc_cols<NCOL>(&tmem_slot);
  tmem_fence_before_sync();
  __syncthreads();
  tmem_fence_after_sync();
  const uint32_t tbase = tmem_slot;
  const uint32_t taddr = tbase + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)((warp >> 2) * CW);

  // element offset of system q's first chunk row in group g (0 if none)
  auto group_first = [&](long long g, int q, bool &act) -> long long {
    const long long gx = g % ngx;
    const long long i1 = g / ngx;
    const long long i0 = gx * W + (PAIR ? 2 * lane + q : 32 * q + lane);
    act = g < ngroups && i0 < p.n0;
    return act ? i0 * p.st0 + i1 * p.st1 + (long long)row0 * stride : 0;
  };

  R pa[S][D], pb[S][D], pc[S][D], pd[S][D];
  long long g = blockIdx.x;
  bool act[S];
  long long first[S], lo[S];
#pragma unroll
  for (int q = 0; q < S; ++q) {
    first[q] = group_first(g, q, act[q]);
    lo[q] = first[q];
  }
  // rows of every system of the thread into window slot k
  auto load_rows = [&](int k, const long long (&off)[S], const bool (&act_)[S], int row) {
    if constexpr (PAIR) {
      wide_load_pair(p, off[0], act_[0] && row < N, row, pa[0][k], pa[1][k], pb[0][k], pb[1][k],
                     pc[0][k], pc[1][k], pd[0][k], pd[1][k]);
    } else {
#pragma unroll
      for (int q = 0; q < S; ++q)
        wide_load_row<R, CR>(p, coef, off[q], act_[q] && row < N, row, pa[q][k], pb[q][k], pc[q][k],
                             pd[q][k]);
    }
  };
#pragma unroll
  for (int j = 0; j < D; ++j) {
    load_rows(j, lo, act, row0 + j);
#pragma unroll
    for (int q = 0; q < S; ++q) lo[q] += stride;
  }

  bool bad = false;
  R racc = R(0);  // pivot_acc of the sweep's pivots
  for (; g < ngroups; g += gridDim.x) {
    bool actn[S];
    long long firstn[S], ln[S];
#pragma unroll
    for (int q = 0; q < S; ++q) {
      firstn[q] = group_first(g + gridDim.x, q, actn[q]);
      ln[q] = firstn[q];
    }

    // forward half of the chunk elimination, streamed row by row; the top
    // reduced row accumulates as x_1 = P + Q x_0 + Sg x_{j+1}
    R ap[S], cp[S], dp[S], a0[S], c0[S], d0[S], P[S], Q[S], Sg[S];
#pragma unroll
    for (int q = 0; q < S; ++q) {
      ap[q] = cp[q] = dp[q] = a0[q] = c0[q] = d0[q] = P[q] = Q[q] = R(0);
      Sg[q] = R(1);
    }
#pragma unroll
    for (int j = 0; j < M; ++j) {
      const int k = j % D;
      R af[S], cfr[S], a_[S], b_[S], c_[S], d_[S], df_[S];
#pragma unroll
      for (int q = 0; q < S; ++q) {
        a_[q] = pa[q][k];
        b_[q] = pb[q][k];
        c_[q] = pc[q][k];
        d_[q] = pd[q][k];
      }
      if (j + D < M) {
        load_rows(k, lo, act, row0 + j + D);
#pragma unroll
        for (int q = 0; q < S; ++q) lo[q] += stride;
      } else {
        load_rows(k, ln, actn, row0 + j + D - M);
#pragma unroll
        for (int q = 0; q < S; ++q) ln[q] += stride;
      }
#pragma unroll
      for (int q = 0; q < S; ++q) {
        const R a = a_[q], b = b_[q], c = c_[q], d = d_[q];
        R df;
        if (j < 2) {
          const R r = rcp_nr(b);
          pivot_acc(racc, r);
          af[q] = a * r;
          cfr[q] = c * r;
          df = d * r;
        } else {
          const R r = rcp_nr(b - a * cp[q]);
          pivot_acc(racc, r);
          df = r * (d - a * dp[q]);
          af[q] = -r * a * ap[q];
          cfr[q] = r * c;
        }
        if constexpr (!PAIR) sdf[(j * S + q) * BS] = df;
        df_[q] = df;
        if (j == 0) {
          a0[q] = af[q];
          c0[q] = cfr[q];
          d0[q] = df;
        } else if (j <= M - 2) {
          P[q] += Sg[q] * df;
          Q[q] -= Sg[q] * af[q];
          Sg[q] = -Sg[q] * cfr[q];
        }
        ap[q] = af[q];
        cp[q] = cfr[q];
        dp[q] = df;
      }
      if constexpr (PAIR) sdf2[j * BS] = make_float2(df_[0], df_[S - 1]);
      tmem_put_row<R, S>(taddr + (uint32_t)(j * CPR), af, cfr);
    }

    // Inc: u of the last block, in flight during the reduced solve
    long long o[S];
    R ucur[S][INC ? B : 1], unext[S][INC ? B : 1];
#pragma unroll
    for (int q = 0; q < S; ++q) o[q] = first[q] + (long long)(M - 1) * stride;
    // u of rows jo - back - i (i < B) into us, o[] being at row jo
    auto load_u = [&](R (&us)[S][INC ? B : 1], int jo, int back) {
      if constexpr (INC) {
#pragma unroll
        for (int i = 0; i < B; ++i) {
          const int j = jo - back - i;
          if constexpr (PAIR) {
            float2 v = make_float2(0.f, 0.f);
            if (act[0] && row0 + j < N)
              v = __ldcg(reinterpret_cast<const float2 *>(p.u + o[0] - (long long)(back + i) * stride));
            us[0][i] = v.x;
            us[1][i] = v.y;
          } else {
#pragma unroll
            for (int q = 0; q < S; ++q)
              us[q][i] =
                  (act[q] && row0 + j < N) ? __ldcg(p.u + o[q] - (long long)(back + i) * stride) : R(0);
          }
        }
      }
    };
    load_u(ucur, M - 1, 0);
    tmem_wait_st();
    R y[S], z[S];
#pragma unroll
    for (int q = 0; q < S; ++q) {
      const R r0 = rcp(R(1) + c0[q] * Q[q]);
      bad |= !finite_rcp(r0);
      const Row<R> top{r0 * a0[q], r0 * c0[q] * Sg[q], r0 * (d0[q] - c0[q] * P[q])};
      const Row<R> bot{ap[q], cp[q], dp[q]};
      block_reduced_solve<R, 2>(red, top, bot, lane, t, T, 32, y[q], z[q], bad);
    }

    // back-substitution with the parked rows, block by block from the
    // chunk's last row up, stored as it goes
    R x[S];
#pragma unroll
    for (int q = 0; q < S; ++q) x[q] = z[q];
#pragma unroll
    for (int bb = M / B - 1; bb >= 0; --bb) {
      uint32_t v[NV];
      tmem_get(taddr + (uint32_t)(bb * B * CPR), v);
      // o[] is at row bb * B + B - 1 here: the next block starts B rows up
      if constexpr (INC) {
        if (bb > 0) load_u(unext, bb * B + B - 1, B);
      }
      tmem_wait_ld(v);
#pragma unroll
      for (int i = B - 1; i >= 0; --i) {
        const int j = bb * B + i;
        R dj[S];
        if (j > 0 && j < M - 1) {
          if constexpr (PAIR) {
            const float2 dv = sdf2[j * BS];
            dj[0] = dv.x;
            dj[S - 1] = dv.y;
          } else {
#pragma unroll
            for (int q = 0; q < S; ++q) dj[q] = sdf[(j * S + q) * BS];
          }
        }
#pragma unroll
        for (int q = 0; q < S; ++q) {
          if (j < M - 1) {
            if (j == 0) {
              x[q] = y[q];
            } else {
              R af, cfq;
              tmem_row<R, S, NV>(v, i, q, af, cfq);
              x[q] = dj[q] - af * y[q] - cfq * x[q];
            }
          }
        }
        if constexpr (PAIR) {
          if (act[0] && row0 + j < N) {
            float2 xv = make_float2(x[0], x[S - 1]);
            if constexpr (INC) {
              xv.x += ucur[0][B - 1 - i];
              xv.y += ucur[S - 1][B - 1 - i];
              *reinterpret_cast<float2 *>(p.u + o[0]) = xv;
            } else {
              *reinterpret_cast<float2 *>(p.d_out + o[0]) = xv;
            }
          }
        } else {
#pragma unroll
          for (int q = 0; q < S; ++q) {
            if (act[q] && row0 + j < N) {
              if constexpr (INC)
                p.u[o[q]] = ucur[q][B - 1 - i] + x[q];
              else
                p.d_out[o[q]] = x[q];
            }
          }
        }
#pragma unroll
        for (int q = 0; q < S; ++q) o[q] -= stride;
      }
      if constexpr (INC) {
#pragma unroll
        for (int q = 0; q < S; ++q)
#pragma unroll
          for (int i = 0; i < B; ++i) ucur[q][i] = unext[q][i];
      }
    }
#pragma unroll
    for (int q = 0; q < S; ++q) {
      first[q] = firstn[q];
      act[q] = actn[q];
      lo[q] = ln[q];
    }
  }
  bad |= racc != racc;
  report_bad_pivot(bad, p.flag);

  tmem_fence_before_sync();
  __syncthreads();
  tmem_fence_after_sync();
  if (warp == 0) tmem_dealloc_cols<NCOL>(tbase);
}

template <typename R> int wide_width() { return wide_w<R>(); }

// FP32 batches that take the paired form: systems contiguous along the
// fastest dimension, whole groups, even offsets and 8-byte aligned arrays.
template <typename R> bool wide_pairs(const BatchArgs<R> &p) {
  if (sizeof(R) != 4) return false;
  auto al8 = [](const void *q) { return (reinterpret_cast<uintptr_t>(q) & 7u) == 0; };
  return p.st0 == 1 && p.n0 % wide_w<R>() == 0 && p.st1 % 2 == 0 && p.stride % 2 == 0 && al8(p.a) &&
         al8(p.b) && al8(p.c) && al8(p.d_in) && al8(p.d_out) && (!p.u || al8(p.u));
}

// Chunks (warps) per system and rows per chunk for a system of N rows
// (64 < N <= 512; 0 if none), `pairs` when the batch takes the paired form.
//   - Systems of up to 256 rows: 8 chunks of up to 32 rows, 256-thread CTAs
//     with 256 TMEM columns each, two per SM (FP64 256^3 z: 0.129 -> 0.114
//     ms against 16 chunks of 16 rows at one CTA per SM);
//   - paired FP32 systems of 129-256 rows: 16 chunks of 16 rows, one CTA
//     per SM with an 8-row window (fraction of the copy bandwidth at 256^3,
//     y / y Inc / z / z Inc: 0.83 / 0.85 / 0.82 / 0.83, against 0.81 / 0.81
//     / 0.79 / 0.78 with two CTAs of 8 chunks: 1024 groups fill 6.9 rounds
//     of 148 CTAs but only 3.5 of 296, and the deeper window pays for the
//     reduced solve that no second CTA overlaps);
//   - longer systems: 16 chunks of 32 rows, one 512-thread CTA per SM.
template <typename R> int wide_chunks(int N, bool pairs) {
  if (N <= 64 || N > 512) return 0;
  return N > 256 || (pairs && N > 128) ? 16 : 8;
}
template <typename R> int wide_rows_per_thread(int N, bool pairs) {
  if (N <= 64 || N > 512) return 0;
  if (N <= 128) return 16;
  return N <= 256 && pairs ? 16 : 32;
}

template <typename R, int M, int T, bool INC, typename CR = R>
static cudaError_t launch_wide_m(const BatchArgs<R> &p, cudaStream_t st,
                                 const CoefPtrs<CR> &cf = CoefPtrs<CR>{}) {
  constexpr int W = wide_w<R>();
  constexpr int BS = 32 * T;
  constexpr int CTAS = T == 8 ? 2 : 1;
  // (the 8-row window is for the paired FP32 form; unpaired it spills)
  constexpr int D = (sizeof(R) == 4 && T == 16 && M == 16) ? 8 : 4;
  const size_t red = ((size_t)6 * T * 33 * sizeof(R) + 15) / 16 * 16;
  size_t smem = red + (size_t)M * wide_s<R>() * BS * sizeof(R);
  // the shared-memory request caps the CTAs per SM at CTAS, so every CTA's
  // TMEM allocation is granted without waiting
  const size_t smem_min = CTAS == 2 ? WIDE2_SMEM_MIN : WIDE_SMEM_MIN;
  if (smem < smem_min) smem = smem_min;
  if (CTAS == 2 && smem > WIDE2_SMEM_MAX) return cudaErrorInvalidValue;
  void (*kern)(const BatchArgs<R>, const CoefPtrs<CR>, long long, long long) = nullptr;
  if constexpr (D == 8) {
    // (wide_chunks gives this shape to the paired form only)
    if (!wide_pairs<R>(p)) return cudaErrorInvalidValue;
    kern = strided_wide_kernel<R, M, T, D, INC, CR, CTAS, true>;
  } else {
    kern = strided_wide_kernel<R, M, T, D, INC, CR, CTAS>;
    if constexpr (sizeof(R) == 4 && std::is_same<CR, R>::value) {
      if (wide_pairs<R>(p)) kern = strided_wide_kernel<R, M, T, D, INC, CR, CTAS, true>;
    }
  }
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const long long ngx = (p.n0 + W - 1) / W;
  const long long ngroups = ngx * (p.nsys / p.n0);
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const long long cap = (long long)sms * CTAS;
  const long long grid = ngroups < cap ? ngroups : cap;
  kern<<<(unsigned)grid, BS, smem, st>>>(p, cf, ngx, ngroups);
  return cudaGetLastError();
}

template <typename R, bool INC, typename CR = R>
static cudaError_t launch_wide_n(const BatchArgs<R> &p, cudaStream_t st,
                                 const CoefPtrs<CR> &cf = CoefPtrs<CR>{}) {
  bool pairs = false;
  if constexpr (std::is_same<CR, R>::value) pairs = wide_pairs<R>(p);
  const int T = wide_chunks<R>(p.N, pairs), M = wide_rows_per_thread<R>(p.N, pairs);
  if (T == 8 && M == 16) return launch_wide_m<R, 16, 8, INC, CR>(p, st, cf);
  if (T == 8 && M == 32) return launch_wide_m<R, 32, 8, INC, CR>(p, st, cf);
  if (T == 16 && M == 32) return launch_wide_m<R, 32, 16, INC, CR>(p, st, cf);
  if constexpr (sizeof(R) == 4 && std::is_same<CR, R>::value) {
    if (T == 16 && M == 16) return launch_wide_m<R, 16, 16, INC, CR>(p, st, cf);
  }
  return cudaErrorInvalidValue;
}

template <typename R, bool INC>
cudaError_t launch_strided_wide(const BatchArgs<R> &p, cudaStream_t st) {
  return launch_wide_n<R, INC>(p, st);
}

// Promoted solve: FP64 arithmetic on FP32-stored coefficients (cf), p.a,
// p.b, p.c unused; 64 < N <= 512.
cudaError_t launch_strided_wide_promoted(const BatchArgs<double> &p, const CoefPtrs<float> &cf,
                                         cudaStream_t st) {
  return launch_wide_n<double, false, float>(p, st, cf);
}

template cudaError_t launch_strided_wide<double, false>(const BatchArgs<double> &, cudaStream_t);
template cudaError_t launch_strided_wide<double, true>(const BatchArgs<double> &, cudaStream_t);
template cudaError_t launch_strided_wide<float, false>(const BatchArgs<float> &, cudaStream_t);
template cudaError_t launch_strided_wide<float, true>(const BatchArgs<float> &, cudaStream_t);
template int wide_width<double>();
template int wide_width<float>();
template int wide_rows_per_thread<double>(int, bool);
template int wide_rows_per_thread<float>(int, bool);
template int wide_chunks<double>(int, bool);
template bool wide_pairs<double>(const BatchArgs<double> &);
template bool wide_pairs<float>(const BatchArgs<float> &);
template int wide_chunks<float>(int, bool);

}  // namespace trid
