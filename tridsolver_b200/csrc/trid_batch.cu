// Plan selection and launchers of the batched solve kernels.
#include <cstdio>
#include <cstring>
#include <string>

#include "trid_internal.h"

namespace trid {

std::atomic<unsigned long long> g_launches{0};

std::string Plan::describe() const {
  char buf[96];
  const char *fam = family == TRID_FAMILY_PCR ? "pcr" : family == TRID_FAMILY_LONG ? "long" : "hybrid";
  snprintf(buf, sizeof(buf), "%s M=%d T=%d W=%d%s", fam, M, T, W,
           smem ? " smem" : vec ? " vec" : tma ? " tma" : wide ? (pairs ? " wide pairs" : " wide")
           : streaming ? " stream" : tiles ? " tiles" : "");
  return buf;
}

static int pow2_ceil(long long v) {
  int p = 1;
  while (p < v) p <<= 1;
  return p;
}

template <typename R>
bool vec_aligned(const BatchArgs<R> &p) {
  if (p.stride != 1) return false;
  auto al = [](const void *q) { return (reinterpret_cast<uintptr_t>(q) & 15u) == 0; };
  if (!al(p.a) || !al(p.b) || !al(p.c) || !al(p.d_in) || !al(p.d_out)) return false;
  if (p.u && !al(p.u)) return false;
  if ((p.st0 * (long long)sizeof(R)) % 16 || (p.st1 * (long long)sizeof(R)) % 16) return false;
  return true;
}

// Which hybrid shapes have kernels: contiguous batches keep a system inside
// one warp (T <= 32); strided batches re-deal the reduced rows through shared
// memory, so a system may span up to 128 chunks (KR = 2T/32 reduced rows per
// lane, instantiated for the M listed here).
static bool hybrid_supported(bool contig, int M, int T) {
  if (T <= 32) return true;
  if (contig) return false;
  if (T == 64) return M == 4 || M == 8 || M == 16;
  if (T == 128) return M == 4 || M == 8;
  return false;
}

// Built-in table of rows per thread by system length and layout, from
// measurements on 256^3 and 512^3 grids (the strided streaming kernels set
// their own rows per thread in choose_plan).
template <typename R>
static int default_m(int N, bool contig) {
  if (contig) {
    // FP32 systems of 129-256 rows: 16 lanes of 16 rows with 16-byte loads
    // (two systems per warp) measured faster than a warp per system staged
    // through shared memory (256^3 x: 0.055 vs 0.071 ms, tridAutotune)
    if (sizeof(R) == 4 && N > 128 && N <= 256) return 16;
    if (N <= 256) return 8;
    if (N <= 512) return 16;
    return 32;
  }
  if (sizeof(R) == 8) return 8;
  return N <= 256 ? 8 : 16;
}

template <typename R>
Plan choose_plan(const BatchArgs<R> &p, bool aligned16, bool honour_force) {
  Forces f;
  if (honour_force) {
    const Settings &st = settings();
    f.family = st.force_family;
    f.m = st.force_m;
    f.w = st.force_w;
    f.tma = st.force_tma;
    f.stream = st.force_stream;
  }
  // nothing forced: the autotuner's choice for this shape class, if any
  if (!f.any()) tuned_forces<R>(p, &f);
  return choose_plan_forced<R>(p, aligned16, f);
}

template <typename R>
Plan choose_plan_forced(const BatchArgs<R> &p, bool aligned16, const Forces &f) {
  Plan plan;
  const int N = p.N;
  const bool contig = p.stride == 1;
  int fam = f.family;
  int M = f.m;
  if (fam == TRID_FAMILY_PCR && N > 32) fam = TRID_FAMILY_HYBRID, M = 0;
  if (fam == TRID_FAMILY_PCR) {
    plan.family = fam;
    plan.M = 1;
    plan.T = pow2_ceil(N < 1 ? 1 : N);
    return plan;
  }
  // the long path needs a reduced system (2 rows per chunk) shorter than N
  if (fam == TRID_FAMILY_LONG && N <= 32) fam = TRID_FAMILY_HYBRID, M = 0;
  if (fam != TRID_FAMILY_LONG) {
    if (M == 0) M = default_m<R>(N, contig);
    const int T = pow2_ceil((N + M - 1) / M);
    if (hybrid_supported(contig, M, T) && (sizeof(R) == 4 || M <= 16 || contig == false)) {
      plan.family = TRID_FAMILY_HYBRID;
      plan.M = M;
      plan.T = T;
      if (contig) {
        plan.vec = aligned16 && ((M * (int)sizeof(R)) % 16 == 0);
        plan.smem = plan.vec && T == 32;
      } else {
        // at least 64 contiguous bytes per row: rows of a z solve are a whole
        // plane apart, and z throughput grows with the bytes per row access
        // rows a whole plane apart (>= 64 KiB: z solves) want 128 bytes per
        // row and per warp load, others 64 (measured, see the plan table)
        const int wseg = (p.stride * (long long)sizeof(R) >= (1LL << 16) ? 128 : 64) / (int)sizeof(R);
        int W = 256 / T > wseg ? 256 / T : wseg;
        const int wmin = 32 / T > 1 ? 32 / T : 1;
        const int n0p = pow2_ceil(p.n0);
        if (W > n0p) W = n0p;
        if (f.w > 0) W = f.w;
        if (W < wmin) W = wmin;
        const int tmax = (T > 32 || M * (int)sizeof(R) <= 64) ? 512 : 256;
        if (W * T > tmax) W = tmax / T;
        plan.W = W;
        // persistent streaming kernel for 64 < N <= 512: 128-byte row
        // segments, 512 threads (32 chunks of FP64 rows, 16 of FP32 rows)
        // and loads kept in flight across groups
        const int fs = f.stream;
        const bool want_tma = f.tma == 1;
        const int fm = f.m;
        // the wide form (256-byte groups, state in tensor memory), when at
        // least half a group holds systems, for
        //  - rows a whole plane apart (>= 64 KiB: z solves), where the rate
        //    of row segments limits 128-byte groups: FP64 512^3 z 0.87 vs
        //    1.22 ms, 256^3 0.114 vs 0.125 ms;
        //  - FP64 Inc solves along y (256^3: 0.151 vs 0.165 ms; 512^3 equal);
        //  - FP32 batches in the paired form (two adjacent systems a thread,
        //    8-byte accesses; wide_pairs): z solves (512^3 0.455 vs 0.656 ms,
        //    256^3 0.065 vs 0.071 ms), y solves of up to 256 rows (256^3
        //    0.063 vs 0.069 ms) and Inc y solves (512^3 0.545 vs 0.578 ms).
        //    Unpaired FP32 systems of up to 256 rows measured faster in
        //    128-byte groups, so unpaired FP32 takes it for z solves of
        //    over 256 rows only.
        // Along y without Inc the 128-byte form with L2 prefetch measured
        // faster otherwise (FP64 512^3 0.847 vs 0.871 ms, FP32 0.442 vs
        // 0.454 ms). Forced with tridForceStream(2) wherever it applies.
        const bool pairs = wide_pairs<R>(p);
        const int mw = wide_rows_per_thread<R>(N, pairs);
        const bool zlike = p.stride * (long long)sizeof(R) >= (1LL << 16);
        bool wide_auto;
        if (sizeof(R) == 8)
          wide_auto = zlike || p.u != nullptr;
        else if (pairs)
          wide_auto = zlike || N <= 256 || p.u != nullptr;
        else
          wide_auto = zlike && N > 256;
        if (mw > 0 && fm == 0 && !want_tma &&
            (fs == 2 || (fs == -1 && wide_auto && 2 * p.n0 >= wide_width<R>()))) {
          plan.M = mw;
          plan.T = wide_chunks<R>(N, pairs);  // chunks per system (one warp each)
          plan.W = wide_width<R>();
          plan.wide = true;
          plan.pairs = pairs;
          return plan;
        }
        const int Ts = 32;
        const int m_lo = 4;  // instantiated: 4, 8, 16
        const bool fm_ok = fm == 0 || ((fm == m_lo || fm == 2 * m_lo || fm == 4 * m_lo) && Ts * fm >= N);
        // (groups are always 128 bytes wide: automatic only when at least half
        // of a group holds systems)
        const int Ws = stream_width<R>(p.n0);
        if ((fs >= 1 || (fs == -1 && !want_tma && fm_ok && 2 * p.n0 >= Ws)) && N > 64 && N <= 512) {
          int Ms = N <= Ts * m_lo ? m_lo : N <= 2 * Ts * m_lo ? 2 * m_lo : 4 * m_lo;
          int Tsel = Ts;
          if (fm > 0 && fm_ok) {
            Ms = fm;
          } else if (sizeof(R) == 4 && !p.u && N <= 256) {
            // FP32 systems up to 256 rows: 16 chunks of up to 16 rows, a
            // 512-thread CTA that runs two per SM (the 32-chunk form runs
            // 1024 threads at the 64-register limit, one per SM)
            Tsel = 16;
            Ms = N <= 128 ? 8 : 16;
          }
          plan.M = Ms;
          plan.T = Tsel;
          plan.W = Ws;
          plan.streaming = true;
          return plan;
        }
        // TMA tiles (two stages when they fit), at most 256 threads per CTA.
        // Opt-in: with rows of 32-64 bytes the tile loads are limited by the
        // rate of box rows, and measure slower than per-thread loads.
        const int ft = f.tma;
        if (ft == 1 && (M == 8 || (M == 16 && sizeof(R) == 4)) && T <= 128) {
          const int wmin_tma = 16 / (int)sizeof(R);
          int wt = f.w > 0 ? f.w : 2 * wmin_tma;
          if (!(f.w > 0)) {
            // widest group (up to 16) that keeps two stages and covers n0
            for (int cand = wt * 2; cand <= 16; cand *= 2) {
              int rb, nb, stg;
              size_t sm;
              if (cand * T > 256 || cand > n0p) break;
              if (!tma_geometry<R>(p, p.u != nullptr, cand, rb, nb, stg, sm, T) || stg < 2) break;
              wt = cand;
            }
          }
          if (wt * T < 32) wt = 32 / T;
          int rb, nb, stg;
          size_t sm;
          if (wt * T <= 256 && tma_geometry<R>(p, p.u != nullptr, wt, rb, nb, stg, sm, T)) {
            plan.W = wt;
            plan.tma = true;
          }
        }
      }
      return plan;
    }
    M = 0;
  }
  plan.family = TRID_FAMILY_LONG;
  plan.M = (M == 8 || M == 16) ? M : 16;
  // contiguous systems: warp tiles staged by coalesced copies (trid_long.cu);
  // strided ones: chunks of M rows per thread
  plan.tiles = contig;
  return plan;
}

// ---------------------------------------------------------------------------

template <typename K>
static void allow_smem(K kernel, size_t bytes) {
  if (bytes > 48 * 1024) cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

template <typename R, int M, int KR, bool INC>
static cudaError_t launch_strided(const BatchArgs<R> &p, const Plan &plan, cudaStream_t st) {
  const int threads = plan.W * plan.T;
  const long long ngx = (p.n0 + plan.W - 1) / plan.W;
  const long long n1 = p.nsys / p.n0;
  const long long blocks = ngx * n1;
  const size_t smem = (size_t)6 * plan.T * (plan.W + 1) * sizeof(R);
  allow_smem(strided_kernel<R, M, KR, INC>, smem);
  strided_kernel<R, M, KR, INC><<<(unsigned)blocks, threads, smem, st>>>(p, plan.T, plan.W, ngx);
  return cudaSuccess;
}

template <typename R, int M, bool INC>
static cudaError_t launch_hybrid_m(const BatchArgs<R> &p, const Plan &plan, cudaStream_t st) {
  if (p.stride == 1) {
    const int threads = 128;
    const long long total = p.nsys * plan.T;
    const long long blocks = (total + threads - 1) / threads;
    if (plan.smem) {
      if constexpr ((M * sizeof(R)) % 16 == 0) {
        using L = SmemLayout<R, M>;
        const size_t smem = (size_t)(threads / 32) * (INC ? 5 : 4) * L::BUF * sizeof(R);
        allow_smem(contig_smem_kernel<R, M, INC>, smem);
        contig_smem_kernel<R, M, INC><<<(unsigned)blocks, threads, smem, st>>>(p);
      } else {
        return cudaErrorInvalidValue;
      }
    } else if (plan.vec) {
      if constexpr ((M * sizeof(R)) % 16 == 0) {
        contig_kernel<R, M, INC, true><<<(unsigned)blocks, threads, 0, st>>>(p, plan.T);
      } else {
        return cudaErrorInvalidValue;
      }
    } else {
      contig_kernel<R, M, INC, false><<<(unsigned)blocks, threads, 0, st>>>(p, plan.T);
    }
  } else if (plan.streaming) {
    cudaError_t e = cudaErrorInvalidValue;
    if constexpr (M == 4 || M == 8 || M == 16) e = launch_strided_stream<R, M, INC>(p, plan, st);
    if (e != cudaSuccess) return e;
  } else if (plan.tma) {
    cudaError_t e = cudaErrorInvalidValue;
    if constexpr (M == 8 || (M == 16 && sizeof(R) == 4)) {
      if (plan.T <= 32)
        e = launch_strided_tma<R, M, 2, INC>(p, plan, st);
      else if (plan.T == 64)
        e = launch_strided_tma<R, M, 4, INC>(p, plan, st);
      else if constexpr (M == 8) {
        if (plan.T == 128) e = launch_strided_tma<R, M, 8, INC>(p, plan, st);
      }
    }
    if (e != cudaSuccess) return e;
  } else {
    cudaError_t e = cudaErrorInvalidValue;
    if (plan.T <= 32) {
      e = launch_strided<R, M, 2, INC>(p, plan, st);
    } else if (plan.T == 64) {
      if constexpr (M == 4 || M == 8 || M == 16) e = launch_strided<R, M, 4, INC>(p, plan, st);
    } else if (plan.T == 128) {
      if constexpr (M == 4 || M == 8) e = launch_strided<R, M, 8, INC>(p, plan, st);
    }
    if (e != cudaSuccess) return e;
  }
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return cudaGetLastError();
}

template <typename R, bool INC>
static cudaError_t launch_hybrid(const BatchArgs<R> &p, const Plan &plan, cudaStream_t st) {
  switch (plan.M) {
    case 2: return launch_hybrid_m<R, 2, INC>(p, plan, st);
    case 4: return launch_hybrid_m<R, 4, INC>(p, plan, st);
    case 8: return launch_hybrid_m<R, 8, INC>(p, plan, st);
    case 16: return launch_hybrid_m<R, 16, INC>(p, plan, st);
    case 32: return launch_hybrid_m<R, 32, INC>(p, plan, st);
    default: return cudaErrorInvalidValue;
  }
}

template <typename R, bool INC>
static cudaError_t launch_pcr(const BatchArgs<R> &p, const Plan &plan, cudaStream_t st) {
  const int threads = 128;
  const long long total = p.nsys * plan.T;
  const long long blocks = (total + threads - 1) / threads;
  pcr_kernel<R, INC><<<(unsigned)blocks, threads, 0, st>>>(p, plan.T);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return cudaGetLastError();
}

template <typename R, int M, bool INC>
static cudaError_t launch_long_m(const BatchArgs<R> &p, cudaStream_t st) {
  const long long nc = ((long long)p.N + M - 1) / M;
  if (2 * nc >= p.N) return cudaErrorInvalidValue;  // would not shrink
  const long long nred = p.nsys * 2 * nc;
  R *scratch = nullptr;
  cudaError_t e = scratch_alloc((void **)&scratch, (size_t)nred * 4 * sizeof(R), st);
  if (e != cudaSuccess) return e;
  R *ra = scratch, *rb = ra + nred, *rc = rb + nred, *rd = rc + nred;
  const int threads = 128;
  const long long items = p.nsys * nc;
  const long long blocks = (items + threads - 1) / threads;
  long_reduce_kernel<R, M><<<(unsigned)blocks, threads, 0, st>>>(p, nc, ra, rb, rc, rd);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  e = cudaGetLastError();
  if (e == cudaSuccess) {
    BatchArgs<R> q{};
    q.a = ra;
    q.b = rb;
    q.c = rc;
    q.d_in = rd;
    q.d_out = rd;
    q.u = nullptr;
    q.N = (int)(2 * nc);
    q.nsys = p.nsys;
    q.n0 = p.nsys;
    q.st0 = 2 * nc;
    q.st1 = 0;
    q.stride = 1;
    q.flag = p.flag;
    // the reduced batch always takes the automatic plan: a forced family
    // applies to the caller's problem only
    Plan qp = choose_plan<R>(q, vec_aligned<R>(q), false);
    e = launch_batch<R, false>(q, qp, st);
  }
  if (e == cudaSuccess) {
    long_substitute_kernel<R, M, INC><<<(unsigned)blocks, threads, 0, st>>>(p, nc, rd);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    e = cudaGetLastError();
  }
  cudaError_t ef = scratch_free(scratch, st);
  return e != cudaSuccess ? e : ef;
}

template <typename R, bool INC>
cudaError_t launch_batch(const BatchArgs<R> &p, const Plan &plan, cudaStream_t st) {
  if (p.nsys <= 0 || p.N <= 0) return cudaSuccess;
  switch (plan.family) {
    case TRID_FAMILY_PCR: return launch_pcr<R, INC>(p, plan, st);
    case TRID_FAMILY_LONG:
      if (plan.tiles) return launch_long_tiles<R, INC>(p, st);
      return plan.M == 8 ? launch_long_m<R, 8, INC>(p, st) : launch_long_m<R, 16, INC>(p, st);
    default:
      if (plan.wide) {
        // rows per thread up to 64 (FP32), chosen inside the launcher
        const cudaError_t e = launch_strided_wide<R, INC>(p, st);
        if (e == cudaSuccess) g_launches.fetch_add(1, std::memory_order_relaxed);
        return e;
      }
      return launch_hybrid<R, INC>(p, plan, st);
  }
}

#define INSTANTIATE(R)                                                                  \
  template Plan choose_plan<R>(const BatchArgs<R> &, bool, bool);                           \
  template Plan choose_plan_forced<R>(const BatchArgs<R> &, bool, const Forces &);          \
  template bool vec_aligned<R>(const BatchArgs<R> &);                                 \
  template cudaError_t launch_batch<R, false>(const BatchArgs<R> &, const Plan &,     \
                                              cudaStream_t);                          \
  template cudaError_t launch_batch<R, true>(const BatchArgs<R> &, const Plan &, cudaStream_t);

INSTANTIATE(float)
INSTANTIATE(double)

}  // namespace trid
