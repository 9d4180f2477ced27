// Tiles of a long contiguous system, one warp each: the building blocks
// shared by ragged batches (trid_ragged.cu) and the tiled long path
// (trid_long.cu).
//
// A tile is 32 chunks of tile_m rows (16 FP64, 32 FP32: 512 / 1024 rows, the
// same bytes, registers and shared memory either way), staged in shared
// memory by coalesced copies. Each lane runs the chunk elimination on its
// rows; the warp's reduced solve then runs for three right-hand sides: the
// tile's own, and the unit couplings to the unknown just before the tile
// (x_prev, the previous tile's last) and just after it (x_next, the next
// tile's first). Every reduced unknown of the tile is p + alpha x_prev +
// beta x_next, and the tile's first and last unknowns give it two rows of a
// second-level tridiagonal system over the tiles' first and last unknowns.
#pragma once

#include "trid_kernels.cuh"

namespace trid {

template <typename R> constexpr int tile_m() { return sizeof(R) == 8 ? 16 : 32; }
template <typename R> constexpr int tile_rows() { return 32 * tile_m<R>(); }

// The warp's reduced solve (as reduced_solve, 32 lanes) for three
// right-hand sides sharing the matrix: k = 0 the rows' own D; k = 1 only
// tD1 on the top row (lane 0: the coupling to the unknown before the
// tile); k = 2 only bD2 on the bottom row (lane 31: the coupling to the one
// after it).
template <typename R>
__device__ __forceinline__ void reduced_solve3(const Row<R> &top, const Row<R> &bot, R tD1, R bD2,
                                               int t, R (&y)[3], R (&z)[3], bool &bad) {
  constexpr int T = 32;
  const R tD[3] = {top.D, tD1, R(0)};
  const R bD[3] = {bot.D, R(0), bD2};
  R pA = shfl_up(bot.A, 1, T), pC = shfl_up(bot.C, 1, T);
  R de[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    R pD = shfl_up(bD[k], 1, T);
    if (t == 0) pD = R(0);
    de[k] = tD[k] - top.C * bD[k];
    de[k] -= top.A * pD;
  }
  if (t == 0) {
    pA = R(0);
    pC = R(0);
  }
  R al = -top.A * pA;
  const R be = R(1) - top.A * pC - top.C * bot.A;
  R ga = -top.C * bot.C;
  R r = rcp(be);
  bad |= !finite_rcp(r);
  al *= r;
  ga *= r;
#pragma unroll
  for (int k = 0; k < 3; ++k) de[k] *= r;
#pragma unroll
  for (int s = 1; s < T; s <<= 1) {
    R al_l = shfl_up(al, s, T), ga_l = shfl_up(ga, s, T);
    R al_r = shfl_down(al, s, T), ga_r = shfl_down(ga, s, T);
    R dl[3], dr[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      dl[k] = shfl_up(de[k], s, T);
      dr[k] = shfl_down(de[k], s, T);
    }
    if (t < s) {
      al_l = ga_l = R(0);
#pragma unroll
      for (int k = 0; k < 3; ++k) dl[k] = R(0);
    }
    if (t + s >= T) {
      al_r = ga_r = R(0);
#pragma unroll
      for (int k = 0; k < 3; ++k) dr[k] = R(0);
    }
    r = rcp(R(1) - al * ga_l - ga * al_r);
    bad |= !finite_rcp(r);
#pragma unroll
    for (int k = 0; k < 3; ++k) de[k] = (de[k] - al * dl[k] - ga * dr[k]) * r;
    al = -al * al_l * r;
    ga = -ga * ga_r * r;
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    y[k] = de[k];
    R yn = shfl_down(y[k], 1, T);
    if (t == T - 1) yn = R(0);
    z[k] = bD[k] - bot.A * y[k] - bot.C * yn;
  }
}

// chunk_forward (reciprocal estimates) with the diagonal read from the
// lane's staged row `brow` 16 bytes at a time as the sweep needs it, so b
// takes no registers beyond one vector.
template <typename R, int M>
__device__ __forceinline__ void chunk_forward_staged(R (&a)[M], const R *brow, R (&c)[M], R (&d)[M],
                                                     bool &bad) {
  using Vt = typename Vec16<R>::T;
  constexpr int n = Vec16<R>::n;
  static_assert(M % n == 0 && M >= 2, "whole vectors");
  const Vt *q = reinterpret_cast<const Vt *>(brow);
#pragma unroll
  for (int g = 0; g < M / n; ++g) {
    const Vt v = q[g];
    R bv[n];
    if constexpr (n == 2) {
      bv[0] = v.x;
      bv[1] = v.y;
    } else {
      bv[0] = v.x;
      bv[1] = v.y;
      bv[2] = v.z;
      bv[3] = v.w;
    }
#pragma unroll
    for (int k = 0; k < n; ++k) {
      const int i = g * n + k;
      if (i < 2) {
        const R r = rcp_nr(bv[k]);
        bad |= !finite_rcp(r);
        a[i] *= r;
        c[i] *= r;
        d[i] *= r;
      } else {
        const R r = rcp_nr(bv[k] - a[i] * c[i - 1]);
        bad |= !finite_rcp(r);
        d[i] = r * (d[i] - a[i] * d[i - 1]);
        a[i] = -r * a[i] * a[i - 1];
        c[i] = r * c[i];
      }
    }
  }
}

// Shared memory of one warp's tile: a, b, c, d in padded chunk rows (as
// contig_smem_kernel), d's rows reused for x on the way out.
// TM: rows per lane (tile_m by default).
template <typename R, int TM = tile_m<R>()> struct TileBuf {
  using L = SmemLayout<R, TM>;
  static constexpr int ELEMS = 4 * L::BUF;
  __device__ static __forceinline__ int slot(int e) { return (e / TM) * L::ROW + e % TM; }
};

// Copies rows [0, nt) of the tile starting at element `base` of a, b, c, d
// into the warp's buffer and makes the rows after nt identity rows. 16-byte cp.async units where
// the tile's start is 16-byte aligned (each unit lies inside one lane's
// chunk row, whose padded start is 16-byte aligned), element-sized copies
// otherwise (32 consecutive elements per instruction) and for the tail.
template <typename R, int TM = tile_m<R>()>
__device__ __forceinline__ void stage_tile_rows(const R *a, const R *b, const R *c, const R *d,
                                                bool vec16, long long base, int nt, R *buf,
                                                int lane) {
  using L = SmemLayout<R, TM>;
  using TB = TileBuf<R, TM>;
  constexpr int V = 16 / (int)sizeof(R);
  int e0 = 0;
  if (vec16 && base % V == 0) {
    const int nfull = nt / V;
#pragma unroll 4
    for (int u = lane; u < nfull; u += 32) {
      const int e = u * V;
      const int o = TB::slot(e);
      cp_async16(buf + 0 * L::BUF + o, a + base + e, 16);
      cp_async16(buf + 1 * L::BUF + o, b + base + e, 16);
      cp_async16(buf + 2 * L::BUF + o, c + base + e, 16);
      cp_async16(buf + 3 * L::BUF + o, d + base + e, 16);
    }
    e0 = nfull * V;
  }
#pragma unroll 4
  for (int e = e0 + lane; e < 32 * TM; e += 32) {
    const int o = TB::slot(e);
    if (e < nt) {
      cp_async_elem<R>(buf + 0 * L::BUF + o, a + base + e);
      cp_async_elem<R>(buf + 1 * L::BUF + o, b + base + e);
      cp_async_elem<R>(buf + 2 * L::BUF + o, c + base + e);
      cp_async_elem<R>(buf + 3 * L::BUF + o, d + base + e);
    } else {
      buf[0 * L::BUF + o] = R(0);
      buf[1 * L::BUF + o] = R(1);
      buf[2 * L::BUF + o] = R(0);
      buf[3 * L::BUF + o] = R(0);
    }
  }
  cp_async_wait_all();
  __syncwarp();
}

// The tile's two rows of the second-level system, from its first unknown
// f = pf + af x_prev + bf x_next and its last l = pl + al x_prev + bl x_next:
//   top  A l_{j-1} + f + C l = D        (x_next eliminated)
//   bot  A f + l + C f_{j+1} = D        (x_prev eliminated)
// The system's first tile (no x_prev) and last tile (no x_next), and tiles
// whose coupling vanishes (bl == 0: then bf == 0 too; af == 0: then al == 0),
// take the end-of-system forms.
template <typename R>
__device__ __forceinline__ void second_level_rows(R pf, R af, R bf, R pl, R al, R bl, bool first,
                                                  bool last, Row<R> &top, Row<R> &bot) {
  if (last || bl == R(0)) {
    top = Row<R>{-af, R(0), pf};
  } else {
    const R q = bf / bl;
    top = Row<R>{-af + q * al, -q, pf - q * pl};
  }
  if (first || af == R(0)) {
    bot = Row<R>{R(0), -bl, pl};
  } else {
    const R q = al / af;
    bot = Row<R>{-q, q * bf - bl, pl - q * pf};
  }
}

}  // namespace trid
