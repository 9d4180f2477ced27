/*
 * ORACLE — test infrastructure only. Never linked into, loaded by or called
 * from the product library (tridsolver_b200); only tests/, the smoke check in
 * __graft_entry__.py and bench.py's CPU-baseline leg may use it, and only as
 * the checker (or the timed CPU baseline), never as the thing measured.
 *
 * A plain-C restatement of the reference CPU algorithm for the batched scalar
 * tridiagonal path of OP-DSL/tridsolver:
 *
 *   oracle_thomas_*         trid_scalar<REAL,INC>, scalar/src/cpu/trid_cpu.cpp:312-353
 *                           (reciprocal of the pivot, then multiply; a[0] and
 *                           c[N-1] do not influence the result)
 *   oracle_strided_batch_*  tridMultiDimBatchSolve<REAL,INC>,
 *                           scalar/src/cpu/trid_cpu.cpp:358-455 (system layout
 *                           i0 + i1*pads[0] + i2*pads[0]*pads[1], the stride of
 *                           dimension s is the product of pads below s)
 *   oracle_ragged_*         one trid_scalar per system of a ragged batch whose
 *                           system k occupies [offsets[k], offsets[k+1]); the
 *                           reference has no ragged entry, its exported
 *                           trid_scalarD/S (trid_cpu.cpp:477-482, 526-531) is
 *                           the per-system solve used here
 *   oracle_adjoint_d        the transposed solve T^T dbar = w done with the same
 *                           Thomas recurrence on (a', b', c') = (c shifted,
 *                           b, a shifted), then abar_i = -dbar_i x_{i-1},
 *                           bbar_i = -dbar_i x_i, cbar_i = -dbar_i x_{i+1}
 *   oracle_adi_*            one ADI heat step: 7-point RHS as in
 *                           apps/adi/src/preproc.hpp:173-214 with the
 *                           constant coefficients of the caller, then x and y
 *                           solves overwriting du and a z solve adding into u
 *                           (apps/adi/src/adi_cpu.cpp:209-270)
 *
 * Parity is pinned by tests/test_oracle.py against the golden fixtures that
 * the reference's own generator produced (tests/golden/make_golden.py) and
 * against the reference's CPU library compiled from its sources (oracle/_ref).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define DEFINE_THOMAS(NAME, REAL)                                              \
  /* Solve one system of length n whose rows are `stride` elements apart.     \
   * inc == 0: x overwrites d.  inc != 0: u += x and d is left untouched.      \
   * work must hold 2*n REALs. */                                              \
  static void NAME(const REAL *a, const REAL *b, const REAL *c, REAL *d,       \
                   REAL *u, long n, long stride, int inc, REAL *work) {        \
    if (n <= 0) return;                                                        \
    REAL *cp = work, *dp = work + n;                                           \
    REAL r = (REAL)1 / b[0];                                                   \
    cp[0] = r * c[0];                                                          \
    dp[0] = r * d[0];                                                          \
    for (long i = 1; i < n; ++i) {                                             \
      long k = i * stride;                                                     \
      REAL ai = a[k];                                                          \
      REAL piv = b[k] - ai * cp[i - 1];                                        \
      REAL rhs = d[k] - ai * dp[i - 1];                                        \
      r = (REAL)1 / piv;                                                       \
      cp[i] = r * c[k];                                                        \
      dp[i] = r * rhs;                                                         \
    }                                                                          \
    REAL x = dp[n - 1];                                                        \
    long k = (n - 1) * stride;                                                 \
    if (inc) u[k] += x; else d[k] = x;                                         \
    for (long i = n - 2; i >= 0; --i) {                                        \
      x = dp[i] - cp[i] * x;                                                   \
      k = i * stride;                                                          \
      if (inc) u[k] += x; else d[k] = x;                                       \
    }                                                                          \
  }

DEFINE_THOMAS(thomas_d, double)
DEFINE_THOMAS(thomas_f, float)

void oracle_thomas_d(const double *a, const double *b, const double *c,
                     double *d, double *u, long n, long stride, int inc) {
  double *w = (double *)malloc(sizeof(double) * 2 * (n > 0 ? n : 1));
  thomas_d(a, b, c, d, u, n, stride, inc, w);
  free(w);
}

void oracle_thomas_f(const float *a, const float *b, const float *c, float *d,
                     float *u, long n, long stride, int inc) {
  float *w = (float *)malloc(sizeof(float) * 2 * (n > 0 ? n : 1));
  thomas_f(a, b, c, d, u, n, stride, inc, w);
  free(w);
}

/* Returns 0 on success, 3 (TRID_STATUS_INVALID_VALUE) on a bad argument. */
#define DEFINE_BATCH(NAME, THOMAS, REAL)                                       \
  int NAME(const REAL *a, const REAL *b, const REAL *c, REAL *d, REAL *u,      \
           int inc, int ndim, int solvedim, const int *dims_in,                \
           const int *pads_in) {                                               \
    if (ndim < 1 || ndim > 3 || solvedim < 0 || solvedim >= ndim) return 3;    \
    long dims[3] = {1, 1, 1}, pads[3] = {1, 1, 1};                             \
    for (int i = 0; i < ndim; ++i) {                                           \
      dims[i] = dims_in[i];                                                    \
      pads[i] = pads_in[i];                                                    \
    }                                                                          \
    long stride[3] = {1, pads[0], pads[0] * pads[1]};                          \
    long n = dims[solvedim];                                                   \
    /* the two dimensions that enumerate systems */                            \
    int o0 = solvedim == 0 ? 1 : 0;                                            \
    int o1 = solvedim == 2 ? 1 : 2;                                            \
    long nsys = dims[o0] * dims[o1];                                           \
    if (n <= 0 || nsys <= 0) return 0;                                         \
    _Pragma("omp parallel")                                                    \
    {                                                                          \
      REAL *w = (REAL *)malloc(sizeof(REAL) * 2 * n);                          \
      _Pragma("omp for schedule(static)")                                      \
      for (long s = 0; s < nsys; ++s) {                                        \
        long i0 = s % dims[o0], i1 = s / dims[o0];                             \
        long base = i0 * stride[o0] + i1 * stride[o1];                         \
        THOMAS(a + base, b + base, c + base, d + base,                         \
               inc ? u + base : (REAL *)0, n, stride[solvedim], inc, w);       \
      }                                                                        \
      free(w);                                                                 \
    }                                                                          \
    return 0;                                                                  \
  }

DEFINE_BATCH(oracle_strided_batch_d, thomas_d, double)
DEFINE_BATCH(oracle_strided_batch_f, thomas_f, float)

#define DEFINE_RAGGED(NAME, THOMAS, REAL)                                      \
  int NAME(const REAL *a, const REAL *b, const REAL *c, REAL *d, REAL *u,      \
           int inc, const int64_t *offsets, long nsys) {                       \
    long nmax = 0;                                                             \
    for (long s = 0; s < nsys; ++s) {                                          \
      long n = (long)(offsets[s + 1] - offsets[s]);                            \
      if (n < 0) return 3;                                                     \
      if (n > nmax) nmax = n;                                                  \
    }                                                                          \
    _Pragma("omp parallel")                                                    \
    {                                                                          \
      REAL *w = (REAL *)malloc(sizeof(REAL) * 2 * (nmax > 0 ? nmax : 1));      \
      _Pragma("omp for schedule(dynamic, 64)")                                 \
      for (long s = 0; s < nsys; ++s) {                                        \
        long o = (long)offsets[s];                                             \
        long n = (long)(offsets[s + 1] - offsets[s]);                          \
        THOMAS(a + o, b + o, c + o, d + o, inc ? u + o : (REAL *)0, n, 1,      \
               inc, w);                                                        \
      }                                                                        \
      free(w);                                                                 \
    }                                                                          \
    return 0;                                                                  \
  }

DEFINE_RAGGED(oracle_ragged_d, thomas_d, double)
DEFINE_RAGGED(oracle_ragged_f, thomas_f, float)

/*
 * Adjoint of x = T^{-1} d for a batch along `solvedim`, given w = dL/dx and
 * the forward solution x.  T^T has sub-diagonal c[i-1], diagonal b[i] and
 * super-diagonal a[i+1]; solving T^T dbar = w gives dL/dd, and the partial
 * derivatives of the rows give dL/da, dL/db, dL/dc.  a[0] and c[N-1] do not
 * enter the forward map, so their gradients are zero.
 */
int oracle_adjoint_d(const double *a, const double *b, const double *c,
                     const double *x, const double *w, double *abar,
                     double *bbar, double *cbar, double *dbar, int ndim,
                     int solvedim, const int *dims_in, const int *pads_in) {
  if (ndim < 1 || ndim > 3 || solvedim < 0 || solvedim >= ndim) return 3;
  long dims[3] = {1, 1, 1}, pads[3] = {1, 1, 1};
  for (int i = 0; i < ndim; ++i) {
    dims[i] = dims_in[i];
    pads[i] = pads_in[i];
  }
  long stride[3] = {1, pads[0], pads[0] * pads[1]};
  long n = dims[solvedim];
  int o0 = solvedim == 0 ? 1 : 0;
  int o1 = solvedim == 2 ? 1 : 2;
  long nsys = dims[o0] * dims[o1];
  if (n <= 0 || nsys <= 0) return 0;
  long st = stride[solvedim];
#pragma omp parallel
  {
    double *at = (double *)malloc(sizeof(double) * 6 * n);
    double *bt = at + n, *ct = bt + n, *dt = ct + n, *work = dt + n;
#pragma omp for schedule(static)
    for (long s = 0; s < nsys; ++s) {
      long i0 = s % dims[o0], i1 = s / dims[o0];
      long base = i0 * stride[o0] + i1 * stride[o1];
      for (long i = 0; i < n; ++i) {
        long k = base + i * st;
        at[i] = i > 0 ? c[k - st] : 0.0;
        bt[i] = b[k];
        ct[i] = i < n - 1 ? a[k + st] : 0.0;
        dt[i] = w[k];
      }
      thomas_d(at, bt, ct, dt, (double *)0, n, 1, 0, work);
      for (long i = 0; i < n; ++i) {
        long k = base + i * st;
        double g = dt[i];
        dbar[k] = g;
        abar[k] = i > 0 ? -g * x[k - st] : 0.0;
        bbar[k] = -g * x[k];
        cbar[k] = i < n - 1 ? -g * x[k + st] : 0.0;
      }
    }
    free(at);
  }
  return 0;
}

/*
 * One ADI heat-diffusion step on an nx*ny*nz grid (x fastest, no padding)
 * with constant coefficients a = c = ca, b = cb on interior points and
 * identity rows (a = c = 0, b = 1, rhs = 0) on the Dirichlet boundary:
 *   du = lambda * (sum of the 6 neighbours - 6 u)        (interior)
 *   du <- solve_x(du); du <- solve_y(du); u += solve_z(du).
 * Follows apps/adi/src/preproc.hpp:173-214 and adi_cpu.cpp:209-270; the
 * coefficient values are parameters because callers choose them.
 */
#define DEFINE_ADI(NAME, BATCH, REAL)                                          \
  int NAME(REAL *u, REAL *du, REAL *ax, REAL *bx, REAL *cx, int nx, int ny,    \
           int nz, REAL lambda, REAL ca, REAL cb) {                            \
    long nxy = (long)nx * ny, n = nxy * nz;                                    \
    _Pragma("omp parallel for schedule(static)")                               \
    for (long k = 0; k < nz; ++k)                                              \
      for (long j = 0; j < ny; ++j)                                            \
        for (long i = 0; i < nx; ++i) {                                        \
          long ind = i + j * nx + k * nxy;                                     \
          int bnd = i == 0 || i == nx - 1 || j == 0 || j == ny - 1 ||          \
                    k == 0 || k == nz - 1;                                     \
          if (bnd) {                                                           \
            du[ind] = 0;                                                       \
            ax[ind] = 0;                                                       \
            bx[ind] = 1;                                                       \
            cx[ind] = 0;                                                       \
          } else {                                                             \
            du[ind] = lambda * (u[ind - 1] + u[ind + 1] + u[ind - nx] +        \
                                u[ind + nx] + u[ind - nxy] + u[ind + nxy] -    \
                                (REAL)6 * u[ind]);                             \
            ax[ind] = ca;                                                      \
            bx[ind] = cb;                                                      \
            cx[ind] = ca;                                                      \
          }                                                                    \
        }                                                                      \
    (void)n;                                                                   \
    int dims[3] = {nx, ny, nz};                                                \
    int rc = BATCH(ax, bx, cx, du, (REAL *)0, 0, 3, 0, dims, dims);            \
    if (!rc) rc = BATCH(ax, bx, cx, du, (REAL *)0, 0, 3, 1, dims, dims);       \
    if (!rc) rc = BATCH(ax, bx, cx, du, u, 1, 3, 2, dims, dims);               \
    return rc;                                                                 \
  }

DEFINE_ADI(oracle_adi_step_d, oracle_strided_batch_d, double)
DEFINE_ADI(oracle_adi_step_f, oracle_strided_batch_f, float)
