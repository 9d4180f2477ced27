/*
 * tridsolver_b200 — the drop-in batched scalar tridiagonal C ABI.
 *
 * The four entry points replace, symbol for symbol, the reference's
 * scalar/include/tridsolver.h:39-69 (implemented for the GPU in
 * scalar/src/cuda/trid_cuda.cu:419-454 and for the CPU in
 * scalar/src/cpu/trid_cpu.cpp:459-524). A program linked against
 * libtridcuda links against libtridsolver_b200 instead, unchanged.
 *
 * Problem: every line of an ndim-dimensional array along dimension
 * `solvedim` is one tridiagonal system
 *
 *     a[i] x[i-1] + b[i] x[i] + c[i] x[i+1] = d[i],   i = 0 .. N-1,
 *
 * with N = dims[solvedim]; a[0] and c[N-1] are never used (as in the
 * reference). Element (i0,i1,i2) lives at i0 + i1*pads[0] + i2*pads[0]*pads[1]
 * (x fastest), so `pads` describe padded allocations and a, b, c, d (, u) may
 * point at the first interior element of a padded array. Only elements inside
 * `dims` are read or written.
 *
 * Pointers are DEVICE pointers (cudaMalloc'd or managed). `dims` and `pads`
 * are host arrays of `ndim` ints, 1 <= ndim <= MAXDIM, 0 <= solvedim < ndim.
 *
 * By default each call is blocking, like the reference: it returns after the
 * solve has finished on the GPU (a stream synchronize, not a device-wide
 * one). tridSetStream / tridSetBlocking in tridsolver_b200.h make calls
 * asynchronous on a caller stream, which is what CUDA-graph capture needs.
 */
#ifndef TRIDSOLVER_H__
#define TRIDSOLVER_H__

#include "trid_common.h"
#include "trid_params.h"

/* x overwrites d.  Replaces scalar/include/tridsolver.h:39-42. */
EXTERN_C
tridStatus_t tridDmtsvStridedBatch(const TridParams *ctx, const double *a,
                                   const double *b, const double *c, double *d,
                                   int ndim, int solvedim, const int *dims,
                                   const int *pads);

/* x overwrites d.  Replaces scalar/include/tridsolver.h:44-48. */
EXTERN_C
tridStatus_t tridSmtsvStridedBatch(const TridParams *ctx, const float *a,
                                   const float *b, const float *c, float *d,
                                   int ndim, int solvedim, const int *dims,
                                   const int *pads);

/* u += x; d is read only.  Replaces scalar/include/tridsolver.h:57-62. */
EXTERN_C
tridStatus_t tridDmtsvStridedBatchInc(const TridParams *ctx, const double *a,
                                      const double *b, const double *c,
                                      double *d, double *u, int ndim,
                                      int solvedim, const int *dims,
                                      const int *pads);

/* u += x; d is read only.  Replaces scalar/include/tridsolver.h:64-69. */
EXTERN_C
tridStatus_t tridSmtsvStridedBatchInc(const TridParams *ctx, const float *a,
                                      const float *b, const float *c, float *d,
                                      float *u, int ndim, int solvedim,
                                      const int *dims, const int *pads);

#endif
