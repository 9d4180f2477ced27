/*
 * tridsolver_b200 — extensions beyond the reference's C ABI.
 *
 * Everything here is additive: the four reference entry points in
 * tridsolver.h keep their exact signatures and semantics. These functions
 * have no counterpart in scalar/include/tridsolver.h unless a line says so.
 */
#ifndef TRIDSOLVER_B200_H__
#define TRIDSOLVER_B200_H__

#include <stddef.h>
#include <stdint.h>

#include "tridsolver.h"

/* ---- execution control (per calling thread) ------------------------------
 * The reference runs every solve on the legacy default stream and ends each
 * call with cudaDeviceSynchronize (scalar/src/cuda/trid_cuda.cu:409-410).
 * Here a call runs on the calling thread's stream (default: the legacy
 * default stream, NULL) and, while blocking is on (the default), returns
 * after a cudaStreamSynchronize of that stream. With blocking off, calls only
 * enqueue work, so they can be captured into a CUDA graph. */
EXTERN_C tridStatus_t tridSetStream(void *cuda_stream); /* a cudaStream_t */
EXTERN_C void *tridGetStream(void);
EXTERN_C tridStatus_t tridSetBlocking(int blocking);
EXTERN_C int tridGetBlocking(void);

/* Zero / non-finite pivots seen on the current device since the last call
 * of this function (blocking calls also report them in their own status):
 * TRID_STATUS_ZERO_PIVOT or TRID_STATUS_SUCCESS. Clears the record. */
EXTERN_C tridStatus_t tridGetPivotStatus(void);

/* Number of kernels this library has launched in this process. */
EXTERN_C unsigned long long tridGetLaunchCount(void);

/* Returns the unused memory of the library's scratch pool on the current
 * device to the driver. Long systems and ragged batches take their scratch
 * from that pool, which otherwise keeps it between calls. Memory backing a
 * call still in flight is kept, and later calls refill the pool as needed.
 * Replaces nothing in the reference, whose scratch is static and never freed
 * (scalar/src/cuda/trid_cuda.cu:185-206). */
EXTERN_C tridStatus_t tridReleaseScratch(void);

/* on != 0: every solve call (the strided-batch, batched, ragged, ADI,
 * adjoint and mixed entry points) pushes an NVTX range named after itself
 * for its host-side duration, so Nsight Systems timelines and ncu
 * --nvtx-include filters can pick out the library's calls. Off by default,
 * or on from the first call when TRIDSOLVER_NVTX=1 is set in the
 * environment. Counterpart of the reference's NVTX profiling ranges
 * (BEGIN_PROFILING, scalar/include/cuda_timing.h:58-102), which are chosen
 * at build time there. */
EXTERN_C tridStatus_t tridSetTracing(int on);

/* ---- plan selection ------------------------------------------------------
 * Kernel families, chosen per system length by the built-in table or the
 * autotuner:
 *   TRID_FAMILY_HYBRID  partition hybrid: T threads per system, M rows per
 *                       thread, warp-shuffle PCR on the reduced system
 *                       (T = 1 is thread-per-system Thomas);
 *   TRID_FAMILY_PCR     pure PCR, one row per thread (systems <= 32 rows);
 *   TRID_FAMILY_LONG    multi-block partition for long systems: reduced
 *                       rows to scratch, recursive reduced solve, substitution.
 * tridForcePlan(family, M) pins the choice for the calling thread (testing and
 * tuning); family < 0 restores automatic selection. */
#define TRID_FAMILY_AUTO (-1)
#define TRID_FAMILY_HYBRID 0
#define TRID_FAMILY_PCR 1
#define TRID_FAMILY_LONG 2
EXTERN_C tridStatus_t tridForcePlan(int family, int rows_per_thread);

/* Autotuner. Counterpart of the reference's fixed Thomas-PCR length tables
 * (scalar/src/cuda/trid_thomaspcr.hpp:537-598), measured instead of fixed:
 * times every plan that applies to the given shape (pure PCR; the hybrid at
 * rows per thread 2..32, from thread-per-system Thomas to a warp per system;
 * for strided batches the register-tile kernel, the 128- and 256-byte
 * streaming kernels and TMA tiles; the long multi-block path) on synthetic
 * data of that shape allocated for the call (cudaMalloc; blocking, typically
 * well under a second), and keeps the fastest for the shape's class on the
 * current device: precision, Inc or not (inc != 0), layout (contiguous;
 * strided with rows under 64 KiB apart; strided with rows further apart),
 * whether at least 32 systems run along the fastest dimension, and the
 * length bucket ceil(log2 N). Later automatic plan choices for that class
 * use it (tridForce* settings still take precedence). *best_ms and plan
 * (a tridDescribePlan string, plan_len bytes) receive the winner when not
 * NULL. tridAutotuneReset forgets the current device's choices. */
EXTERN_C tridStatus_t tridAutotune(int dtype_bytes, int ndim, int solvedim, const int *dims,
                                   const int *pads, int inc, float *best_ms, char *plan,
                                   int plan_len);
EXTERN_C tridStatus_t tridAutotuneReset(void);

/* Pins the number of neighbouring systems one thread block of the strided
 * hybrid handles (a power of two; 0 restores the automatic choice). */
EXTERN_C tridStatus_t tridForceSystemsPerBlock(int systems);

/* Strided batches: 1 = load whole tiles with TMA (persistent, double
 * buffered) wherever the alignment and size rules allow; 0 or -1 (default) =
 * per-thread loads, which measure faster for rows of 32-64 bytes. */
EXTERN_C tridStatus_t tridForceTma(int mode);

/* Strided batches of 64 < N <= 512 rows: -1 (default) = automatic: the wide
 * streaming kernel (groups of 256 bytes of neighbouring systems, elimination
 * state parked in tensor memory) when rows are at least 64 KiB apart (z
 * solves), else the persistent streaming kernel (groups of 128 bytes, loads
 * kept in flight across groups), unless TMA is forced; 1 = the 128-byte
 * streaming kernel and 2 = the wide one, wherever they apply; 0 = the
 * register-tile strided kernel. */
EXTERN_C tridStatus_t tridForceStream(int mode);

/* ---- ragged batches -------------------------------------------------------
 * No counterpart in the reference. nsys independent contiguous systems of
 * uneven lengths: system k is rows [offsets[k], offsets[k+1]) of a, b, c, d
 * (device arrays; offsets: nsys+1 non-decreasing int64 on the device).
 * x overwrites d. Bucketed by length on the device, then solved in one
 * persistent launch of independent warps: short systems (up to 256 rows)
 * one per warp with a per-length-class rows-per-lane table (pure PCR up to
 * 32 rows, the partition hybrid beyond), longer ones cut into tiles of 512
 * rows, one warp per tile, joined by a second-level system of two rows per
 * tile (up to 16384 rows per system; a longer system makes a blocking call
 * return TRID_STATUS_MATRIX_TYPE_NOT_SUPPORTED). */
EXTERN_C tridStatus_t tridDmtsvRaggedBatch(const TridParams *ctx, const double *a, const double *b,
                                           const double *c, double *d, const int64_t *offsets,
                                           long long nsys);
EXTERN_C tridStatus_t tridSmtsvRaggedBatch(const TridParams *ctx, const float *a, const float *b,
                                           const float *c, float *d, const int64_t *offsets,
                                           long long nsys);
/* As above, with the batch's element count given by the caller: nelems >=
 * offsets[nsys] - offsets[0] (a larger count only sizes more scratch). The
 * call above reads those two offsets back to size its scratch, a
 * synchronisation; this one reads nothing back, so with blocking off it
 * only enqueues work and can be captured into a CUDA graph (its scratch
 * then comes from the graph's own allocation). A count below the batch's is
 * refused on the device before anything is written: d is left as it was
 * and a blocking call returns TRID_STATUS_INVALID_VALUE (a non-blocking
 * call cannot report it). nelems < 0 returns TRID_STATUS_INVALID_VALUE. */
EXTERN_C tridStatus_t tridDmtsvRaggedBatchSized(const TridParams *ctx, const double *a,
                                                const double *b, const double *c, double *d,
                                                const int64_t *offsets, long long nsys,
                                                long long nelems);
EXTERN_C tridStatus_t tridSmtsvRaggedBatchSized(const TridParams *ctx, const float *a,
                                                const float *b, const float *c, float *d,
                                                const int64_t *offsets, long long nsys,
                                                long long nelems);
/* Times, per length class up to one warp's worth of rows, every
 * rows-per-lane choice of a warp per system and the staged tile path, on
 * this device (uniform synthetic batches, about a second), and keeps the
 * fastest for later ragged calls of that precision on the current device.
 * Longer systems always take tiles (512 rows, N <= 16384). */
EXTERN_C tridStatus_t tridRaggedAutotune(int dtype_bytes);
/* Failure-detection hook (process-wide; tests only). A warp holding one tile
 * of a multi-tile system waits, bounded, for the warp that solves the
 * system's second-level system to publish it. polls sets that bound (each
 * poll sleeps about 128 ns; 0 restores the default of 2^22 polls, about half
 * a second); withhold_publish != 0 makes the solving warp withhold its
 * publication, so every such wait runs out. A wait that gives up leaves its
 * tile unsolved, stops the launch's other waits at once, and makes a
 * blocking ragged call return TRID_STATUS_EXECUTION_FAILED; the device
 * context stays usable and later calls solve normally once the hook is
 * reset. */
EXTERN_C tridStatus_t tridRaggedSetWaitBound(unsigned long long polls, int withhold_publish);

/* Copies the table in use (one entry per length class ceil(log2 N) = 0, 1,
 * ...: rows per lane of a warp per system, or 0 for tiles) and
 * returns the number of classes, or -1. */
EXTERN_C int tridRaggedTable(int dtype_bytes, int *rows_per_lane, int nclasses);

/* ---- distributed solve ---------------------------------------------------
 * Counterpart of the reference's MPI/NCCL build, which links the same four
 * strided-batch entry points (scalar/src/cuda/trid_cuda_mpi.cu:773-817) and
 * reads its distributed parameters from ctx->mpi_params (MpiSolverParams,
 * scalar/include/trid_mpi_solver_params.hpp:47-181). Every system is split
 * along solvedim over nranks ranks; each rank passes its own local block
 * (dims[solvedim] = its row count, at least 2) and rank is its position
 * along solvedim. The partition method with the reference's ALLGATHER
 * strategy: each rank reduces its segment of every system to two boundary
 * rows, the rows are all-gathered, every rank solves the reduced systems,
 * then its local segments. The exchange is the caller's allgather callback
 * (an NCCL all-gather over NVLink from torch.distributed, or any host code):
 *   allgather(send, recv, bytes_per_rank, user, cuda_stream)
 * must gather bytes_per_rank bytes of device memory at `send` from every
 * rank into `recv` in rank order (recv holds nranks * bytes_per_rank bytes),
 * ordered after the work enqueued on cuda_stream and before later work on
 * it; it returns 0 on success (non-zero makes the solve return
 * TRID_STATUS_EXECUTION_FAILED after releasing its scratch).
 * ctx->mpi_params is used only when it points at parameters registered by
 * tridDistInit (the pointer is compared, never dereferenced otherwise, so an
 * uninitialised mpi_params stays harmless as in the single-GPU library).
 * The reference's other strategies (Jacobi, PCR across ranks, latency
 * hiding by mini-batches) solve the same reduced system; this library
 * always gathers it whole (6 values per system and rank). */
typedef int (*tridAllgatherFn)(const void *send, void *recv, size_t bytes_per_rank, void *user,
                               void *cuda_stream);
typedef struct tridDistParams {
  int solvedim; /* the split dimension; calls along other dimensions are refused */
  int rank;     /* position along solvedim, 0 .. nranks - 1 */
  int nranks;
  tridAllgatherFn allgather;
  void *user;
} tridDistParams;
EXTERN_C tridStatus_t tridDistInit(tridDistParams *params, int solvedim, int rank, int nranks,
                                   tridAllgatherFn allgather, void *user);
EXTERN_C tridStatus_t tridDistFinalize(tridDistParams *params);
/* Bytes one rank contributes to the exchange of a call (6 values per
 * system), or -1 for invalid arguments. */
EXTERN_C long long tridDistExchangeBytes(int dtype_bytes, int ndim, int solvedim, const int *dims);

/* ---- ADI heat-diffusion timestep -----------------------------------------
 * No single counterpart in the reference: one timestep of its ADI
 * application (apps/adi/src/adi_cuda.cu:282-326, preproc.cu:40-90) on an
 * nx*ny*nz grid of device arrays (x fastest, no padding):
 *   du = lambda*(sum of 6 neighbours - 6u) inside, 0 on the boundary;
 *   a = c = -alpha*lambda, b = 1 + 2*alpha*lambda inside, identity rows on
 *   the boundary (alpha = 1: a = c = -lambda, b = 1 + 2*lambda; alpha = 0.5:
 *   the reference application's coefficients);
 *   du <- x solve; du <- y solve; u += z solve.
 * lambda = lam[*step] read on the device (lam[0] when step is NULL), and
 * *step += 1 at the end, so one captured CUDA graph of a timestep replays a
 * sequence of per-step lambdas. du is caller scratch of nx*ny*nz, and so are
 * a, b, c when given (the reference application's coefficient arrays: a
 * preprocessing kernel and three array solves, 21 words of memory traffic
 * per point). With a, b, c all NULL the coefficients stay three scalars:
 * each kernel factors the shared interior matrix once and sweeps only
 * right-hand sides, and the 7-point stencil is formed inside the x solve
 * (three kernels, 7 words per point; grids with an edge above 512 use the
 * array form on library scratch instead). */
EXTERN_C tridStatus_t tridDADIStep(double *u, double *du, double *a, double *b, double *c,
                                   const double *lam, int *step, double alpha, int nx, int ny,
                                   int nz);
EXTERN_C tridStatus_t tridSADIStep(float *u, float *du, float *a, float *b, float *c,
                                   const float *lam, int *step, float alpha, int nx, int ny,
                                   int nz);

/* Adjoint of one timestep of tridDADIStep / tridSADIStep (lambda = lam[0]:
 * pass lam + k for the k-th step), for differentiating a multi-step run:
 * given u (the step's input field, nx*ny*nz device array) and g = dL/du' (u'
 * the step's output), writes ubar = dL/du (a separate array) and adds
 * dL/dlambda to lambar[0] (a device scalar). The forward intermediates are
 * recomputed from u (the coefficient-array form of the step), then the three
 * transposed solves and the stencil transpose run, with the lambda
 * derivative reduced in FP64 on the device; the scratch (seven arrays of the
 * grid) comes from the library's pool. Edges up to 1024; no counterpart in
 * the reference. */
EXTERN_C tridStatus_t tridDADIStepAdjoint(const double *u, const double *g, double *ubar,
                                          double *lambar, const double *lam, double alpha, int nx,
                                          int ny, int nz);
EXTERN_C tridStatus_t tridSADIStepAdjoint(const float *u, const float *g, float *ubar,
                                          float *lambar, const float *lam, float alpha, int nx,
                                          int ny, int nz);

/* ---- adjoint ------------------------------------------------------------
 * No counterpart in the reference. For x = T^{-1} d solved along `solvedim`
 * (the forward call's arguments) and w = dL/dx, writes
 *   dbar = T^{-T} w,  abar_i = -dbar_i x_{i-1},  bbar_i = -dbar_i x_i,
 *   cbar_i = -dbar_i x_{i+1}   (abar = 0 on the first, cbar on the last row).
 * abar, bbar, cbar may each be NULL (x is then not read if all three are);
 * dbar may alias w. One pass, systems up to N = 1024 (longer ones return
 * TRID_STATUS_MATRIX_TYPE_NOT_SUPPORTED). Layout rules as tridDmtsvStridedBatch. */
EXTERN_C tridStatus_t tridDmtsvStridedBatchAdjoint(const TridParams *ctx, const double *a,
                                                   const double *b, const double *c,
                                                   const double *x, const double *w, double *dbar,
                                                   double *abar, double *bbar, double *cbar,
                                                   int ndim, int solvedim, const int *dims,
                                                   const int *pads);
EXTERN_C tridStatus_t tridSmtsvStridedBatchAdjoint(const TridParams *ctx, const float *a,
                                                   const float *b, const float *c, const float *x,
                                                   const float *w, float *dbar, float *abar,
                                                   float *bbar, float *cbar, int ndim,
                                                   int solvedim, const int *dims, const int *pads);

/* ---- generic strided batch -------------------------------------------------
 * The surface of the reference's solveBatchedTrid
 * (scalar/src/cuda/trid_thomaspcr.hpp:794-832, a C++ template there): numTrids
 * systems of `length` rows, rows stride1 elements apart; system k starts at
 * k*stride2 when stride1 == 1, else at (k / subBatchSize)*subBatchStride +
 * (k % subBatchSize)*stride2 (e.g. a y solve of an X*Y*Z cube: stride1 = X,
 * stride2 = 1, subBatchSize = X, subBatchStride = X*Y). d is read and x
 * written (Inc: x += solution); a[0] and c[length-1] are treated as zero.
 * Unlike the reference, any combination of strides is accepted (it requires
 * stride1 == 1 or stride2 == 1), a last partial sub-batch is allowed, and a
 * status is returned instead of 0/1. */
EXTERN_C tridStatus_t tridDsolveBatchedTrid(const TridParams *ctx, int numTrids, int length,
                                            int stride1, int stride2, int subBatchSize,
                                            int subBatchStride, const double *a, const double *b,
                                            const double *c, const double *d, double *x);
EXTERN_C tridStatus_t tridSsolveBatchedTrid(const TridParams *ctx, int numTrids, int length,
                                            int stride1, int stride2, int subBatchSize,
                                            int subBatchStride, const float *a, const float *b,
                                            const float *c, const float *d, float *x);
EXTERN_C tridStatus_t tridDsolveBatchedTridInc(const TridParams *ctx, int numTrids, int length,
                                               int stride1, int stride2, int subBatchSize,
                                               int subBatchStride, const double *a,
                                               const double *b, const double *c, const double *d,
                                               double *x);
EXTERN_C tridStatus_t tridSsolveBatchedTridInc(const TridParams *ctx, int numTrids, int length,
                                               int stride1, int stride2, int subBatchSize,
                                               int subBatchStride, const float *a, const float *b,
                                               const float *c, const float *d, float *x);

/* ---- FP32 storage, FP64 accuracy -----------------------------------------
 * No counterpart in the reference. Solves T x = d where a, b, c are stored in
 * FP32 (the system is exactly those values, promoted to FP64) and d is FP64;
 * x overwrites d. The solve runs in FP32; only the residual r = d - T x and
 * the accumulation x += dx run in FP64. The FP32 factorisation is computed
 * once and reused by every refinement pass, all on chip, until the estimated
 * relative error of x is at most tol for every system, or max_iters FP32
 * solves. The estimate is the a-posteriori bound of a contraction:
 * rho / (1 - rho) * max|dx_k| / max|x|, with rho = max|dx_k| / max|dx_{k-1}|
 * (max|dx_k| / max|x| itself while rho is unknown or >= 1/2). One pass over
 * memory: 28 bytes per element against 40 for tridDmtsvStridedBatch.
 * Blocking calls report the largest iteration count and the largest final
 * error estimate over all systems in *iters_out / *correction_out (-1 when
 * not blocking). Supports N <= 512 (longer systems return
 * TRID_STATUS_MATRIX_TYPE_NOT_SUPPORTED).
 * By default, wherever a direct kernel exists, the system is instead solved
 * in FP64 arithmetic straight from the FP32 values (no refinement needed,
 * *iters_out = 0 and *correction_out = 0; the result is the FP64 solve of
 * the promoted system bit for bit): strided batches of 64 < N <= 512 rows
 * (the streaming kernel reading a, b, c as FP32; about twice as fast as the
 * refinement there, whose per-row state does not fit on chip, but slower
 * than tridDmtsvStridedBatch on FP64 arrays because the FP32 rows of a
 * 16-system group are 64-byte segments) and 16-byte-aligned contiguous
 * systems of 129 to 512 rows (a, b, c staged in shared memory as FP32;
 * faster than both the refinement and the FP64 solve). Both move 28 bytes
 * per element. tridSetMixedMode (per calling thread) chooses: 0 = that
 * automatic choice (default), 1 = always the FP32 solve with FP64
 * refinement, 2 = the same as 0. */
EXTERN_C tridStatus_t tridSetMixedMode(int mode);
EXTERN_C tridStatus_t tridDmtsvStridedBatchMixed(const TridParams *ctx, const float *a,
                                                 const float *b, const float *c, double *d,
                                                 int ndim, int solvedim, const int *dims,
                                                 const int *pads, int max_iters, double tol,
                                                 int *iters_out, double *correction_out);

/* ---- FP32 factorisation, FP64-specified system ----------------------------
 * No counterpart in the reference. Solves T x = d for an FP64-specified
 * system (a, b, c, d FP64 arrays; x overwrites d) by iterative refinement:
 * the FP32 factorisation of the coefficients rounded to FP32 is computed
 * once, on chip, and every pass forms the residual r = d - T x in FP64 with
 * the FP64 coefficients, solves T dx = r with the FP32 factors and
 * accumulates x += dx in FP64, until the estimated relative error (the
 * contraction estimate of tridDmtsvStridedBatchMixed) is at most tol for
 * every system, or max_iters FP32 solves. The result converges to the
 * solution of the FP64 system itself (tridDmtsvStridedBatchMixed instead
 * solves the system of its FP32 values exactly). One pass over memory: a, b,
 * c, d read once and x written once, 40 bytes per element, the same as
 * tridDmtsvStridedBatch, so it is not faster than the direct FP64 solve; it
 * exists for callers that want the FP32 factorisation with an FP64 error
 * bound and iteration count per call. Blocking calls report the largest
 * iteration count and error estimate in *iters_out / *correction_out (-1
 * when not blocking). N <= 512 (longer systems return
 * TRID_STATUS_MATRIX_TYPE_NOT_SUPPORTED). */
EXTERN_C tridStatus_t tridDmtsvStridedBatchRefine(const TridParams *ctx, const double *a,
                                                  const double *b, const double *c, double *d,
                                                  int ndim, int solvedim, const int *dims,
                                                  const int *pads, int max_iters, double tol,
                                                  int *iters_out, double *correction_out);

/* ---- solve without allocating ------------------------------------------
 * No counterpart in the reference. tridDmtsvStridedBatch with the same
 * arguments and results, for callers that cannot allocate device memory
 * (services that reserve and account for all device memory up front,
 * real-time loops where an allocation's latency or failure is not
 * acceptable): the regular entry point allocates scratch for systems longer
 * than one warp holds and pins a host word on first use; this one allocates
 * nothing. Its scratch is one fixed 16 MiB array in device memory that every
 * GPU loading the library holds until exit. Problems whose long-system
 * scratch would exceed it return TRID_STATUS_INVALID_VALUE (with a message on
 * stderr); systems short enough for one warp per system (N <= 512 along x,
 * N <= 1024 along y or z) need none. All calls share the array, so calls that
 * overlap on the GPU race; the first call on a device looks up the array's
 * address and should come before any stream capture, and a cudaDeviceReset
 * after it is not supported. Zero pivots are reported in blocking mode only.
 * The plan is always the automatic one (tridForce* settings are ignored), and
 * a ctx whose mpi_params were registered by tridDistInit is refused with
 * TRID_STATUS_INVALID_VALUE: the distributed solve is not available here. */
EXTERN_C tridStatus_t tridDmtsvStridedBatchNoAlloc(const TridParams *ctx, const double *a,
                                                   const double *b, const double *c, double *d,
                                                   int ndim, int solvedim, const int *dims,
                                                   const int *pads);

/* Describes the plan the next solve of this shape would use, e.g.
 * "hybrid M=16 T=32 W=1 vec" (for logs and tests). Returns the length. */
EXTERN_C int tridDescribePlan(int dtype_bytes, int ndim, int solvedim, const int *dims,
                              const int *pads, char *buf, int buflen);

/* As tridDescribePlan, for the Inc variant of the solve when inc != 0 (its
 * plan may differ: u is a fifth stream of every row). Arrays are taken as
 * aligned. Returns the length. */
EXTERN_C int tridDescribePlanInc(int dtype_bytes, int ndim, int solvedim, const int *dims,
                                 const int *pads, int inc, char *buf, int buflen);

#endif
