// Host-side internals shared by the translation units of libtridsolver_b200.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <string>

#include "trid_kernels.cuh"
#include "tridsolver_b200.h"

namespace trid {

struct Plan {
  int family = TRID_FAMILY_HYBRID;  // TRID_FAMILY_*
  int M = 8;                        // rows per thread (hybrid, long)
  int T = 1;                        // threads per system (hybrid, pcr)
  int W = 1;                        // systems per block (strided hybrid)
  bool vec = false;                 // 16-byte vector loads (contiguous hybrid)
  bool smem = false;                // warp-per-system staging through shared memory
  bool tma = false;                 // strided: TMA tiles, persistent, double-buffered
  bool streaming = false;           // strided: persistent streaming kernel (T = 32)
  bool wide = false;                // strided: wide streaming kernel (256-byte groups)
  bool tiles = false;               // long, contiguous: warp tiles of 512 / 1024 rows
  bool pairs = false;               // wide, FP32: two adjacent systems per thread
  std::string describe() const;
};

// Per-thread execution settings (see tridsolver_b200.h).
struct Settings {
  cudaStream_t stream = nullptr;
  bool blocking = true;
  int force_family = TRID_FAMILY_AUTO;
  int force_m = 0;
  int force_w = 0;
  int force_tma = -1;  // -1 automatic, 0 off, 1 on where it applies
  int force_stream = -1;  // -1 automatic, 0 off, 1 128-byte groups, 2 256-byte groups
  int mixed_mode = 0;     // tridSetMixedMode: 0 automatic, 1 refinement, 2 promoted
};
Settings &settings();

extern std::atomic<unsigned long long> g_launches;

// Stream-ordered scratch from the library's own pool (trid_pool.cu).
cudaError_t scratch_alloc(void **ptr, size_t bytes, cudaStream_t st);
cudaError_t scratch_free(void *ptr, cudaStream_t st);
cudaError_t scratch_release();

// An NVTX range named after one library call, for Nsight Systems timelines
// and ncu range filters, while tracing is on (tridSetTracing, or
// TRIDSOLVER_NVTX=1 in the environment at the first call); nothing
// otherwise. Ranges are per host thread.
class TraceScope {
 public:
  explicit TraceScope(const char *name);
  ~TraceScope();
  TraceScope(const TraceScope &) = delete;
  TraceScope &operator=(const TraceScope &) = delete;

 private:
  bool on_;
};

// Host-mapped zero-pivot word of the current device (device pointer), or
// nullptr if it could not be set up.
unsigned *pivot_flag_device();
bool pivot_flag_take();  // reads and clears the word of the current device

// CUDA error -> library status (trid_api.cu).
tridStatus_t status_of(cudaError_t e);
// The current device is an sm_100 GPU (trid_api.cu).
tridStatus_t check_device();
// Validates the strided-batch arguments and fills a BatchArgs; SUCCESS with
// *empty = true when there is nothing to solve (trid_api.cu).
template <typename R>
tridStatus_t make_batch(const R *a, const R *b, const R *c, R *d, R *u, bool inc, int ndim,
                        int solvedim, const int *dims_p, const int *pads_p, BatchArgs<R> *out,
                        bool *empty);

// Plan choices that override the built-in table: the calling thread's
// tridForce* settings, or an autotuned recipe (family, rows per thread,
// streaming form, TMA; all automatic by default).
struct Forces {
  int family = TRID_FAMILY_AUTO;
  int m = 0;
  int w = 0;
  int tma = -1;
  int stream = -1;
  bool any() const { return family != TRID_FAMILY_AUTO || m != 0 || w != 0 || tma != -1 || stream != -1; }
};

// honour_force: apply the calling thread's tridForce* settings (top-level
// calls only; internal recursions do not). With nothing forced, the
// autotuner's recipe for the batch's shape class is used when one exists
// (tridAutotune), else the built-in table.
template <typename R>
Plan choose_plan(const BatchArgs<R> &p, bool aligned16, bool honour_force = true);
template <typename R>
Plan choose_plan_forced(const BatchArgs<R> &p, bool aligned16, const Forces &f);
// The autotuned recipe for p's shape class on the current device (trid_autotune.cu);
// leaves *f untouched when there is none.
template <typename R>
void tuned_forces(const BatchArgs<R> &p, Forces *f);

// Enqueues the solve of batch p on `st` (no synchronisation).
template <typename R, bool INC>
cudaError_t launch_batch(const BatchArgs<R> &p, const Plan &plan, cudaStream_t st);

// TMA tile geometry of a strided batch (trid_strided_tma.cu); false when TMA
// does not apply (alignment, strides, length, shared-memory size).
template <typename R>
bool tma_geometry(const BatchArgs<R> &p, bool inc, int W, int &rows_box, int &nbox, int &stages,
                  size_t &smem, int T);
template <typename R, int M, int KR, bool INC>
cudaError_t launch_strided_tma(const BatchArgs<R> &p, const Plan &plan, cudaStream_t st);

// Streaming strided kernel (trid_strided_stream.cu): group width for n0
// systems along the fastest dimension, and its launcher.
template <typename R> int stream_width(long long n0);
template <typename R> struct AdjointOut {
  R *abar = nullptr, *bbar = nullptr, *cbar = nullptr;
};
template <typename R, int M>
cudaError_t launch_strided_stream_adjoint(const BatchArgs<R> &p, const AdjointOut<R> &q,
                                          cudaStream_t st);
template <typename R, int M, bool INC>
cudaError_t launch_strided_stream(const BatchArgs<R> &p, const Plan &plan, cudaStream_t st);
// Wide streaming kernel (trid_strided_wide.cu): 256-byte groups with the
// elimination state parked in tensor memory; rows per thread and chunks
// per system for N rows (0 when it does not apply), group width, launcher.
template <typename R> int wide_rows_per_thread(int N, bool pairs);
template <typename R> int wide_chunks(int N, bool pairs);
template <typename R> bool wide_pairs(const BatchArgs<R> &p);
template <typename R> int wide_width();
template <typename R, bool INC>
cudaError_t launch_strided_wide(const BatchArgs<R> &p, cudaStream_t st);
// Long contiguous systems in warp tiles (trid_long.cu): reduction of every
// tile to two second-level rows, recursive solve of those, substitution.
template <typename R, bool INC>
cudaError_t launch_long_tiles(const BatchArgs<R> &p, cudaStream_t st);
// The wide kernel in FP64 arithmetic on FP32-stored a, b, c.
cudaError_t launch_strided_wide_promoted(const BatchArgs<double> &p, const CoefPtrs<float> &cf,
                                         cudaStream_t st);
// The streaming kernel in FP64 arithmetic on FP32-stored a, b, c.
template <int M>
cudaError_t launch_strided_stream_promoted(const BatchArgs<double> &p, const CoefPtrs<float> &cf,
                                           cudaStream_t st);

// The ADI step's preprocessing kernel (trid_adi.cu): du = lambda L u on
// interior points, 0 on the boundary, and one shared set of coefficient
// arrays (identity rows on the boundary).
template <typename R>
cudaError_t launch_adi_preproc(const R *u, R *du, R *a, R *b, R *c, const R *lam, const int *step,
                               R alpha, int nx, int ny, int nz, cudaStream_t st);
// Solves of the fused ADI timestep (trid_adi_fused.cu): the x solve with the
// 7-point stencil of u formed on the fly (du written), 1 <= nx <= 512; the y
// or z solve of du in place (INC: u += solution), 1 <= N <= 512.
template <typename R>
cudaError_t launch_adi_x(const R *u, R *du, const ConstCoef<R> &k, unsigned *flag, int nx, int ny,
                         int nz, cudaStream_t st);
template <typename R, bool INC>
cudaError_t launch_adi_yz(const BatchArgs<R> &p, const ConstCoef<R> &k, cudaStream_t st);
// Transposed solves of the step's matrices, in place (the step's adjoint):
// interior rows of interior systems solved, rows 0 and N - 1 and boundary
// systems left as they are (1 <= N <= 512).
template <typename R>
cudaError_t launch_adi_x_transposed(R *w, const ConstCoef<R> &k, int nx, int ny, int nz,
                                    cudaStream_t st);
template <typename R>
cudaError_t launch_adi_yz_transposed(const BatchArgs<R> &p, const ConstCoef<R> &k, cudaStream_t st);

// Distributed solve (trid_dist.cu): whether ctx->mpi_params was registered
// by tridDistInit, and the solve of this rank's block.
bool dist_registered(const void *params);
template <typename R, bool INC>
tridStatus_t dist_solve(const tridDistParams *dp, const BatchArgs<R> &p, int solvedim,
                        cudaStream_t st, bool blocking);

// Whether every pointer and every system start allows 16-byte vector access
// (contiguous systems only).
template <typename R>
bool vec_aligned(const BatchArgs<R> &p);

}  // namespace trid
