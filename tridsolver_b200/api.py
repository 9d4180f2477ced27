"""Python mirror of the reference's C API, over the in-tree C-ABI library.

Two levels:

* The reference's four entry points under their own names
  (tridDmtsvStridedBatch, tridSmtsvStridedBatch, ...Inc), taking device
  pointers (ints) or CUDA tensors, returning the tridStatus_t code exactly as
  the C functions do (scalar/include/tridsolver.h:39-69). These are blocking
  by default, like the reference.
* ``strided_batch`` / ``solve``: the same solve on torch CUDA tensors,
  enqueued on torch's current stream without blocking, raising TridError on
  a non-success status.

Layout is the reference's: element (i0, i1, i2) at i0 + i1*pads[0] +
i2*pads[0]*pads[1]. A C-contiguous torch tensor of shape (n2, n1, n0) has
exactly that layout with dims = [n0, n1, n2], so torch dimension k is the
reference's solvedim = ndim - 1 - k.
"""

import ctypes
import enum

from . import _lib


class TridStatus(enum.IntEnum):
    """tridStatus_t (scalar/include/trid_common.h:64-75)."""
    SUCCESS = 0
    NOT_INITIALIZED = 1
    ALLOC_FAILED = 2
    INVALID_VALUE = 3
    ARCH_MISMATCH = 4
    MAPPING_ERROR = 5
    EXECUTION_FAILED = 6
    INTERNAL_ERROR = 7
    MATRIX_TYPE_NOT_SUPPORTED = 8
    ZERO_PIVOT = 9


class TridError(RuntimeError):
    def __init__(self, status, what=""):
        self.status = TridStatus(status)
        super().__init__(f"{what}: {self.status.name}" if what else self.status.name)


MAXDIM = 3


class TridParams(ctypes.Structure):
    """struct TridParams (scalar/include/trid_params.h:31-35)."""
    _fields_ = [("mpi_params", ctypes.c_void_p),
                ("opts", ctypes.c_int * MAXDIM),
                ("sync", ctypes.c_int)]


FAMILY_AUTO, FAMILY_HYBRID, FAMILY_PCR, FAMILY_LONG = -1, 0, 1, 2


def _addr(x):
    if x is None:
        return None
    if hasattr(x, "data_ptr"):
        return x.data_ptr()
    return int(x)


def _ctx(ctx):
    if ctx is None:
        return None
    if isinstance(ctx, TridParams):
        return ctypes.addressof(ctx)
    return int(ctx)


def _ints(vals):
    vals = list(vals)
    return (ctypes.c_int * max(1, len(vals)))(*[int(v) for v in vals])


# ---- the reference's entry points ------------------------------------------

def tridDmtsvStridedBatch(ctx, a, b, c, d, ndim, solvedim, dims, pads):
    return _lib.load().tridDmtsvStridedBatch(_ctx(ctx), _addr(a), _addr(b), _addr(c), _addr(d),
                                             int(ndim), int(solvedim), _ints(dims), _ints(pads))


def tridSmtsvStridedBatch(ctx, a, b, c, d, ndim, solvedim, dims, pads):
    return _lib.load().tridSmtsvStridedBatch(_ctx(ctx), _addr(a), _addr(b), _addr(c), _addr(d),
                                             int(ndim), int(solvedim), _ints(dims), _ints(pads))


def tridDmtsvStridedBatchInc(ctx, a, b, c, d, u, ndim, solvedim, dims, pads):
    return _lib.load().tridDmtsvStridedBatchInc(_ctx(ctx), _addr(a), _addr(b), _addr(c), _addr(d),
                                                _addr(u), int(ndim), int(solvedim), _ints(dims),
                                                _ints(pads))


def tridSmtsvStridedBatchInc(ctx, a, b, c, d, u, ndim, solvedim, dims, pads):
    return _lib.load().tridSmtsvStridedBatchInc(_ctx(ctx), _addr(a), _addr(b), _addr(c), _addr(d),
                                                _addr(u), int(ndim), int(solvedim), _ints(dims),
                                                _ints(pads))


def solve_batched_trid(num_trids, length, stride1, stride2, sub_batch_size, sub_batch_stride, a, b,
                       c, d, x, inc=False, ctx=None):
    """The reference's solveBatchedTrid surface (include/tridsolver_b200.h):
    FP64 or FP32 by the tensors' dtype; x receives the solution (x += it
    when inc). Returns the status."""
    f64 = getattr(a, "dtype", None) is None or str(a.dtype).endswith("float64")
    name = ("tridDsolveBatchedTrid" if f64 else "tridSsolveBatchedTrid") + ("Inc" if inc else "")
    return getattr(_lib.load(), name)(_ctx(ctx), int(num_trids), int(length), int(stride1),
                                      int(stride2), int(sub_batch_size), int(sub_batch_stride),
                                      _addr(a), _addr(b), _addr(c), _addr(d), _addr(x))


def tridDmtsvStridedBatchMixed(ctx, a, b, c, d, ndim, solvedim, dims, pads, max_iters=10,
                               tol=1e-12):
    """FP32-stored a, b, c; FP64 d (x overwrites it); FP32 solves refined in
    FP64 on chip (include/tridsolver_b200.h). Returns (status, iterations,
    final relative correction); the last two are -1 unless blocking."""
    it = ctypes.c_int(-1)
    corr = ctypes.c_double(-1.0)
    st = _lib.load().tridDmtsvStridedBatchMixed(_ctx(ctx), _addr(a), _addr(b), _addr(c), _addr(d),
                                                int(ndim), int(solvedim), _ints(dims), _ints(pads),
                                                int(max_iters), float(tol), ctypes.byref(it),
                                                ctypes.byref(corr))
    return st, it.value, corr.value


def tridDmtsvStridedBatchRefine(ctx, a, b, c, d, ndim, solvedim, dims, pads, max_iters=10,
                                tol=1e-12):
    """FP64-specified a, b, c, d (x overwrites d): FP32 factorisation of the
    rounded coefficients, refined with the FP64 residual of the FP64 system
    on chip (include/tridsolver_b200.h). Returns (status, iterations,
    estimated relative error); the last two are -1 unless blocking."""
    it = ctypes.c_int(-1)
    corr = ctypes.c_double(-1.0)
    st = _lib.load().tridDmtsvStridedBatchRefine(_ctx(ctx), _addr(a), _addr(b), _addr(c), _addr(d),
                                                 int(ndim), int(solvedim), _ints(dims),
                                                 _ints(pads), int(max_iters), float(tol),
                                                 ctypes.byref(it), ctypes.byref(corr))
    return st, it.value, corr.value


def tridDmtsvStridedBatchAdjoint(ctx, a, b, c, x, w, dbar, abar, bbar, cbar, ndim, solvedim, dims,
                                 pads):
    """Adjoint of the strided solve (include/tridsolver_b200.h); abar, bbar,
    cbar may be None. Returns the status code."""
    return _lib.load().tridDmtsvStridedBatchAdjoint(
        _ctx(ctx), _addr(a), _addr(b), _addr(c), _addr(x), _addr(w), _addr(dbar), _addr(abar),
        _addr(bbar), _addr(cbar), int(ndim), int(solvedim), _ints(dims), _ints(pads))


def tridSmtsvStridedBatchAdjoint(ctx, a, b, c, x, w, dbar, abar, bbar, cbar, ndim, solvedim, dims,
                                 pads):
    return _lib.load().tridSmtsvStridedBatchAdjoint(
        _ctx(ctx), _addr(a), _addr(b), _addr(c), _addr(x), _addr(w), _addr(dbar), _addr(abar),
        _addr(bbar), _addr(cbar), int(ndim), int(solvedim), _ints(dims), _ints(pads))


def tridDmtsvRaggedBatch(ctx, a, b, c, d, offsets, nsys):
    """Ragged batch (include/tridsolver_b200.h): offsets is a device int64
    array of nsys + 1 entries. Returns the status code."""
    return _lib.load().tridDmtsvRaggedBatch(_ctx(ctx), _addr(a), _addr(b), _addr(c), _addr(d),
                                            _addr(offsets), int(nsys))


def tridSmtsvRaggedBatch(ctx, a, b, c, d, offsets, nsys):
    return _lib.load().tridSmtsvRaggedBatch(_ctx(ctx), _addr(a), _addr(b), _addr(c), _addr(d),
                                            _addr(offsets), int(nsys))


def tridDmtsvRaggedBatchSized(ctx, a, b, c, d, offsets, nsys, nelems):
    """Ragged batch with the element count given (nelems >= offsets[nsys] -
    offsets[0]): nothing is read back, so the call can be captured into a
    CUDA graph with blocking off. Returns the status code."""
    return _lib.load().tridDmtsvRaggedBatchSized(_ctx(ctx), _addr(a), _addr(b), _addr(c),
                                                 _addr(d), _addr(offsets), int(nsys), int(nelems))


def tridSmtsvRaggedBatchSized(ctx, a, b, c, d, offsets, nsys, nelems):
    return _lib.load().tridSmtsvRaggedBatchSized(_ctx(ctx), _addr(a), _addr(b), _addr(c),
                                                 _addr(d), _addr(offsets), int(nsys), int(nelems))


def ragged_autotune(dtype_bytes):
    st = _lib.load().tridRaggedAutotune(int(dtype_bytes))
    if st != 0:
        raise TridError(st, "tridRaggedAutotune")


def autotune(dtype_bytes, dims, solvedim, pads=None, inc=False):
    """tridAutotune: time every applicable plan for this shape on the current
    device and keep the fastest for its shape class. Returns (ms, plan)."""
    pads = dims if pads is None else pads
    ms = ctypes.c_float(-1.0)
    buf = ctypes.create_string_buffer(96)
    st = _lib.load().tridAutotune(int(dtype_bytes), len(dims), int(solvedim), _ints(dims),
                                  _ints(pads), int(bool(inc)), ctypes.byref(ms), buf, 96)
    if st != 0:
        raise TridError(st, "tridAutotune")
    return ms.value, buf.value.decode()


def autotune_reset():
    """tridAutotuneReset: forget the current device's tuned choices."""
    st = _lib.load().tridAutotuneReset()
    if st != 0:
        raise TridError(st, "tridAutotuneReset")


def ragged_table(dtype_bytes):
    """Rows per lane by length class (index = ceil(log2 N)) for warp items."""
    buf = (ctypes.c_int * 32)()
    n = _lib.load().tridRaggedTable(int(dtype_bytes), buf, 32)
    if n < 0:
        raise TridError(TridStatus.INVALID_VALUE, "tridRaggedTable")
    return list(buf[:n])


# ---- execution control -------------------------------------------------------

def set_stream(stream):
    """stream: a torch.cuda.Stream, a raw cudaStream_t (int) or None."""
    raw = getattr(stream, "cuda_stream", stream)
    _lib.load().tridSetStream(None if raw in (None, 0) else int(raw))


def set_blocking(blocking):
    _lib.load().tridSetBlocking(1 if blocking else 0)


def get_blocking():
    return bool(_lib.load().tridGetBlocking())


def pivot_status():
    return TridStatus(_lib.load().tridGetPivotStatus())


def launch_count():
    return int(_lib.load().tridGetLaunchCount())


def set_tracing(on=True):
    """NVTX ranges around the library's solve calls (tridSetTracing)."""
    _lib.load().tridSetTracing(1 if on else 0)


def release_scratch():
    """Return the unused memory of the library's scratch pool on the current
    device to the driver (tridReleaseScratch)."""
    st = _lib.load().tridReleaseScratch()
    if st != 0:
        raise TridError(st, "tridReleaseScratch")


def force_plan(family=FAMILY_AUTO, rows_per_thread=0):
    st = _lib.load().tridForcePlan(int(family), int(rows_per_thread))
    if st != 0:
        raise TridError(st, "tridForcePlan")


def force_systems_per_block(systems=0):
    st = _lib.load().tridForceSystemsPerBlock(int(systems))
    if st != 0:
        raise TridError(st, "tridForceSystemsPerBlock")


def force_tma(mode=-1):
    """1: TMA tiles for strided batches wherever allowed; 0 / -1 (default): not."""
    st = _lib.load().tridForceTma(int(mode))
    if st != 0:
        raise TridError(st, "tridForceTma")


def force_stream(mode=-1):
    """Strided batches of 64 < N <= 512: -1 (default) automatic (the wide
    streaming kernel with 256-byte groups for rows a plane apart, else the
    streaming kernel with 128-byte groups, unless TMA is forced); 1 the
    128-byte streaming kernel, 2 the wide one, wherever they apply; 0 the
    register-tile kernel."""
    st = _lib.load().tridForceStream(int(mode))
    if st != 0:
        raise TridError(st, "tridForceStream")


def set_mixed_mode(mode=0):
    """tridDmtsvStridedBatchMixed strategy for this thread: 0 automatic (the
    direct FP64 solve of the FP32 values where a direct kernel exists:
    strided 64 < N <= 512 and aligned contiguous 129 <= N <= 512; FP32 with
    FP64 refinement otherwise), 1 always refinement, 2 the same as 0."""
    st = _lib.load().tridSetMixedMode(int(mode))
    if st != 0:
        raise TridError(st, "tridSetMixedMode")


def describe_plan(dtype_bytes, dims, solvedim, pads=None, inc=False):
    pads = dims if pads is None else pads
    buf = ctypes.create_string_buffer(128)
    n = _lib.load().tridDescribePlanInc(int(dtype_bytes), len(dims), int(solvedim), _ints(dims),
                                        _ints(pads), int(bool(inc)), buf, 128)
    if n < 0:
        raise TridError(TridStatus.INVALID_VALUE, "tridDescribePlan")
    return buf.value.decode()


class on_stream:
    """Context manager: run library calls on `stream` (default: torch's current
    stream) with the given blocking mode, restoring the previous settings."""

    def __init__(self, stream=None, blocking=False):
        self.stream = stream
        self.blocking = blocking

    def __enter__(self):
        import torch
        lib = _lib.load()
        self._prev = (lib.tridGetStream(), lib.tridGetBlocking())
        s = self.stream if self.stream is not None else torch.cuda.current_stream()
        set_stream(s)
        set_blocking(self.blocking)
        return self

    def __exit__(self, *exc):
        lib = _lib.load()
        lib.tridSetStream(self._prev[0])
        lib.tridSetBlocking(self._prev[1])
        return False


# ---- torch-tensor interface ------------------------------------------------------

def strided_batch(a, b, c, d, solvedim, dims, pads=None, u=None, ctx=None):
    """Solve along `solvedim` of the reference layout on CUDA tensors (any shape,
    addressed through dims/pads from their first element). d <- x, or u += x
    when u is given. Enqueued on torch's current stream; raises TridError."""
    import torch
    pads = list(dims) if pads is None else list(pads)
    dt = d.dtype
    if dt not in (torch.float64, torch.float32):
        raise TypeError("float32 or float64 tensors only")
    for t in (a, b, c, d) + ((u,) if u is not None else ()):
        if t.dtype != dt or not t.is_cuda:
            raise TypeError("all arrays must be CUDA tensors of one dtype")
    with torch.cuda.device(d.device), on_stream(blocking=False):
        if dt == torch.float64:
            st = (tridDmtsvStridedBatch(ctx, a, b, c, d, len(dims), solvedim, dims, pads) if u is None
                  else tridDmtsvStridedBatchInc(ctx, a, b, c, d, u, len(dims), solvedim, dims, pads))
        else:
            st = (tridSmtsvStridedBatch(ctx, a, b, c, d, len(dims), solvedim, dims, pads) if u is None
                  else tridSmtsvStridedBatchInc(ctx, a, b, c, d, u, len(dims), solvedim, dims, pads))
    if st != 0:
        raise TridError(st, "strided batch solve")


def solve(a, b, c, d, dim=-1, u=None):
    """Solve along torch dimension `dim` of C-contiguous tensors of one shape
    (ndim <= 3). d <- x in place, or u += x when u is given."""
    shape = tuple(d.shape)
    nd = len(shape)
    if not 1 <= nd <= MAXDIM:
        raise ValueError("1 to 3 dimensions")
    for t in (a, b, c, d) + ((u,) if u is not None else ()):
        if tuple(t.shape) != shape or not t.is_contiguous():
            raise ValueError("contiguous tensors of one shape")
    dims = list(reversed(shape))
    solvedim = nd - 1 - (dim % nd)
    strided_batch(a, b, c, d, solvedim, dims, dims, u=u)
