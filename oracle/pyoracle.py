"""ctypes bindings of the CPU checkers built by oracle/Makefile.

ORACLE — test infrastructure only (checkers and the baseline legs of bench.py):

* ``Restatement``: oracle/_build/liboracle.so, the plain-C restatement of the
  reference algorithm (trid_oracle.c, each function cites the reference).
* ``Reference``: oracle/_ref/libtridcpu_ref_{avx512,avx2}.so, the reference's
  own scalar/src/cpu/trid_cpu.cpp compiled from its sources with the API
  symbols renamed ref_*. The AVX-512 build is used when this CPU has avx512f.
* ``ReferenceGPU``: oracle/_ref/libtridcuda_ref.so, the reference's own CUDA
  library built for sm_100a: a same-box comparator for the benchmark,
  itself checked against the two above by tests/test_reference_gpu.py.

All arrays are numpy, x-fastest (Fortran order for an ndim-shaped array).
"""

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")

_dp = ctypes.POINTER(ctypes.c_double)
_fp = ctypes.POINTER(ctypes.c_float)
_ip = ctypes.POINTER(ctypes.c_int)
_i64p = ctypes.POINTER(ctypes.c_int64)


def _ptr(arr):
    if arr is None:
        return None
    if arr.dtype == np.float64:
        return arr.ctypes.data_as(_dp)
    if arr.dtype == np.float32:
        return arr.ctypes.data_as(_fp)
    raise TypeError(arr.dtype)


def _ints(vals):
    return (ctypes.c_int * len(vals))(*[int(v) for v in vals])


def cpu_has_avx512():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    return " avx512f " in f" {line.split(':', 1)[1].strip()} "
    except OSError:
        pass
    return False


def _check(arrs, dtype):
    for a in arrs:
        if a is None:
            continue
        if a.dtype != dtype or not a.flags.c_contiguous:
            raise TypeError("arrays must be contiguous and of one dtype")


class Restatement:
    """The plain-C restatement (oracle/trid_oracle.c)."""

    def __init__(self, path=ORACLE_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle`")
        self.lib = ctypes.CDLL(path)

    def strided_batch(self, a, b, c, d, dims, solvedim, pads=None, u=None):
        """Solve in place: d <- x (u is None) or u += x."""
        dt = d.dtype
        _check((a, b, c, d, u), dt)
        pads = dims if pads is None else pads
        fn = self.lib.oracle_strided_batch_d if dt == np.float64 else self.lib.oracle_strided_batch_f
        rc = fn(_ptr(a), _ptr(b), _ptr(c), _ptr(d), _ptr(u), int(u is not None),
                len(dims), int(solvedim), _ints(dims), _ints(pads))
        if rc != 0:
            raise ValueError(f"oracle_strided_batch rc={rc}")

    def ragged(self, a, b, c, d, offsets, u=None):
        dt = d.dtype
        _check((a, b, c, d, u), dt)
        offsets = np.ascontiguousarray(offsets, dtype=np.int64)
        fn = self.lib.oracle_ragged_d if dt == np.float64 else self.lib.oracle_ragged_f
        rc = fn(_ptr(a), _ptr(b), _ptr(c), _ptr(d), _ptr(u), int(u is not None),
                offsets.ctypes.data_as(_i64p), ctypes.c_long(len(offsets) - 1))
        if rc != 0:
            raise ValueError(f"oracle_ragged rc={rc}")

    def adjoint(self, a, b, c, x, w, dims, solvedim, pads=None):
        """Return (abar, bbar, cbar, dbar) for L = sum(w * x), x = T^{-1} d."""
        _check((a, b, c, x, w), np.float64)
        pads = dims if pads is None else pads
        outs = [np.zeros_like(x) for _ in range(4)]
        rc = self.lib.oracle_adjoint_d(_ptr(a), _ptr(b), _ptr(c), _ptr(x), _ptr(w),
                                       *[_ptr(o) for o in outs], len(dims),
                                       int(solvedim), _ints(dims), _ints(pads))
        if rc != 0:
            raise ValueError(f"oracle_adjoint rc={rc}")
        return tuple(outs)

    def adi_step(self, u, lam, ca, cb, nx, ny, nz):
        """One ADI heat step on u (x fastest) in place; returns du."""
        dt = u.dtype
        du = np.zeros_like(u)
        ax, bx, cx = (np.zeros_like(u) for _ in range(3))
        fn = self.lib.oracle_adi_step_d if dt == np.float64 else self.lib.oracle_adi_step_f
        ctype = ctypes.c_double if dt == np.float64 else ctypes.c_float
        fn.argtypes = None
        rc = fn(_ptr(u), _ptr(du), _ptr(ax), _ptr(bx), _ptr(cx), int(nx), int(ny),
                int(nz), ctype(lam), ctype(ca), ctype(cb))
        if rc != 0:
            raise ValueError(f"oracle_adi_step rc={rc}")
        return du


class Reference:
    """The reference's CPU library, compiled from its own sources."""

    def __init__(self, isa=None):
        isa = isa or ("avx512" if cpu_has_avx512() else "avx2")
        path = os.path.join(REF_DIR, f"libtridcpu_ref_{isa}.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle` where the reference tree exists")
        # trid_cpu.cpp keeps 2*N_MAX SIMD vectors on each worker's stack
        os.environ.setdefault("OMP_STACKSIZE", "32M")
        self.isa = isa
        self.path = path
        self.lib = ctypes.CDLL(path)
        for name in ("ref_tridDmtsvStridedBatch", "ref_tridSmtsvStridedBatch",
                     "ref_tridDmtsvStridedBatchInc", "ref_tridSmtsvStridedBatchInc"):
            getattr(self.lib, name).restype = ctypes.c_int

    def strided_batch(self, a, b, c, d, dims, solvedim, pads=None, u=None):
        dt = d.dtype
        _check((a, b, c, d, u), dt)
        pads = dims if pads is None else pads
        p = "D" if dt == np.float64 else "S"
        if u is None:
            rc = getattr(self.lib, f"ref_trid{p}mtsvStridedBatch")(
                None, _ptr(a), _ptr(b), _ptr(c), _ptr(d), len(dims), int(solvedim),
                _ints(dims), _ints(pads))
        else:
            rc = getattr(self.lib, f"ref_trid{p}mtsvStridedBatchInc")(
                None, _ptr(a), _ptr(b), _ptr(c), _ptr(d), _ptr(u), len(dims),
                int(solvedim), _ints(dims), _ints(pads))
        if rc != 0:
            raise ValueError(f"reference rc={rc}")

    def scalar(self, a, b, c, d, n, stride=1):
        """trid_scalar{D,S}: one system of n rows, `stride` apart, in place."""
        p = "D" if d.dtype == np.float64 else "S"
        getattr(self.lib, f"ref_trid_scalar{p}")(_ptr(a), _ptr(b), _ptr(c), _ptr(d),
                                                 int(n), int(stride))


def normwise_error(x, ref):
    """max|x - ref| / max|ref|, the parity measure for whole batches."""
    x = np.asarray(x, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    den = np.max(np.abs(ref)) if ref.size else 1.0
    return float(np.max(np.abs(x - ref)) / (den if den > 0 else 1.0)) if ref.size else 0.0


class _RefTridParams(ctypes.Structure):
    """struct TridParams (scalar/include/trid_params.h:31-35)."""
    _fields_ = [("mpi_params", ctypes.c_void_p), ("opts", ctypes.c_int * 3), ("sync", ctypes.c_int)]


class ReferenceGPU:
    """The reference's own CUDA library, scalar/src/cuda/trid_cuda.cu compiled
    for sm_100a from its sources (oracle/_ref/libtridcuda_ref.so, API symbols
    renamed ref_gpu_*). Takes device pointers; every call ends with the
    library's own cudaDeviceSynchronize. Its x path keeps transpose scratch
    sized in an int, so arrays must stay below 2^31 bytes; its vectorised
    y/z path assumes a system count divisible by 4 (FP32) or 2 (FP64) and
    dims[0] * sizeof a multiple of 16 whenever the pointers are aligned."""

    def __init__(self, path=None):
        path = path or os.path.join(REF_DIR, "libtridcuda_ref.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle` where the reference tree exists")
        self.path = path
        self.lib = ctypes.CDLL(path)
        for name in ("ref_gpu_tridDmtsvStridedBatch", "ref_gpu_tridSmtsvStridedBatch",
                     "ref_gpu_tridDmtsvStridedBatchInc", "ref_gpu_tridSmtsvStridedBatchInc"):
            fn = getattr(self.lib, name)
            fn.restype = ctypes.c_int
        self.ctx = _RefTridParams()  # opts 0: the library's defaults

    def strided_batch(self, a, b, c, d, dims, solvedim, dtype_bytes, pads=None, u=None, opts=None):
        """a, b, c, d, u: device addresses (ints). d <- x, or u += x."""
        pads = dims if pads is None else pads
        n = 1
        for v in pads:
            n *= int(v)
        if n * dtype_bytes >= 2 ** 31:
            raise ValueError("arrays of 2^31 bytes or more overflow the reference's scratch size")
        if opts is not None:
            for i, v in enumerate(opts):
                self.ctx.opts[i] = int(v)
        p = "D" if dtype_bytes == 8 else "S"
        vp = ctypes.c_void_p
        if u is None:
            rc = getattr(self.lib, f"ref_gpu_trid{p}mtsvStridedBatch")(
                ctypes.byref(self.ctx), vp(a), vp(b), vp(c), vp(d), len(dims), int(solvedim),
                _ints(dims), _ints(pads))
        else:
            rc = getattr(self.lib, f"ref_gpu_trid{p}mtsvStridedBatchInc")(
                ctypes.byref(self.ctx), vp(a), vp(b), vp(c), vp(d), vp(u), len(dims),
                int(solvedim), _ints(dims), _ints(pads))
        if rc != 0:
            raise ValueError(f"reference GPU rc={rc}")
