"""CPU: the C-ABI library loads, exports every declared symbol and rejects bad
arguments before touching a device (no compute calls here)."""

import ctypes
import subprocess

import pytest

import tridsolver_b200 as tb
from tridsolver_b200 import _lib
from tridsolver_b200.api import TridParams, TridStatus


@pytest.mark.parametrize("compiler,flags", [("gcc", ["-std=c99", "-x", "c"]),
                                            ("g++", ["-std=c++11", "-x", "c++"])])
def test_headers_compile_for_c_and_cxx_callers(compiler, flags, tmp_path):
    """include/*.h is the drop-in boundary: a C or C++ caller includes it
    as the reference's tridsolver.h, with the extensions beside it."""
    import os
    import shutil
    if shutil.which(compiler) is None:
        pytest.skip(f"{compiler} not installed")
    inc = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include")
    src = tmp_path / "caller.c"
    src.write_text('#include "tridsolver.h"\n#include "tridsolver_b200.h"\n'
                   "typedef tridStatus_t (*solve_fn)(const TridParams *, const double *,\n"
                   "    const double *, const double *, double *, int, int, const int *,\n"
                   "    const int *);\n"
                   "int main(void) { tridDistParams p; TridParams ctx; solve_fn f =\n"
                   "  tridDmtsvStridedBatch; (void)p; (void)ctx; (void)f; return 0; }\n")
    r = subprocess.run([compiler, *flags, "-Wall", "-Werror", "-fsyntax-only", "-I", inc, str(src)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_c_caller_links_and_runs_without_device(tmp_path):
    """A C program written against the reference's header links against the
    library in its place (-ltridsolver_b200 instead of -ltridcuda) and runs:
    argument errors and empty problems are answered before any device is
    touched, and a real solve without a usable device returns an error
    status instead of exiting."""
    import os
    import shutil
    import torch
    if shutil.which("gcc") is None:
        pytest.skip("gcc not installed")
    if torch.cuda.is_available():
        pytest.skip("a device is present: the GPU tests run real solves")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    libdir = os.path.dirname(_lib.LIB_PATH)
    src = tmp_path / "caller.c"
    src.write_text(
        '#include <stdio.h>\n#include "tridsolver.h"\n'
        "int main(void) {\n"
        "  double buf[8] = {0};\n"
        "  int dims[1] = {8}, pads[1] = {8}, empty[1] = {0};\n"
        "  TridParams ctx = {0};\n"
        "  tridStatus_t bad = tridDmtsvStridedBatch(&ctx, buf, buf, buf, buf, 1, 1, dims, pads);\n"
        "  tridStatus_t none = tridDmtsvStridedBatch(&ctx, buf, buf, buf, buf, 1, 0, empty, empty);\n"
        "  tridStatus_t real = tridDmtsvStridedBatch(&ctx, buf, buf, buf, buf, 1, 0, dims, pads);\n"
        '  printf("%d %d %d\\n", (int)bad, (int)none, (int)real);\n'
        "  return 0;\n}\n")
    exe = tmp_path / "caller"
    r = subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I", os.path.join(root, "include"),
                        str(src), "-o", str(exe), "-L", libdir, "-ltridsolver_b200",
                        f"-Wl,-rpath,{libdir}"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stderr
    bad, none, real = (int(v) for v in r.stdout.split())
    assert bad == TridStatus.INVALID_VALUE
    assert none == TridStatus.SUCCESS
    assert real not in (TridStatus.SUCCESS, TridStatus.INVALID_VALUE)


def test_library_loads():
    lib = _lib.load()
    assert lib is not None


def test_exports_every_header_symbol():
    declared = _lib.header_symbols()
    # the reference's four entry points are among them
    for name in ("tridDmtsvStridedBatch", "tridSmtsvStridedBatch", "tridDmtsvStridedBatchInc",
                 "tridSmtsvStridedBatchInc"):
        assert name in declared
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    missing = [n for n in declared if n not in exported]
    assert not missing, missing


def test_tridparams_layout_matches_reference():
    # struct TridParams {void *mpi_params; int opts[MAXDIM]; int sync;}
    assert ctypes.sizeof(TridParams) == 24
    assert TridParams.opts.offset == 8 and TridParams.sync.offset == 20


BAD = [
    dict(ndim=0, solvedim=0, dims=[4], pads=[4]),
    dict(ndim=4, solvedim=0, dims=[4, 4, 4, 4], pads=[4, 4, 4, 4]),
    dict(ndim=2, solvedim=2, dims=[4, 4], pads=[4, 4]),
    dict(ndim=2, solvedim=-1, dims=[4, 4], pads=[4, 4]),
    dict(ndim=2, solvedim=0, dims=[4, 4], pads=[3, 4]),     # pads[0] < dims[0]
    dict(ndim=3, solvedim=1, dims=[4, 4, 4], pads=[4, 2, 4]),
    dict(ndim=2, solvedim=0, dims=[-1, 4], pads=[4, 4]),
]


@pytest.mark.parametrize("case", BAD)
@pytest.mark.parametrize("fn", ["tridDmtsvStridedBatch", "tridSmtsvStridedBatch"])
def test_invalid_arguments(fn, case):
    dummy = 4096  # never dereferenced: validation fails first
    st = getattr(tb, fn)(None, dummy, dummy, dummy, dummy, case["ndim"], case["solvedim"],
                         case["dims"], case["pads"])
    assert st == TridStatus.INVALID_VALUE


def test_null_pointer_rejected():
    st = tb.tridDmtsvStridedBatch(None, None, 4096, 4096, 4096, 1, 0, [8], [8])
    assert st == TridStatus.INVALID_VALUE
    st = tb.tridDmtsvStridedBatchInc(None, 4096, 4096, 4096, 4096, None, 1, 0, [8], [8])
    assert st == TridStatus.INVALID_VALUE


def test_empty_problem_is_success_without_device():
    st = tb.tridDmtsvStridedBatch(None, None, None, None, None, 2, 1, [0, 5], [0, 5])
    assert st == TridStatus.SUCCESS
    ctx = TridParams()
    ctx.opts[0] = 4
    st = tb.tridSmtsvStridedBatchInc(ctx, None, None, None, None, None, 3, 2, [3, 0, 2], [3, 1, 2])
    assert st == TridStatus.SUCCESS


def test_tracing_ranges_wrap_calls():
    """With NVTX tracing on, calls still answer as before (the ranges are
    host-side and need no device)."""
    tb.set_tracing(True)
    try:
        st = tb.tridDmtsvStridedBatch(None, None, 4096, 4096, 4096, 1, 0, [8], [8])
        assert st == TridStatus.INVALID_VALUE
        st = tb.tridSmtsvStridedBatchInc(None, None, None, None, None, None, 2, 1, [0, 5], [0, 5])
        assert st == TridStatus.SUCCESS
    finally:
        tb.set_tracing(False)


def test_release_scratch_reports_missing_device():
    """Without a usable device the release returns an error status (raised
    as TridError), it does not crash."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present: the GPU tests cover the release")
    st = tb.load_library().tridReleaseScratch()
    assert st != TridStatus.SUCCESS
    with pytest.raises(tb.TridError):
        tb.release_scratch()


@pytest.mark.parametrize("dtype_bytes,dims,solvedim,expect", [
    (8, [512, 512, 512], 0, "hybrid M=16 T=32 W=1 smem"),
    (8, [512, 512, 512], 2, "hybrid M=32 T=16 W=32 wide"),
    (8, [512, 512, 512], 1, "hybrid M=16 T=32 W=16 stream"),
    (8, [256, 256, 256], 2, "hybrid M=32 T=8 W=32 wide"),
    (8, [16, 512, 300], 2, "hybrid M=32 T=16 W=32 wide"),
    (8, [15, 512, 300], 2, "hybrid M=16 T=32 W=16 stream"),
    (8, [7, 512, 3], 1, "hybrid M=8 T=64 W=8"),
    (8, [8, 512, 3], 1, "hybrid M=16 T=32 W=16 stream"),
    (4, [512, 512, 512], 2, "hybrid M=32 T=16 W=64 wide pairs"),
    (4, [256, 256, 256], 2, "hybrid M=16 T=16 W=64 wide pairs"),
    (4, [512, 512, 512], 1, "hybrid M=16 T=32 W=32 stream"),
    (4, [256, 256, 256], 1, "hybrid M=16 T=16 W=64 wide pairs"),
    (4, [128, 100, 2], 1, "hybrid M=16 T=8 W=64 wide pairs"),
    (4, [96, 100, 2], 1, "hybrid M=8 T=16 W=32 stream"),
    (4, [96, 200, 2], 1, "hybrid M=16 T=16 W=32 stream"),
    (4, [3, 100, 2], 1, "hybrid M=8 T=16 W=4"),
    (4, [16, 100, 2], 1, "hybrid M=8 T=16 W=32 stream"),
    (8, [256, 256, 256], 1, "hybrid M=8 T=32 W=16 stream"),
    (8, [64, 65], 1, "hybrid M=4 T=32 W=16 stream"),
    (8, [64, 64], 1, "hybrid M=8 T=8 W=32"),
    (8, [8, 8, 1024], 2, "hybrid M=8 T=128 W=4"),
    (4, [1024, 8], 0, "hybrid M=32 T=32"),
    (4, [256, 256, 256], 0, "hybrid M=16 T=16 W=1 vec"),
    (4, [128, 256, 2], 0, "hybrid M=8 T=16 W=1 vec"),
    (8, [256, 256, 256], 0, "hybrid M=8 T=32 W=1 smem"),
    (8, [100000], 0, "long"),
    (8, [5, 7], 1, "hybrid M=8 T=1"),
])
def test_plan_table(dtype_bytes, dims, solvedim, expect):
    assert tb.describe_plan(dtype_bytes, dims, solvedim).startswith(expect)


@pytest.mark.parametrize("dtype_bytes,dims,solvedim,expect", [
    (4, [512, 512, 512], 1, "hybrid M=32 T=16 W=64 wide pairs"),
    (8, [512, 512, 512], 1, "hybrid M=32 T=16 W=32 wide"),
    (8, [512, 512, 512], 2, "hybrid M=32 T=16 W=32 wide"),
    (4, [96, 200, 2], 1, "hybrid M=8 T=32 W=32 stream"),
])
def test_plan_table_inc(dtype_bytes, dims, solvedim, expect):
    """The Inc variant's plan (u a fifth stream): the wide kernel takes FP64
    and paired FP32 Inc solves along y too."""
    assert tb.describe_plan(dtype_bytes, dims, solvedim, inc=True).startswith(expect)


def test_force_plan_round_trip():
    tb.force_plan(tb.FAMILY_PCR)
    assert tb.describe_plan(8, [20, 10], 0).startswith("pcr M=1 T=32")
    tb.force_plan(tb.FAMILY_LONG, 8)
    assert tb.describe_plan(8, [100, 10], 0).startswith("long M=8")
    # too short for the multi-block path: falls back to the hybrid
    assert tb.describe_plan(8, [20, 10], 0).startswith("hybrid")
    tb.force_plan(tb.FAMILY_HYBRID, 4)
    assert tb.describe_plan(8, [20, 10], 0).startswith("hybrid M=4 T=8")
    tb.force_plan()
    with pytest.raises(tb.TridError):
        tb.force_plan(tb.FAMILY_HYBRID, 3)


def test_blocking_and_stream_settings():
    assert tb.get_blocking() is True
    tb.set_blocking(False)
    assert tb.get_blocking() is False
    tb.set_blocking(True)
    tb.set_stream(None)
    assert _lib.load().tridGetStream() in (None, 0)


def test_no_alloc_entry_refuses_a_distributed_ctx():
    """tridDmtsvStridedBatchNoAlloc has no distributed solve: a ctx whose
    mpi_params were registered by tridDistInit is refused before any device
    is touched, instead of solving only the local block."""
    import numpy as np
    from tridsolver_b200.distributed import DistContext

    fn = _lib.load().tridDmtsvStridedBatchNoAlloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p] * 5 + [ctypes.c_int, ctypes.c_int,
                                            ctypes.POINTER(ctypes.c_int),
                                            ctypes.POINTER(ctypes.c_int)]
    buf = np.zeros(64)
    ptr = buf.ctypes.data
    dims = (ctypes.c_int * 2)(8, 8)
    with DistContext(1, rank=0, nranks=1, allgather=lambda *a: None) as dc:
        st = fn(ctypes.addressof(dc.ctx), ptr, ptr, ptr, ptr, 2, 1, dims, dims)
    assert st == TridStatus.INVALID_VALUE
    assert not buf.any()


def test_sized_ragged_call_checks_its_count_without_device():
    """The sized ragged entry points refuse a negative element count, and an
    empty batch succeeds, before any device is touched."""
    for fn in (tb.tridDmtsvRaggedBatchSized, tb.tridSmtsvRaggedBatchSized):
        assert fn(None, None, None, None, None, None, 0, -1) == TridStatus.INVALID_VALUE
        assert fn(None, None, None, None, None, None, 0, 0) == TridStatus.SUCCESS
        assert fn(None, None, None, None, None, None, -3, 0) == TridStatus.INVALID_VALUE
