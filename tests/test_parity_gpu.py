"""GPU parity: the CUDA path, called through the C ABI, against the oracle.

* the reference generator's golden fixtures, plain and padded, with the
  reference tests' tolerances (scalar/test/test_cuda.cu:38-174);
* seeded batches of every layout, odd and tiny sizes, Inc, unaligned and
  padded pointers, against the plain-C restatement and the reference's own
  CPU library: normwise relative error <= 1e-12 (FP64) / 1e-5 (FP32);
* every kernel family (hybrid for each rows-per-thread, pure PCR, the long
  multi-block path) forced on the same problems;
* the full benchmark grids (256^3, 512^3 FP64) through size-independent
  checks: the residual of T x = d, and sampled systems against the oracle.
"""

import numpy as np
import pytest
import torch

import tridsolver_b200 as tb
from fixtures import CASE_NAMES, allclose_ref, load_case
from helpers import from_padded, make_system, normwise, pad_offset, padded_index, to_padded
from oracle.pyoracle import Reference, Restatement

pytestmark = pytest.mark.gpu

DEV = "cuda:0"
TOL = {np.float64: 1e-12, np.float32: 1e-5}
TORCH = {np.float64: torch.float64, np.float32: torch.float32}


@pytest.fixture(scope="module")
def oracle():
    return Restatement()


@pytest.fixture(scope="module")
def reference():
    try:
        return Reference()
    except FileNotFoundError:
        return None


@pytest.fixture(autouse=True)
def _reset_plan():
    tb.force_plan()
    yield
    tb.force_plan()


def gpu(x):
    return torch.from_numpy(np.ascontiguousarray(x)).to(DEV)


def run_gpu(a, b, c, d, dims, solvedim, pads=None, u=None, offset=0, ctx=None):
    """Copy to the device, solve through the C ABI (blocking), copy back."""
    pads = dims if pads is None else pads
    ta, tb_, tc, td = (gpu(v) for v in (a, b, c, d))
    tu = gpu(u) if u is not None else None
    es = ta.element_size()
    ptr = lambda t: t.data_ptr() + offset * es  # noqa: E731
    dbl = d.dtype == np.float64
    if u is None:
        fn = tb.tridDmtsvStridedBatch if dbl else tb.tridSmtsvStridedBatch
        st = fn(ctx, ptr(ta), ptr(tb_), ptr(tc), ptr(td), len(dims), solvedim, dims, pads)
    else:
        fn = tb.tridDmtsvStridedBatchInc if dbl else tb.tridSmtsvStridedBatchInc
        st = fn(ctx, ptr(ta), ptr(tb_), ptr(tc), ptr(td), ptr(tu), len(dims), solvedim, dims, pads)
    torch.cuda.synchronize()
    return st, td.cpu().numpy(), (tu.cpu().numpy() if tu is not None else None)


# ---- golden fixtures ------------------------------------------------------------

@pytest.mark.parametrize("dt", [np.float64, np.float32])
@pytest.mark.parametrize("name", CASE_NAMES)
def test_golden(name, dt):
    case = load_case(name)
    a, b, c, d = (case[k].astype(dt) for k in "abcd")
    ctx = tb.TridParams()
    ctx.opts[0] = 1 if len(case["dims"]) == 1 else 0  # as scalar/test/test_cuda.cu:18
    st, out, _ = run_gpu(a, b, c, d, case["dims"], case["solvedim"], ctx=ctx)
    assert st == 0
    exp = case["u"] if dt == np.float64 else case["u_float"]
    ok, worst, diff = allclose_ref(exp, out, dt)
    assert ok, (worst, diff)


@pytest.mark.parametrize("dt", [np.float64, np.float32])
@pytest.mark.parametrize("name", CASE_NAMES)
def test_golden_padded(name, dt):
    case = load_case(name)
    dims = case["dims"]
    pads = [n + 2 for n in dims]
    arrs = [to_padded(case[k].astype(dt), dims, pads, fill=7.0) for k in "abcd"]
    st, out, _ = run_gpu(*arrs, dims, case["solvedim"], pads=pads, offset=pad_offset(pads))
    assert st == 0
    exp = case["u"] if dt == np.float64 else case["u_float"]
    ok, worst, diff = allclose_ref(exp, from_padded(out, dims, pads), dt)
    assert ok, (worst, diff)
    mask = np.ones(out.size, bool)
    mask[padded_index(dims, pads)] = False
    assert np.all(out[mask] == 7.0), "padding was written"


# ---- seeded batches against the oracle --------------------------------------------

SHAPES = [([1], 0), ([2], 0), ([3], 0), ([31], 0), ([33], 0), ([200], 0), ([201], 0), ([1000], 0),
          ([1023], 0), ([1, 1, 1000], 2),
          ([5, 3], 1), ([33, 31], 0), ([33, 31], 1), ([9, 10, 11], 0), ([9, 10, 11], 1),
          ([9, 10, 11], 2), ([64, 48, 40], 0), ([64, 48, 40], 1), ([64, 48, 40], 2),
          ([256, 16, 8], 0), ([7, 512, 3], 1), ([4, 3, 512], 2), ([1, 1, 700], 2),
          ([511, 2, 2], 0), ([3, 257, 5], 1),
          # strided: reduced rows per lane 2, 4 and 8, a partial group of
          # systems, lengths that do not fill the chunks
          ([50, 3, 200], 2), ([17, 700, 2], 1), ([33, 5, 400], 2), ([40, 130], 1)]


def _check(dims, solvedim, dt, inc, oracle, reference, pads=None, offset=0, seed=0):
    a, b, c, d = make_system(dims, solvedim, dt, seed=seed)
    u0 = np.random.default_rng(seed + 1).standard_normal(d.size).astype(dt) if inc else None
    want_d = d.copy()
    want_u = u0.copy() if inc else None
    oracle.strided_batch(a, b, c, want_d, dims, solvedim, u=want_u)
    want = want_u if inc else want_d
    if pads is not None:
        arrs = [to_padded(v, dims, pads, fill=3.0) for v in (a, b, c, d)]
        up = to_padded(u0, dims, pads, fill=3.0) if inc else None
        st, od, ou = run_gpu(*arrs, dims, solvedim, pads=pads, u=up, offset=pad_offset(pads))
        got = from_padded(ou if inc else od, dims, pads)
        if inc:
            assert np.array_equal(from_padded(od, dims, pads), d)
    else:
        pre = [np.concatenate([np.full(offset, 5.0, dt), v]) for v in (a, b, c, d)]
        up = np.concatenate([np.full(offset, 5.0, dt), u0]) if inc else None
        st, od, ou = run_gpu(*pre, dims, solvedim, u=up, offset=offset)
        got = (ou if inc else od)[offset:]
        if inc:
            assert np.array_equal(od[offset:], d), "Inc must leave d untouched"
    assert st == 0, st
    err = normwise(got, want)
    assert err <= TOL[dt], err
    if reference is not None and max(dims) <= 16384:
        rd = d.copy()
        ru = u0.copy() if inc else None
        reference.strided_batch(a, b, c, rd, dims, solvedim, u=ru)
        assert normwise(got, ru if inc else rd) <= TOL[dt]


@pytest.mark.parametrize("dt", [np.float64, np.float32])
@pytest.mark.parametrize("inc", [False, True])
@pytest.mark.parametrize("dims,solvedim", SHAPES)
def test_random_against_oracle(dims, solvedim, inc, dt, oracle, reference):
    _check(dims, solvedim, dt, inc, oracle, reference, seed=sum(dims) + solvedim)


@pytest.mark.parametrize("dt", [np.float64, np.float32])
@pytest.mark.parametrize("dims,solvedim", [([64, 48, 40], 0), ([64, 48, 40], 1), ([64, 48, 40], 2),
                                           ([256, 16, 8], 0), ([30, 200], 0)])
def test_unaligned_pointers(dims, solvedim, dt, oracle, reference):
    """Interior pointers one element off any 16-byte boundary (no vector path)."""
    _check(dims, solvedim, dt, False, oracle, reference, offset=1)


@pytest.mark.parametrize("dt", [np.float64, np.float32])
@pytest.mark.parametrize("inc", [False, True])
@pytest.mark.parametrize("dims,solvedim,extra", [([64, 48, 40], 0, [2, 3, 1]), ([64, 48, 40], 1, [2, 3, 1]),
                                                 ([64, 48, 40], 2, [5, 1, 4]), ([256, 6], 0, [0, 4]),
                                                 ([100, 20, 3], 1, [28, 0, 0])])
def test_padded(dims, solvedim, extra, inc, dt, oracle, reference):
    pads = [n + e for n, e in zip(dims, extra)]
    _check(dims, solvedim, dt, inc, oracle, reference, pads=pads)


FORCED = [(tb.FAMILY_HYBRID, m) for m in (2, 4, 8, 16, 32)] + \
         [(tb.FAMILY_PCR, 0), (tb.FAMILY_LONG, 8), (tb.FAMILY_LONG, 16)]


@pytest.mark.parametrize("dt", [np.float64, np.float32])
@pytest.mark.parametrize("family,m", FORCED)
@pytest.mark.parametrize("dims,solvedim", [([32, 20, 6], 0), ([12, 29, 7], 1), ([9, 5, 30], 2),
                                           ([130, 40], 0), ([40, 130], 1)])
def test_every_family(dims, solvedim, family, m, dt, oracle, reference):
    tb.force_plan(family, m)
    _check(dims, solvedim, dt, solvedim == 2, oracle, reference, seed=family * 10 + m)


@pytest.mark.parametrize("dt", [np.float64, np.float32])
@pytest.mark.parametrize("inc", [False, True])
@pytest.mark.parametrize("tma", [1, 0])
@pytest.mark.parametrize("dims,solvedim", [([48, 37, 20], 1), ([48, 37, 20], 2), ([24, 300, 3], 1),
                                           ([20, 3, 260], 2), ([12, 7, 513], 2), ([64, 40], 1),
                                           ([8, 9, 16], 2)])
def test_tma_tiles(dims, solvedim, tma, inc, dt, oracle, reference):
    """TMA tile path against the per-thread-load path and the oracle: partial
    groups of systems, lengths that end inside a box, two and three boxes."""
    tb.force_tma(tma)
    try:
        _check(dims, solvedim, dt, inc, oracle, reference, seed=tma + 2 * inc)
    finally:
        tb.force_tma(-1)


@pytest.mark.parametrize("inc", [False, True])
@pytest.mark.parametrize("offset", [0, 2, 1])
@pytest.mark.parametrize("dims,solvedim", [([64, 7, 100], 2), ([128, 3, 200], 2), ([64, 300, 3], 1),
                                           ([128, 5, 511], 2), ([64, 257], 1), ([192, 66], 1),
                                           ([64, 2, 256], 2), ([64, 129, 2], 1)])
def test_wide_pairs(dims, solvedim, inc, offset, oracle, reference):
    """FP32 wide kernel in the paired form (two adjacent systems a thread,
    8-byte accesses): every chunk count and size (8 x 16, 8 x 32, 16 x 32
    rows), lengths that end inside a chunk; an odd offset (arrays not 8-byte
    aligned) takes the unpaired form."""
    tb.force_stream(2)
    try:
        _check(dims, solvedim, np.float32, inc, oracle, reference, offset=offset,
               seed=11 + offset + 2 * inc + solvedim)
    finally:
        tb.force_stream(-1)


@pytest.mark.parametrize("inc", [False, True])
@pytest.mark.parametrize("dims,pads,solvedim", [([64, 30, 100], [66, 32, 100], 2),
                                                ([64, 30, 100], [65, 31, 100], 2),
                                                ([128, 150, 3], [130, 150, 3], 1)])
def test_wide_pairs_padded(dims, pads, solvedim, inc, oracle, reference):
    """Padded FP32 batches in the wide kernel. In the reference's layout the
    arrays start at element (1, 1, 1) of the padded grid, an odd offset for
    any pads that keep the strides even, so these take the unpaired form."""
    tb.force_stream(2)
    try:
        _check(dims, solvedim, np.float32, inc, oracle, reference, pads=pads, seed=21 + 2 * inc)
    finally:
        tb.force_stream(-1)


@pytest.mark.parametrize("dt", [np.float64, np.float32])
@pytest.mark.parametrize("inc", [False, True])
@pytest.mark.parametrize("stream", [2, 1, 0])
@pytest.mark.parametrize("dims,solvedim", [([48, 37, 100], 2), ([24, 300, 3], 1), ([20, 3, 260], 2),
                                           ([7, 130, 5], 1), ([64, 65], 1), ([5, 9, 512], 2),
                                           ([33, 17, 129], 2), ([40, 257], 1), ([70, 3, 300], 2),
                                           ([96, 2, 511], 2), ([200, 129], 1)])
def test_streaming_kernel(dims, solvedim, stream, inc, dt, oracle, reference):
    """Persistent streaming strided kernels (2: 256-byte groups with the state
    in tensor memory, 1: 128-byte groups) against the register-tile kernel
    and the oracle: partial groups, every chunk size, lengths that end inside
    a chunk, groups fewer than the grid and many per CTA."""
    tb.force_stream(stream)
    try:
        _check(dims, solvedim, dt, inc, oracle, reference, seed=3 + stream + 2 * inc)
    finally:
        tb.force_stream(-1)


@pytest.mark.parametrize("dt", [np.float64, np.float32])
@pytest.mark.parametrize("dims,solvedim", [([100000], 0), ([3, 20000], 1), ([2, 2, 9000], 2),
                                           ([70000, 3], 0)])
def test_long_systems(dims, solvedim, dt, oracle, reference):
    _check(dims, solvedim, dt, True, oracle, None, seed=5)


@pytest.mark.parametrize("dt", [np.float64, np.float32])
@pytest.mark.parametrize("inc", [False, True])
@pytest.mark.parametrize("dims,solvedim,pads", [([513, 3], 0, None), ([1025, 2], 0, None),
                                                ([1537, 5], 0, None), ([70001, 2], 0, None),
                                                ([4097, 3, 2], 0, [4099, 3, 2]),
                                                ([2048, 4], 0, [2051, 4]), ([600, 33], 0, None)])
def test_long_contiguous_tiles(dims, solvedim, pads, inc, dt, oracle, reference):
    """Long contiguous systems in warp tiles (two passes around the
    second-level solve): partial last tiles, one to 137 tiles per system,
    system starts off the 16-byte grid (odd padding), Inc."""
    assert "tiles" in tb.describe_plan(np.dtype(dt).itemsize, dims, solvedim, pads) or \
        dims[0] <= (512 if dt == np.float64 else 1024)
    _check(dims, solvedim, dt, inc, oracle, reference if pads is None else None, pads=pads, seed=21)


def test_zero_pivot_reported(oracle):
    a, b, c, d = make_system([16, 8], 0, np.float64)
    a[:] = 0.0
    c[:] = 0.0
    b[37] = 0.0
    st, out, _ = run_gpu(a, b, c, d, [16, 8], 0)
    assert st == tb.TridStatus.ZERO_PIVOT
    a, b, c, d = make_system([16, 8], 0, np.float64)
    st, out, _ = run_gpu(a, b, c, d, [16, 8], 0)
    assert st == 0


@pytest.mark.parametrize("dt,emax", [(np.float64, 1000), (np.float32, 120)])
@pytest.mark.parametrize("n", [256, 512])
def test_contiguous_reciprocal_within_one_ulp(n, dt, emax):
    """Contiguous systems invert their pivots with the hardware reciprocal
    estimate (FP64: refined by two Newton-Raphson steps). With a = c = 0 and
    d = 1 the solution is that reciprocal itself, which must lie within one
    unit in the last place of the correctly rounded 1/b, over pivots from
    2^-emax to 2^emax of either sign. A zero pivot on the same path is still
    reported."""
    dims = [n, 64]
    # the warp-per-system shared-memory kernel (FP32 systems of 256 rows
    # take two per warp by default)
    tb.force_plan(tb.FAMILY_HYBRID, n // 32)
    assert "smem" in tb.describe_plan(np.dtype(dt).itemsize, dims, 0)
    rng = np.random.default_rng(n)
    count = n * 64
    b = rng.uniform(1.0, 2.0, count) * np.exp2(rng.integers(-emax, emax, count).astype(np.float64))
    b = (b * rng.choice([-1.0, 1.0], count)).astype(dt)
    a = np.zeros(count, dt)
    c = np.zeros(count, dt)
    d = np.ones(count, dt)
    st, out, _ = run_gpu(a, b, c, d, dims, 0)
    assert st == 0
    want = (1.0 / b.astype(np.float64)).astype(dt)
    ulps = np.abs(out.astype(np.float64) - want) / np.spacing(np.abs(want)).astype(np.float64)
    assert ulps.max() <= 1.0, ulps.max()
    b[n + 77] = 0.0
    st, out, _ = run_gpu(a, b, c, d, dims, 0)
    assert st == tb.TridStatus.ZERO_PIVOT


def test_solve_with_tracing_on(oracle):
    """NVTX ranges around the calls change nothing in the results."""
    dims, sd = [64, 48, 40], 2
    a, b, c, d = make_system(dims, sd, np.float64, seed=11)
    tb.set_tracing(True)
    try:
        st, out, _ = run_gpu(a, b, c, d, dims, sd)
    finally:
        tb.set_tracing(False)
    assert st == 0
    want = d.copy()
    oracle.strided_batch(a, b, c, want, dims, sd)
    assert normwise(out, want) <= 1e-12


def test_async_stream_matches_blocking(oracle):
    dims, sd = [64, 48, 40], 1
    a, b, c, d = make_system(dims, sd, np.float64, seed=9)
    ta, tb_, tc, td = (gpu(v) for v in (a, b, c, d))
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        tb.strided_batch(ta, tb_, tc, td, sd, dims)
    s.synchronize()
    want = d.copy()
    oracle.strided_batch(a, b, c, want, dims, sd)
    assert normwise(td.cpu().numpy(), want) <= 1e-12


def test_torch_solve_dim_mapping(oracle):
    x = torch.randn(6, 7, 8, dtype=torch.float64, device=DEV)
    for dim in range(3):
        a = torch.rand_like(x) - 0.5
        c = torch.rand_like(x) - 0.5
        b = 1 + a.abs() + c.abs() + torch.rand_like(x)
        d = x.clone()
        tb.solve(a, b, c, d, dim=dim)
        torch.cuda.synchronize()
        dims = [8, 7, 6]
        want = x.cpu().numpy().reshape(-1).copy()
        oracle.strided_batch(*(t.cpu().numpy().reshape(-1).copy() for t in (a, b, c)), want,
                             dims, 2 - dim)
        assert normwise(d.cpu().numpy().reshape(-1), want) <= 1e-12


# ---- full-size grids: size-independent properties ------------------------------------------

def _residual(a, b, c, x, d, tdim):
    """max |T x - d| / max |d| along torch dim tdim (a[0], c[N-1] ignored)."""
    n = x.shape[tdim]
    xm = torch.zeros_like(x)
    xp = torch.zeros_like(x)
    xm.narrow(tdim, 1, n - 1).copy_(x.narrow(tdim, 0, n - 1))
    xp.narrow(tdim, 0, n - 1).copy_(x.narrow(tdim, 1, n - 1))
    r = b * x + a * xm + c * xp - d
    return (r.abs().max() / d.abs().max()).item()


@pytest.mark.parametrize("n", [256, 512])
@pytest.mark.parametrize("solvedim", [0, 1, 2])
def test_full_grid_fp64(n, solvedim, oracle):
    g = torch.Generator(device=DEV).manual_seed(n + solvedim)
    shape = (n, n, n)
    tdim = 2 - solvedim
    a = torch.rand(shape, generator=g, device=DEV, dtype=torch.float64) - 0.5
    c = torch.rand(shape, generator=g, device=DEV, dtype=torch.float64) - 0.5
    b = 1 + a.abs() + c.abs() + torch.rand(shape, generator=g, device=DEV, dtype=torch.float64)
    a.narrow(tdim, 0, 1).zero_()
    c.narrow(tdim, n - 1, 1).zero_()
    d = torch.randn(shape, generator=g, device=DEV, dtype=torch.float64)
    x = d.clone()
    st = tb.tridDmtsvStridedBatch(None, a, b, c, x, 3, solvedim, [n] * 3, [n] * 3)
    assert st == 0
    assert _residual(a, b, c, x, d, tdim) <= 1e-13
    # 64 sampled systems against the oracle
    idx = torch.randint(0, n * n, (64,), generator=g, device=DEV)
    lines = [t.movedim(tdim, -1).reshape(-1, n).index_select(0, idx).cpu().numpy()
             for t in (a, b, c, d, x)]
    sa, sb, sc, sd, sx = (np.ascontiguousarray(v.reshape(-1)) for v in lines)
    want = sd.copy()
    oracle.strided_batch(sa, sb, sc, want, [n, 64], 0)
    assert normwise(sx, want) <= 1e-12
    del a, b, c, d, x
    torch.cuda.empty_cache()
