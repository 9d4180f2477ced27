"""CPU: pin the oracle before trusting it.

The plain-C restatement (oracle/trid_oracle.c) and the reference's own CPU
library compiled from its sources (oracle/_ref) must both reproduce the golden
fixtures made by the reference's generator, with the reference tests'
tolerances and padded layouts (scalar/test/test_cpu.cpp:68-128, 175-352), and
must agree with each other on seeded batches of every layout, odd sizes and
the Inc variant.
"""

import numpy as np
import pytest

from fixtures import CASE_NAMES, allclose_ref, load_case
from helpers import from_padded, make_system, normwise, pad_offset, to_padded
from oracle.pyoracle import Reference, Restatement

DTYPES = [np.float64, np.float32]


@pytest.fixture(scope="module")
def restatement():
    return Restatement()


@pytest.fixture(scope="module")
def reference():
    try:
        return Reference()
    except FileNotFoundError as e:  # the reference tree is not here
        pytest.skip(str(e))


def _expected(case, dt):
    return case["u"] if dt == np.float64 else case["u_float"]


@pytest.mark.parametrize("dt", DTYPES)
@pytest.mark.parametrize("name", CASE_NAMES)
@pytest.mark.parametrize("which", ["restatement", "reference"])
def test_golden(which, name, dt, request):
    lib = request.getfixturevalue(which)
    case = load_case(name)
    a, b, c, d = (np.ascontiguousarray(case[k].astype(dt)) for k in "abcd")
    lib.strided_batch(a, b, c, d, case["dims"], case["solvedim"])
    ok, worst, diff = allclose_ref(_expected(case, dt), d, dt)
    assert ok, f"{which} {name} worst index {worst} diff {diff}"


@pytest.mark.parametrize("dt", DTYPES)
@pytest.mark.parametrize("name", CASE_NAMES)
@pytest.mark.parametrize("which", ["restatement", "reference"])
def test_golden_padded(which, name, dt, request):
    """Every dimension padded by 2, pointers offset to the first interior
    element (scalar/test/test_cpu.cpp:86-128)."""
    lib = request.getfixturevalue(which)
    case = load_case(name)
    dims = case["dims"]
    pads = [n + 2 for n in dims]
    arrs = [to_padded(case[k].astype(dt), dims, pads, fill=0.0) for k in "abcd"]
    off = pad_offset(pads)
    views = [v[off:] for v in arrs]
    lib.strided_batch(*views, dims, case["solvedim"], pads=pads)
    out = from_padded(arrs[3], dims, pads)
    ok, worst, diff = allclose_ref(_expected(case, dt), out, dt)
    assert ok, f"{which} {name} worst index {worst} diff {diff}"
    # padding untouched
    mask = np.ones(arrs[3].size, bool)
    from helpers import padded_index
    mask[padded_index(dims, pads)] = False
    assert np.all(arrs[3][mask] == 0.0)


SHAPES = [([1], 0), ([7], 0), ([33, 5], 0), ([33, 5], 1), ([9, 10, 11], 0), ([9, 10, 11], 1),
          ([9, 10, 11], 2), ([64, 64, 64], 0), ([64, 64, 64], 1), ([64, 64, 64], 2),
          ([3, 1000], 1), ([1000, 2], 0)]


@pytest.mark.parametrize("dt", DTYPES)
@pytest.mark.parametrize("inc", [False, True])
@pytest.mark.parametrize("dims,solvedim", SHAPES)
def test_restatement_matches_reference(dims, solvedim, inc, dt, restatement, reference):
    a, b, c, d = make_system(dims, solvedim, dt, seed=len(dims) * 7 + solvedim)
    u0 = np.random.default_rng(3).standard_normal(d.size).astype(dt) if inc else None
    outs = []
    for lib in (restatement, reference):
        dd = d.copy()
        uu = u0.copy() if inc else None
        lib.strided_batch(a, b, c, dd, dims, solvedim, u=uu)
        outs.append(uu if inc else dd)
        if inc:
            assert np.array_equal(dd, d), "Inc must leave d untouched"
    tol = 1e-13 if dt == np.float64 else 2e-6
    assert normwise(outs[0], outs[1]) <= tol


def test_ragged_oracle_matches_reference_scalar(restatement, reference):
    rng = np.random.default_rng(11)
    lens = rng.integers(1, 300, size=40)
    offs = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
    n = int(offs[-1])
    a, b, c, d = make_system([n], 0, np.float64, seed=5)
    d1 = d.copy()
    restatement.ragged(a, b, c, d1, offs)
    d2 = d.copy()
    for k in range(len(lens)):
        s, e = offs[k], offs[k + 1]
        seg = [np.ascontiguousarray(v[s:e]) for v in (a, b, c)]
        dd = np.ascontiguousarray(d2[s:e])
        reference.scalar(*seg, dd, e - s)
        d2[s:e] = dd
    assert normwise(d1, d2) <= 1e-13


def test_adjoint_oracle_against_finite_differences(restatement):
    dims, sd = [6, 20, 5], 1
    a, b, c, d = make_system(dims, sd, np.float64, seed=21)
    w = np.random.default_rng(2).standard_normal(d.size)
    x = d.copy()
    restatement.strided_batch(a, b, c, x, dims, sd)
    abar, bbar, cbar, dbar = restatement.adjoint(a, b, c, x, w, dims, sd)

    def loss(aa, bb, cc, dd):
        xx = dd.copy()
        restatement.strided_batch(aa, bb, cc, xx, dims, sd)
        return float(np.dot(w, xx))

    rng = np.random.default_rng(4)
    h = 1e-6
    for which, grad in (("a", abar), ("b", bbar), ("c", cbar), ("d", dbar)):
        for idx in rng.integers(0, d.size, 20):
            arrs = {"a": a, "b": b, "c": c, "d": d}
            p = {k: v.copy() for k, v in arrs.items()}
            m = {k: v.copy() for k, v in arrs.items()}
            p[which][idx] += h
            m[which][idx] -= h
            fd = (loss(p["a"], p["b"], p["c"], p["d"]) - loss(m["a"], m["b"], m["c"], m["d"])) / (2 * h)
            assert abs(fd - grad[idx]) <= 1e-6 * max(1.0, abs(fd)), (which, idx, fd, grad[idx])


def test_invalid_arguments_rejected(restatement):
    a, b, c, d = make_system([4, 4], 0)
    with pytest.raises(ValueError):
        restatement.strided_batch(a, b, c, d, [4, 4], 2)


try:
    from hypothesis import HealthCheck, given, settings
    from hypothesis import strategies as hs
except ImportError:  # pragma: no cover
    given = None


if given is not None:
    @settings(max_examples=300, deadline=None, suppress_health_check=[HealthCheck.function_scoped_fixture])
    @given(data=hs.data())
    def test_fuzz_restatement_against_reference(data, restatement, reference):
        """Random shapes, system directions, paddings (pointer at the first
        interior element, as scalar/test/test_cpu.cpp:86-128 does), Inc and
        precision: the restatement and the reference's own library agree on
        the interior, and Inc leaves d as it was."""
        ndim = data.draw(hs.integers(1, 3))
        dims = [data.draw(hs.integers(1, 24)) for _ in range(ndim)]
        solvedim = data.draw(hs.integers(0, ndim - 1))
        pads = [n + data.draw(hs.integers(0, 2)) for n in dims]
        inc = data.draw(hs.booleans())
        dt = data.draw(hs.sampled_from(DTYPES))
        seed = data.draw(hs.integers(0, 2 ** 31 - 1))
        a, b, c, d = make_system(dims, solvedim, dt, seed=seed)
        u0 = np.random.default_rng(seed + 1).standard_normal(d.size).astype(dt) if inc else None
        off = pad_offset(pads)
        span = off + int(np.prod(pads))

        def padded(v, fill=3.0):
            # the whole padded extent from the interior pointer on: the
            # reference's vectorised x sweep (pads[0] a multiple of the SIMD
            # width) reads every padded row in full, beyond the last interior
            # row's end, and solves the padded rows as part of the system
            # (pads[0] rows, not dims[0]). With c = 0 on the last interior row
            # the interior does not depend on them, as long as they are a
            # nonsingular continuation: a = c = 0 there, b = d = 3 (a = b =
            # c = 3 gives a zero pivot on the second padded row, and its NaN
            # reaches the interior through 0 * NaN)
            full = to_padded(v, dims, pads, fill=fill)
            return np.concatenate([full, np.full(max(0, span - full.size), fill, dt)])

        outs = []
        for lib in (restatement, reference):
            arrs = [padded(v, f) for v, f in zip((a, b, c, d), (0.0, 3.0, 0.0, 3.0))]
            up = padded(u0) if inc else None
            lib.strided_batch(*(v[off:] for v in arrs), dims, solvedim, pads=pads,
                              u=up[off:] if inc else None)
            got = from_padded(up if inc else arrs[3], dims, pads)
            outs.append(got)
            if inc:
                assert np.array_equal(from_padded(arrs[3], dims, pads), d)
        tol = 1e-13 if dt == np.float64 else 2e-6
        assert normwise(outs[0], outs[1]) <= tol, (dims, solvedim, pads, inc, dt)


@pytest.mark.parametrize("dt", DTYPES)
@pytest.mark.parametrize("shape", [(9, 7, 6), (17, 12, 10), (3, 3, 3)])
def test_adi_oracle_matches_reference_solves(shape, dt, restatement, reference):
    """The ADI oracle step (stencil, then x and y solves overwriting du and a
    z solve adding into u) equals the same step built from numpy's 7-point
    stencil and the reference library's own tridDmtsvStridedBatch / ...Inc,
    the structure of apps/adi/src/adi_cpu.cpp:209-270 with the RHS of
    apps/adi/src/preproc.hpp:173-214 (identity rows on the boundary)."""
    nx, ny, nz = shape
    rng = np.random.default_rng(nx * 100 + ny)
    lam = 0.37
    ca, cb = -lam, 1 + 2 * lam
    u0 = np.zeros((nz, ny, nx))
    u0[1:-1, 1:-1, 1:-1] = rng.standard_normal((nz - 2, ny - 2, nx - 2))
    u0 = u0.astype(dt)

    u_oracle = u0.ravel().copy()
    restatement.adi_step(u_oracle, lam, ca, cb, nx, ny, nz)

    u = u0.astype(np.float64)
    du = np.zeros_like(u)
    du[1:-1, 1:-1, 1:-1] = lam * (u[1:-1, 1:-1, :-2] + u[1:-1, 1:-1, 2:] + u[1:-1, :-2, 1:-1]
                                  + u[1:-1, 2:, 1:-1] + u[:-2, 1:-1, 1:-1] + u[2:, 1:-1, 1:-1]
                                  - 6 * u[1:-1, 1:-1, 1:-1])
    inner = np.zeros_like(u, dtype=bool)
    inner[1:-1, 1:-1, 1:-1] = True
    a = np.where(inner, ca, 0.0).astype(dt).ravel()
    b = np.where(inner, cb, 1.0).astype(dt).ravel()
    c = a.copy()
    d = du.astype(dt).ravel()
    dims = [nx, ny, nz]
    reference.strided_batch(a, b, c, d, dims, 0)
    reference.strided_batch(a, b, c, d, dims, 1)
    u_ref = u0.ravel().copy()
    reference.strided_batch(a, b, c, d, dims, 2, u=u_ref)
    tol = 1e-13 if dt == np.float64 else 2e-6
    assert normwise(u_oracle, u_ref) <= tol


@pytest.mark.parametrize("dims,sd", [([12, 7, 5], 0), ([6, 20, 5], 1), ([5, 6, 17], 2), ([40], 0)])
def test_adjoint_oracle_against_reference_transposed_solve(dims, sd, restatement, reference):
    """The adjoint oracle against a gradient built from the reference's own
    CPU solver: dbar solves T^T dbar = w, which is the tridiagonal system
    with sub-diagonal c one row up and super-diagonal a one row down; then
    abar_i = -dbar_i x_{i-1}, bbar_i = -dbar_i x_i, cbar_i = -dbar_i x_{i+1}."""
    a, b, c, d = make_system(dims, sd, np.float64, seed=sum(dims) + sd)
    w = np.random.default_rng(5).standard_normal(d.size)
    x = d.copy()
    reference.strided_batch(a, b, c, x, dims, sd)
    abar, bbar, cbar, dbar = restatement.adjoint(a, b, c, x, w, dims, sd)

    shape = tuple(reversed(dims))
    ax = len(dims) - 1 - sd
    first = [slice(None)] * len(dims)
    first[ax] = 0
    last = [slice(None)] * len(dims)
    last[ax] = -1
    A, C, X = (v.reshape(shape) for v in (a, c, x))
    at = np.roll(C, 1, axis=ax)
    at[tuple(first)] = 0.0
    ct = np.roll(A, -1, axis=ax)
    ct[tuple(last)] = 0.0
    dref = w.copy()
    reference.strided_batch(at.ravel().copy(), b, ct.ravel().copy(), dref, dims, sd)
    Dr = dref.reshape(shape)
    xm = np.roll(X, 1, axis=ax)
    xm[tuple(first)] = 0.0
    xp = np.roll(X, -1, axis=ax)
    xp[tuple(last)] = 0.0
    want = {"abar": (-Dr * xm).ravel(), "bbar": (-Dr * X).ravel(), "cbar": (-Dr * xp).ravel(),
            "dbar": dref}
    for name, got in (("abar", abar), ("bbar", bbar), ("cbar", cbar), ("dbar", dbar)):
        assert normwise(got, want[name]) <= 1e-13, name


if given is not None:
    @settings(max_examples=100, deadline=None, suppress_health_check=[HealthCheck.function_scoped_fixture])
    @given(n=hs.integers(1, 40), seed=hs.integers(0, 2 ** 31 - 1))
    def test_fuzz_restatement_against_dense_solve(n, seed, restatement):
        """One system against numpy's dense LU solve of the same matrix, a
        check independent of both Thomas implementations (a[0] and c[n-1]
        are outside the matrix and must not matter)."""
        rng = np.random.default_rng(seed)
        a = rng.uniform(-0.5, 0.5, n)
        c = rng.uniform(-0.5, 0.5, n)
        b = 1 + np.abs(a) + np.abs(c) + rng.uniform(0, 1, n)
        d = rng.standard_normal(n)
        a[0] = rng.uniform(-5, 5)
        c[-1] = rng.uniform(-5, 5)
        T = np.diag(b) + np.diag(a[1:], -1) + np.diag(c[:-1], 1)
        want = np.linalg.solve(T, d)
        got = d.copy()
        restatement.strided_batch(a, b, c, got, [n], 0)
        assert normwise(got, want) <= 1e-13
