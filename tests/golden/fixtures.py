"""Load the reference's known-answer fixtures (tests/golden/reference_fixtures.npz).

The committed file holds the golden solutions that the reference's own
generator (scalar/test/gen_testcases.py) produced, see make_golden.py. The
inputs are regenerated here: gen_testcases.py seeds numpy's legacy MT19937
stream with 1 (:2) and draws, per case and in order (:76-80),

    a = -1 + rand(shape) * 0.1,  b = 2 + rand(shape),
    c = -1 + rand(shape) * 0.1,  d = rand(shape),

then writes every value rounded to 15 decimals in Fortran order (:44-74),
which is x-fastest, the layout of the C API. The regenerated inputs are
checked against the SHA-256 stored with each case, so a drift in numpy's
stream or in the rounding would fail loudly instead of comparing against
the wrong problem.

Tolerances are the reference tests' (scalar/test/utils.hpp:14-17) with its
elementwise rule |exp - act| <= abs + rel * min(|exp|, |act|)
(scalar/test/catch_utils.hpp:62-80).
"""

import hashlib
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURES = os.path.join(HERE, "reference_fixtures.npz")

CASE_ORDER = [
    ("one_dim_small", [5], 0),
    ("one_dim_large", [200], 0),
    ("two_dim_small_solve0", [8, 8], 0),
    ("two_dim_small_solve1", [8, 8], 1),
    ("two_dim_large_solve0", [32, 32], 0),
    ("two_dim_large_solve1", [32, 32], 1),
    ("three_dim_large_solve0", [32, 32, 32], 0),
    ("three_dim_large_solve1", [32, 32, 32], 1),
    ("three_dim_large_solve2", [32, 32, 32], 2),
]
CASE_NAMES = [c[0] for c in CASE_ORDER]

ABS_TOL = {np.float64: 1e-11, np.float32: 1e-6}
REL_TOL = {np.float64: 1e-11, np.float32: 1e-5}

_inputs_cache = None


def _regenerate_all():
    global _inputs_cache
    if _inputs_cache is None:
        rs = np.random.RandomState(1)
        out = {}
        for name, shape, _ in CASE_ORDER:
            a = -1 + rs.rand(*shape) * 0.1
            b = 2 + rs.rand(*shape)
            c = -1 + rs.rand(*shape) * 0.1
            d = rs.rand(*shape)
            out[name] = [np.round(v, 15).flatten(order="F") for v in (a, b, c, d)]
        _inputs_cache = out
    return _inputs_cache


def load_case(name):
    """Return dict(dims, solvedim, a, b, c, d, u, u_float) for one fixture.

    a..d and u are float64 flat arrays in x-fastest order; u_float is the
    6-decimal solution of the 6-decimal-rounded inputs, as the reference's
    float tests use it.
    """
    z = np.load(FIXTURES)
    a, b, c, d = _regenerate_all()[name]
    h = hashlib.sha256()
    for arr in (a, b, c, d):
        h.update(np.ascontiguousarray(arr, dtype=np.float64).tobytes())
    want = str(z[f"{name}/inputs_sha256"])
    if h.hexdigest() != want:
        raise AssertionError(f"regenerated inputs of {name} do not match the fixture")
    return {
        "dims": [int(v) for v in z[f"{name}/dims"]],
        "solvedim": int(z[f"{name}/solvedim"]),
        "a": a, "b": b, "c": c, "d": d,
        "u": z[f"{name}/u"],
        "u_float": z[f"{name}/u_float_micro"] / 1e6,
    }


def allclose_ref(expected, actual, dtype):
    """The reference tests' elementwise check; returns (ok, worst index, diff)."""
    e = np.asarray(expected, dtype=np.float64)
    a = np.asarray(actual, dtype=np.float64)
    tol = ABS_TOL[dtype] + REL_TOL[dtype] * np.minimum(np.abs(e), np.abs(a))
    diff = np.abs(e - a)
    bad = diff > tol
    worst = int(np.argmax(diff - tol)) if diff.size else 0
    return (not bad.any()), worst, float(diff.max() if diff.size else 0.0)
