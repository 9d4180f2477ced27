"""Generate tests/golden/reference_fixtures.npz from the reference's own
fixture generator, scalar/test/gen_testcases.py (seed pinned at :2).

Run here, where the reference tree exists (it does not exist where the GPU
tests run, which is why its output is committed):

    python tests/golden/make_golden.py /path/to/reference

The generator draws a, b, c, d with numpy's legacy MT19937 stream
(gen_testcases.py:76-80), solves every system with scipy's spsolve
(:33-40) and writes text files (:44-74) that the reference's C++ tests read
(scalar/test/utils.hpp:207-247). This script runs the generator's own
gen_testcase() for every case up to three dimensions, in the order of its
main() (:95-104) so the random stream is the same, lets it write its text
files into a temporary directory, and parses them back exactly as the C++
loader does. The four-dimensional cases (:105-108) are skipped: the
reference library is built with MAXDIM=3 and its 4-D tests are compiled
out (scalar/test/test_cuda.cu:176), and they come after every case kept
here, so skipping them does not shift the random stream.

Stored per case: dims, solvedim, the double solution row `u` (15 decimals),
the float solution row (6 decimals) as integer micro-units (exact), and a
SHA-256 of the inputs as written. The inputs themselves are regenerated at
test time by tests/golden/fixtures.py and checked against that hash.
"""

import contextlib
import hashlib
import io
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

# (file name, shape, solvedim) in the order of gen_testcases.py main()
CASES = [
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


def parse_case_file(path):
    """Read a fixture text file the way scalar/test/utils.hpp:207-247 does."""
    with open(path) as f:
        lines = f.read().split("\n")
    ndim, solvedim = (int(v) for v in lines[0].split())
    dims = [int(v) for v in lines[1].split()]
    rows = [np.array([float(v) for v in line.split()], dtype=np.float64)
            for line in lines[2:8]]
    assert len(dims) == ndim
    n = int(np.prod(dims))
    assert all(r.size == n for r in rows)
    a, b, c, d, u, u_float = rows
    return dims, solvedim, a, b, c, d, u, u_float


def inputs_digest(a, b, c, d):
    h = hashlib.sha256()
    for arr in (a, b, c, d):
        h.update(np.ascontiguousarray(arr, dtype=np.float64).tobytes())
    return h.hexdigest()


def main(ref_root):
    """ref_root: the reference checkout whose scalar/test/gen_testcases.py
    generates the fixtures."""
    test_dir = os.path.join(ref_root, "scalar", "test")
    sys.path.insert(0, test_dir)
    import gen_testcases as gen  # noqa: E402  (its import seeds the stream)

    out = {}
    with tempfile.TemporaryDirectory() as tmp:
        cwd = os.getcwd()
        os.chdir(tmp)
        try:
            with contextlib.redirect_stdout(io.StringIO()):
                for name, shape, solvedim in CASES:
                    gen.gen_testcase(name, shape, solvedim)
            for name, shape, solvedim in CASES:
                dims, sd, a, b, c, d, u, u_float = parse_case_file(name)
                assert dims == shape and sd == solvedim
                micro = np.rint(u_float * 1e6).astype(np.int64)
                assert np.array_equal(micro / 1e6, u_float)
                out[f"{name}/dims"] = np.array(dims, dtype=np.int64)
                out[f"{name}/solvedim"] = np.array(solvedim, dtype=np.int64)
                out[f"{name}/u"] = u
                out[f"{name}/u_float_micro"] = micro
                out[f"{name}/inputs_sha256"] = np.array(inputs_digest(a, b, c, d))
        finally:
            os.chdir(cwd)
    path = os.path.join(HERE, "reference_fixtures.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")

    # the test-time regeneration must reproduce the inputs bit for bit
    sys.path.insert(0, HERE)
    from fixtures import load_case  # noqa: E402
    for name, _, _ in CASES:
        load_case(name)
    print("regenerated inputs match the written fixtures")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py /path/to/reference")
    main(sys.argv[1])
