"""GPU: the reference's own callers, unmodified, linked against this library.

oracle/Makefile compiles, from the reference's sources where they lie, with
this repository's include/ searched first and libtridsolver_b200.so linked
in place of the reference's libtridcuda:

* scalar/test/test_cuda.cu with catch_main.cpp: the reference's Catch2 GPU
  tests (x, y, z solves of its known-answer fixtures, plain and padded, FP32
  and FP64, at its own tolerances). They read ./files/<case>; the fixture
  files are written here, in the generator's text format
  (scalar/test/gen_testcases.py:44-74), from the committed golden data
  (tests/golden/), which reproduces the generator's files value for value;
* apps/adi/src/adi_cuda.cu with preproc.cu: the ADI heat application (its
  preprocessing kernel, then x and y tridDmtsvStridedBatch and a z
  tridDmtsvStridedBatchInc per iteration). Its printed sum of u must match
  the same application's CPU build (apps/adi/src/adi_cpu.cpp) linked to the
  reference's own CPU solver.
"""

import os
import re
import subprocess

import numpy as np
import pytest

from fixtures import CASE_NAMES, load_case

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CALLERS = os.path.join(ROOT, "oracle", "_ref", "callers")


def _binary(name):
    path = os.path.join(CALLERS, name)
    if not os.path.exists(path):
        pytest.skip(f"{path} not built (make -C oracle where the reference tree exists)")
    return path


def _fmt(values, decimals):
    return " ".join(str(round(float(v), decimals)) for v in values)


def write_fixture_files(directory):
    """files/<case> for every golden case, as gen_testcases.py writes them."""
    files = os.path.join(directory, "files")
    os.makedirs(files, exist_ok=True)
    for name in CASE_NAMES:
        case = load_case(name)
        with open(os.path.join(files, name), "w") as f:
            f.write(f"{len(case['dims'])} {case['solvedim']}\n")
            f.write(" ".join(str(v) for v in case["dims"]) + "\n")
            for key in "abcd":
                f.write(_fmt(case[key], 15) + "\n")
            f.write(_fmt(case["u"], 15) + "\n")
            f.write(_fmt(case["u_float"], 6) + "\n")


def test_reference_catch2_gpu_tests_pass(tmp_path):
    exe = _binary("cuda_tests")
    write_fixture_files(str(tmp_path))
    r = subprocess.run([exe], cwd=str(tmp_path), capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-4000:] + r.stderr[-2000:]
    assert "All tests passed" in r.stdout, r.stdout[-2000:]


def _adi_sum(cmd, env=None):
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-2000:]
    m = re.search(r"end h_u sum = (\S+)", r.stdout)
    assert m, r.stdout[-2000:]
    return float(m.group(1))


@pytest.mark.parametrize("n,iters", [(64, 10), (128, 20), (256, 10)])
def test_reference_adi_application_matches_its_cpu_build(n, iters):
    gpu = _binary("adi_cuda")
    cpu = _binary("adi_cpu")
    args = ["-nx", str(n), "-ny", str(n), "-nz", str(n), "-iter", str(iters), "-prof", "0"]
    env = dict(os.environ, OMP_NUM_THREADS=str(len(os.sched_getaffinity(0))))
    s_gpu = _adi_sum([gpu] + args)
    s_cpu = _adi_sum([cpu] + args, env)
    # the applications print the sum with %lg (6 significant digits)
    assert np.isfinite(s_gpu) and s_gpu != 0.0
    assert abs(s_gpu - s_cpu) <= 1e-5 * abs(s_cpu), (s_gpu, s_cpu)
