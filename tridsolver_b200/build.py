"""Build libtridsolver_b200.so in-tree (tridsolver_b200/lib/) with nvcc for sm_100a.

    python -m tridsolver_b200.build [--verbose-ptxas] [-j N]

Each .cu file under csrc/ is compiled to an object in parallel, then linked
into one shared library with the CUDA runtime linked statically, so the
library needs only the driver on the machine that loads it.
"""

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
OBJDIR = os.path.join(HERE, "_build")
LIBDIR = os.path.join(HERE, "lib")
LIBNAME = "libtridsolver_b200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O2",
    "--expt-relaxed-constexpr", "-I", INCLUDE, "-I", CSRC,
    "-ccbin", "g++",
]


def nvcc():
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(path):
        raise RuntimeError("nvcc not found")
    return path


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def headers():
    out = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    out += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h")]
    return out


def _compile(src, verbose_ptxas):
    obj = os.path.join(OBJDIR, os.path.basename(src)[:-3] + ".o")
    dep_mtime = max(os.path.getmtime(h) for h in headers() + [src, __file__])
    if os.path.exists(obj) and os.path.getmtime(obj) >= dep_mtime and not verbose_ptxas:
        return obj, ""
    cmd = [nvcc()] + NVCC_FLAGS + (["-Xptxas", "-v"] if verbose_ptxas else []) + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


def build(verbose_ptxas=False, jobs=None):
    """Compile every csrc/*.cu for sm_100a and link lib/libtridsolver_b200.so."""
    os.makedirs(OBJDIR, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    srcs = sources()
    jobs = jobs or min(len(srcs), os.cpu_count() or 4)
    with cf.ThreadPoolExecutor(jobs) as ex:
        results = list(ex.map(lambda s: _compile(s, verbose_ptxas), srcs))
    objs = [r[0] for r in results]
    lib = os.path.join(LIBDIR, LIBNAME)
    newest = max(os.path.getmtime(o) for o in objs)
    if not os.path.exists(lib) or os.path.getmtime(lib) < newest:
        cmd = [nvcc()] + ARCH + ["-shared", "-o", lib] + objs + ["-ccbin", "g++"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return lib, "".join(r[1] for r in results)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose-ptxas", action="store_true")
    ap.add_argument("-j", type=int, default=None)
    args = ap.parse_args(argv)
    lib, log = build(args.verbose_ptxas, args.j)
    if log:
        sys.stderr.write(log)
    print(lib)


if __name__ == "__main__":
    main()
