"""Build libxkblas.so (sm_100a kernels + C++ host runtime) in-tree.

    python -m xkblas_b200.build [--force] [--jobs N]

Every CUDA source is compiled with
``nvcc -gencode arch=compute_100a,code=sm_100a -lineinfo -O3``; host C++ is
compiled by nvcc as well.  The CUDA runtime is linked statically and the
driver is reached through cudaGetDriverEntryPoint, so the library loads on a
machine without a GPU driver (entry points then report ENODEV).
Objects go to xkblas_b200/_build/, the library to xkblas_b200/libxkblas.so.
The Fortran-77 BLAS names (f77/xkblas_f77.cpp) are linked into a second
library, xkblas_b200/libxkblas_blas.so, on top of libxkblas.so: loading it
replaces the system BLAS level 3 for an unmodified application, so it is
kept out of libxkblas.so itself.
"""
import argparse
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libxkblas.so")
F77_SRC = os.path.join(HERE, "f77", "xkblas_f77.cpp")
F77_LIB = os.path.join(HERE, "libxkblas_blas.so")
CXX = os.environ.get("CXX", "g++")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-fvisibility=default",
          "-I" + os.path.join(ROOT, "include"), "-I" + CSRC]


def sources():
    out = []
    for f in sorted(os.listdir(CSRC)):
        if f.endswith(".cu") or f.endswith(".cpp"):
            out.append(os.path.join(CSRC, f))
    return out


def _deps_mtime(src):
    # headers in csrc/ and include/ count as dependencies of every source
    m = os.path.getmtime(src)
    for d in (CSRC, os.path.join(ROOT, "include")):
        for f in os.listdir(d):
            if f.endswith((".h", ".hpp", ".cuh")):
                m = max(m, os.path.getmtime(os.path.join(d, f)))
    return m


def _compile(src, force):
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    if not force and os.path.exists(obj) and os.path.getmtime(obj) >= _deps_mtime(src):
        return obj, None
    cmd = [NVCC] + ARCH + COMMON + ["-c", src, "-o", obj]
    if src.endswith(".cpp"):
        cmd = [NVCC, "-x", "cu"] + ARCH + COMMON + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        return obj, (" ".join(cmd) + "\n" + r.stdout + r.stderr)
    return obj, None


def build(force=False, jobs=None, verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    srcs = sources()
    jobs = jobs or min(len(srcs), os.cpu_count() or 4)
    with ThreadPoolExecutor(max_workers=jobs) as ex:
        results = list(ex.map(lambda s: _compile(s, force), srcs))
    errs = [e for _, e in results if e]
    if errs:
        raise RuntimeError("nvcc failed:\n" + "\n".join(errs))
    objs = [o for o, _ in results]
    if force or not os.path.exists(LIB) or any(
            os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", LIB] + objs + ["-ldl", "-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
        if verbose:
            print("linked", LIB)
    if force or not os.path.exists(F77_LIB) or max(
            os.path.getmtime(LIB), _deps_mtime(F77_SRC)) > os.path.getmtime(F77_LIB):
        cmd = [CXX, "-O2", "-std=c++17", "-fPIC", "-shared", "-I" + os.path.join(ROOT, "include"),
               F77_SRC, "-o", F77_LIB, "-L" + HERE, "-lxkblas", "-Wl,-rpath,$ORIGIN"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
        if verbose:
            print("linked", F77_LIB)
    return LIB


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=None)
    a = ap.parse_args(argv)
    print(build(force=a.force, jobs=a.jobs, verbose=True))


if __name__ == "__main__":
    sys.exit(main())
