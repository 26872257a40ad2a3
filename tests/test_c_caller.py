"""A C caller compiled against include/xkblas.h with the system C compiler
and linked with libxkblas.so (tests/c/caller.c): the drop-in boundary as a
C program sees it -- header helpers, -i argument codes, ENODEV without a
GPU (CPU test) and a correct product with one (GPU test)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "xkblas_b200")


def _build(tmp_path):
    cc = shutil.which("cc") or shutil.which("gcc")
    if not cc:
        pytest.skip("no C compiler")
    exe = str(tmp_path / "caller")
    r = subprocess.run([cc, "-std=c99", "-O1", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                        os.path.join(ROOT, "tests", "c", "caller.c"), "-o", exe,
                        "-L" + LIBDIR, "-lxkblas", "-Wl,-rpath," + LIBDIR, "-lm"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except ImportError:
        return False


def test_c_caller_without_gpu(tmp_path):
    if _has_gpu():
        pytest.skip("a GPU is present (the GPU variant covers it)")
    exe = _build(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "caller ok" in r.stdout


@pytest.mark.gpu
def test_c_caller_on_gpu(tmp_path):
    exe = _build(tmp_path)
    r = subprocess.run([exe, "gpu"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "caller ok" in r.stdout


def test_header_compiles_as_cxx(tmp_path):
    """The same header from C++ (std::complex scalars)."""
    cxx = shutil.which("c++") or shutil.which("g++")
    if not cxx:
        pytest.skip("no C++ compiler")
    src = tmp_path / "h.cpp"
    src.write_text('#include "xkblas.h"\n#include "xkb_cuda.h"\n'
                   'int f() { return xkblas_blas2cblas_fill("U") + xkblas_blas2cblas_diag("n"); }\n')
    r = subprocess.run([cxx, "-std=c++17", "-Wall", "-Werror", "-fsyntax-only",
                        "-I", os.path.join(ROOT, "include"), str(src)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
