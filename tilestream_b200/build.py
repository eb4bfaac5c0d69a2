"""Builds libtilestream_b200.so in-tree for sm_100a (nvcc for the kernels, g++ for the host).

`build()` is incremental: a stamp holds the SHA-256 of every source, header and flag, and the
library is rebuilt only when that changes. The result is tilestream_b200/libtilestream_b200.so,
which the Python package loads with ctypes, and libtilestream_b200.a (the same objects) for
C++ programs that link the library statically; nothing is installed outside the repository.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import hashlib
import os
import shutil
import subprocess

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libtilestream_b200.so")
# The same objects as a static archive, for C++ programs that link the library into one
# executable with one CUDA runtime (the reference's test suites, tests/reference_suite).
ARCHIVE = os.path.join(PKG, "libtilestream_b200.a")

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# Calibration keeps IEEE binary32 semantics: no fast math, no FMA contraction, no FTZ.
NVCC_FLAGS = ARCH + ["-O3", "-std=c++17", "-lineinfo", "--fmad=false", "-ftz=false",
                     "-prec-div=true", "-prec-sqrt=true", "-Xcompiler", "-fPIC",
                     "-I" + INCLUDE, "-I" + CSRC]
CXX_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-Wall", "-Wextra", "-ffp-contract=off",
             "-I" + INCLUDE, "-I" + CSRC, "-I" + os.path.join(CUDA_HOME, "include")]
LINK_FLAGS = ["-shared", "-cudart", "static", "-Xlinker", "-Bsymbolic-functions",
              "-lz", "-lpthread", "-ldl", "-lrt"]


def sources():
    cu = sorted(glob.glob(os.path.join(CSRC, "kernels", "*.cu")))
    cpp = sorted(glob.glob(os.path.join(CSRC, "host", "*.cpp")))
    headers = sorted(glob.glob(os.path.join(CSRC, "**", "*.h"), recursive=True) +
                     glob.glob(os.path.join(CSRC, "**", "*.cuh"), recursive=True) +
                     glob.glob(os.path.join(INCLUDE, "**", "*.h"), recursive=True))
    return cu, cpp, headers


def fingerprint() -> str:
    cu, cpp, headers = sources()
    h = hashlib.sha256()
    for path in cu + cpp + headers:
        h.update(os.path.relpath(path, ROOT).encode())
        with open(path, "rb") as f:
            h.update(f.read())
    # Flags name absolute include paths; hash them relative to the repository root so that a
    # copy of the tree elsewhere (with its built library) is still up to date.
    h.update(" ".join(NVCC_FLAGS + CXX_FLAGS + LINK_FLAGS).replace(ROOT, "<root>").encode())
    return h.hexdigest()


def up_to_date() -> bool:
    stamp = os.path.join(BUILD, "stamp")
    if not os.path.exists(LIB) or not os.path.exists(ARCHIVE) or not os.path.exists(stamp):
        return False
    with open(stamp) as f:
        return f.read().strip() == fingerprint()


def _compile(src: str) -> str:
    obj = os.path.join(BUILD, os.path.relpath(src, CSRC).replace(os.sep, "_") + ".o")
    if src.endswith(".cu"):
        cmd = [NVCC] + NVCC_FLAGS + ["-c", src, "-o", obj]
    else:
        cmd = [os.environ.get("CXX", "g++")] + CXX_FLAGS + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return obj


def build(force: bool = False, verbose: bool = False) -> str:
    """Compiles and links the library when a source changed; returns its path."""
    if not force and up_to_date():
        return LIB
    if shutil.which(NVCC) is None and not os.path.exists(NVCC):
        raise RuntimeError(f"nvcc not found at {NVCC}")
    os.makedirs(BUILD, exist_ok=True)
    cu, cpp, _ = sources()
    with cf.ThreadPoolExecutor(max_workers=max(2, os.cpu_count() or 2)) as pool:
        objs = list(pool.map(_compile, cu + cpp))
    tmp = LIB + ".tmp"
    cmd = [NVCC] + ARCH + ["-o", tmp] + objs + LINK_FLAGS
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, LIB)
    if os.path.exists(ARCHIVE):
        os.remove(ARCHIVE)
    r = subprocess.run(["ar", "rcs", ARCHIVE] + objs, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"archive failed: {r.stdout}\n{r.stderr}")
    with open(os.path.join(BUILD, "stamp"), "w") as f:
        f.write(fingerprint())
    if verbose:
        print(f"built {LIB}")
    return LIB


if __name__ == "__main__":
    build(force=True, verbose=True)
