"""Build libstz_b200.so (CUDA kernels + C++ host + C ABI) for sm_100a, in-tree.

Usage: python sc25-stz2_b200/build.py [--force]

Objects go to sc25-stz2_b200/_build/, the library to sc25-stz2_b200/lib/.
Sources are recompiled only when they (or any header) change.
"""
from __future__ import annotations

import concurrent.futures as cf
import hashlib
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libstz_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-Wall", "-I", CSRC, "-I", os.path.join(ROOT, "include")]
# Every FP operation of the predictor/quantizer is explicit PTX; these flags
# make the remaining compiler-generated arithmetic follow the same rules.
CUDA_FLAGS = ARCH + ["-fmad=false", "-ftz=true", "-prec-div=true", "-prec-sqrt=true", "-Xptxas", "-v"]
SOURCES = ["levels.cu", "huffman.cu", "roi.cu", "api.cu", "server.cu", "noalloc.cu", "train.cu", "learned.cu", "host.cpp"]


def _digest() -> str:
    h = hashlib.sha256()
    for d in (CSRC, os.path.join(ROOT, "include", "stz")):
        for name in sorted(os.listdir(d)):
            with open(os.path.join(d, name), "rb") as f:
                h.update(name.encode() + f.read())
    h.update(" ".join(COMMON + CUDA_FLAGS).encode())
    return h.hexdigest()


def _compile(src: str) -> tuple[str, str]:
    obj = os.path.join(BUILD, os.path.splitext(src)[0] + ".o")
    cmd = [NVCC, "-c", os.path.join(CSRC, src), "-o", obj] + COMMON
    if src.endswith(".cu"):
        cmd += CUDA_FLAGS
    else:
        cmd += ["-x", "c++"] + ARCH
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stderr}")
    return obj, r.stderr


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    stamp = os.path.join(BUILD, "stamp")
    dig = _digest()
    if not force and os.path.exists(LIB) and os.path.exists(stamp) and open(stamp).read() == dig:
        return LIB
    with cf.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        results = list(ex.map(_compile, SOURCES))
    if verbose:
        for _, log in results:
            sys.stderr.write(log)
    objs = [o for o, _ in results]
    cmd = [NVCC, "-shared", "-o", LIB + ".tmp"] + ARCH + objs + ["-l:libzstd.so.1", "-lpthread"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stderr}")
    os.replace(LIB + ".tmp", LIB)
    with open(stamp, "w") as f:
        f.write(dig)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
