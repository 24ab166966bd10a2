"""Build recipe for libbldm.so (sm_100a) — compiles bnmf-algs_b200/csrc/*.cu in-tree.

Usage: python bnmf-algs_b200/build.py [--force] [--verbose-ptxas]
"""

import argparse
import concurrent.futures
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libbldm.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
if not os.path.exists(NVCC):
    NVCC = shutil.which("nvcc") or NVCC
HOST_CXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-ccbin", HOST_CXX,
         "--expt-relaxed-constexpr", "-I", os.path.join(HERE, "..", "include")]


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC)
                  if f.endswith(".cu") or f.endswith(".cpp"))


def headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hs.append(os.path.join(HERE, "..", "include", "bldm.h"))
    return hs


def _newest(paths):
    return max(os.path.getmtime(p) for p in paths)


def _compile(src, verbose_ptxas):
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    cmd = [NVCC] + ARCH + FLAGS + ["-c", src, "-o", obj]
    if verbose_ptxas:
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


def build(force=False, verbose_ptxas=False, jobs=None):
    """Compile every .cu into libbldm.so; returns the library path."""
    os.makedirs(BUILD, exist_ok=True)
    srcs = sources()
    if (not force and os.path.exists(LIB)
            and os.path.getmtime(LIB) >= _newest(srcs + headers() + [__file__])):
        return LIB
    jobs = jobs or min(len(srcs), os.cpu_count() or 4)
    logs = []
    with concurrent.futures.ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = []
        for obj, log in ex.map(lambda s: _compile(s, verbose_ptxas), srcs):
            objs.append(obj)
            logs.append(log)
    cmd = [NVCC] + ARCH + ["-shared", "-ccbin", HOST_CXX, "-o", LIB] + objs + ["-lcudart"]
    subprocess.run(cmd, check=True)
    if verbose_ptxas:
        sys.stderr.write("".join(logs))
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose-ptxas", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose_ptxas=a.verbose_ptxas))
