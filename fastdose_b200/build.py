"""Builds libfd2.so (the CUDA kernels and the C ABI) in-tree for sm_100a.

    python -m fastdose_b200.build            # incremental
    python -m fastdose_b200.build --force    # rebuild everything
    python -m fastdose_b200.build --ptxas-v  # print register / shared-memory use

Objects go to fastdose_b200/_build/, the library to fastdose_b200/libfd2.so.
"""
import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libfd2.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
              "--expt-relaxed-constexpr", "-I", INCLUDE]


def _nvcc():
    return shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"


def _deps():
    return sorted(glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(INCLUDE, "*.h")))


# Translation units compiled with the reference's math flags: the cone-direction
# table must reproduce the reference's single-precision bits.
FAST_MATH_UNITS = {"cccs_dirs.cu"}


def _compile(src, force, ptxas_v):
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    newest = max([os.path.getmtime(src)] + [os.path.getmtime(d) for d in _deps()] + [os.path.getmtime(__file__)])
    if not force and os.path.exists(obj) and os.path.getmtime(obj) >= newest:
        return obj, ""
    cmd = [_nvcc(), "-c", src, "-o", obj] + ARCH + NVCC_FLAGS
    if os.path.basename(src) in FAST_MATH_UNITS:
        cmd += ["-use_fast_math"]
    if ptxas_v:
        cmd += ["-Xptxas", "-v"]
    p = subprocess.run(cmd, capture_output=True, text=True)
    if p.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{p.stdout}\n{p.stderr}")
    return obj, p.stderr


def build(force=False, ptxas_v=False, verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    with cf.ThreadPoolExecutor(max(1, min(8, os.cpu_count() or 1))) as ex:
        results = list(ex.map(lambda s: _compile(s, force, ptxas_v), srcs))
    objs = [r[0] for r in results]
    if verbose or ptxas_v:
        for s, (_, log) in zip(srcs, results):
            if log.strip():
                print(f"--- {os.path.basename(s)}\n{log}", file=sys.stderr)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        tmp = LIB + ".tmp"
        cmd = [_nvcc(), "-shared", "-o", tmp] + objs + ARCH + ["-lcudart"]
        p = subprocess.run(cmd, capture_output=True, text=True)
        if p.returncode != 0:
            raise RuntimeError(f"link failed:\n{p.stdout}\n{p.stderr}")
        os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--ptxas-v", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.ptxas_v, verbose=True))
