"""In-tree build of the package's native libraries.

* ``lib/libgrhd2host.so``  host-side problem setup (g++, C++17)
* ``lib/libgrhd2gpu.so``   the CUDA C-ABI: sm_100a kernels (nvcc -gencode
  arch=compute_100a,code=sm_100a), FP64 parity kernels built without FMA contraction

Run ``python -m grhd_b200.build`` (or ``__graft_entry__.build()``).  nvcc cross-compiles
for sm_100a without a GPU.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "lib")
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _cxx() -> str:
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"


def _nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else (shutil.which("nvcc") or "nvcc")


def _newer(out: str, srcs) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(s) > t for s in srcs)


def _sources(sub: str, exts):
    out = []
    for dp, _, fs in os.walk(os.path.join(CSRC, sub)):
        out += [os.path.join(dp, f) for f in fs if f.endswith(exts)]
    return sorted(out)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build_host(force=False, verbose=False) -> str:
    os.makedirs(LIB, exist_ok=True)
    out = os.path.join(LIB, "libgrhd2host.so")
    srcs = _sources("host", (".cpp",))
    hdrs = [os.path.join(INCLUDE, "grhd2_host.h"), os.path.join(INCLUDE, "grhd2_gpu.h")]
    if force or _newer(out, srcs + hdrs):
        _run([_cxx(), "-O2", "-std=c++17", "-fPIC", "-shared", "-Wall", "-I" + INCLUDE,
              "-o", out] + srcs, verbose)
    return out


def build_gpu(force=False, verbose=False) -> str:
    os.makedirs(LIB, exist_ok=True)
    out = os.path.join(LIB, "libgrhd2gpu.so")
    srcs = _sources("gpu", (".cu",))
    deps = srcs + _sources("gpu", (".cuh", ".h")) + [os.path.join(INCLUDE, "grhd2_gpu.h")]
    if not srcs:
        raise RuntimeError("no CUDA sources under grhd_b200/csrc/gpu")
    if force or _newer(out, deps):
        cmd = [_nvcc()] + ARCH + [
            "-O3", "-lineinfo", "-std=c++17", "--fmad=false", "-Xcompiler", "-fPIC",
            "-shared", "-I" + INCLUDE, "-I" + os.path.join(CSRC, "gpu"),
            "-ccbin", _cxx(), "-o", out] + srcs
        _run(cmd, verbose)
    return out


def build_all(force=False, verbose=False):
    build_host(force, verbose)
    build_gpu(force, verbose)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv, verbose=True)
