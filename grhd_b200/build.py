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
    hdrs = [os.path.join(INCLUDE, "grhd2_host.h"), os.path.join(INCLUDE, "grhd2_gpu.h"),
            os.path.join(CSRC, "gpu", "metric_eval.h")]
    if force or _newer(out, srcs + hdrs):
        _run([_cxx(), "-O2", "-std=c++17", "-fPIC", "-shared", "-Wall", "-I" + INCLUDE,
              "-I" + os.path.join(CSRC, "gpu"), "-o", out] + srcs, verbose)
    return out


def _precision_flags(src: str):
    """FP64 translation units keep every multiply and add separately rounded (the parity
    path follows the reference's operation order).  The *_fp32.cu units hold only the
    single-precision kernels of the mixed policy (reconstruction, Riemann, the cell update
    with its FP64 con2prim, the persistent step), whose bar is an L1 tolerance, not bitwise
    parity: they contract to FMA and use the approximate single-precision division and
    square root."""
    flags = ["--fmad=true", "-prec-div=false", "-prec-sqrt=false"] if "_fp32" in src else ["--fmad=false"]
    if os.path.basename(src).startswith("persistent_"):
        # the persistent kernel reads state that other blocks write during the launch:
        # plain loads bypass L1 (the primitives' loads use ld.global.cg explicitly)
        flags += ["-Xptxas", "-dlcm=cg"]
    return flags


def build_gpu(force=False, verbose=False) -> str:
    """Each .cu compiles to its own object in parallel, then one shared library links them.
    --fmad=false keeps every multiply and add separately rounded (the FP64 parity path
    must follow the reference's operation order)."""
    os.makedirs(LIB, exist_ok=True)
    obj_dir = os.path.join(HERE, "_build")
    os.makedirs(obj_dir, exist_ok=True)
    out = os.path.join(LIB, "libgrhd2gpu.so")
    srcs = _sources("gpu", (".cu",))
    headers = _sources("gpu", (".cuh", ".h")) + [os.path.join(INCLUDE, "grhd2_gpu.h")]
    if not srcs:
        raise RuntimeError("no CUDA sources under grhd_b200/csrc/gpu")
    common = [_nvcc()] + ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                                 "-I" + INCLUDE, "-I" + os.path.join(CSRC, "gpu"), "-ccbin", _cxx()]
    objs, jobs = [], []
    for s in srcs:
        o = os.path.join(obj_dir, os.path.splitext(os.path.basename(s))[0] + ".o")
        objs.append(o)
        if force or _newer(o, [s] + headers):
            jobs.append(common + _precision_flags(s) + ["-c", "-o", o, s])
    if jobs:
        from concurrent.futures import ThreadPoolExecutor
        with ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 4)) as ex:
            list(ex.map(lambda c: _run(c, verbose), jobs))
    if force or jobs or _newer(out, objs):
        _run([_nvcc()] + ARCH + ["-shared", "-ccbin", _cxx(), "-o", out] + objs, verbose)
    return out


def build_all(force=False, verbose=False):
    build_host(force, verbose)
    build_gpu(force, verbose)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv, verbose=True)
