"""Build libgft_b200.so in-tree with nvcc for sm_100a (B200).

The reference-arithmetic kernels are compiled with ``-fmad=false`` so that no
multiply-add is contracted (they reproduce the reference's FP64 operation
order); the throughput kernels use the default contraction.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libgft_b200.so")
HOST_RUN = os.path.join(HERE, "gft_run")  # GFTEvolver's main() over the C ABI (host/gft_run.cpp)

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
          "-I", os.path.join(ROOT, "include"), "--expt-relaxed-constexpr"]

# (source, extra flags)
SOURCES = [
    ("gft_ref_kernels.cu", ["-fmad=false"]),
    ("gft_fast_kernels.cu", []),
    ("gft_tiled_kernels.cu", []),
    ("gft_aux_kernels.cu", []),
    ("gft_static_observe.cu", []),
    ("gft_ensemble.cu", []),
    ("gft_slab_nccl.cu", []),
    ("gft_abi.cu", []),
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _deps_mtime() -> float:
    m = 0.0
    for d in (CSRC, os.path.join(ROOT, "include"), os.path.join(HERE, "host")):
        for f in os.listdir(d):
            m = max(m, os.path.getmtime(os.path.join(d, f)))
    return m


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> str:
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= _deps_mtime() and not ptxas_info:
        if not os.path.exists(HOST_RUN) or os.path.getmtime(HOST_RUN) < _deps_mtime():
            build_host()
        return LIB
    os.makedirs(BUILD, exist_ok=True)
    cc = nvcc()

    def compile_one(item):
        src, extra = item
        obj = os.path.join(BUILD, src.replace(".cu", ".o"))
        cmd = [cc, *ARCH, *COMMON, *extra, "-c", os.path.join(CSRC, src), "-o", obj]
        if ptxas_info:
            cmd.insert(1, "-Xptxas=-v")
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}")
        return obj, r.stdout

    with ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        results = list(ex.map(compile_one, SOURCES))
    if ptxas_info:
        for _, out in results:
            sys.stdout.write(out)
    objs = [o for o, _ in results]
    tmp = LIB + ".tmp"
    r = subprocess.run([cc, *ARCH, "-shared", "-o", tmp, *objs], stdout=subprocess.PIPE, stderr=subprocess.STDOUT,
                       text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc link failed:\n{r.stdout}")
    os.replace(tmp, LIB)
    build_host()
    return LIB


def build_host() -> str:
    """The gft_run program (g++, linked against the in-tree library with an $ORIGIN rpath)."""
    cxx = os.environ.get("CXX", "g++")
    cmd = [cxx, "-O2", "-std=c++17", "-pthread", "-I", os.path.join(ROOT, "include"),
           os.path.join(HERE, "host", "gft_run.cpp"), "-L", HERE, "-lgft_b200", "-Wl,-rpath,$ORIGIN", "-o", HOST_RUN]
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"host program build failed:\n{r.stdout}")
    return HOST_RUN


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv, ptxas_info="--ptxas" in sys.argv))
