"""Build libnnpe.so in-tree with nvcc for sm_100a (no JIT, no torch extension cache).

The kernels that restate the reference's float arithmetic (list, pair, bonded, integrator,
g(r)) are compiled with -fmad=false so that no multiply-add is contracted; the network kernels
use the default contraction.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "lib")
LIB = os.path.join(OUT, "libnnpe.so")
DRIVER = os.path.join(OUT, "nnpe_run")
CXX = os.environ.get("CXX", "g++")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off", "--expt-relaxed-constexpr",
          "-I" + os.path.join(HERE, "..", "include")]
EXACT = ["-fmad=false"]
UNITS = {
    "ctx.cu": EXACT,
    "rebuild.cu": EXACT,
    "forces.cu": EXACT,
    "force_step_noalloc.cu": EXACT,
    "integrate.cu": EXACT,
    "gr.cu": EXACT,
    "rmdf.cu": EXACT,
    "sqd.cu": EXACT,
    "serve.cu": [],
    "nnp.cu": [],
    "nnp_tc.cu": [],
}


def _compile(unit: str, flags, verbose: bool) -> str:
    src = os.path.join(CSRC, unit)
    obj = os.path.join(OUT, unit.replace(".cu", ".o"))
    cmd = [NVCC] + ARCH + COMMON + flags + ["-c", src, "-o", obj]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {unit}:\n{r.stderr}")
    if verbose:
        sys.stderr.write(r.stderr)
    return obj


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(OUT, exist_ok=True)
    srcs = [os.path.join(CSRC, u) for u in UNITS] + [os.path.join(CSRC, "internal.cuh"), os.path.join(CSRC, "nnp.cuh"), os.path.join(CSRC, "tc_util.cuh"),
                                                     os.path.join(HERE, "..", "include", "nnpe.h"), os.path.join(CSRC, "nnpe_run.cpp")]
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) > max(os.path.getmtime(s) for s in srcs):
        return LIB
    with ThreadPoolExecutor(max_workers=8) as ex:
        objs = list(ex.map(lambda kv: _compile(kv[0], kv[1], verbose), UNITS.items()))
    cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed:\n" + r.stderr)
    # the run-file driver: plain C++ host code over the C ABI, found next to the library at run time
    cmd = [CXX, "-std=c++17", "-O2", "-Wall", "-o", DRIVER, os.path.join(CSRC, "nnpe_run.cpp"), "-L" + OUT, "-lnnpe",
           "-Wl,-rpath,$ORIGIN"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nnpe_run failed to build:\n" + r.stderr)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force=True))
