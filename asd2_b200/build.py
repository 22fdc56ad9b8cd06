"""Build recipe for the asd2g shared library (sm_100a only).

``python -m asd2_b200.build`` compiles every CUDA translation unit under
csrc/ with nvcc for sm_100a into asd2_b200/libasd2g.so (in-tree, so the built
library travels with the source tree).  The FP64 parity kernels are compiled
with -fmad=false: no multiply is fused into an add, which keeps their results
bit-identical to the reference's x86-64 build.  The FP32 level-set unit
(levelset32.cu, the mixed-precision path) is built with fused multiply-adds.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libasd2g.so")
DROPIN = os.path.join(HERE, "dropin")
DROPIN_LIB = os.path.join(HERE, "libasd2_dropin.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# translation unit -> extra flags
UNITS = {
    "bc.cu": ["-fmad=false"],
    "levelset.cu": ["-fmad=false"],
    "momentum.cu": ["-fmad=false"],
    "axisym.cu": ["-fmad=false"],
    "pressure.cu": ["-fmad=false"],
    "api.cu": [],
    "pcg_static.cu": ["-fmad=false"],
    "pcg_cluster.cu": ["-fmad=false"],
    "pcg_persist.cu": ["-fmad=false"],
    "mg.cu": [],
    "mg_persist.cu": [],
    "levelset32.cu": [],
    "weno32.cu": [],
    "reinit32.cu": [],
    "batch.cu": [],
    "unet.cu": [],
    "unet_net.cu": [],
}


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def _stale(out: str, deps: list) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def gxx() -> str:
    for cand in (os.environ.get("ASD2_CXX"), "/usr/bin/g++", "g++"):
        if cand and (not os.path.isabs(cand) or os.path.exists(cand)):
            return cand
    return "g++"


def build_dropin(verbose: bool = False) -> str:
    """The C++ classes with the reference's interfaces, linked against libasd2g.so."""
    srcs = sorted(os.path.join(DROPIN, f) for f in os.listdir(DROPIN) if f.endswith(".cpp"))
    hdrs = [os.path.join(DROPIN, f) for f in os.listdir(DROPIN) if f.endswith(".h")]
    hdrs.append(os.path.join(ROOT, "include", "asd2g.h"))
    if not _stale(DROPIN_LIB, srcs + hdrs + [LIB, __file__]):
        return DROPIN_LIB
    cmd = [gxx(), "-std=c++17", "-O2", "-fPIC", "-shared", "-Wall", "-Wno-unused-function",
           "-I", os.path.join(ROOT, "include"), "-I", DROPIN, *srcs, "-o", DROPIN_LIB,
           "-L", HERE, "-lasd2g", "-Wl,-rpath,$ORIGIN"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return DROPIN_LIB


def build(verbose: bool = False, ptxas_v: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers.append(os.path.join(ROOT, "include", "asd2g.h"))
    objs, cmds = [], []
    for unit, extra in UNITS.items():
        src = os.path.join(CSRC, unit)
        obj = os.path.join(BUILD, unit.replace(".cu", ".o"))
        objs.append(obj)
        if not _stale(obj, [src, __file__] + headers):
            continue
        cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-rdc=false",
               "-I", os.path.join(ROOT, "include"), "-I", CSRC, *extra, "-c", src, "-o", obj]
        if ptxas_v:
            cmd.insert(1, "-Xptxas=-v")
        cmds.append(cmd)
    # the translation units are independent: compile them concurrently
    jobs = max(1, min(len(cmds), os.cpu_count() or 1))

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    if cmds:
        with ThreadPoolExecutor(jobs) as ex:
            list(ex.map(run, cmds))
    if _stale(LIB, objs):
        cmd = [nvcc(), *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    build_dropin(verbose)
    return LIB


if __name__ == "__main__":
    build(verbose=True, ptxas_v="-v" in sys.argv)
