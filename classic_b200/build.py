"""In-tree build of the CUDA library (sm_100a) and of the CPU oracle.

``build_library()`` compiles classic_b200/csrc/claw_b200.cu with nvcc into
classic_b200/libclawb200.so.  The FP64 path is built with --fmad=false so
each multiply and add rounds separately, in the reference's operation order.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libclawb200.so")
ARCH = "-gencode=arch=compute_100a,code=sm_100a"


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC)
                  if f.endswith((".cu", ".cuh")))


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    hdr = os.path.join(os.path.dirname(HERE), "include", "claw_b200.h")
    return all(os.path.getmtime(s) <= t for s in sources() + [hdr])


# Translation units and their arithmetic flags: the reference-order FP64 path
# rounds every multiply and add separately; the characteristic-variable path
# (fast2d.cu) contracts to fused multiply-adds.
UNITS = [("claw_b200.cu", "--fmad=false"), ("noalloc.cu", "--fmad=false"),
         ("fast2d.cu", "--fmad=true"), ("claw3d.cu", "--fmad=false"),
         ("batch2d.cu", "--fmad=false"), ("nn.cu", "--fmad=true"),
         ("fast3d.cu", "--fmad=true"), ("split2d.cu", "--fmad=false"),
         ("split2d_fast.cu", "--fmad=true"), ("probe.cu", "--fmad=true"),
         ("fma2d.cu", "--fmad=true"), ("batch2d_fast.cu", "--fmad=true"),
         ("fast2d_minmod.cu", "--fmad=true"), ("fast2d_superbee.cu", "--fmad=true"),
         ("fast2d_vanleer.cu", "--fmad=true"), ("fast2d_pairs_minmod.cu", "--fmad=true"),
         ("fast2d_pairs_superbee.cu", "--fmad=true"), ("fast2d_pairs_vanleer.cu", "--fmad=true"),
         ("fast2d_pairs_mc.cu", "--fmad=true"), ("split2d_char.cu", "--fmad=true")]


def build_library(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return LIB
    obj_dir = os.path.join(HERE, "_build")
    os.makedirs(obj_dir, exist_ok=True)
    objs, procs = [], []
    for src, fmad in UNITS:  # the units compile in parallel
        obj = os.path.join(obj_dir, src.replace(".cu", ".o"))
        cmd = [_nvcc(), ARCH, "-O3", "-lineinfo", fmad, "-std=c++17", "-Xcompiler", "-fPIC",
               "-c", "-o", obj, os.path.join(CSRC, src)]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
            print(" ".join(cmd), file=sys.stderr)
        procs.append((cmd, subprocess.Popen(cmd)))
        objs.append(obj)
    for cmd, p in procs:
        if p.wait() != 0:
            raise subprocess.CalledProcessError(p.returncode, cmd)
    subprocess.run([_nvcc(), ARCH, "-shared", "-o", LIB] + objs, check=True)
    return LIB


def build_oracle():
    root = os.path.dirname(HERE)
    subprocess.run(["make", "-s", "-C", os.path.join(root, "oracle")], check=True)


if __name__ == "__main__":
    build_library(force="--force" in sys.argv, verbose="-v" in sys.argv)
    build_oracle()
