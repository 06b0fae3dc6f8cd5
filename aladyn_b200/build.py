"""Build the in-tree device library ``aladyn_b200/libaladyn_gpu.so``.

Every translation unit is compiled by nvcc for sm_100a only.  The FP64 form
and the host bookkeeping are compiled with ``-fmad=false`` so that no
multiply-add is contracted (the reference's arithmetic order is kept bit for
bit); the FP32 split form is compiled with contraction on.

Usage: ``python -m aladyn_b200.build [--force] [--verbose]``
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libaladyn_gpu.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
          "-I", INCLUDE, "-ccbin", "g++"]

# (source, extra flags)
UNITS = [
    ("agpu_fp64.cu", ["-fmad=false"]),
    ("agpu_util.cu", ["-fmad=false"]),
    ("agpu_api.cu", ["-fmad=false"]),
    ("agpu_fp32.cu", ["-fmad=true"]),
    ("agpu_tile64.cu", ["-fmad=false"]),
    ("agpu_tile32.cu", ["-fmad=true"]),
    ("agpu_tile32c.cu", ["-fmad=true"]),
    ("agpu_bin.cu", ["-fmad=false"]),
    ("agpu_noalloc.cu", ["-fmad=false"]),
    ("agpu_envar.cu", ["-fmad=false"]),
    ("agpu_env.cu", ["-fmad=false"]),
    ("agpu_beam.cu", ["-fmad=false"]),
    ("agpu_ionz.cpp", []),
    ("agpu_batch.cpp", ["-Xcompiler", "-pthread"]),
]
HEADERS = ["agpu_common.cuh", "agpu_kernels.h", "agpu_util.h", "agpu_yee.cuh", "agpu_ionz.h", "agpu_bin.cuh",
           "agpu_tile.h", "agpu_select.cuh", "agpu_beam.h", "agpu_multi.h", "agpu_yee_fused.cuh", "agpu_env.h",
           "agpu_fp64_dep.cuh"]


def _mtime(p: str) -> float:
    return os.path.getmtime(p) if os.path.exists(p) else 0.0


def build(force: bool = False, verbose: bool = False, ptxas_verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    hdr_time = max([_mtime(os.path.join(CSRC, h)) for h in HEADERS] +
                   [_mtime(os.path.join(INCLUDE, "aladyn_gpu.h"))])
    objs = []
    rebuilt = False
    for src, extra in UNITS:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src + ".o")
        objs.append(o)
        if force or _mtime(o) < max(_mtime(s), hdr_time, _mtime(__file__)):
            cmd = [NVCC, *ARCH, *COMMON, *extra, "-c", s, "-o", o]
            if ptxas_verbose and src.endswith(".cu"):
                cmd.insert(1, "-Xptxas=-v")
            if src.endswith(".cpp"):
                cmd[cmd.index("-c"):cmd.index("-c")] = ["-x", "c++"]
            if verbose:
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)
            rebuilt = True
    if rebuilt or force or not os.path.exists(LIB):
        cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart", "-lcufft", "-Xcompiler", "-pthread",
               "-Xlinker", "-rpath=/usr/local/cuda/lib64"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return LIB


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas", action="store_true", help="print ptxas register/spill usage")
    a = ap.parse_args(argv)
    print(build(a.force, a.verbose, a.ptxas))


if __name__ == "__main__":
    sys.exit(main())
