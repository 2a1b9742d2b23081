"""Builds the sm_100a shared library lowmachfhd_b200/_fhd_b200.so in place
with nvcc (no JIT, no torch extension: the library exports a plain C ABI)."""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_fhd_b200.so")
SOURCES = ["fhd_solver.cu", "fhd_step.cu", "fhd_capi.cu", "fhd_noalloc.cu", "fhd_mass.cu", "fhd_server.cu",
           "fhd_sk.cu", "fhd_mass_f32.cu", "fhd_batch.cu"]
# translation units whose FP32 arithmetic may contract into FMA (tolerance-
# checked, no FP64 parity path inside)
FMA_SOURCES = {"fhd_mass_f32.cu"}
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    # FP64 parity with the CPU restatement: no contraction into FMA
    "--fmad=false",
    "-Xcompiler", "-fPIC", "-shared",
    "--expt-relaxed-constexpr",
]


def nvcc() -> str:
    for p in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if p and (os.path.sep not in p or os.path.exists(p)):
            return p
    return "nvcc"


def build(verbose: bool = False, extra: list[str] | None = None) -> str:
    srcs = [os.path.join(SRC, s) for s in SOURCES]
    newest = max(os.path.getmtime(p) for p in srcs + [os.path.join(SRC, h) for h in os.listdir(SRC)]
                 + [os.path.join(HERE, "..", "include", "fhd_b200.h")])
    if os.path.exists(OUT) and os.path.getmtime(OUT) >= newest and not extra:
        return OUT
    # one nvcc per translation unit, in parallel, then one link
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    cflags = [f for f in NVCC_FLAGS if f != "-shared"] + (extra or [])
    objs = [os.path.join(objdir, os.path.splitext(os.path.basename(p))[0] + ".o") for p in srcs]
    def flags_for(src):
        if os.path.basename(src) in FMA_SOURCES:
            return ["--fmad=true" if f == "--fmad=false" else f for f in cflags]
        return cflags
    cmds = [[nvcc()] + flags_for(src) + ["-c", src, "-o", obj] for src, obj in zip(srcs, objs)]
    if verbose:
        for c in cmds:
            print(" ".join(c), flush=True)
    with ThreadPoolExecutor(max_workers=min(len(cmds), os.cpu_count() or 1)) as ex:
        for r in list(ex.map(lambda c: subprocess.run(c), cmds)):
            if r.returncode:
                raise subprocess.CalledProcessError(r.returncode, r.args)
    link = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-Xcompiler", "-fPIC",
            "-o", OUT + ".tmp"] + objs + ["-lcufft", "-lcudart"]
    if verbose:
        print(" ".join(link), flush=True)
    subprocess.run(link, check=True)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    print(build(verbose=True, extra=sys.argv[1:] or None))
