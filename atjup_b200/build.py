"""Build the in-tree CUDA library atjup_b200/libatjup_gpu.so for sm_100a (B200).

    python -m atjup_b200.build

nvcc cross-compiles without a GPU. The library is the product: every CUDA kernel and the C ABI
declared in include/atjup_gpu.h. It is built in-tree so it travels with the repository.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "libatjup_gpu.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3", "--expt-relaxed-constexpr",
         "-I", str(ROOT / "include")]


# The microphysics decide branches on exact cancellations (a rain flux that evaporates completely
# is 0, not +-1 ulp; a saturation test sits on its threshold): these files keep the reference's
# rounding by being compiled without FMA contraction, as the reference is. So does the projection
# around the obstacle, whose SOR stopping test decides the sweep count on the last bits of phi, and
# the filters and the column balance, which then equal the reference's to the bit.
PER_FILE = {"satadj.cu": ["-fmad=false"], "micro.cu": ["-fmad=false"], "mca.cu": ["-fmad=false"],
            "cone.cu": ["-fmad=false"], "filters.cu": ["-fmad=false"]}


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(CSRC.glob("*.cu"))


def build(force: bool = False, verbose: bool = False, extra=()) -> Path:
    srcs = sources()
    deps = srcs + sorted(CSRC.glob("*.cuh")) + [ROOT / "include" / "atjup_gpu.h"]
    if LIB.exists() and not force and all(LIB.stat().st_mtime >= p.stat().st_mtime for p in deps):
        return LIB
    objdir = PKG / "_build"
    objdir.mkdir(exist_ok=True)
    objs = []
    procs = []
    for s in srcs:
        o = objdir / (s.stem + ".o")
        cmd = [nvcc(), *ARCH, *FLAGS, *PER_FILE.get(s.name, []), *extra, "-c", str(s), "-o", str(o)]
        if verbose:
            print(" ".join(cmd))
        procs.append((subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT), s))
        objs.append(o)
    failed = []
    for p, s in procs:
        out = p.communicate()[0].decode()
        if verbose and out:
            print(out)
        if p.returncode != 0:
            failed.append((s, out))
    if failed:
        raise RuntimeError("nvcc failed:\n" + "\n".join(f"{s}:\n{o}" for s, o in failed))
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc(), *ARCH, "-shared", "-o", str(tmp), *map(str, objs)]
    subprocess.run(cmd, check=True, capture_output=not verbose)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=["-Xptxas", "-v"] if "--ptxas" in sys.argv else ())
    print(LIB)
