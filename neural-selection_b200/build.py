"""Build recipe for the B200 library: nvcc, sm_100a only.

Produces neural-selection_b200/libns_b200.so in-tree (git-ignored; it travels
with the source tree to the GPU host). Flags: --fmad=false keeps every binary32
multiply and add separately rounded, as the reference arithmetic requires;
divisions and square roots stay IEEE (no fast-math); the host side is compiled
with -ffp-contract=off for the same reason.
"""
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
INCLUDE = PKG.parent / "include"
LIB = PKG / "libns_b200.so"
SOURCES = sorted(CSRC.glob("*.cu"))
HEADERS = sorted(list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h")))
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc():
    exe = os.environ.get("NVCC") or shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(exe).exists() and not shutil.which(exe):
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libns_b200.so")
    return exe


def flags(extra=()):
    return ["-O3", "-std=c++17", "--fmad=false", "-lineinfo", *ARCH, "-Xcompiler", "-fPIC,-ffp-contract=off",
            "-I", str(CSRC), "-I", str(INCLUDE), *extra]


def build(force=False, verbose=False, ptxas_info=False):
    newest = max(p.stat().st_mtime for p in SOURCES + HEADERS)
    if LIB.exists() and not force and LIB.stat().st_mtime >= newest:
        return LIB
    objs = []
    build_dir = PKG / "_build"
    build_dir.mkdir(exist_ok=True)
    for src in SOURCES:
        obj = build_dir / (src.stem + ".o")
        cmd = [nvcc(), *flags(["-Xptxas", "-v"] if ptxas_info else []), "-c", str(src), "-o", str(obj)]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src.name}:\n{res.stderr}")
        if verbose or ptxas_info:
            sys.stderr.write(res.stderr)
        objs.append(str(obj))
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc(), *ARCH, "-shared", *objs, "-o", str(tmp)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"link failed:\n{res.stderr}")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True, ptxas_info="--ptxas" in sys.argv))
