"""ORACLE — test infrastructure only. Build recipe for the checker.

Outputs (all git-ignored):
  oracle/_build/libns_oracle.so       C restatement, exp/log correctly rounded
  oracle/_build/libns_oracle_libm.so  C restatement, glibc expf/logf
  oracle/_build/exhaustive_math       exhaustive exp/log agreement checker
  oracle/_ref/libns_ref.so            the reference host executor
                                      (gym_adapter/native.cpp), built from the
                                      reference sources in place
  oracle/_ref/libns_ref_cr.so         same sources, exp/log correctly rounded
  oracle/_ref/libns_ref_gpu.so        the reference CUDA batch
                                      (gym_adapter/gpu.cu) for sm_100a with the
                                      reference's flags (gym_adapter/gpu.py:19)
  oracle/_ref/libns_ref_world.so      the reference world simulator's neural
                                      kernels (src/main.cu) with its own flags
  oracle/_ref/libns_ref_world_cr.so   the same kernels with IEEE arithmetic and
                                      correctly rounded exp/log
The _ref targets need the reference tree (REFERENCE_ROOT, default: a directory
named "reference" beside this repository) and are skipped when it is absent; prebuilt files are used as
they are.
"""
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
REPO = HERE.parent
BUILD = HERE / "_build"
REF_OUT = HERE / "_ref"
CSRC = REPO / "neural-selection_b200" / "csrc"
REFERENCE = Path(os.environ.get("REFERENCE_ROOT", REPO.parent / "reference"))

CFLAGS = ["-O2", "-fPIC", "-ffp-contract=off", "-fno-fast-math"]


def _run(cmd):
    subprocess.run([str(c) for c in cmd], check=True)


def _stale(target, sources):
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(s).stat().st_mtime > t for s in sources)


def build_oracle(verbose=False):
    BUILD.mkdir(exist_ok=True)
    cr_obj = BUILD / "or_crmath.o"
    if _stale(cr_obj, [HERE / "or_crmath.c"]):
        _run(["gcc", *CFLAGS, "-c", HERE / "or_crmath.c", "-o", cr_obj])
    srcs = [HERE / "ns_oracle.c", HERE / "or_episode.c", HERE / "ns_oracle.h", cr_obj]
    for name, extra in (("libns_oracle.so", []), ("libns_oracle_libm.so", ["-DOR_LIBM"])):
        out = BUILD / name
        if _stale(out, srcs):
            _run(["gcc", *CFLAGS, *extra, "-shared", HERE / "ns_oracle.c", HERE / "or_episode.c", cr_obj,
                  "-o", out, "-lquadmath", "-lm"])
    ex = BUILD / "exhaustive_math"
    if _stale(ex, [HERE / "exhaustive_math.cpp", cr_obj, CSRC / "ns_crmath.h"]):
        _run(["g++", "-O2", "-std=c++17", "-mfma", "-ffp-contract=off", "-I", CSRC,
              HERE / "exhaustive_math.cpp", cr_obj, "-lquadmath", "-lpthread", "-o", ex])
    return BUILD


def build_ref(verbose=False, gpu=True):
    """Compile the reference's own sources (never copied) into oracle/_ref."""
    native = REFERENCE / "gym_adapter" / "native.cpp"
    if not native.exists():
        return None
    REF_OUT.mkdir(exist_ok=True)
    build_oracle()
    inc = ["-I", REFERENCE / "src", "-I", REFERENCE / "gym_adapter"]
    deps = [native, REFERENCE / "gym_adapter" / "core.cuh", REFERENCE / "src" / "physiology.cuh",
            HERE / "ref_harness.cpp", HERE / "ref_cr_shim.h"]
    # Same flags as the reference's own build (gym_adapter/adapter.py:22).
    base = ["g++", "-O3", "-std=c++17", "-shared", "-fPIC", "-Wno-macro-redefined", *inc]
    out = REF_OUT / "libns_ref.so"
    if _stale(out, deps):
        _run([c for c in base if c != "-Wno-macro-redefined"] + [HERE / "ref_harness.cpp", "-o", out])
    out = REF_OUT / "libns_ref_cr.so"
    if _stale(out, deps):
        _run([c for c in base if c != "-Wno-macro-redefined"] +
             ["-include", HERE / "ref_cr_shim.h", HERE / "ref_harness.cpp", BUILD / "or_crmath.o",
              "-o", out, "-lquadmath"])
    if gpu and shutil.which("nvcc"):
        gpu_src = REFERENCE / "gym_adapter" / "gpu.cu"
        out = REF_OUT / "libns_ref_gpu.so"
        if _stale(out, [gpu_src, native]):
            # Flags of gym_adapter/gpu.py:19 with the arch pinned to sm_100a.
            _run(["nvcc", "-O3", "-std=c++17", "--fmad=false", "--prec-div=true", "--prec-sqrt=true",
                  "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-Xcompiler", "-fPIC",
                  *inc, gpu_src, "-o", out, "--cudart", "shared"])
        # The world simulator's neural kernels (src/main.cu) with the world
        # binary's flags (CMakeLists.txt:8), for timing only.
        world_src = REFERENCE / "src" / "main.cu"
        out = REF_OUT / "libns_ref_world.so"
        if _stale(out, [world_src, HERE / "ref_world_harness.cu"]):
            stub = REF_OUT / "stub_include"
            stub.mkdir(exist_ok=True)
            (stub / "png.h").write_text(
                "/* stub: the timing harness never writes images */\n#pragma once\n"
                "typedef struct { unsigned version, width, height, format; char message[64]; } png_image;\n"
                "#define PNG_IMAGE_VERSION 1\n#define PNG_FORMAT_RGB 2\n"
                "static inline int png_image_write_to_file(png_image *, const char *, int, const void *, int,"
                " const void *) { return 1; }\n")
            _run(["nvcc", "-O3", "-std=c++17", "--use_fast_math", "-gencode", "arch=compute_100a,code=sm_100a",
                  "-shared", "-Xcompiler", "-fPIC", "-I", stub, "-I", REFERENCE / "src",
                  "-DLIVE_ASSET_DIR=\"/nonexistent\"", HERE / "ref_world_harness.cu", REFERENCE / "src" / "live_view.cpp",
                  "-o", out, "-lz"])
        # The same kernels for the bit-exact comparison: IEEE division and
        # square root, no FMA contraction, exp/log correctly rounded.
        out = REF_OUT / "libns_ref_world_cr.so"
        if _stale(out, [world_src, HERE / "ref_world_harness.cu", HERE / "ref_cr_shim_cuda.h", CSRC / "ns_crmath.h"]):
            stub = REF_OUT / "stub_include"
            # -maxrregcount=128: the reference launches 512-thread CTAs
            # (NEURAL_BLOCK), which can hold at most 128 registers per thread.
            _run(["nvcc", "-O3", "-std=c++17", "--fmad=false", "--prec-div=true", "--prec-sqrt=true",
                  "-maxrregcount=128", "-gencode", "arch=compute_100a,code=sm_100a", "-shared",
                  "-Xcompiler", "-fPIC,-ffp-contract=off",
                  "-I", stub, "-I", REFERENCE / "src", "-I", CSRC, "-include", HERE / "ref_cr_shim_cuda.h",
                  "-DLIVE_ASSET_DIR=\"/nonexistent\"", HERE / "ref_world_harness.cu", REFERENCE / "src" / "live_view.cpp",
                  "-o", out, "-lz"])
    return REF_OUT


if __name__ == "__main__":
    build_oracle()
    r = build_ref(gpu="--no-gpu" not in sys.argv)
    print("oracle built;", "reference built" if r else "reference tree absent")
