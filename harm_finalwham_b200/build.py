"""Build the sm_100a shared library libharmgpu.so in-tree.

    python -m harm_finalwham_b200.build

nvcc compiles csrc/harm_gpu.cu (kernels and C ABI), csrc/serve.cu (the
serving loop, host code), csrc/rdump.cu (restart dumps, host code) for sm_100a only (-gencode
arch=compute_100a,code=sm_100a) with -fmad=false so that the FP64 path keeps
the reference's floating-point operation order (the reference CPU build uses
-ffp-contract=off), and csrc/flux_f32.cu (the FP32 kernels of the mixed
precision path) with FMA contraction and fast FP32 division/square root.
The objects go to _build/ and are linked into lib/libharmgpu.so, whose
plain C ABI is include/harmgpu.h.
"""
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIBDIR = os.path.join(PKG, "lib")
LIB = os.path.join(LIBDIR, "libharmgpu.so")
SOURCES = ["harm_gpu.cu", "serve.cu", "rdump.cu", "flux_f32.cu"]
HEADERS = ["harm_device.cuh", "weno5.cuh", "common.cuh", os.path.join(ROOT, "include", "harmgpu.h")]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
                 "-diag-suppress", "177,550"]
# FP64 path: no contraction, so every operation rounds as in the reference build
NVCC_FLAGS = COMMON + ["-fmad=false"]
# FP32 kernels of the mixed-precision path: contraction and fast FP32 division
# and square root (these flags do not affect FP64 arithmetic)
NVCC_FLAGS_F32 = COMMON + ["-fmad=true", "-prec-div=false", "-prec-sqrt=false", "-ftz=true"]
FAST_SOURCES = {"flux_f32.cu"}
OBJDIR = os.path.join(PKG, "_build")


def _newest_input():
    paths = [os.path.join(CSRC, s) for s in SOURCES] + [h if os.path.isabs(h) else os.path.join(CSRC, h) for h in HEADERS]
    return max(os.path.getmtime(p) for p in paths)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed building libharmgpu.so")


def build(force=False, verbose=False):
    os.makedirs(LIBDIR, exist_ok=True)
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= _newest_input():
        return LIB
    nvcc = os.environ.get("NVCC", "nvcc")
    os.makedirs(OBJDIR, exist_ok=True)
    inc = ["-I" + os.path.join(ROOT, "include")]
    objs = []
    for src in SOURCES:
        obj = os.path.join(OBJDIR, src.replace(".cu", ".o"))
        flags = NVCC_FLAGS_F32 if src in FAST_SOURCES else NVCC_FLAGS
        _run([nvcc] + flags + inc + ["-c", "-o", obj, os.path.join(CSRC, src)], verbose)
        objs.append(obj)
    _run([nvcc] + ARCH + ["-shared", "-o", LIB] + objs, verbose)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
