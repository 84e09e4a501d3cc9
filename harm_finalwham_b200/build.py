"""Build the sm_100a shared library libharmgpu.so in-tree.

    python -m harm_finalwham_b200.build

nvcc compiles csrc/harm_gpu.cu for sm_100a only (-gencode
arch=compute_100a,code=sm_100a) with -fmad=false so that the FP64 path keeps
the reference's floating-point operation order (the reference CPU build uses
-ffp-contract=off).  The library has a plain C ABI (include/harmgpu.h).
"""
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIBDIR = os.path.join(PKG, "lib")
LIB = os.path.join(LIBDIR, "libharmgpu.so")
SOURCES = ["harm_gpu.cu"]
HEADERS = ["harm_device.cuh", "weno5.cuh", os.path.join(ROOT, "include", "harmgpu.h")]

NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
              "-fmad=false", "-Xcompiler", "-fPIC", "-shared", "--expt-relaxed-constexpr",
              "-diag-suppress", "177"]


def _newest_input():
    paths = [os.path.join(CSRC, s) for s in SOURCES] + [h if os.path.isabs(h) else os.path.join(CSRC, h) for h in HEADERS]
    return max(os.path.getmtime(p) for p in paths)


def build(force=False, verbose=False):
    os.makedirs(LIBDIR, exist_ok=True)
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= _newest_input():
        return LIB
    nvcc = os.environ.get("NVCC", "nvcc")
    cmd = [nvcc] + NVCC_FLAGS + ["-I" + os.path.join(ROOT, "include"), "-o", LIB] + \
          [os.path.join(CSRC, s) for s in SOURCES]
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed building libharmgpu.so")
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
