"""The C-ABI library loads and exports every entry point include/harmgpu.h
declares (no GPU needed: nothing here launches work)."""
import ctypes
import os
import re
import subprocess

from harm_finalwham_b200 import build as hbuild
from harm_finalwham_b200.gpu import load_library

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    txt = open(os.path.join(ROOT, "include", "harmgpu.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(hgpu_[a-z_0-9]+)\s*\(", txt)))


def test_library_builds_and_loads():
    path = hbuild.build()
    assert os.path.exists(path)
    L = load_library()
    hdr = open(os.path.join(ROOT, "include", "harmgpu.h")).read()
    assert L.hgpu_abi_version() == int(re.search(r"#define HGPU_ABI_VERSION (\d+)", hdr).group(1))


def test_every_declared_symbol_is_exported():
    names = declared_functions()
    assert len(names) >= 14
    out = subprocess.run(["nm", "-D", "--defined-only", hbuild.LIB], capture_output=True, text=True, check=True).stdout
    exported = set(line.split()[-1] for line in out.splitlines() if " T " in line)
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    L = ctypes.CDLL(hbuild.LIB)
    for n in names:
        getattr(L, n)


def test_library_is_sm100a_only():
    out = subprocess.run(["cuobjdump", "--list-elf", hbuild.LIB], capture_output=True, text=True)
    if out.returncode != 0:
        return  # tool absent: nothing to check
    assert "sm_100a" in out.stdout


def test_invalid_config_is_rejected_without_gpu_work():
    from harm_finalwham_b200.gpu import HarmGPU, HarmGPUError
    import pytest
    with pytest.raises((HarmGPUError, ValueError)):
        HarmGPU(16, 16, 1, 1, (0.1, 0.1, 1.0))  # ng < 2 is invalid before any device call
