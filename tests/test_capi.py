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


def test_configuration_validation_on_the_host():
    # hgpu_context_bytes runs the same validation as hgpu_create and
    # touches no device: 0 means rejected
    from harm_finalwham_b200.gpu import context_bytes, make_config

    def ok(**kw):
        base = dict(n=(32, 32, 1), ng=3, dx=(0.1, 0.1, 1.0))
        base.update(kw)
        n, ng, dx = base.pop("n"), base.pop("ng"), base.pop("dx")
        return context_bytes(make_config(n, ng, dx, **base)) > 0

    assert ok()
    assert ok(lim="PARA") and not ok(lim="PARA", ng=2)          # PARA reads 3 zones out
    assert ok(lim="WENO5", ng=6) and not ok(lim="WENO5", ng=5)  # WENO5 reads 6
    assert ok(timeorder=4) and ok(timeorder=1) and not ok(timeorder=5)
    assert ok(utoprim="JON") and not ok(utoprim=7)
    assert ok(doenoflux="ENOFINITEVOLUME", ng=11, n=(32, 32, 1)) and not ok(doenoflux=2)
    assert not ok(n=(32, 2, 1))                                  # reflections need n2 >= ng
    # the finite-volume scheme keeps a second conserved array; RK3/RK4 a second intermediate state
    base = context_bytes(make_config((32, 32, 1), 3, (0.1, 0.1, 1.0)))
    assert context_bytes(make_config((32, 32, 1), 3, (0.1, 0.1, 1.0), doenoflux="ENOFINITEVOLUME")) > base
    assert context_bytes(make_config((32, 32, 1), 3, (0.1, 0.1, 1.0), timeorder=4)) > base


def test_split_entry_points_reject_bad_arguments_without_gpu_work():
    # every x3-split entry point validates its arguments before touching the
    # device: a NULL context (or NULL output) is HGPU_E_INVALID
    HGPU_E_INVALID = 1
    L = load_library()
    buf = ctypes.create_string_buffer(64)
    nb = ctypes.c_size_t()
    st = ctypes.c_void_p()
    assert L.hgpu_halo_bytes(None, ctypes.byref(nb)) == HGPU_E_INVALID
    for side in (0, 1):
        assert L.hgpu_halo_pack(None, 0, side, 1, ctypes.addressof(buf)) == HGPU_E_INVALID
        assert L.hgpu_halo_unpack(None, 0, side, 0, ctypes.addressof(buf)) == HGPU_E_INVALID
    assert L.hgpu_stats_clear(None) == HGPU_E_INVALID
    assert L.hgpu_stats_read(None, None) == HGPU_E_INVALID
    assert L.hgpu_stage_advance(None, 0) == HGPU_E_INVALID
    assert L.hgpu_stage_fixup(None, 0) == HGPU_E_INVALID
    assert L.hgpu_post_fixup(None, 1, None) == HGPU_E_INVALID
    assert L.hgpu_dt_probe(None) == HGPU_E_INVALID
    assert L.hgpu_step_end(None, 1) == HGPU_E_INVALID
    assert L.hgpu_ndt_pack(None, ctypes.addressof(buf)) == HGPU_E_INVALID
    assert L.hgpu_ndt_unpack(None, ctypes.addressof(buf)) == HGPU_E_INVALID
    assert L.hgpu_stream(None, ctypes.byref(st)) == HGPU_E_INVALID
    assert L.hgpu_autotune(None, None) == HGPU_E_INVALID
