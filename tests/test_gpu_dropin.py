"""The reference's own program driving the GPU through the drop-in step_ch.

oracle/_ref/harm_ref_*_gpushim is the reference's C sources (its init, its
arrays, the step loop of oracle/ref_harness.c that main.c:33-49 runs) with
harm_finalwham_b200/dropin/step_ch_gpu.c linked in place of its CPU step_ch
(step_ch.c:16).  Its dumps must equal the reference's own CPU run bit for
bit: the 64x64 torus configuration for its 200 steps (the record of the
reference's run), the 3D WENO5 + HLL torus with azimuthal modes, a strongly
magnetised torus (failed inversions, b^2 flags) and the finite-volume scheme
(PARA, RK4, Jon's inverter) against their golden fixtures, and the restart
dump the reference's restart_write makes from the GPU state equals the one
of its CPU run byte for byte."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from oracle.pyoracle import LIBDIR, RefDump
from tests.fixtures import load, load_record, same

pytestmark = pytest.mark.gpu


def run_shim(binary, nsteps, dumps, args=()):
    exe = os.path.join(LIBDIR, binary)
    assert os.path.exists(exe), f"{exe} is missing: __graft_entry__.build() builds it"
    tmp = tempfile.TemporaryDirectory()
    out = os.path.join(tmp.name, "out")
    r = subprocess.run([exe] + list(args) + [out, str(nsteps)] + [str(d) for d in dumps], cwd=tmp.name,
                       capture_output=True, text=True)
    assert r.returncode == 0, f"{binary} failed: {r.stderr[-2000:]}"
    return tmp, RefDump(out)


def test_reference_loop_on_gpu_matches_reference_run_64x64():
    rec = load_record("torus2d_64x64_mc_hll_200")
    tmp, rd = run_shim("harm_ref_64x64x1_MC_HLL_gpushim", 200, [1])
    with tmp:
        for s in (1, 200):
            tag = f"s{s}"
            p = rd.crop(rd.p(tag), 0)
            f = rd.crop(rd.pflag(tag), 0)[..., 0]
            m = rd.meta_of(tag)
            assert same(p, rec[f"{tag}_p"]), f"primitives differ from the reference's run after step {s}"
            assert np.array_equal(f, rec[f"{tag}_pflag"]), f"failure flags differ after step {s}"
            assert m["t"] == float(rec[f"{tag}_t"]) and m["dt"] == float(rec[f"{tag}_dt"])
            assert m["nstroke"] == float(rec[f"{tag}_nstroke"])


@pytest.mark.parametrize("binary,fixture,args", [
    ("harm_ref_12x12x6_WENO5_HLL_gpushim", "torus3d_12x12x6_weno5_hll", ["--phimodes", "1"]),
    ("harm_ref_16x16x1_MC_HLL_beta0.0001_gpushim", "torus2d_16x16_mc_hll_beta1e-4", []),
    ("harm_ref_16x16x1_PARA_HLL_rk4_jon_fv_gpushim", "torus2d_16x16_para_hll_rk4_jon_fv", []),
])
def test_reference_loop_on_gpu_matches_golden(binary, fixture, args):
    pr, ref = load(fixture)
    steps = sorted(ref)
    # --rdump: the reference's own restart_write after the last step, through
    # the shim's wrapper that brings unew from the device (a run without
    # dump_ener, as the fixture's dump was made)
    tmp, rd = run_shim(binary, steps[-1], [], ["--rdump"] + list(args))
    with tmp:
        with open(os.path.join(tmp.name, "dumps", "rdump-0"), "rb") as f:
            assert f.read() == pr.rdump, "the restart dump differs from the reference's"
    # --ener --ffc: dump_ener, whose wrapper adds the device's failure and
    # floor counters to the reference's failfloorcount, before every dump
    tmp, rd = run_shim(binary, steps[-1], steps[:-1], ["--ener", "--ffc"] + list(args))
    with tmp:
        for s in steps:
            tag = f"s{s}"
            r = ref[s]
            assert same(rd.crop(rd.p(tag), pr.ng), r["p"]), f"primitives differ after step {s}"
            assert np.array_equal(rd.crop(rd.pflag(tag), pr.ng)[..., 0], r["pflag"])
            assert np.array_equal(rd.crop(rd.pflag(tag), pr.ng)[..., 2:4], r["bsq"])
            act = pr.active
            assert np.array_equal(act(rd.crop(rd.ffc(tag), pr.ng)), act(r["ffc"])), \
                f"failure/floor counters differ after step {s}"
            m = rd.meta_of(tag)
            assert m["t"] == r["t"] and m["dt"] == r["dt"] and m["nstroke"] == r["nstroke"]
            if r["u"] is not None:
                assert same(act(rd.crop(rd.unew(tag), pr.ng)), act(r["u"])), f"unew differs after step {s}"


def test_reference_bondi_flow_on_gpu_tracks_its_cpu_run():
    # the generic init.c's Bondi flow (TESTNUMBER 153) with its Bondi-integral
    # x1 boundaries and the generic polar axis, through the drop-in built
    # with -DHARMGPU_GENERIC_BOUNDS; pow in the boundaries makes the bar a
    # tolerance (the device's own runs: tests/test_gpu_bondi_bc.py)
    pr, ref = load("bondi2d_16x16_mc_hll")
    exe = os.path.join(LIBDIR, "harm_bondi_16x16x1_MC_HLL_jon_gpushim")
    assert os.path.exists(exe), f"{exe} is missing: __graft_entry__.build() builds it"
    steps = sorted(ref)
    with tempfile.TemporaryDirectory() as tmp:
        with open(os.path.join(tmp, "bondigrid16.dat"), "wb") as f:
            f.write(pr.bondigrid_dat)
        out = os.path.join(tmp, "out")
        r = subprocess.run([exe, out, str(steps[-1])] + [str(s) for s in steps[:-1]], cwd=tmp,
                           capture_output=True, text=True)
        assert r.returncode == 0, r.stderr[-2000:]
        rd = RefDump(out)
        act = pr.active
        for s in steps:
            p = act(rd.crop(rd.p(f"s{s}"), pr.ng))
            want = act(ref[s]["p"])
            for q, tol in ((0, 1e-13), (1, 1e-13), (2, 1e-13), (3, 1e-11)):
                l1 = float(np.sum(np.abs(p[..., q] - want[..., q])) / np.sum(np.abs(want[..., q])))
                assert l1 < tol, f"primitive {q}: relative L1 {l1:.3e} after {s} steps"
            m = rd.meta_of(f"s{s}")
            assert abs(m["t"] - ref[s]["t"]) <= 1e-13 * ref[s]["t"]


def test_reference_shock_tube_on_gpu_matches_its_cpu_run():
    # the generic init.c's relativistic shock tube 6.1 (TESTNUMBER 106: failed
    # inversions, the Lorentz-factor limit, checksolution) on the Minkowski
    # line, the drop-in built with -DHARMGPU_GENERIC_BOUNDS
    pr, ref = load("ram106_400_mc_hll")
    steps = sorted(ref)
    tmp, rd = run_shim("harm_ram106_400x1x1_MC_HLL_jon_gpushim", steps[-1], steps[:-1])
    with tmp:
        for s in steps:
            tag = f"s{s}"
            r = ref[s]
            assert same(rd.crop(rd.p(tag), pr.ng), r["p"]), f"primitives differ after step {s}"
            assert np.array_equal(rd.crop(rd.pflag(tag), pr.ng)[..., 0], r["pflag"])
            m = rd.meta_of(tag)
            assert m["t"] == r["t"] and m["dt"] == r["dt"] and m["nstroke"] == r["nstroke"]

