"""The FP64 GPU path against the reference at the benchmark configurations'
own sizes and step counts.

The reference binary of each configuration (oracle/_ref, built from the
reference's sources by __graft_entry__.build) writes its initial state and
geometry; the GPU runs the configuration's steps from it, and the result is
compared with the record of the reference's own run of the same steps
(tests/golden/records, made by tests/golden/make_golden.py):

* the initial state equals the one the record was made from (same binary,
  same seed);
* the primitives and the failure-flag map of the active zones hash to the
  reference's (SHA-256: bit-identical), and t, dt and the Newton iteration
  count agree exactly;
* on a mismatch the test reports the relative L1 per primitive (over every
  zone where the record holds the whole state, else over its sample
  lattice) against the gates: 1e-12 after one step, 1e-8 after the
  configuration's step count.
"""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from harm_finalwham_b200.gpu import HarmGPU
from oracle.pyoracle import LIBDIR, RefDump
from tests.fixtures import load_record, summarise

pytestmark = pytest.mark.gpu

# record -> (reference binary, ghost zones on the GPU)
CONFIGS = {
    # 2D FM torus 64x64, MC + HLL + flux-CT, RK2, CFL 0.8, 200 steps
    "torus2d_64x64_mc_hll_200": ("harm_ref_64x64x1_MC_HLL", 3),
    # 3D torus 128x64x32 with azimuthal density modes, WENO5 + HLL, 500 steps
    "torus3d_128x64x32_weno5_hll_500": ("harm_ref_128x64x32_WENO5_HLL", 6),
    # precision-at-scale torus 256x128x128, WENO5 + HLL, first 5 steps
    "torus3d_256x128x128_weno5_hll_5": ("harm_ref_256x128x128_WENO5_HLL", 6),
    # the FM torus problem file's own scheme (PARA, RK4, Jon, finite volume,
    # all 11 MAXBND ghosts) on the 3D torus 64x32x32, 20 steps
    "torus3d_64x32x32_para_hll_rk4_jon_fv_20": ("harm_ref_64x32x32_PARA_HLL_rk4_jon_fv", 11),
}


def reference_init(name):
    """Initial state and geometry written by the configuration's reference binary."""
    exe, ng = CONFIGS[name]
    exe = os.path.join(LIBDIR, exe)
    assert os.path.exists(exe), f"{exe} is missing: __graft_entry__.build() builds it"
    rec = load_record(name)
    args = str(rec["harness_args"]).split()
    with tempfile.TemporaryDirectory() as tmp:
        out = os.path.join(tmp, "init")
        subprocess.run([exe] + args + [out, "0"], cwd=tmp, check=True, stdout=subprocess.DEVNULL,
                       stderr=subprocess.DEVNULL)
        pr = RefDump(out).to_problem(ng, "init")
    return pr, rec


def rel_l1(got, ref):
    """Relative L1 per primitive (sum |got - ref| / sum |ref| over zones)."""
    axes = tuple(range(ref.ndim - 1))
    return np.abs(got - ref).sum(axis=axes) / np.maximum(np.abs(ref).sum(axis=axes), 1e-300)


@pytest.mark.parametrize("name", list(CONFIGS))
def test_configuration_matches_reference_run(name):
    pr, rec = reference_init(name)
    stride = tuple(int(s) for s in rec["stride"])
    s0 = summarise(pr.active(pr.p), pr.active(pr.pflag), stride)
    assert s0["sha_p"] == str(rec["init_sha_p"]), "the reference binary wrote a different initial state"
    assert pr.t == float(rec["init_t"]) and pr.dt == float(rec["init_dt"])
    steps = [int(s) for s in rec["steps"]]
    with HarmGPU.from_problem(pr) as g:
        done = 0
        for s in steps:
            if s - done > 1:
                g.step_ch(s - done - 1)
            st = g.step_ch(1)
            done = s
            p, pf, t, dt = g.download_state()
            pa, fa = g.active(p), g.active(pf)
            got = summarise(pa, fa, stride)
            tag = f"s{s}"
            whole = f"{tag}_p" in rec
            ref = rec[f"{tag}_p"] if whole else rec[f"{tag}_sample"]
            rel = rel_l1(pa if whole else got["sample"], ref)
            bar = 1e-12 if s == 1 else 1e-8
            where = "all zones" if whole else "the sample lattice"
            assert (rel <= bar).all(), f"step {s}: relative L1 per primitive over {where} {rel} above {bar}"
            assert got["sha_pflag"] == str(rec[f"{tag}_sha_pflag"]), f"step {s}: failure-flag map differs"
            assert got["sha_p"] == str(rec[f"{tag}_sha_p"]), \
                f"step {s}: not bit-identical (relative L1 over {where} {rel}, within the {bar} gate)"
            assert t == float(rec[f"{tag}_t"]) and dt == float(rec[f"{tag}_dt"])
            assert st.newton_iters == float(rec[f"{tag}_nstroke"])
            assert st.err == 0
