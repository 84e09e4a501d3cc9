"""The CPU restatement (oracle/) reproduces the reference's own outputs bit for
bit on the golden fixtures generated from the reference build."""
import numpy as np
import pytest

from oracle.pyoracle import Oracle
from tests.fixtures import CASES, load, same


@pytest.fixture(scope="module")
def orc():
    return Oracle()


@pytest.mark.parametrize("name", CASES)
def test_oracle_matches_reference(orc, name):
    pr, ref = load(name)
    done = 0
    for s in sorted(ref):
        orc.step(pr, s - done)
        done = s
        r = ref[s]
        assert same(pr.p, r["p"]), f"primitives differ after step {s}"
        assert np.array_equal(pr.pflag, r["pflag"]), f"pflag map differs after step {s}"
        assert pr.dt == r["dt"] and pr.t == r["t"]
        if r["u"] is not None:
            # the finite-volume scheme's evolved conserved state (unew) in the active zones
            act = pr.active
            assert same(act(pr.u), act(r["u"])), f"conserved state differs after step {s}"


@pytest.mark.parametrize("name", CASES)
def test_oracle_newton_iterations_match_reference(orc, name):
    # the reference counts Newton iterations per step in nstroke (main.c:35)
    pr, ref = load(name)
    done = 0
    for s in sorted(ref):
        if s - done != 1:
            orc.step(pr, s - done - 1)
        st = orc.step(pr, 1)
        done = s
        assert st.newton_iters == ref[s]["nstroke"]


@pytest.mark.parametrize("name", CASES)
def test_divb_roundoff_in_reference_and_oracle(orc, name):
    # flux-CT keeps the corner-centred div B at round-off (global.h:1586-1645)
    from tests.divb import divb_max
    pr, ref = load(name)
    for s in sorted(ref):
        assert divb_max(ref[s]["p"], pr.gdet, pr.ng, pr.dx, pr.n) < 1e-12
    orc.step(pr, 10)
    assert divb_max(pr.p, pr.gdet, pr.ng, pr.dx, pr.n) < 1e-12


@pytest.mark.parametrize("inv", ["2DFINAL", "JON"])
def test_oracle_utoprim_zones_match_reference(orc, inv):
    # the reference's Utoprimgen run zone by zone through the harness
    # (oracle/ref_harness.c --invert) on seeded zones, both inverters
    from tests.fixtures import load_zones
    z = load_zones()
    pr, pf, it = orc.utoprim(z["U"], z["gcov"], z["gcon"], z["gdet"], z["guess"], z["gam"], z["gammafail"],
                             version=inv)
    assert np.array_equal(pf, z[f"pflag_{inv}"])
    assert same(pr, z[f"pr_{inv}"])
    assert it == int(z[f"iters_{inv}"].sum())
    # the fixture covers converged, failed-Newton and negative-energy zones
    flags = set(np.unique(pf).tolist())
    assert {0, 101, 10} <= flags


def test_oracle_pi2u_matches_reference_init():
    # pi2Uavg (initbase.c:1833): the finite-volume scheme's initial unew
    pr, _ = load("torus2d_16x16_para_hll_rk4_jon_fv")
    assert same(Oracle().pi2u(pr), pr.u)


def test_oracle_matches_reference_run_of_the_64x64_torus(orc):
    # the 2D FM torus 64x64 configuration (MC + HLL + flux-CT, RK2, CFL 0.8)
    # for its 200 steps, against the record of the reference's own run; the
    # initial state comes from the same reference binary
    import os
    import subprocess
    import tempfile

    from oracle.pyoracle import LIBDIR, RefDump
    from tests.fixtures import load_record, summarise
    exe = os.path.join(LIBDIR, "harm_ref_64x64x1_MC_HLL")
    if not os.path.exists(exe):
        pytest.skip("reference binary not built (__graft_entry__.build builds it where the reference tree is)")
    rec = load_record("torus2d_64x64_mc_hll_200")
    with tempfile.TemporaryDirectory() as tmp:
        out = os.path.join(tmp, "init")
        subprocess.run([exe, out, "0"], cwd=tmp, check=True, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        pr = RefDump(out).to_problem(3, "init")
    assert summarise(pr.active(pr.p), pr.active(pr.pflag), (1, 1, 1))["sha_p"] == str(rec["init_sha_p"])
    done = 0
    for s in [int(x) for x in rec["steps"]]:
        orc.step(pr, s - done)
        done = s
        assert same(pr.active(pr.p), rec[f"s{s}_p"]), f"primitives differ after step {s}"
        assert np.array_equal(pr.active(pr.pflag), rec[f"s{s}_pflag"])
        assert pr.t == float(rec[f"s{s}_t"]) and pr.dt == float(rec[f"s{s}_dt"])
