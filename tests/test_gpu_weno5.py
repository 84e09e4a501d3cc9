"""WENO5 (lim=WENO5) FP64 GPU path vs the oracle, which test_oracle_golden pins
to the reference's own WENO5 build bit for bit.  Exact comparisons."""
import numpy as np
import pytest

from harm_finalwham_b200 import torus
from harm_finalwham_b200.gpu import HarmGPU
from oracle.pyoracle import Oracle, Problem
from tests.fixtures import load, same

pytestmark = pytest.mark.gpu


def problem_of(dom):
    pr = Problem(*dom.n, dom.ng, dom.dx, gam=dom.gam, cour=dom.cour, lim=dom.lim, flux=dom.flux, bc=dom.bc,
                 safe=dom.safe, defcon=dom.defcon, tf=dom.tf, rhominlimit=dom.rhominlimit,
                 uuminlimit=dom.uuminlimit, gammamax=dom.gammamax, gammafail=dom.gammafail)
    for k in ("gcov", "gcon", "gcovpert", "gdet", "conn", "floors", "p", "pflag"):
        getattr(pr, k)[...] = getattr(dom, k)
    pr.t, pr.dt = dom.t, dom.dt
    return pr


def test_weno5_long_run_2d_matches_oracle():
    pr, _ = load("torus2d_16x16_weno5_hll")
    q = pr.copy()
    with HarmGPU.from_problem(pr) as g:
        g.step_ch(100)
        p, pf, t, dt = g.download_state()
    Oracle().step(q, 100)
    assert same(p, q.p)
    assert np.array_equal(pf, q.pflag)
    assert t == q.t and dt == q.dt


@pytest.mark.parametrize("flux", ["HLL", "LAXF"])
def test_weno5_3d_torus_matches_oracle(flux):
    dom = torus.fm_torus(32, 32, 16, ng=6, lim="WENO5", flux=flux, seed=11)
    pr = problem_of(dom)
    q = pr.copy()
    with HarmGPU.from_problem(pr) as g:
        g.init_dt()
        _, _, _, dt0 = g.download_state()
        q.dt = dt0
        st = g.step_ch(3)
        p, pf, t, dt = g.download_state()
    Oracle().step(q, 3)
    assert st.err == 0
    assert same(p, q.p), f"{int(np.count_nonzero(p != q.p))} values differ"
    assert np.array_equal(pf, q.pflag)
    assert t == q.t and dt == q.dt


def test_weno5_rejects_too_few_ghosts():
    from harm_finalwham_b200.gpu import HarmGPUError
    with pytest.raises(HarmGPUError):
        HarmGPU(16, 16, 1, 3, (0.1, 0.1, 0.1), lim="WENO5")
