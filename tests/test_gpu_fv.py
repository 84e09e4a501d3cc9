"""Finite-volume scheme (DOENOFLUX = ENOFINITEVOLUME, avgscheme = DONOR) on
the GPU: the FM torus problem file's own scheme (PARA, HLL, RK4, Jon's
inverter).  The golden fixtures (test_gpu_parity) pin the first steps to the
reference build; these compare longer runs with the oracle, which
test_oracle_golden pins to the reference, and check that a restart from
(p, unew) continues bit for bit."""
import numpy as np
import pytest

from harm_finalwham_b200.gpu import HarmGPU
from oracle.pyoracle import Oracle
from tests.fixtures import load, same

pytestmark = pytest.mark.gpu


def test_fv_default_scheme_long_run_matches_oracle():
    pr, _ = load("torus2d_16x16_para_hll_rk4_jon_fv")
    q = pr.copy()
    with HarmGPU.from_problem(pr) as g:
        g.step_ch(60)
        p, pf, t, dt = g.download_state()
        u = g.download_conserved()
    Oracle().step(q, 60)
    assert same(p, q.p)
    assert np.array_equal(pf, q.pflag)
    assert t == q.t and dt == q.dt
    assert same(g.active(u), q.active(q.u))


def test_fv_starts_from_pi2u_without_stored_unew():
    # upload_state alone sets unew = U(p) (init_conservatives), which is
    # what the reference's init dumps
    pr, _ = load("torus2d_16x16_mc_hll_fv")
    q = pr.copy()
    q.u = None
    with HarmGPU.from_problem(q) as g:
        u0 = g.download_conserved()
    assert same(u0, pr.u)


def test_fv_restart_from_p_and_unew_continues_bit_for_bit():
    pr, _ = load("torus3d_12x12x6_para_laxf_rk4_jon_fv")
    with HarmGPU.from_problem(pr) as g:
        g.step_ch(3)
        p3, pf3, t3, dt3 = g.download_state()
        u3 = g.download_conserved()
        g.step_ch(3)
        p6, pf6, t6, dt6 = g.download_state()
        u6 = g.download_conserved()
    r = pr.copy()
    r.p[...] = p3
    r.pflag[...] = pf3
    r.t, r.dt = t3, dt3
    r.u = u3
    with HarmGPU.from_problem(r) as g:
        g.step_ch(3)
        p, pf, t, dt = g.download_state()
        u = g.download_conserved()
    assert same(p, p6) and np.array_equal(pf, pf6) and t == t6 and dt == dt6
    assert same(g.active(u), g.active(u6))
