"""The reference's own relativistic shock tube (the generic init.c's
TESTNUMBER 101, the RAM paper's first problem: 400 zones, rho 10 | 1,
p 13.33 | 1e-8, Gamma 5/3, CFL 0.5, OUTFLOW copies at both ends, its
density floors), run by the reference build (tests/golden, made by
tests/golden/make_golden.py) and on the device: as a single 1D domain and
as one instance of a batch of uneven problems advanced by shared launches,
bit for bit after 1, 50 and 200 steps, with the same failure and floor
counters."""
import numpy as np
import pytest

from harm_finalwham_b200 import riemann
from harm_finalwham_b200.gpu import HarmBatch, HarmGPU
from tests.fixtures import load, same

pytestmark = pytest.mark.gpu

NAME = "ram101_400_mc_hll"


def test_reference_shock_tube_on_one_domain():
    pr, ref = load(NAME)
    with HarmGPU.from_problem(pr) as g:
        done = 0
        for s in sorted(ref):
            st = g.step_ch(s - done)
            done = s
            p, pf, t, dt = g.download_state()
            r = ref[s]
            assert same(p, r["p"]), f"primitives differ after step {s}"
            assert np.array_equal(pf, r["pflag"]) and t == r["t"] and dt == r["dt"]
            assert st.err == 0
            c = g.active(g.download_failfloorcount())
            assert np.array_equal(c, pr.active(r["ffc"]) - pr.active(pr.ffc_init)), f"counters after step {s}"


def test_reference_shock_tube_as_a_batch_instance():
    pr, ref = load(NAME)
    n, ng = pr.n[0], pr.ng
    others = riemann.draw(3, seed=5, nmin=60, nmax=300)
    n1s = [n] + [q.n for q in others]
    dxs = [pr.dx[0]] + [q.dx for q in others]
    gams = [pr.gam] + [q.gam for q in others]
    tfs = [pr.tf] + [0.4] * len(others)
    b = HarmBatch(n1s, dxs, gams, tfs, ng=ng, lim=pr.lim, flux=pr.flux, cour=pr.cour, safe=pr.safe,
                  defcon=pr.defcon, rhominlimit=pr.rhominlimit, uuminlimit=pr.uuminlimit, gammamax=pr.gammamax,
                  gammafail=pr.gammafail, utoprim=pr.utoprim, timeorder=pr.timeorder)
    try:
        geo = list(riemann.minkowski_geometry(b.nt[0]))
        # instance 0 carries the reference's own geometry and density floors
        # (the floors of its zones are the reference's set_density_floors)
        for q, a in enumerate((pr.gcov, pr.gcon, pr.gcovpert, pr.gdet, pr.conn, pr.floors)):
            seg = b.split(geo[q][:-1] if geo[q].shape[0] == b.nt[0] + 1 else geo[q])[0]
            seg[...] = a[:n + 2 * ng]
        b.upload_geometry(*geo)
        b.upload_state(b.join([pr.p] + [riemann.primitives(q, ng) for q in others]), None, 0.0, 0.0)
        b.init_dt()
        t0, dt0, _, _ = b.status()
        dt0[0] = pr.dt           # the reference's start-up dt (its set_dt)
        b.set_time(t0, dt0)
        done = 0
        for s in sorted(ref):
            b.step_ch(s - done)
            done = s
            p, pf, _, _ = b.download_state()
            t, dt, _, _ = b.status()
            r = ref[s]
            assert same(b.split(p)[0], r["p"]), f"the batch instance differs from the reference after step {s}"
            assert np.array_equal(b.split(pf)[0][ng:ng + n], r["pflag"][ng:ng + n])
            assert t[0] == r["t"] and dt[0] == r["dt"]
    finally:
        b.close()
