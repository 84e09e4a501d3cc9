"""The reference's own relativistic shock tubes (the generic init.c's
TESTNUMBER 101, 102, 103 and 106: the RAM paper's problems 1, 2, 3 and 6.1
on 400 zones, CFL 0.5, OUTFLOW copies at both ends, the reference's density
floors and Jon's inverter; 6.1 trips failed inversions, the Lorentz-factor
limit and checksolution), run by the reference build (tests/golden, made by
tests/golden/make_golden.py) and on the device: each as a single 1D domain,
and all four together as instances of one batch of uneven problems advanced
by shared launches, bit for bit after every dumped step, with the same
failure and floor counters."""
import numpy as np
import pytest

from harm_finalwham_b200 import riemann
from harm_finalwham_b200.gpu import HarmBatch, HarmGPU
from tests.fixtures import load, same

pytestmark = pytest.mark.gpu

NAMES = ["ram101_400_mc_hll", "ram102_400_mc_hll", "ram103_400_mc_hll", "ram106_400_mc_hll"]


@pytest.mark.parametrize("name", NAMES)
def test_reference_shock_tube_on_one_domain(name):
    pr, ref = load(name)
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


def test_reference_shock_tubes_as_batch_instances():
    probs = [load(n) for n in NAMES]
    pr0 = probs[0][0]
    ng = pr0.ng
    others = riemann.draw(3, seed=5, nmin=60, nmax=300)
    n1s = [pr.n[0] for pr, _ in probs] + [q.n for q in others]
    b = HarmBatch(n1s, [pr.dx[0] for pr, _ in probs] + [q.dx for q in others],
                  [pr.gam for pr, _ in probs] + [q.gam for q in others],
                  [pr.tf for pr, _ in probs] + [0.4] * len(others), ng=ng, lim=pr0.lim, flux=pr0.flux,
                  cour=pr0.cour, safe=pr0.safe, defcon=pr0.defcon, rhominlimit=pr0.rhominlimit,
                  uuminlimit=pr0.uuminlimit, gammamax=pr0.gammamax, gammafail=pr0.gammafail, utoprim=pr0.utoprim,
                  timeorder=pr0.timeorder)
    try:
        geo = list(riemann.minkowski_geometry(b.nt[0]))
        # the reference problems' instances carry their own geometry and
        # density floors (the reference's set_density_floors)
        for q, (pr, _) in enumerate(probs):
            n = pr.n[0]
            for k, a in enumerate((pr.gcov, pr.gcon, pr.gcovpert, pr.gdet, pr.conn, pr.floors)):
                b.split(geo[k][:-1])[q][...] = a[:n + 2 * ng]
        b.upload_geometry(*geo)
        b.upload_state(b.join([pr.p for pr, _ in probs] + [riemann.primitives(q, ng) for q in others]), None,
                       0.0, 0.0)
        b.init_dt()
        t0, dt0, _, _ = b.status()
        for q, (pr, _) in enumerate(probs):
            dt0[q] = pr.dt           # the reference's start-up dt (its set_dt)
        b.set_time(t0, dt0)
        steps = sorted({s for _, ref in probs for s in ref})
        done = 0
        for s in steps:
            b.step_ch(s - done)
            done = s
            p, pf, _, _ = b.download_state()
            t, dt, _, _ = b.status()
            for q, (pr, ref) in enumerate(probs):
                if s not in ref:
                    continue
                r, n = ref[s], pr.n[0]
                assert same(b.split(p)[q], r["p"]), f"instance {q} ({NAMES[q]}) differs after step {s}"
                assert np.array_equal(b.split(pf)[q][ng:ng + n], r["pflag"][ng:ng + n])
                assert t[q] == r["t"] and dt[q] == r["dt"]
    finally:
        b.close()
