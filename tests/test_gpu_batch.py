"""Batched 1D relativistic-MHD Riemann problems (hgpu_create_batch): every
instance of a batch, advanced by shared launches with its own gamma, dx, t
and dt until its own end time, is bit-identical to the oracle running that
instance alone (the oracle's physics is pinned to the reference build)."""
import numpy as np
import pytest

from harm_finalwham_b200 import riemann
from harm_finalwham_b200.gpu import HarmBatch, HarmGPU
from oracle.pyoracle import BC_OUTFLOW, BC_OUTFLOW_COPY, Oracle, Problem
from tests.fixtures import same

pytestmark = pytest.mark.gpu


def oracle_problem(pb, ng, lim, flux, tf, dt):
    pr = Problem(pb.n, 1, 1, ng, (pb.dx, 1.0, 1.0), gam=pb.gam, cour=0.5, lim=lim, flux=flux,
                 bc=(BC_OUTFLOW_COPY, BC_OUTFLOW_COPY) + (BC_OUTFLOW,) * 4, tf=tf)
    for k, a in zip(("gcov", "gcon", "gcovpert", "gdet", "conn", "floors"), riemann.minkowski_geometry(pb.n + 2 * ng)):
        getattr(pr, k)[...] = a
    pr.p[...] = riemann.primitives(pb, ng)
    pr.dt = dt
    return pr


def make_batch(probs, ng, lim, flux, tfs, precision="fp64"):
    b = HarmBatch([p.n for p in probs], [p.dx for p in probs], [p.gam for p in probs], tfs, ng=ng, lim=lim,
                  flux=flux, precision=precision)
    b.upload_geometry(*riemann.minkowski_geometry(b.nt[0]))
    b.upload_state(b.join([riemann.primitives(p, ng) for p in probs]), None, 0.0, 0.0)
    b.init_dt()
    return b


@pytest.mark.parametrize("lim,flux,ng", [("MC", "HLL", 3), ("WENO5", "LAXF", 6), ("PARA", "HLL", 3)])
def test_batch_instances_match_oracle(lim, flux, ng):
    probs = riemann.draw(6, seed=3, nmin=40, nmax=120)
    tfs = [0.4, 0.05, 0.4, 0.2, 0.4, 0.1]
    b = make_batch(probs, ng, lim, flux, tfs)
    try:
        _, dt0, _, _ = b.status()
        steps, _, per, _ = b.run(check_every=7)
        t, _, done, ndone = b.status()
        assert ndone == len(probs) and np.all(done == 1)
        p, pf, _, _ = b.download_state()
    finally:
        b.close()
    assert steps < 200
    orc = Oracle()
    for q, (pb, tf) in enumerate(zip(probs, tfs)):
        pr = oracle_problem(pb, ng, lim, flux, tf, dt0[q])
        n = 0
        while pr.t < tf and n < 10000:
            orc.step(pr, 1)
            n += 1
        assert t[q] == pr.t
        mine = b.split(p)[q]
        assert same(mine, pr.p), f"instance {q} (n={pb.n}) differs"
        assert np.array_equal(b.split(pf)[q], pr.pflag)


def test_batch_graph_equals_plain_steps():
    probs = riemann.draw(4, seed=9, nmin=30, nmax=60)
    tfs = [0.4] * 4
    b1 = make_batch(probs, 3, "MC", "HLL", tfs)
    b2 = make_batch(probs, 3, "MC", "HLL", tfs)
    try:
        b1.step_ch(20)
        b2.step_graph(20)
        assert same(b1.download_state()[0], b2.download_state()[0])
        assert np.array_equal(b1.status()[0], b2.status()[0])
    finally:
        b1.close()
        b2.close()


def test_single_context_with_outflow_copy_matches_oracle():
    pb = riemann.draw(1, seed=4, nmin=50, nmax=50)[0]
    ng = 3
    g = HarmGPU(pb.n, 1, 1, ng, (pb.dx, 1.0, 1.0), lim="MC", flux="HLL",
                bc=("OUTFLOW_COPY", "OUTFLOW_COPY", "OUTFLOW", "OUTFLOW", "OUTFLOW", "OUTFLOW"), gam=pb.gam, cour=0.5,
                tf=0.4)
    try:
        g.upload_geometry(*riemann.minkowski_geometry(pb.n + 2 * ng))
        g.upload_state(riemann.primitives(pb, ng), None, 0.0, 0.0)
        dt0 = g.init_dt()
        g.step_ch(10)
        p, pf, t, dt = g.download_state()
    finally:
        g.close()
    pr = oracle_problem(pb, ng, "MC", "HLL", 0.4, dt0)
    Oracle().step(pr, 10)
    assert same(p, pr.p) and t == pr.t and dt == pr.dt


def test_batch_autotune_keeps_state_and_results():
    probs = riemann.draw(5, seed=21, nmin=40, nmax=90)
    tfs = [0.4, 0.1, 0.4, 0.25, 0.4]
    b1 = make_batch(probs, 3, "MC", "HLL", tfs)
    b2 = make_batch(probs, 3, "MC", "HLL", tfs)
    try:
        before = b2.status()
        tun = b2.autotune()
        after = b2.status()
        for x, y in zip(before, after):
            assert np.array_equal(np.asarray(x), np.asarray(y))
        assert set(tun) >= {"flux", "update", "invert"}
        r1 = b1.run(check_every=5)
        r2 = b2.run(check_every=5)
        assert r1[0] == r2[0] and np.array_equal(r1[2], r2[2])
        assert same(b1.download_state()[0], b2.download_state()[0])
        assert np.array_equal(b1.status()[0], b2.status()[0])
    finally:
        b1.close()
        b2.close()
