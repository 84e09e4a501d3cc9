"""The seeded Riemann-problem generator and the oracle on it (CPU)."""
import numpy as np

from harm_finalwham_b200 import riemann
from oracle.pyoracle import BC_OUTFLOW, BC_OUTFLOW_COPY, Oracle, Problem


def test_draw_distributions():
    probs = riemann.draw(200, seed=1)
    ns = np.array([p.n for p in probs])
    assert ns.min() >= 200 and ns.max() <= 2000
    for p in probs:
        for s in (p.left, p.right):
            assert 0.1 <= s[0] <= 10 and 0.01 <= s[1] <= 100
            assert np.sqrt(np.sum(s[2:5] ** 2)) <= 0.95 + 1e-12
            assert -5 <= s[6] <= 5 and -5 <= s[7] <= 5
        assert p.left[5] == p.right[5] and p.gam in (4.0 / 3.0, 5.0 / 3.0)
    assert riemann.draw(3, seed=5)[2].n == riemann.draw(3, seed=5)[2].n


def test_primitives_layout():
    pb = riemann.draw(1, seed=2, nmin=20, nmax=20)[0]
    p = riemann.primitives(pb, 3)
    assert p.shape == (26, 1, 1, 8)
    assert np.all(p[:3] == p[3]) and np.all(p[-3:] == p[-4])
    assert p[3, 0, 0, 0] == pb.left[0] and p[-4, 0, 0, 0] == pb.right[0]


def test_oracle_runs_a_riemann_problem_to_the_end():
    pb = riemann.draw(1, seed=7, nmin=60, nmax=60)[0]
    ng = 3
    pr = Problem(pb.n, 1, 1, ng, (pb.dx, 1.0, 1.0), gam=pb.gam, cour=0.5, lim="MC", flux="HLL",
                 bc=(BC_OUTFLOW_COPY, BC_OUTFLOW_COPY) + (BC_OUTFLOW,) * 4, tf=0.4)
    for k, a in zip(("gcov", "gcon", "gcovpert", "gdet", "conn", "floors"), riemann.minkowski_geometry(pb.n + 2 * ng)):
        getattr(pr, k)[...] = a
    pr.p[...] = riemann.primitives(pb, ng)
    pr.dt = 0.25 * pb.dx
    orc = Oracle()
    n = 0
    while pr.t < 0.4 and n < 1000:
        st = orc.step(pr, 1)
        n += 1
    assert pr.t == 0.4 and st.err == 0
    assert 0.6 * pb.n < n < 1.2 * pb.n
    assert np.all(np.isfinite(pr.p))
