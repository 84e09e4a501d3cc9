"""The CPU restatement of the Bondi-integral x1 boundaries (oracle/bondi_bc.py)
reproduces, bit for bit, the ghost zones the reference build writes for its
Bondi flow (the generic init.c's TESTNUMBER 153 with bounds.c:140-156,
295-308), at init and after 1, 10 and 100 steps; the x2 ghost rows mirror
the x1 ghosts with u~2 and B2 negated (bounds.c:477-489)."""
import numpy as np
import pytest

from oracle import bondi_bc as bb
from tests.fixtures import load

CENT = 7


def ghosts(pr, p):
    """The x1 ghosts of active j from the active edge zones of p."""
    g1, g2 = pr.g[0], pr.g[1]
    n1, n2 = pr.n[0], pr.n[1]
    out = {}
    for side in (0, 1):
        i0 = 0 if side == 0 else n1 - 1
        for j in range(n2):
            z = (i0 + g1, j + g2)
            geo = pr.bcgeom[z]
            C1, C2, K = bb.integrals(p[z + (0,)].tolist(), pr.gcov[z + (CENT,)].tolist(),
                                     pr.gcon[z + (CENT,)].tolist(), geo[1:17].reshape(4, 4).tolist(), geo[0], pr.gam)
            if side == 1:
                C2, K = bb.C2X, bb.KX
            for q in range(1, g1 + 1):
                i = -q if side == 0 else n1 - 1 + q
                zg = (i + g1, j + g2)
                gg = pr.bcgeom[zg]
                out[(i, j)] = bb.generate(C1, C2, K, pr.gam, gg[0], gg[17:33].reshape(4, 4).tolist(),
                                          gg[33:49].reshape(4, 4).tolist(), pr.gcon[zg + (CENT,)].tolist())
    return out


@pytest.mark.parametrize("step", [0, 1, 10, 100])
def test_bondi_ghosts_restated_bit_for_bit(step):
    pr, ref = load("bondi2d_16x16_mc_hll")
    p = pr.p if step == 0 else ref[step]["p"]
    g1, g2 = pr.g[0], pr.g[1]
    for (i, j), want in ghosts(pr, p).items():
        got = p[i + g1, j + g2, 0]
        assert np.array_equal(np.array(want), got), f"ghost ({i}, {j}) after step {step}: {want} vs {got.tolist()}"
    # x2 ghosts (every i): the mirror row with u~2 and B2 negated
    n2 = pr.n[1]
    for jg in range(1, g2 + 1):
        for jn, js in ((-jg, jg - 1), (n2 - 1 + jg, n2 - jg)):
            a = p[:, jn + g2, 0].copy()
            b = p[:, js + g2, 0].copy()
            b[:, 3] *= -1.
            b[:, 6] *= -1.
            assert np.array_equal(a, b), f"x2 ghost row {jn} after step {step}"
