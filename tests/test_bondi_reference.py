"""The serving loop's Bondi solutions (harm_finalwham_b200/bondi.py, which
solves the transonic Michel flow directly) against the reference's own
tabulated solutions, bondigrid{32,64,128,256}.dat (readin_bondi_solution,
init.c:350-460; Schwarzschild, Gamma = 4/3, sonic point r = 8M), kept as
tests/golden/bondigrid.npz.  The temperature p/rho and the radial
4-velocity do not depend on the polytrope's normalisation; both agree with
every row of every table, ghost rows included, to 1e-12."""
import os

import numpy as np
import pytest

from harm_finalwham_b200 import bondi

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "bondigrid.npz")


@pytest.mark.parametrize("n", [32, 64, 128, 256])
def test_bondi_profile_matches_reference_table(n):
    d = np.load(GOLDEN)
    gam, rcr, uu1cr, rhocr, nx, rin, rout = d[f"n{n}_head"]
    rows = d[f"n{n}_rows"]
    i, x, r, rho_t, uu1_t, u_t = rows.T
    assert int(nx) == n and gam == pytest.approx(4.0 / 3.0) and rcr == 8.0
    rho, ur = bondi.solution(r, gam, rcr)
    th_t = (gam - 1.0) * u_t / rho_t
    th = rho ** (gam - 1.0)                    # p = K rho^Gamma with K = 1
    assert np.max(np.abs(th / th_t - 1.0)) < 1e-12
    assert np.max(np.abs(ur / (-uu1_t) - 1.0)) < 1e-12
    # the table's own sonic conditions
    assert uu1cr == -0.25 and abs(rcr * rcr * rhocr * 0.25 - rho_t[0] * (-uu1_t[0]) * r[0] ** 2) < 1e-12
