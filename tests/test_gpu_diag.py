"""Device diagnostics (hgpu_diagnostics) against the same quantities computed
on the host from the downloaded state."""
import numpy as np
import pytest

from harm_finalwham_b200.gpu import HarmGPU
from tests.divb import divb_maxavg
from tests.fixtures import load

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["torus2d_16x16_mc_hll", "torus3d_12x12x6_weno5_laxf"])
def test_diagnostics(name):
    pr, _ = load(name)
    with HarmGPU.from_problem(pr) as g:
        g.step_ch(5)
        dg = g.diagnostics()
        p, pf, t, dt = g.download_state()
        unew = g.download_conserved()
    assert dg["nsteps"] == 5 and dg["t"] == t and dg["dt"] == dt
    mx, av = divb_maxavg(p, pr.gdet, pr.ng, pr.dx, pr.n)
    assert dg["divb_max"] == pytest.approx(mx, rel=1e-12, abs=1e-300)
    assert dg["divb_avg"] == pytest.approx(av, rel=1e-9, abs=1e-300)
    # the corners flux-CT constrains stay at round-off
    mi = divb_maxavg(p, pr.gdet, pr.ng, pr.dx, pr.n, interior=True)
    assert dg["divb_max_interior"] == pytest.approx(mi, rel=1e-12, abs=1e-300)
    assert dg["divb_max_interior"] < 1e-12
    # mass: sum of gdet rho u^t dV over active zones
    a = g.active(p)
    ga = pr.g
    n = pr.n
    gcov = pr.gcov[ga[0]:ga[0] + n[0], ga[1]:ga[1] + n[1], 7][:, :, None]
    gcon = pr.gcon[ga[0]:ga[0] + n[0], ga[1]:ga[1] + n[1], 7][:, :, None]
    gd = pr.gdet[ga[0]:ga[0] + n[0], ga[1]:ga[1] + n[1], 7][:, :, None]
    ut = a[..., 2:5]
    qsq = np.einsum("...i,...ij,...j->...", ut, gcov[..., 1:4, 1:4], ut)
    gamma = np.sqrt(1.0 + qsq)
    alpha = 1.0 / np.sqrt(-gcon[..., 0, 0])
    mass = float(np.sum(gd * a[..., 0] * gamma / alpha) * pr.dx[0] * pr.dx[1] * pr.dx[2])
    assert dg["integral"][0] == pytest.approx(mass, rel=1e-12)
    assert dg["nfail"] == int(np.count_nonzero(g.active(pf) > 0))
    # unew (the conserved state the step produced) inverts to p: its mass integral agrees
    umass = float(np.sum(g.active(unew)[..., 0]) * pr.dx[0] * pr.dx[1] * pr.dx[2])
    assert umass == pytest.approx(mass, rel=1e-3)  # floors and fixups change p after the inversion
