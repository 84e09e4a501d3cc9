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


@pytest.mark.parametrize("name", ["torus2d_16x16_mc_hll", "torus3d_12x12x6_weno5_hll", "torus2d_16x16_mc_hll_beta1e-4",
                                  "torus2d_16x16_para_hll_rk4_jon_fv"])
def test_diagnostics_match_reference_ener_out(name):
    # the reference's own ener.out (dump_ener.c:287-295, written by its
    # dump_ener through the harness at init and after each dumped step):
    # t, realnstep, the conserved integrals U_tot (constotal dump_ener.c:596,
    # U with gdet times dx1 dx2 dx3 over the active zones; unew for the
    # finite-volume scheme), ..., divbmax, divbavg (divbmaxavg :482).  The
    # file prints 15 significant digits and sums in loop order, the device
    # in a fixed tree order: integrals agree to 1e-13 of the mass integral's
    # scale, the div B maximum to the print precision.
    pr, ref = load(name)
    assert pr.ener_init is not None, "fixture lacks the reference's ener.out"
    npr = 8
    ncol = 2 + npr + 2 * 6 * npr + 2 * npr

    def check(dg, line, step):
        assert line[0] == pytest.approx(dg["t"], rel=1e-14, abs=1e-300)
        scale = abs(line[2])
        for q in range(npr):
            assert dg["integral"][q] == pytest.approx(line[2 + q], rel=1e-13, abs=1e-13 * scale), \
                f"step {step}: integral {q}: {dg['integral'][q]!r} vs ener.out {line[2 + q]!r}"
        assert dg["divb_max"] == pytest.approx(line[ncol], rel=1e-13, abs=1e-300)
        assert dg["divb_avg"] == pytest.approx(line[ncol + 1], rel=1e-12, abs=1e-300)

    with HarmGPU.from_problem(pr) as g:
        check(g.diagnostics(), pr.ener_init, 0)
        done = 0
        for s in sorted(ref):
            g.step_ch(s - done)
            done = s
            check(g.diagnostics(), ref[s]["ener"], s)
