"""FP64 GPU path vs the reference: bit-identical primitives, pflag maps, dt.

The golden fixtures hold the reference build's own outputs (tests/golden);
larger cases compare against the CPU oracle, which test_oracle_golden pins to
the reference.  Comparisons are exact (==), sign of zero aside."""
import numpy as np
import pytest

from harm_finalwham_b200.gpu import HarmGPU, utoprim_batch
from oracle.pyoracle import Oracle
from tests.fixtures import CASES, load, same

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", CASES)
def test_step_ch_bit_identical_to_reference(name):
    pr, ref = load(name)
    with HarmGPU.from_problem(pr) as g:
        done = 0
        for s in sorted(ref):
            st = g.step_ch(s - done)
            done = s
            p, pf, t, dt = g.download_state()
            r = ref[s]
            nbad = int(np.count_nonzero(~((p == r["p"]) | (np.isnan(p) & np.isnan(r["p"])))))
            assert nbad == 0, f"{nbad} primitive values differ after step {s}"
            assert np.array_equal(pf, r["pflag"]), f"pflag map differs after step {s}"
            assert t == r["t"] and dt == r["dt"]
            assert st.err == 0
            # the conserved state unew, active zones: evolved by the
            # finite-volume scheme, the last stage's update otherwise
            u = g.download_conserved()
            assert same(g.active(u), g.active(r["unew"])), f"conserved state differs after step {s}"


@pytest.mark.parametrize("name", CASES)
def test_failure_floor_counters_match_reference(name):
    # failfloorcount (fixup.c:206) per zone and category: the reference's
    # counts after each dumped step less its counts at init (init's own
    # fixup counts too; the device starts from zero at upload)
    pr, ref = load(name)
    with HarmGPU.from_problem(pr) as g:
        done = 0
        for s in sorted(ref):
            g.step_ch(s - done)
            done = s
            c = g.active(g.download_failfloorcount())
            want = g.active(ref[s]["ffc"]) - g.active(pr.ffc_init)
            bad = np.argwhere(c != want)
            assert bad.size == 0, (f"{len(bad)} counters differ after step {s}, first (i, j, k, category) "
                                   f"{tuple(bad[0])}: {c[tuple(bad[0])]} vs {want[tuple(bad[0])]}")


@pytest.mark.parametrize("name", CASES)
def test_newton_iterations_match_reference(name):
    pr, ref = load(name)
    with HarmGPU.from_problem(pr) as g:
        done = 0
        for s in sorted(ref):
            if s - done > 1:
                g.step_ch(s - done - 1)
            st = g.step_ch(1)
            done = s
            assert st.newton_iters == ref[s]["nstroke"]


def test_stage_by_stage_matches_oracle():
    pr, _ = load("torus3d_12x12x6_mc_laxf")
    orc = Oracle()
    q = pr.copy()
    orc.step(q, 9)  # a state with failures in the next step
    with HarmGPU.from_problem(q) as g:
        ndt0, st0 = g.advance_stage(0)
        ndt1, st1 = g.advance_stage(1)
        p, pf, _, _ = g.download_state()
    orc.step(q, 1)
    assert same(g.active(p), q.active(q.p))
    assert np.array_equal(g.active(pf), q.active(q.pflag))
    assert st1.nfail > 0 and st1.nfixed > 0


def test_long_run_2d_matches_oracle():
    pr, _ = load("torus2d_16x16_mc_hll")
    orc = Oracle()
    q = pr.copy()
    with HarmGPU.from_problem(pr) as g:
        g.step_ch(100)
        p, pf, t, dt = g.download_state()
    orc.step(q, 100)
    assert same(p, q.p)
    assert np.array_equal(pf, q.pflag)
    assert t == q.t and dt == q.dt


def test_utoprim_batch_matches_oracle():
    pr, ref = load("torus3d_12x12x6_mc_laxf")
    rng = np.random.default_rng(7)
    # CENT metrics of the fixture, primitives of the reference state after 10 steps
    g0 = pr.g
    p = ref[10]["p"][g0[0]:g0[0] + pr.n[0], g0[1]:g0[1] + pr.n[1], g0[2]:g0[2] + pr.n[2]].reshape(-1, 8)
    ii, jj = np.meshgrid(np.arange(pr.n[0]), np.arange(pr.n[1]), indexing="ij")
    gi = (ii + g0[0]).ravel().repeat(pr.n[2])
    gj = (jj + g0[1]).ravel().repeat(pr.n[2])
    gcov = pr.gcov[gi, gj, 7].reshape(-1, 16)
    gcon = pr.gcon[gi, gj, 7].reshape(-1, 16)
    gdet = pr.gdet[gi, gj, 7].copy()
    # conserved from a GPU/oracle-independent source: perturb the state and use the
    # oracle's own step outputs is not needed; any U exercises the inversion
    U = p * gdet[:, None] * (1.0 + 0.05 * rng.standard_normal(p.shape))
    U[:, 1] = -np.abs(U[:, 1]) - U[:, 0]  # T^t_t < 0 with rest mass removed
    guess = p * (1.0 + 0.01 * rng.standard_normal(p.shape))
    a, fa, ia = utoprim_batch(U, gcov, gcon, gdet, guess, pr.gam, pr.gammafail)
    b, fb, ib = Oracle().utoprim(U, gcov, gcon, gdet, guess, pr.gam, pr.gammafail)
    assert np.array_equal(fa, fb)
    assert same(a, b)
    assert ia == ib


@pytest.mark.parametrize("inv", ["2DFINAL", "JON"])
def test_utoprim_zones_match_reference(inv):
    # zone-level fixture: the reference's Utoprimgen on seeded zones with
    # Lorentz factors up to 2000, b^2/rho up to 1e3 and perturbed energies
    from tests.fixtures import load_zones
    z = load_zones()
    pr, pf, it = utoprim_batch(z["U"], z["gcov"], z["gcon"], z["gdet"], z["guess"], z["gam"], z["gammafail"],
                               version=inv)
    assert np.array_equal(pf, z[f"pflag_{inv}"])
    assert same(pr, z[f"pr_{inv}"])
    assert it == int(z[f"iters_{inv}"].sum())


@pytest.mark.parametrize("name", [c for c in CASES if c.startswith("torus")])
def test_bsq_flags_match_reference(name):
    # pre_fixup's b^2/rho and b^2/u flags (pflag slots FLAGBSQORHO and
    # FLAGBSQOU, get_bsqflags fixup.c:1751) as the reference leaves them
    pr, ref = load(name)
    with HarmGPU.from_problem(pr) as g:
        done = 0
        for s in sorted(ref):
            g.step_ch(s - done)
            done = s
            bsq = ref[s]["bsq"]
            assert bsq is not None, "fixture lacks the b^2 flags"
            got = g.download_bsqflags()
            assert np.array_equal(got, bsq), f"{int(np.count_nonzero(got != bsq))} flags differ after step {s}"


@pytest.mark.parametrize("name", ["torus2d_16x16_mc_hll_beta1e-4", "torus3d_12x12x6_weno5_hll",
                                  "torus2d_16x16_para_hll_rk4_jon", "bondi2d_16x16_mc_hll"])
def test_active_zone_transfers_keep_the_run_bit_identical(name):
    # hgpu_upload_active / hgpu_download_active every step (the host holds
    # only active zones; bound_prim on the device rebuilds the ghosts) give
    # the run that keeps the state on the device
    pr, ref = load(name)
    with HarmGPU.from_problem(pr) as g, HarmGPU.from_problem(pr) as h:
        steps = max(ref)
        # both start from the device's own ghosts (the Bondi-integral ones
        # differ from the reference's in pow's last bits)
        g.bound_prim(0)
        g.step_ch(steps)
        for _ in range(steps):
            p, f, t, dt = h.download_active()
            h.upload_active(p, t, dt)
            h.step_ch(1)
        pg, fg, tg, dtg = g.download_state()
        pa, fa, ta, dta = h.download_active()
        assert same(g.active(pg), pa) and np.array_equal(g.active(fg), fa) and tg == ta and dtg == dta
        ph, fh, _, _ = h.download_state()
        assert same(pg, ph)
