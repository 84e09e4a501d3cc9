"""fixup_checksolution's visiting order, on the CPU.

The reference visits its candidates in (i, j, k) order and each visit may
flag the zone for its later neighbours; the device resolves this with the
formulation of tests/checksol_model.py (independent candidates final at
once, a fixpoint over the rest).  Here: the sequential restatement equals
the oracle's checksolution on states drawn to be rich in candidates, and
the device formulation equals the sequential loop on many random grids (1D,
2D, 3D; dense candidates, long chains, every flag code, zero and negative u,
NaN gamma), whatever order the candidates are listed and swept in."""
import numpy as np
import pytest

from oracle.pyoracle import Oracle
from tests.checksol_model import FAIL_CODES, REF_FAIL_CODES, craft, device_scheme, sequential
from tests.fixtures import load


@pytest.mark.parametrize("name", ["torus2d_16x16_mc_hll", "torus3d_12x12x6_mc_hll"])
def test_sequential_restatement_matches_oracle(name):
    orc = Oracle()
    for seed in range(4):
        pr, _ = load(name)
        craft(pr, 2000 + seed, REF_FAIL_CODES)
        flags0 = pr.pflag.copy()
        err, gam = orc.checksolution(pr)
        assert err == 0
        want = sequential(flags0, gam, pr.p[..., 1], pr.n, pr.g, pr.s)
        assert np.array_equal(pr.pflag, want)
        assert np.count_nonzero(pr.pflag != flags0) > 0


def _random_grid(rng, n, dense):
    s = tuple(1 if x > 1 else 0 for x in n)
    g = tuple(2 if x > 1 else 0 for x in n)
    nt = tuple(x + 2 * y for x, y in zip(n, g))
    gam_choices = [1.0, 1.5, 1.99, 2.0, 2.5, 3.9, 4.0, 4.1, 8.0, 8.1, 16.5, np.nan]
    p = [.02, .04, .04, .1, .15, .1, .1, .1, .1, .1, .1, .05] if dense else \
        [.2, .2, .1, .1, .1, .05, .05, .05, .05, .05, .04, .01]
    gam = rng.choice(gam_choices, size=nt, p=p)
    uu = 10.0 ** rng.uniform(-3.0, 1.0, size=nt)
    uu[rng.random(nt) < 0.03] = 0.0
    uu[rng.random(nt) < 0.03] *= -1.0
    fail = rng.random(nt) < rng.uniform(0.05, 0.5)
    flags = np.where(fail, rng.choice(FAIL_CODES, size=nt), 0).astype(np.int32)
    return flags, gam, uu, g, s


@pytest.mark.parametrize("n", [(400, 1, 1), (20, 20, 1), (10, 9, 4)])
def test_device_formulation_equals_sequential_loop(n):
    rng = np.random.default_rng(7)
    ndep = nchanged = norder = 0
    for trial in range(40):
        flags, gam, uu, g, s = _random_grid(rng, n, dense=trial % 2 == 0)
        want = sequential(flags, gam, uu, n, g, s)
        for jacobi in (False, True):
            got, m = device_scheme(flags, gam, uu, n, g, s, rng, jacobi=jacobi)
            assert np.array_equal(got, want), f"trial {trial} jacobi {jacobi}"
            ndep += m
        nchanged += int(np.count_nonzero(want != flags))
        norder += int(np.count_nonzero(want != sequential(flags, gam, uu, n, g, s, order_free=True)))
    # the grids exercise the votes, the visiting order and the dependent
    # candidates
    assert nchanged > 0
    if n[1] > 1:
        assert norder > 0
    if n[1] > 1:
        assert ndep > 0


def test_device_formulation_on_a_long_chain():
    # a diagonal of candidates each voted failed by its neighbours, so every
    # decision waits for the one before it
    n = (40, 40, 1)
    g, s = (2, 2, 0), (1, 1, 0)
    nt = (44, 44, 1)
    gam = np.full(nt, 1.0)
    uu = np.ones(nt)
    for d in range(40):
        gam[d + 2, d + 2, 0] = 2.5
        gam[d + 2, min(d + 3, 43), 0] = 8.0
    flags = np.zeros(nt, dtype=np.int32)
    rng = np.random.default_rng(3)
    want = sequential(flags, gam, uu, n, g, s)
    assert np.count_nonzero(want != sequential(flags, gam, uu, n, g, s, order_free=True)) > 30
    for jacobi in (False, True):
        got, m = device_scheme(flags, gam, uu, n, g, s, rng, jacobi=jacobi)
        assert m > 30
        assert np.array_equal(got, want)


@pytest.mark.parametrize("build,finalstep", [("harm_ref_16x16x1_MC_HLL", 1), ("harm_ref_16x16x1_MC_HLL", 0),
                                             ("harm_ref_12x12x6_MC_LAXF", 1)])
def test_oracle_post_fixup_matches_reference_on_crafted_states(build, finalstep):
    # the reference's own post_fixup (fixup.c:37-96, through the harness's
    # --postfixup) on the candidate-rich states the GPU test uses: pins the
    # oracle there, beyond what the stepped fixtures reach
    import os
    import tempfile

    from oracle.pyoracle import LIBDIR
    from tests.fixtures import reference_on_state, reference_problem
    exe = os.path.join(LIBDIR, build)
    if not os.path.exists(exe):
        pytest.skip("reference binary not built (__graft_entry__.build builds it where the reference tree is)")
    orc = Oracle()
    with tempfile.TemporaryDirectory() as tmp:
        for seed in range(3):
            pr = reference_problem(exe, tmp)
            craft(pr, 4000 + seed, REF_FAIL_CODES)
            p_out, f_out = reference_on_state(exe, tmp, "--postfixup", pr, (finalstep,), with_flags=True)
            q = pr.copy()
            assert orc.post_fixup(q, finalstep) == 0
            assert np.array_equal(q.pflag, f_out), f"seed {seed}: {np.count_nonzero(q.pflag != f_out)} flags differ"
            same = (q.p == p_out) | (np.isnan(q.p) & np.isnan(p_out))
            assert same.all(), f"seed {seed}: {np.count_nonzero(~same)} primitive values differ"
            assert np.count_nonzero(f_out != pr.pflag) > 0
