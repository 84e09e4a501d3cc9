"""post_fixup (fixup.c:37-96) on crafted states, GPU against the oracle.

fixup_checksolution (fixup.c:460-560) visits its candidates (active zones with
gamma >= 2) in loop order and each visit may flag the zone, which later
visits of its neighbours read; the device resolves that order dependence with
a fixpoint over the candidates whose earlier neighbours can change their
vote.  The torus steps of the other tests produce few candidates, so these
states are drawn to make many: Lorentz factors from 1.1 to 9 and internal
energies over four decades zone by zone (every vote threshold is crossed),
and failure codes on a quarter of the zones.  A plain-Python restatement of
the loop (tests/checksol_model.py) shows that the sequential result differs
from an order-free one on these states, i.e. the chains are exercised; the
device's post_fixup (checksolution, then fixup_utoprim's neighbour averages)
must equal the oracle's bit for bit."""
import numpy as np
import pytest

from harm_finalwham_b200.gpu import HarmGPU
from oracle.pyoracle import Oracle
from tests.checksol_model import FAIL_CODES, REF_FAIL_CODES, craft, sequential
from tests.fixtures import load

pytestmark = pytest.mark.gpu

CASES = [("torus2d_16x16_mc_hll", 1), ("torus2d_16x16_mc_hll", 0), ("torus3d_12x12x6_mc_hll", 1)]


@pytest.mark.parametrize("codes", ["reference", "with_fixed"])
@pytest.mark.parametrize("name,finalstep", CASES)
def test_post_fixup_matches_oracle_on_crafted_states(name, finalstep, codes):
    # "reference": the failure codes the reference's fixup_utoprim accepts,
    # where the oracle's post_fixup is pinned to the reference's own
    # (tests/test_checksol_order.py); "with_fixed" adds -1
    orc = Oracle()
    order_dependent = 0
    for seed in range(6):
        pr, _ = load(name)
        craft(pr, 1000 + seed, REF_FAIL_CODES if codes == "reference" else FAIL_CODES)
        # the sequential loop against an order-free pass (every neighbour's
        # original flag): where they differ, the visiting order matters
        _, gam = orc.checksolution(pr.copy())
        seq = sequential(pr.pflag, gam, pr.p[..., 1], pr.n, pr.g, pr.s)
        free = sequential(pr.pflag, gam, pr.p[..., 1], pr.n, pr.g, pr.s, order_free=True)
        order_dependent += int(np.count_nonzero(seq != free))
        with HarmGPU.from_problem(pr) as gpu:
            gpu.upload_state(pr.p, pr.pflag, pr.t, pr.dt)
            st = gpu.post_fixup(finalstep)
            p, pf, _, _ = gpu.download_state()
        q = pr.copy()
        assert orc.post_fixup(q, finalstep) == 0
        assert st.err == 0
        assert np.array_equal(pf, q.pflag), f"seed {seed}: {np.count_nonzero(pf != q.pflag)} flags differ"
        same = (p == q.p) | (np.isnan(p) & np.isnan(q.p))
        assert same.all(), f"seed {seed}: {np.count_nonzero(~same)} primitive values differ"
    # the drawn states do make checksolution's visiting order matter
    assert order_dependent > 0


def test_post_fixup_finite_volume_corrects_unew():
    # with the finite-volume scheme a final step's fixups carry every
    # primitive change into the evolved conserved state (diag_fixup,
    # fixup.c:240-250); unew is compared on the active zones it is defined on
    orc = Oracle()
    for seed in range(3):
        pr, _ = load("torus2d_16x16_mc_hll_fv")
        craft(pr, 3000 + seed)
        pr.u = orc.pi2u(pr)
        with HarmGPU.from_problem(pr) as gpu:
            gpu.upload_state(pr.p, pr.pflag, pr.t, pr.dt)
            gpu.upload_conserved(pr.u)
            st = gpu.post_fixup(1)
            p, pf, _, _ = gpu.download_state()
            u = gpu.active(gpu.download_conserved())
        q = pr.copy()
        assert orc.post_fixup(q, 1) == 0
        assert st.err == 0 and st.nfixed > 0
        assert np.array_equal(pf, q.pflag)
        assert ((p == q.p) | (np.isnan(p) & np.isnan(q.p))).all()
        uq = q.active(q.u)
        assert ((u == uq) | (np.isnan(u) & np.isnan(uq))).all()
        assert not np.array_equal(uq, pr.active(pr.u))
