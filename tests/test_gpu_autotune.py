"""The autotuner (hgpu_autotune) picks resident-block variants of the heavy
FP64 kernels on the context's own state; the state is left as it was and
the results stay bit-identical to the reference whatever it picks."""
import numpy as np
import pytest

from harm_finalwham_b200.gpu import HarmGPU
from tests.fixtures import load, same

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["torus3d_12x12x6_weno5_laxf", "torus2d_16x16_para_hll_rk4_jon_fv"])
def test_autotune_keeps_state_and_results(name):
    pr, ref = load(name)
    with HarmGPU.from_problem(pr) as g:
        p0, pf0, t0, dt0 = g.download_state()
        tu = g.autotune()
        p1, pf1, t1, dt1 = g.download_state()
        assert same(p0, p1) and np.array_equal(pf0, pf1) and t0 == t1 and dt0 == dt1
        for fam in ("flux", "update", "invert"):
            assert tu[fam]["minb"] in [int(c) for c in tu[fam]["ms"]]
            assert all(v > 0 for v in tu[fam]["ms"].values())
        s = sorted(ref)[-1]
        g.step_ch(s)
        p, pf, t, dt = g.download_state()
    r = ref[s]
    assert same(p, r["p"]) and np.array_equal(pf, r["pflag"]) and t == r["t"] and dt == r["dt"]


def test_set_tuning_applies_a_known_choice():
    pr, ref = load("torus2d_16x16_mc_hll")
    with HarmGPU.from_problem(pr) as g:
        g.set_tuning({"flux": 3, "weno": 3, "update": 3, "invert": 2})
        s = sorted(ref)[-1]
        g.step_ch(s)
        p, pf, t, dt = g.download_state()
        with pytest.raises(Exception):
            g.set_tuning({"flux": 7, "weno": 8, "update": 1, "invert": 1})
    r = ref[s]
    assert same(p, r["p"]) and np.array_equal(pf, r["pflag"]) and t == r["t"] and dt == r["dt"]
