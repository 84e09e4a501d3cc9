"""Mixed precision (HGPU_PREC_MIXED) against the FP64 path, which is
bit-identical to the reference.  With WENO5 the reconstruction runs in FP32
(on differences from each cell's own value, with the FP64 epsilons) and the
Riemann fluxes in FP64; with MC/PARA the Riemann kernel, which reconstructs
too, runs in FP32.  Flux-CT, the conserved update and the inversion stay
FP64.  The mixed path is not bit-compatible by design; these tests state and
bound its error."""
import numpy as np
import pytest

from harm_finalwham_b200 import torus
from harm_finalwham_b200.gpu import HarmGPU
from tests.divb import divb_max

pytestmark = pytest.mark.gpu


def run(dom, precision, nsteps):
    g = HarmGPU(*dom.n, dom.ng, dom.dx, lim=dom.lim, flux=dom.flux, precision=precision, gam=dom.gam, cour=dom.cour)
    try:
        g.upload_geometry(dom.gcov, dom.gcon, dom.gcovpert, dom.gdet, dom.conn, dom.floors)
        g.upload_state(dom.p, dom.pflag, 0.0, 0.0)
        g.init_dt()
        st = g.step_ch(nsteps)
        p, pf, t, dt = g.download_state()
        return g.active(p), g.active(pf), t, st, divb_max(p, dom.gdet, dom.ng, dom.dx, dom.n)
    finally:
        g.close()


def rel_l1(a, b):
    return np.abs(a - b).sum() / np.abs(b).sum()


@pytest.mark.parametrize("lim", ["WENO5", "MC"])
def test_mixed_tracks_fp64(lim):
    dom = torus.fm_torus(32, 32, 16, ng=6 if lim == "WENO5" else 3, lim=lim, flux="HLL", seed=5)
    p64, f64, t64, s64, d64 = run(dom, "fp64", 10)
    p32, f32, t32, s32, d32 = run(dom, "mixed", 10)
    assert s64.err == 0 and s32.err == 0
    # flux-CT runs in FP64 in both modes: div B stays at round-off
    assert d64 < 1e-12 and d32 < 1e-12
    assert np.all(np.isfinite(p32))
    errs = {name: rel_l1(p32[..., q], p64[..., q]) for name, q in (("rho", 0), ("u", 1), ("B1", 5), ("B2", 6))}
    print(lim, "mixed vs fp64 after 10 steps, relative L1:", {k: f"{v:.2e}" for k, v in errs.items()})
    assert errs["rho"] < 1e-5 and errs["u"] < 1e-4
    assert abs(t32 - t64) < 1e-5 * t64
    # failure maps: the same zones fail in both, up to a handful
    assert abs(int(np.count_nonzero(f32)) - int(np.count_nonzero(f64))) <= max(4, np.count_nonzero(f64) // 20)


def test_mixed_finite_volume_default_scheme():
    # the FM torus problem file's own scheme (PARA, RK4, Jon, finite volume
    # over all 11 MAXBND ghosts) in mixed precision against FP64
    from tests.fixtures import load
    pr, _ = load("torus2d_16x16_para_hll_rk4_jon_fv")
    out = {}
    for prec in ("fp64", "mixed"):
        with HarmGPU.from_problem(pr, precision=prec) as g:
            st = g.step_ch(20)
            p, pf, t, dt = g.download_state()
            assert st.err == 0
            out[prec] = (g.active(p), t)
    p64, t64 = out["fp64"]
    p32, t32 = out["mixed"]
    assert np.all(np.isfinite(p32))
    assert rel_l1(p32[..., 0], p64[..., 0]) < 1e-4
    assert abs(t32 - t64) < 1e-4 * t64


def test_mixed_weno5_within_1e5_of_fp64_at_scale():
    # the precision-at-scale torus 256x128x128 (WENO5 + HLL + flux-CT), 200
    # steps: the benchmark's bound is relative L1(rho) <= 1e-5 against FP64
    dom = torus.fm_torus(256, 128, 128, ng=6, lim="WENO5", flux="HLL", seed=7)
    p64, f64, t64, s64, d64 = run(dom, "fp64", 200)
    p32, f32, t32, s32, d32 = run(dom, "mixed", 200)
    assert s64.err == 0 and s32.err == 0
    errs = {name: rel_l1(p32[..., q], p64[..., q]) for name, q in (("rho", 0), ("u", 1), ("B1", 5), ("B2", 6),
                                                                     ("B3", 7))}
    print("WENO5 mixed vs fp64 after 200 steps at 256x128x128, relative L1:",
          {k: f"{v:.2e}" for k, v in errs.items()})
    assert all(v <= 1e-5 for v in errs.values()), errs
    assert d32 < 1e-12
