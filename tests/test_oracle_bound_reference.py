"""bound_prim of the oracle against the reference's own on drawn states.

The stepped fixtures reach the boundaries only with the torus's own flow.
Here every active zone gets random primitives, with radial velocities of
both signs and Lorentz factors up to ~30 (so the outflow boundaries' inflow
check, fixup.c:2271, and its gamma limit, fixup.c:1859, both act at each x1
edge) and transverse velocities and fields of both signs (the polar axis
reflection flips u2 and B2, bounds.fishmon.c:213-324; the 3D case adds the
periodic x3 copy).  The reference build runs its bound_prim on the same
state through oracle/ref_harness.c --boundprim; the ghosts must agree bit
for bit."""
import os
import tempfile

import numpy as np
import pytest

from oracle.pyoracle import CENT, LIBDIR, Oracle
from tests.fixtures import reference_on_state, reference_problem


def draw_boundary_state(pr, seed):
    rng = np.random.default_rng(seed)
    nt = pr.nt
    g = pr.g
    act = tuple(slice(gg, gg + n) for gg, n in zip(g, pr.n))
    shape = tuple(pr.n)
    # the metric does not depend on x3
    g11 = pr.gcov[:nt[0], :nt[1], CENT, 1, 1][act[:2]][:, :, None]
    g22 = pr.gcov[:nt[0], :nt[1], CENT, 2, 2][act[:2]][:, :, None]
    q = 10.0 ** rng.uniform(-2.0, 1.5, size=shape)
    p = pr.p
    p[act + (0,)] = 10.0 ** rng.uniform(-3.0, 0.0, size=shape)
    p[act + (1,)] = p[act + (0,)] * 10.0 ** rng.uniform(-3.0, 0.0, size=shape)
    p[act + (2,)] = rng.choice([-1.0, 1.0], size=shape) * q / np.sqrt(g11)
    p[act + (3,)] = rng.uniform(-1.0, 1.0, size=shape) / np.sqrt(g22)
    p[act + (4,)] = rng.uniform(-0.5, 0.5, size=shape)
    for v in (5, 6, 7):
        p[act + (v,)] = rng.uniform(-1e-2, 1e-2, size=shape)
    pr.p = np.ascontiguousarray(p)


@pytest.mark.parametrize("build", ["harm_ref_16x16x1_MC_HLL", "harm_ref_12x12x6_MC_LAXF"])
def test_oracle_bound_prim_matches_reference_on_drawn_states(build):
    exe = os.path.join(LIBDIR, build)
    if not os.path.exists(exe):
        pytest.skip("reference binary not built (__graft_entry__.build builds it where the reference tree is)")
    orc = Oracle()
    with tempfile.TemporaryDirectory() as tmp:
        changed = 0
        for seed in range(4):
            pr = reference_problem(exe, tmp)
            draw_boundary_state(pr, 5000 + seed)
            p_ref = reference_on_state(exe, tmp, "--boundprim", pr)
            q = pr.copy()
            assert orc.bound_prim(q) == 0
            same = (q.p == p_ref) | (np.isnan(q.p) & np.isnan(p_ref))
            assert same.all(), f"seed {seed}: {np.count_nonzero(~same)} values differ"
            changed += int(np.count_nonzero(q.p != pr.p))
        assert changed > 0
