"""The reference's restart dump (restart_write, restart.c:206-245), as its
own build writes it: the fixtures' rdump is a header line (write_restart_header,
restart.c:640-800) and then, for every active zone with k outermost and i
fastest (DUMPGENLOOP, global.h:1411-1432), p[0..7] and unew[0..7] each as
"%21.15g " (myfwrite's text branch, mpi_fileio.c:2134-2143) and a newline.
This pins the layout hgpu_write_rdump writes against the reference's own
file, on the CPU."""
import os
import subprocess
import tempfile

import pytest

from oracle.pyoracle import LIBDIR
from tests.fixtures import load

RDUMP_CASES = ["torus2d_16x16_mc_hll", "torus2d_16x16_mc_hll_beta1e-4", "torus2d_16x16_para_hll_rk4_jon_fv",
               "torus3d_12x12x6_weno5_hll"]


def rdump_body(pr, p, unew):
    """The body the reference writes for active-zone arrays p and unew."""
    act = pr.active
    p, u = act(p), act(unew)
    n1, n2, n3 = pr.n
    out = []
    for k in range(n3):
        for j in range(n2):
            for i in range(n1):
                out.append("".join("%21.15g " % v for v in p[i, j, k]) +
                           "".join("%21.15g " % v for v in u[i, j, k]) + "\n")
    return "".join(out).encode()


@pytest.mark.parametrize("name", RDUMP_CASES)
def test_reference_rdump_body_is_p_then_unew_in_dump_order(name):
    pr, ref = load(name)
    assert pr.rdump is not None
    header, body = pr.rdump.split(b"\n", 1)
    r = ref[max(ref)]
    assert body == rdump_body(pr, r["p"], r["unew"])
    # the header starts with the grid size (restart.c:788-790: totalsize[1..3])
    assert [int(v) for v in header.split()[:3]] == list(pr.n)


def test_reference_rdump_is_reproducible():
    # the header holds no uninitialised or time-dependent field in a run
    # without dump_ener: the same run writes the same bytes
    exe = os.path.join(LIBDIR, "harm_ref_16x16x1_MC_HLL")
    if not os.path.exists(exe):
        pytest.skip("reference build missing (__graft_entry__.build() makes it)")
    pr, ref = load("torus2d_16x16_mc_hll")
    with tempfile.TemporaryDirectory() as tmp:
        subprocess.run([exe, "--rdump", "-", str(max(ref))], cwd=tmp, check=True, capture_output=True)
        with open(os.path.join(tmp, "dumps", "rdump-0"), "rb") as f:
            assert f.read() == pr.rdump
