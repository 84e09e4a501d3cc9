"""Restart dumps written from and read into device state (hgpu_write_rdump,
hgpu_read_rdump): the file the device writes after the reference's step
count is byte for byte the one the reference build writes (restart_write,
restart.c:206-245; its header passed through), a binary dump read back
reproduces the state exactly, and a run continued from it equals the
uninterrupted run bit for bit."""
import os
import tempfile

import numpy as np
import pytest

from harm_finalwham_b200.gpu import HarmGPU
from tests.fixtures import load, same
from tests.test_rdump_format import RDUMP_CASES

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", RDUMP_CASES)
def test_rdump_from_device_equals_reference_file(name):
    pr, ref = load(name)
    header = pr.rdump[:pr.rdump.index(b"\n") + 1]
    with HarmGPU.from_problem(pr) as g, tempfile.TemporaryDirectory() as tmp:
        g.step_ch(max(ref))
        path = os.path.join(tmp, "rdump-0")
        g.write_rdump(path, header)
        with open(path, "rb") as f:
            got = f.read()
    assert len(got) == len(pr.rdump)
    if got != pr.rdump:
        bad = next(i for i, (a, b) in enumerate(zip(got, pr.rdump)) if a != b)
        pytest.fail(f"restart dump differs from the reference's at byte {bad}: "
                    f"{got[max(0, bad - 40):bad + 40]!r} vs {pr.rdump[max(0, bad - 40):bad + 40]!r}")


@pytest.mark.parametrize("name", ["torus2d_16x16_mc_hll", "torus2d_16x16_para_hll_rk4_jon_fv"])
def test_binary_rdump_round_trip_and_continuation(name):
    pr, ref = load(name)
    with tempfile.TemporaryDirectory() as tmp:
        a, b = os.path.join(tmp, "a.bin"), os.path.join(tmp, "b.bin")
        with HarmGPU.from_problem(pr) as g, HarmGPU.from_problem(pr) as h:
            g.step_ch(3)
            g.write_rdump(a, b"HDR\n", binary=True)
            _, _, t, dt = g.download_state()
            h.read_rdump(a, t, dt, header_bytes=4, binary=True)
            h.write_rdump(b, b"HDR\n", binary=True)
            with open(a, "rb") as fa, open(b, "rb") as fb:
                assert fa.read() == fb.read()
            # the state read back is the state written: ghosts by bound_prim
            # reproduce the step's own boundary pass
            pg, fg, _, _ = g.download_state()
            ph, fh, _, _ = h.download_state()
            assert same(pg, ph)
            g.step_ch(2)
            h.step_ch(2)
            pg, fg, tg, dtg = g.download_state()
            ph, fh, th, dth = h.download_state()
            assert same(pg, ph) and np.array_equal(fg, fh) and tg == th and dtg == dth
            assert same(g.active(g.download_conserved()), h.active(h.download_conserved()))


def test_text_rdump_reads_fifteen_digits():
    pr, ref = load("torus2d_16x16_mc_hll")
    with tempfile.TemporaryDirectory() as tmp, HarmGPU.from_problem(pr) as g:
        path = os.path.join(tmp, "rdump-0")
        g.step_ch(1)
        p0, _, t, dt = g.download_state()
        g.write_rdump(path)
        g.read_rdump(path, t, dt)
        p1, _, _, _ = g.download_state()
        act = g.active
        want = np.vectorize(lambda v: float("%21.15g" % v))(act(p0))
        assert same(act(p1), want)


def test_rdump_errors_are_reported():
    pr, ref = load("torus2d_16x16_mc_hll")
    with tempfile.TemporaryDirectory() as tmp, HarmGPU.from_problem(pr) as g:
        short = os.path.join(tmp, "short")
        with open(short, "wb") as f:
            f.write(b"1 2 3\n")
        with pytest.raises(RuntimeError, match="short or malformed"):
            g.read_rdump(short, 0.0, 0.0)
        with pytest.raises(RuntimeError, match="cannot open"):
            g.read_rdump(os.path.join(tmp, "missing"), 0.0, 0.0)
