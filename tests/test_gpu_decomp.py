"""A domain split along x3 (the reference's MPI decomposition over ncpux3
ranks, boundmpi.c:6-180) reproduces the whole-domain run bit for bit: the
slabs of one torus run as separate contexts on one device, their ghost planes
and ndt minima moved between phases by device copies."""
import numpy as np
import pytest

from harm_finalwham_b200.decomp import SplitRun
from harm_finalwham_b200.gpu import HarmGPU
from harm_finalwham_b200.torus import fm_torus

pytestmark = pytest.mark.gpu


def _torus(n, ng, lim, flux, timeorder=2, utoprim="2DFINAL", doenoflux="NOENOFLUX"):
    dom = fm_torus(*n, ng=ng, lim=lim, flux=flux)
    dom.timeorder, dom.utoprim, dom.doenoflux = timeorder, utoprim, doenoflux
    return dom


def _same_bits(a, b):
    return np.array_equal(np.asarray(a).view(np.uint8), np.asarray(b).view(np.uint8))


SCHEMES = [
    ("mc_hll_rk2", dict(n=(32, 16, 16), ng=3, lim="MC", flux="HLL")),
    ("para_laxf_rk4_jon_fv", dict(n=(32, 16, 16), ng=3, lim="PARA", flux="LAXF", timeorder=4, utoprim="JON",
                                  doenoflux="ENOFINITEVOLUME")),
    ("weno5_hll_rk3", dict(n=(24, 16, 24), ng=6, lim="WENO5", flux="HLL", timeorder=3)),
    # the FM torus problem file's own scheme with all MAXBND = 11 ghosts
    ("fishmon_maxbnd11", dict(n=(24, 16, 44), ng=11, lim="PARA", flux="HLL", timeorder=4, utoprim="JON",
                              doenoflux="ENOFINITEVOLUME")),
]


@pytest.mark.parametrize("name,kw", SCHEMES, ids=[s[0] for s in SCHEMES])
@pytest.mark.parametrize("nslabs", [1, 2, 4])
def test_split_run_matches_whole_domain(name, kw, nslabs):
    _split_vs_whole(kw, nslabs, "fp64")


@pytest.mark.parametrize("nslabs", [2, 4])
def test_split_run_matches_whole_domain_mixed_precision(nslabs):
    _split_vs_whole(SCHEMES[2][1], nslabs, "mixed")


def _split_vs_whole(kw, nslabs, precision):
    dom = _torus(**kw)
    if dom.n[2] // nslabs < dom.g[2]:
        pytest.skip("slab thinner than the ghost planes")
    nsteps = 6
    with HarmGPU.from_problem(dom, precision=precision) as whole:
        # the generator's ghost planes are evaluated, not copied: start both
        # runs from bound_prim, as the reference's init does
        whole.bound_prim(0)
        dt0 = whole.init_dt()
        st_w = whole.step_ch(nsteps)
        p_w, f_w, t_w, dt_w = whole.download_state()
        p_w, f_w = whole.active(p_w), whole.active(f_w)
    run = SplitRun.local(dom, nslabs, precision=precision, init_dt=True)
    try:
        _, _, _, dt_s0 = run.download()
        assert dt_s0 == dt0
        st_s = run.step(nsteps)
        p_s, f_s, t_s, dt_s = run.download()
    finally:
        run.close()
    assert (t_s, dt_s) == (t_w, dt_w)
    assert _same_bits(p_s, p_w), np.abs(p_s - p_w).max()
    assert np.array_equal(f_s, f_w)
    assert st_s.newton_iters == st_w.newton_iters
    assert st_s.err == st_w.err == 0



def test_collective_transport_on_one_rank_matches_whole_domain():
    """The multi-GPU transport with one rank (no process group): the planes
    wrap onto the same context on its own stream, no host synchronisation."""
    from harm_finalwham_b200.decomp import CollectiveTransport, SlabContext
    dom = _torus(n=(32, 16, 16), ng=3, lim="PARA", flux="HLL", timeorder=4, utoprim="JON",
                 doenoflux="ENOFINITEVOLUME")
    with HarmGPU.from_problem(dom) as whole:
        whole.bound_prim(0)
        whole.init_dt()
        whole.step_ch(5)
        p_w, f_w, t_w, dt_w = whole.download_state()
    g = HarmGPU.from_problem(dom)
    run = SplitRun([g], CollectiveTransport(SlabContext(g)))
    try:
        run.start(init_dt=True)
        run.step(5)
        p_s, f_s, t_s, dt_s = run.download()
    finally:
        run.close()
    assert (t_s, dt_s) == (t_w, dt_w)
    assert _same_bits(p_s, p_w[3:-3, 3:-3, 3:-3])
    assert np.array_equal(f_s, f_w[3:-3, 3:-3, 3:-3])


def _gloo_rank(rank, world, port, kw, nsteps, out):
    import datetime
    import os

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        from harm_finalwham_b200.decomp import CollectiveTransport, SlabContext, split_x3
        dom = _torus(**kw)
        g = HarmGPU.from_problem(split_x3(dom, world, rank))
        tr = CollectiveTransport(SlabContext(g))
        assert tr.staged and tr.world == world
        run = SplitRun([g], tr)
        try:
            run.start(init_dt=True)
            st = run.step(nsteps)
            p, f, t, dt = run.download()
        finally:
            run.close()
        out[rank] = (p, f, t, dt, st.newton_iters)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_processes_through_the_collective_transport_match_whole_domain():
    """Two ranks (processes) on one GPU, each with its own slab context; the
    planes and the ndt minima go through torch.distributed (gloo, through
    pinned host copies), so no kernel ever waits on the other process."""
    import socket

    import torch.multiprocessing as mp
    kw, nsteps, world = SCHEMES[0][1], 4, 2
    dom = _torus(**kw)
    with HarmGPU.from_problem(dom) as whole:
        whole.bound_prim(0)
        whole.init_dt()
        st_w = whole.step_ch(nsteps)
        p_w, f_w, t_w, dt_w = whole.download_state()
        p_w, f_w = whole.active(p_w), whole.active(f_w)
    sock = socket.socket()
    sock.bind(("127.0.0.1", 0))
    port = sock.getsockname()[1]
    sock.close()
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    procs = [ctx.Process(target=_gloo_rank, args=(r, world, port, kw, nsteps, out)) for r in range(world)]
    for pr in procs:
        pr.start()
    for pr in procs:
        pr.join(300)
        assert pr.exitcode == 0
    p_s = np.concatenate([out[r][0] for r in range(world)], axis=2)
    f_s = np.concatenate([out[r][1] for r in range(world)], axis=2)
    assert all((out[r][2], out[r][3]) == (t_w, dt_w) for r in range(world))
    assert _same_bits(p_s, p_w)
    assert np.array_equal(f_s, f_w)
    assert sum(out[r][4] for r in range(world)) == st_w.newton_iters
