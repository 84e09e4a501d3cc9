"""Serving loop (hgpu_server_*): solves of different kinds (Kerr tori in 2D
and 3D, Bondi accretion, 1D shock tubes) and sizes that
arrive while others run are admitted as memory frees up, run overlapped on
the device, and each result is bit-identical to running that solve alone."""
import numpy as np
import pytest

from harm_finalwham_b200 import bondi, riemann, torus
from harm_finalwham_b200.gpu import HarmGPU, HarmServer, context_bytes, make_config
from tests.fixtures import same

pytestmark = pytest.mark.gpu

TF = 0.25


def requests():
    return [torus.fm_torus(32, 32, 1, ng=3, a=0.5, beta=50.0, seed=1),
            bondi.bondi(32, 32, ng=3, beta=30.0, seed=2),
            torus.fm_torus(16, 16, 8, ng=3, a=0.9, beta=200.0, seed=3),
            torus.fm_torus(24, 16, 1, ng=6, lim="WENO5", seed=4),
            bondi.bondi(48, 32, ng=3, beta=300.0, seed=5),
            torus.fm_torus(32, 16, 1, ng=3, a=0.2, seed=6)] + \
        [riemann.domain(p) for p in riemann.draw(2, seed=9, nmin=100, nmax=300)]


def run_alone(dom, tf):
    inv = {0: "OUTFLOW", 4: "POLARAXIS", 7: "PERIODIC", 1000: "OUTFLOW_COPY"}
    g = HarmGPU(*dom.n, dom.ng, dom.dx, lim=dom.lim, flux=dom.flux, bc=tuple(inv[b] for b in dom.bc), gam=dom.gam,
                cour=dom.cour, tf=tf)
    try:
        g.upload_geometry(dom.gcov, dom.gcon, dom.gcovpert, dom.gdet, dom.conn, dom.floors)
        g.upload_state(dom.p, None, 0.0, 0.0)
        g.init_dt()
        for _ in range(2000):
            g.step_ch(1, stats=False)
            if g.time()[0] >= tf:
                break
        return g.download_state()
    finally:
        g.close()


def test_serve_matches_alone():
    reqs = requests()
    inv = {0: "OUTFLOW", 4: "POLARAXIS", 7: "PERIODIC", 1000: "OUTFLOW_COPY"}
    sizes = [context_bytes(make_config(d.n, d.ng, d.dx, lim=d.lim, bc=tuple(inv[b] for b in d.bc))) for d in reqs]
    assert min(sizes) > 0
    # room for about two solves at a time: the rest queue and are admitted as memory frees up
    srv = HarmServer(max_device_bytes=int(2.2 * max(sizes)), max_active=4, steps_per_chunk=3)
    try:
        ids = [srv.submit(d, TF) for d in reqs[:3]]
        seen_queue = False
        for it in range(200000):
            pend, act, fin = srv.poll()
            seen_queue |= pend > 0 and act > 0
            if it == 20:
                ids += [srv.submit(d, TF) for d in reqs[3:]]
            if len(ids) == len(reqs) and fin == len(reqs):
                break
        assert fin == len(reqs)
        assert seen_queue
        for rid, d in zip(ids, reqs):
            p, pf, t, steps, qms, rms = srv.result(rid)
            pa, pfa, ta, _ = run_alone(d, TF)
            assert t == ta and t >= TF and steps > 0
            assert same(p, pa), f"request {rid} differs from its run alone"
            assert np.array_equal(pf, pfa)
    finally:
        srv.close()


def test_context_frozen_after_end_time():
    # steps past tf leave primitives, flags and t unchanged (the reference stops at t >= tf)
    dom = requests()[3]
    inv = {0: "OUTFLOW", 4: "POLARAXIS", 7: "PERIODIC", 1000: "OUTFLOW_COPY"}
    g = HarmGPU(*dom.n, dom.ng, dom.dx, lim=dom.lim, flux=dom.flux, bc=tuple(inv[b] for b in dom.bc), gam=dom.gam,
                cour=dom.cour, tf=TF)
    try:
        g.upload_geometry(dom.gcov, dom.gcon, dom.gcovpert, dom.gdet, dom.conn, dom.floors)
        g.upload_state(dom.p, None, 0.0, 0.0)
        g.init_dt()
        while g.time()[0] < TF:
            g.step_ch(1, stats=False)
        a = g.download_state()
        g.step_ch(4, stats=False)
        b = g.download_state()
    finally:
        g.close()
    assert same(a[0], b[0]) and np.array_equal(a[1], b[1]) and a[2] == b[2] and a[2] >= TF


def test_reconfigured_context_equals_fresh_context():
    # hgpu_reconfigure: a context reused for another solve of the same
    # allocation shape (another spin, so another dx, and another end time)
    # gives the fresh context's result bit for bit, in plain and graph steps
    a = torus.fm_torus(32, 32, 1, ng=3, a=0.5, beta=50.0, seed=1)
    b = torus.fm_torus(32, 32, 1, ng=3, a=0.9, beta=200.0, seed=7)
    assert a.dx != b.dx
    ref = run_alone(b, 0.3)
    inv = {0: "OUTFLOW", 4: "POLARAXIS", 7: "PERIODIC", 1000: "OUTFLOW_COPY"}
    g = HarmGPU(*a.n, a.ng, a.dx, lim=a.lim, flux=a.flux, bc=tuple(inv[q] for q in a.bc), gam=a.gam, cour=a.cour,
                tf=TF)
    try:
        for use_graph in (False, True):
            for dom, tf in ((a, TF), (b, 0.3)):
                g.reconfigure(dx=dom.dx, gam=dom.gam, cour=dom.cour, tf=tf)
                g.upload_geometry(dom.gcov, dom.gcon, dom.gcovpert, dom.gdet, dom.conn, dom.floors)
                g.upload_state(dom.p, None, 0.0, 0.0)
                g.init_dt()
                for _ in range(2000):
                    if use_graph:
                        g.step_graph(1, stats=False)
                    else:
                        g.step_ch(1, stats=False)
                    if g.time()[0] >= tf:
                        break
            p, pf, t, dt = g.download_state()
            assert same(p, ref[0]) and np.array_equal(pf, ref[1]) and t == ref[2] and dt == ref[3]
        # another allocation shape is refused
        import ctypes
        from harm_finalwham_b200.gpu import hgpu_config
        c = hgpu_config.from_buffer_copy(g.cfg)
        c.n1 = 64
        assert g.L.hgpu_reconfigure(g.h, ctypes.byref(c)) != 0
    finally:
        g.close()
