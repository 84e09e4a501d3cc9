"""Python bindings for the CPU oracle and loaders for reference dumps.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's cpu_baseline leg, never by the product package.

- ``build_oracle()`` compiles oracle/harm_oracle.c into oracle/_ref/libharm_oracle.so
  with the precision flags the reference is built with (gcc -O2
  -ffp-contract=off -fno-fast-math).
- ``RefDump`` reads the raw arrays written by oracle/ref_harness.c.
- ``Oracle`` wraps hgo_step / hgo_substep / hgo_utoprim_batch.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBDIR = os.path.join(HERE, "_ref")
LIB = os.path.join(LIBDIR, "libharm_oracle.so")

NPR = 8
LOCS = 8
CENT = 7

LIM = {"DONOR": 0, "VANL": 1, "MINM": 2, "MC": 3, "PARA": 4, "WENO5": 9}
FLUX = {"LAXF": 0, "HLL": 1}
UTOPRIM = {"2DFINAL": 6, "JON": 8, "JONNONRELCOMPAT": 8}   # global.h:283-287
DOENOFLUX = {"NOENOFLUX": 0, "ENOFINITEVOLUME": 3}           # global.h:188-191
BC_OUTFLOW, BC_POLARAXIS, BC_PERIODIC, BC_OUTFLOW_COPY = 0, 4, 7, 1000


def build_oracle(force=False):
    src = os.path.join(HERE, "harm_oracle.c")
    os.makedirs(LIBDIR, exist_ok=True)
    if (not force and os.path.exists(LIB)
            and os.path.getmtime(LIB) >= max(os.path.getmtime(src), os.path.getmtime(os.path.join(HERE, "harm_oracle.h")))):
        return LIB
    cmd = ["gcc", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared", "-o", LIB, src, "-lm"]
    subprocess.run(cmd, check=True)
    return LIB


class hgo_config(ctypes.Structure):
    _fields_ = [("n1", ctypes.c_int), ("n2", ctypes.c_int), ("n3", ctypes.c_int), ("ng", ctypes.c_int),
                ("lim", ctypes.c_int), ("fluxmethod", ctypes.c_int), ("bc", ctypes.c_int * 6),
                ("dx", ctypes.c_double * 4), ("gam", ctypes.c_double), ("cour", ctypes.c_double),
                ("safe", ctypes.c_double), ("defcon", ctypes.c_double), ("tf", ctypes.c_double),
                ("rhominlimit", ctypes.c_double), ("uuminlimit", ctypes.c_double),
                ("gammamax", ctypes.c_double), ("gammafail", ctypes.c_double), ("timeorder", ctypes.c_int),
                ("utoprimversion", ctypes.c_int), ("doenoflux", ctypes.c_int)]


class hgo_geometry(ctypes.Structure):
    _fields_ = [(n, ctypes.POINTER(ctypes.c_double)) for n in ("gcov", "gcon", "gcovpert", "gdet", "conn", "floors")]


class hgo_stats(ctypes.Structure):
    _fields_ = [("newton_iters", ctypes.c_long), ("err", ctypes.c_int), ("nfail_final", ctypes.c_int)]


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


class Problem:
    """A domain: config scalars, per-(i,j) geometry, and the zone arrays."""

    def __init__(self, n1, n2, n3, ng, dx, gam=4.0 / 3.0, cour=0.8, lim="MC", flux="HLL",
                 bc=(BC_OUTFLOW, BC_OUTFLOW, BC_POLARAXIS, BC_POLARAXIS, BC_PERIODIC, BC_PERIODIC),
                 safe=1.3, defcon=1.0, tf=2000.0, rhominlimit=1e-20, uuminlimit=1e-20, gammamax=25.0,
                 gammafail=2500.0, timeorder=2, utoprim="2DFINAL", doenoflux="NOENOFLUX"):
        self.n = (n1, n2, n3)
        self.timeorder = timeorder
        self.utoprim = utoprim
        self.doenoflux = doenoflux
        self.u = None   # evolved conserved state (unew) of the finite-volume scheme
        self.ng = ng
        self.g = tuple(ng if n > 1 else 0 for n in self.n)
        self.s = tuple(1 if n > 1 else 0 for n in self.n)
        self.nt = tuple(n + 2 * g for n, g in zip(self.n, self.g))
        self.gt = (self.nt[0] + self.s[0], self.nt[1] + self.s[1])
        self.dx = tuple(dx)
        self.gam, self.cour, self.lim, self.flux = gam, cour, lim, flux
        self.bc = tuple(bc)
        self.safe, self.defcon, self.tf = safe, defcon, tf
        self.rhominlimit, self.uuminlimit = rhominlimit, uuminlimit
        self.gammamax, self.gammafail = gammamax, gammafail
        gt = self.gt
        self.gcov = np.zeros(gt + (LOCS, 4, 4))
        self.gcon = np.zeros(gt + (LOCS, 4, 4))
        self.gcovpert = np.zeros(gt + (LOCS, 4))
        self.gdet = np.zeros(gt + (LOCS,))
        self.conn = np.zeros(gt + (4, 4, 4))
        self.floors = np.zeros(gt + (2,))
        self.p = np.zeros(self.nt + (NPR,))
        self.pflag = np.zeros(self.nt, dtype=np.int32)
        self.t = 0.0
        self.dt = 0.0

    def active(self, a):
        g = self.g
        return a[g[0]:g[0] + self.n[0], g[1]:g[1] + self.n[1], g[2]:g[2] + self.n[2]]

    def config(self):
        c = hgo_config()
        c.n1, c.n2, c.n3 = self.n
        c.ng = self.ng
        c.lim = LIM[self.lim]
        c.fluxmethod = FLUX[self.flux]
        # BCtype order X1UP, X1DN, X2UP, X2DN, X3UP, X3DN (global.h:467-472)
        for i, b in enumerate(self.bc):
            c.bc[i] = b
        c.dx[0] = 0.0
        for i in range(3):
            c.dx[i + 1] = self.dx[i]
        c.gam, c.cour, c.safe, c.defcon, c.tf = self.gam, self.cour, self.safe, self.defcon, self.tf
        c.rhominlimit, c.uuminlimit = self.rhominlimit, self.uuminlimit
        c.gammamax, c.gammafail = self.gammamax, self.gammafail
        c.timeorder = getattr(self, "timeorder", 2)
        c.utoprimversion = UTOPRIM[getattr(self, "utoprim", "2DFINAL")]
        c.doenoflux = DOENOFLUX[getattr(self, "doenoflux", "NOENOFLUX")]
        return c

    def copy(self):
        import copy
        q = copy.copy(self)
        q.p = self.p.copy()
        q.pflag = self.pflag.copy()
        if getattr(self, "u", None) is not None:
            q.u = self.u.copy()
        return q


def _meta(path):
    m = {}
    with open(path) as f:
        for line in f:
            k, v = line.split()
            try:
                m[k] = int(v)
            except ValueError:
                m[k] = float(v)
    return m


class RefDump:
    """Arrays written by oracle/ref_harness.c (the reference's own layout)."""

    def __init__(self, outdir):
        self.dir = outdir
        m = self.meta = _meta(os.path.join(outdir, "init_meta.txt"))
        self.N = (m["N1"], m["N2"], m["N3"])
        B = m["MAXBND"]
        self.bnd = tuple(B if n > 1 else 0 for n in self.N)
        self.sh = (m["SHIFT1"], m["SHIFT2"], m["SHIFT3"])
        self.NM = tuple(n + 2 * b for n, b in zip(self.N, self.bnd))

    def _f(self, tag, name, dtype=np.float64):
        return np.fromfile(os.path.join(self.dir, f"{tag}_{name}.bin"), dtype=dtype)

    def meta_of(self, tag):
        return _meta(os.path.join(self.dir, f"{tag}_meta.txt"))

    def p(self, tag):
        return self._f(tag, "p").reshape(self.NM + (NPR,))

    def pflag(self, tag):
        return self._f(tag, "pflag", np.int32).reshape(self.NM + (5,))

    def flux(self, tag, d):
        return self._f(tag, f"F{d}").reshape(self.NM + (NPR,))

    def unew(self, tag):
        return self._f(tag, "unew").reshape(self.NM + (NPR,))

    def ffc(self, tag):
        """failfloorcount of the first time scale: [N1M][N2M][N3M][9]."""
        return self._f(tag, "ffc").reshape(self.NM + (9,))

    def pk(self, tag):
        return self._f(tag, "pk").reshape((2,) + self.NM + (NPR,))

    def geom(self, name):
        """Geometry array, x3 extent 1 when the harness wrote only the first
        x3 plane (--geomplane)."""
        gm = tuple(n + s for n, s in zip(self.NM, self.sh))
        nm = self.NM
        if self.meta.get("GEOMPLANE", 0):
            gm = gm[:2] + (1,)
            nm = nm[:2] + (1,)
        shapes = {"gcov": (LOCS, 4, 4), "gcon": (LOCS, 4, 4), "gcovpert": (LOCS, 4), "gdet": (LOCS,),
                  "conn": (4, 4, 4)}
        if name in shapes:
            a = self._f("init", name)
            full = (nm if name == "conn" else gm) + shapes[name]
            if a.size == int(np.prod(shapes[name])):
                # a constant metric (CARTMINKMETRIC: the reference stores one
                # point, defs.h:214) holds everywhere
                return np.broadcast_to(a.reshape((1, 1, 1) + shapes[name]), full).copy()
            return a.reshape(full)
        if name == "floors":
            return self._f("init", name).reshape(nm + (2,))
        raise KeyError(name)

    def to_problem(self, ng, tag="init"):
        """Crop the reference arrays to `ng` ghosts into a Problem."""
        m = self.meta
        lim = {v: k for k, v in LIM.items()}[m["lim"]]
        flux = {v: k for k, v in FLUX.items()}[m["fluxmethod"]]
        bc = tuple(m[f"BCtype{i}"] for i in range(6))
        utoprim = {v: k for k, v in UTOPRIM.items() if k != "JONNONRELCOMPAT"}[m["UTOPRIMVERSION"]]
        doenoflux = {v: k for k, v in DOENOFLUX.items()}[m["DOENOFLUX"]]
        pr = Problem(self.N[0], self.N[1], self.N[2], ng, (m["dx1"], m["dx2"], m["dx3"]), gam=m["gam"],
                     cour=m["cour"], lim=lim, flux=flux, bc=bc, safe=m["SAFE"], defcon=m["defcon"], tf=m["tf"],
                     rhominlimit=m["RHOMINLIMIT"], uuminlimit=m["UUMINLIMIT"], gammamax=m["GAMMAMAX"],
                     gammafail=m["GAMMAFAIL"], timeorder=int(m["TIMEORDER"]), utoprim=utoprim, doenoflux=doenoflux)
        off = tuple(b - g for b, g in zip(self.bnd, pr.g))
        sl = tuple(slice(o, o + nt) for o, nt in zip(off, pr.nt))
        gsl = tuple(slice(o, o + gt) for o, gt in zip(off[:2], pr.gt))
        k0 = 0  # the metric does not depend on x3; take the first plane
        for name in ("gcov", "gcon", "gcovpert", "gdet"):
            getattr(pr, name)[...] = self.geom(name)[gsl[0], gsl[1], k0]
        conn = self.geom("conn")
        fl = self.geom("floors")
        nconn = conn[sl[0], sl[1], k0]
        pr.conn[:nconn.shape[0], :nconn.shape[1]] = nconn
        pr.floors[:nconn.shape[0], :nconn.shape[1]] = fl[sl[0], sl[1], k0]
        pr.p[...] = self.p(tag)[sl]
        pr.pflag[...] = self.pflag(tag)[sl][..., 0]
        if doenoflux == "ENOFINITEVOLUME":
            pr.u = np.ascontiguousarray(self.unew(tag)[sl])
        mm = self.meta_of(tag)
        pr.t, pr.dt = mm["t"], mm["dt"]
        return pr

    def crop(self, arr, ng):
        g = tuple(ng if n > 1 else 0 for n in self.N)
        off = tuple(b - gg for b, gg in zip(self.bnd, g))
        nt = tuple(n + 2 * gg for n, gg in zip(self.N, g))
        return arr[off[0]:off[0] + nt[0], off[1]:off[1] + nt[1], off[2]:off[2] + nt[2]]


class Oracle:
    def __init__(self):
        self.lib = ctypes.CDLL(build_oracle())
        L = self.lib
        L.hgo_step.argtypes = [ctypes.POINTER(hgo_config), ctypes.POINTER(hgo_geometry),
                               ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int),
                               ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double), ctypes.c_int,
                               ctypes.POINTER(hgo_stats)]
        L.hgo_step.restype = ctypes.c_int
        L.hgo_step_u.argtypes = [ctypes.POINTER(hgo_config), ctypes.POINTER(hgo_geometry),
                                 ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int),
                                 ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                                 ctypes.POINTER(ctypes.c_double), ctypes.c_int, ctypes.POINTER(hgo_stats)]
        L.hgo_step_u.restype = ctypes.c_int
        L.hgo_pi2u.argtypes = [ctypes.POINTER(hgo_config), ctypes.POINTER(hgo_geometry),
                               ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]
        L.hgo_pi2u.restype = ctypes.c_int
        L.hgo_post_fixup.argtypes = [ctypes.POINTER(hgo_config), ctypes.POINTER(hgo_geometry),
                                     ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int), ctypes.c_int,
                                     ctypes.POINTER(ctypes.c_double)]
        L.hgo_post_fixup.restype = ctypes.c_int
        L.hgo_fluxcalc.argtypes = [ctypes.POINTER(hgo_config), ctypes.POINTER(hgo_geometry)] + \
            [ctypes.POINTER(ctypes.c_double)] * 5
        L.hgo_fluxcalc.restype = ctypes.c_int
        L.hgo_bound_prim.argtypes = [ctypes.POINTER(hgo_config), ctypes.POINTER(hgo_geometry),
                                     ctypes.POINTER(ctypes.c_double)]
        L.hgo_bound_prim.restype = ctypes.c_int
        L.hgo_checksolution.argtypes = [ctypes.POINTER(hgo_config), ctypes.POINTER(hgo_geometry),
                                        ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int),
                                        ctypes.POINTER(ctypes.c_double)]
        L.hgo_checksolution.restype = ctypes.c_int
        L.hgo_utoprim_batch.argtypes = [ctypes.POINTER(ctypes.c_double)] * 5 + [ctypes.POINTER(ctypes.c_int),
                                        ctypes.c_long, ctypes.c_double, ctypes.c_double,
                                        ctypes.POINTER(ctypes.c_long)]
        L.hgo_utoprim_batch.restype = ctypes.c_int
        L.hgo_utoprim_batch_v.argtypes = [ctypes.POINTER(ctypes.c_double)] * 5 + [ctypes.POINTER(ctypes.c_int),
                                          ctypes.c_long, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                          ctypes.POINTER(ctypes.c_long)]
        L.hgo_utoprim_batch_v.restype = ctypes.c_int

    @staticmethod
    def geometry(pr):
        for n in ("gcov", "gcon", "gcovpert", "gdet", "conn", "floors"):
            a = getattr(pr, n)
            assert a.flags.c_contiguous and a.dtype == np.float64
        g = hgo_geometry()
        g.gcov, g.gcon, g.gcovpert = _dp(pr.gcov), _dp(pr.gcon), _dp(pr.gcovpert)
        g.gdet, g.conn, g.floors = _dp(pr.gdet), _dp(pr.conn), _dp(pr.floors)
        return g

    def step(self, pr, nsteps=1):
        """Advance `pr` in place; returns hgo_stats."""
        c = pr.config()
        g = self.geometry(pr)
        st = hgo_stats()
        t = ctypes.c_double(pr.t)
        dt = ctypes.c_double(pr.dt)
        assert pr.p.flags.c_contiguous and pr.pflag.flags.c_contiguous
        if c.doenoflux == DOENOFLUX["ENOFINITEVOLUME"]:
            if getattr(pr, "u", None) is None:
                pr.u = self.pi2u(pr)
            self.lib.hgo_step_u(ctypes.byref(c), ctypes.byref(g), _dp(pr.p), _ip(pr.pflag), _dp(pr.u),
                                ctypes.byref(t), ctypes.byref(dt), nsteps, ctypes.byref(st))
        else:
            self.lib.hgo_step(ctypes.byref(c), ctypes.byref(g), _dp(pr.p), _ip(pr.pflag), ctypes.byref(t),
                              ctypes.byref(dt), nsteps, ctypes.byref(st))
        pr.t, pr.dt = t.value, dt.value
        return st

    def post_fixup(self, pr, finalstep=1):
        """post_fixup (fixup.c:37-96) on pr.p / pr.pflag in place; returns the
        error bits."""
        assert pr.p.flags.c_contiguous and pr.pflag.flags.c_contiguous
        u = getattr(pr, "u", None)
        return self.lib.hgo_post_fixup(ctypes.byref(pr.config()), ctypes.byref(self.geometry(pr)), _dp(pr.p),
                                       _ip(pr.pflag), int(finalstep), _dp(u) if u is not None else None)

    def fluxcalc(self, pr, fill=0.0):
        """fluxcalc + flux_ct on pr.p: (error bits, [F1, F2, F3], [ndt1, ndt2,
        ndt3]); faces the update does not read keep `fill`."""
        assert pr.p.flags.c_contiguous
        F = [np.full(pr.p.shape, fill) for _ in range(3)]
        ndt = np.zeros(3)
        e = self.lib.hgo_fluxcalc(ctypes.byref(pr.config()), ctypes.byref(self.geometry(pr)), _dp(pr.p), _dp(F[0]),
                                  _dp(F[1]), _dp(F[2]), _dp(ndt))
        return e, F, list(ndt)

    def bound_prim(self, pr):
        """bound_prim (the problem file's boundaries) on pr.p in place;
        returns the error bits."""
        assert pr.p.flags.c_contiguous
        return self.lib.hgo_bound_prim(ctypes.byref(pr.config()), ctypes.byref(self.geometry(pr)), _dp(pr.p))

    def checksolution(self, pr):
        """fixup_checksolution (fixup.c:460-560) alone on pr.pflag in place;
        returns (error bits, the Lorentz factors it compared)."""
        assert pr.p.flags.c_contiguous and pr.pflag.flags.c_contiguous
        gam = np.zeros(pr.pflag.shape)
        e = self.lib.hgo_checksolution(ctypes.byref(pr.config()), ctypes.byref(self.geometry(pr)), _dp(pr.p),
                                       _ip(pr.pflag), _dp(gam))
        return e, gam

    def pi2u(self, pr):
        """pi2Uavg: the conserved state U(p) in every zone (init_conservatives)."""
        u = np.zeros_like(pr.p)
        self.lib.hgo_pi2u(ctypes.byref(pr.config()), ctypes.byref(self.geometry(pr)), _dp(pr.p), _dp(u))
        return u

    def utoprim(self, U, gcov, gcon, gdet, guess, gam, gammafail, version="2DFINAL"):
        U = np.ascontiguousarray(U, dtype=np.float64)
        gcov = np.ascontiguousarray(gcov, dtype=np.float64)
        gcon = np.ascontiguousarray(gcon, dtype=np.float64)
        gdet = np.ascontiguousarray(gdet, dtype=np.float64)
        pr = np.array(guess, dtype=np.float64, order="C", copy=True)
        n = U.shape[0]
        pflag = np.zeros(n, dtype=np.int32)
        it = ctypes.c_long(0)
        self.lib.hgo_utoprim_batch_v(_dp(U), _dp(gcov), _dp(gcon), _dp(gdet), _dp(pr), _ip(pflag), n, gam, gammafail,
                                     UTOPRIM[version], ctypes.byref(it))
        return pr, pflag, it.value
