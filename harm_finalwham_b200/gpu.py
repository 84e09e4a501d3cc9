"""ctypes bindings of the C ABI in include/harmgpu.h.

The class mirrors the reference's entry points for the per-zone update:
``step_ch`` (step_ch.c:16), ``advance_stage`` (advance.c:16 plus the per-stage
bound/post_fixup sequence of step_ch.c:94-186), ``fluxcalc`` (flux.c:7 with
flux_ct fluxct.c:10), ``bound_prim`` (step_ch.c:568) and ``utoprim_batch``
(utoprimgen.c:23, batched).  Host arrays use the reference's layouts; errors
are raised as HarmGPUError carrying the library's return code and message.
There is no CPU fallback: if the library or a GPU is missing, calls fail.
"""
import ctypes
import os

import numpy as np

from . import build as _build

NPR = 8
LIM = {"DONOR": 0, "VANL": 1, "MINM": 2, "MC": 3, "PARA": 4, "WENO5": 9}
FLUX = {"LAXF": 0, "HLL": 1}
BC = {"OUTFLOW": 0, "POLARAXIS": 4, "PERIODIC": 7, "OUTFLOW_COPY": 1000, "POLARAXIS_FLIP": 1001,
      "BONDIMDOTOUTFLOW": 109, "BONDIINTOUTFLOW": 110}
PREC = {"fp64": 0, "mixed": 1}
UTOPRIM = {"2DFINAL": 6, "JON": 8, "JONNONRELCOMPAT": 8}
DOENOFLUX = {"NOENOFLUX": 0, "ENOFINITEVOLUME": 3}

_lib = None


class HarmGPUError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"libharmgpu error {code}: {msg}")
        self.code = code


class hgpu_config(ctypes.Structure):
    _fields_ = [("n1", ctypes.c_int), ("n2", ctypes.c_int), ("n3", ctypes.c_int), ("ng", ctypes.c_int),
                ("lim", ctypes.c_int), ("fluxmethod", ctypes.c_int), ("bc", ctypes.c_int * 6),
                ("precision", ctypes.c_int), ("dx", ctypes.c_double * 4), ("gam", ctypes.c_double),
                ("cour", ctypes.c_double), ("safe", ctypes.c_double), ("defcon", ctypes.c_double),
                ("tf", ctypes.c_double), ("rhominlimit", ctypes.c_double), ("uuminlimit", ctypes.c_double),
                ("gammamax", ctypes.c_double), ("gammafail", ctypes.c_double), ("timeorder", ctypes.c_int),
                ("utoprimversion", ctypes.c_int), ("doenoflux", ctypes.c_int)]


class hgpu_tuning(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in ("flux_minb", "weno_minb", "update_minb", "invert_minb")] + \
               [(n, ctypes.c_int * 2) for n in ("flux_cand", "weno_cand", "update_cand", "invert_cand")] + \
               [(n, ctypes.c_float * 2) for n in ("flux_ms", "weno_ms", "update_ms", "invert_ms")] + \
               [("weno_lb", ctypes.c_int * 4), ("weno_lines", ctypes.c_int * 4), ("weno_tile_ms", ctypes.c_float * 4)]


class hgpu_diag(ctypes.Structure):
    _fields_ = [("t", ctypes.c_double), ("dt", ctypes.c_double), ("integral", ctypes.c_double * 8),
                ("divb_max", ctypes.c_double), ("divb_avg", ctypes.c_double), ("nfail", ctypes.c_int),
                ("nfloor", ctypes.c_longlong), ("nsteps", ctypes.c_longlong),
                ("divb_max_interior", ctypes.c_double)]


class hgpu_stats(ctypes.Structure):
    _fields_ = [("newton_iters", ctypes.c_longlong), ("err", ctypes.c_int), ("nfail", ctypes.c_int),
                ("nfixed", ctypes.c_int)]


_P = ctypes.POINTER
_dp = _P(ctypes.c_double)
_ip = _P(ctypes.c_int)


def load_library(path=None):
    """Load libharmgpu.so (building it in-tree first if sources are newer)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    if path is None:
        path = _build.LIB
        if not os.path.exists(path):
            path = _build.build()
    L = ctypes.CDLL(path)
    L.hgpu_abi_version.restype = ctypes.c_int
    L.hgpu_set_device.argtypes = [ctypes.c_int]
    L.hgpu_set_device.restype = ctypes.c_int
    L.hgpu_last_error.restype = ctypes.c_char_p
    L.hgpu_create.argtypes = [_P(hgpu_config), _P(ctypes.c_void_p)]
    L.hgpu_destroy.argtypes = [ctypes.c_void_p]
    L.hgpu_destroy.restype = None
    L.hgpu_upload_geometry.argtypes = [ctypes.c_void_p] + [_dp] * 6
    L.hgpu_upload_state.argtypes = [ctypes.c_void_p, _dp, _ip, ctypes.c_double, ctypes.c_double]
    L.hgpu_download_state.argtypes = [ctypes.c_void_p, _dp, _ip, _dp, _dp]
    L.hgpu_step_ch.argtypes = [ctypes.c_void_p, ctypes.c_int, _P(hgpu_stats)]
    L.hgpu_advance_stage.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, _P(hgpu_stats)]
    L.hgpu_fluxcalc.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, _dp, _dp, _dp, _dp, _dp]
    L.hgpu_bound_prim.argtypes = [ctypes.c_void_p, ctypes.c_int]
    L.hgpu_post_fixup.argtypes = [ctypes.c_void_p, ctypes.c_int, _P(hgpu_stats)]
    L.hgpu_utoprim_batch.argtypes = [_dp, _dp, _dp, _dp, _dp, _ip, ctypes.c_longlong, ctypes.c_double,
                                     ctypes.c_double, _P(ctypes.c_longlong)]
    L.hgpu_utoprimgen_batch.argtypes = [_dp, _dp, _dp, _dp, _dp, _ip, ctypes.c_longlong, ctypes.c_double,
                                        ctypes.c_double, ctypes.c_int, _P(ctypes.c_longlong)]
    L.hgpu_device_prims.argtypes = [ctypes.c_void_p, ctypes.c_int, _P(ctypes.c_void_p)]
    L.hgpu_sync.argtypes = [ctypes.c_void_p]
    L.hgpu_init_dt.argtypes = [ctypes.c_void_p, _dp]
    L.hgpu_step_ch_timed.argtypes = [ctypes.c_void_p, ctypes.c_int, _P(ctypes.c_float), _P(hgpu_stats)]
    L.hgpu_set_profiling.argtypes = [ctypes.c_void_p, ctypes.c_int]
    L.hgpu_kernel_times.argtypes = [ctypes.c_void_p, _P(ctypes.c_char_p), _dp, _P(ctypes.c_longlong), ctypes.c_int]
    L.hgpu_launch_count.argtypes = [ctypes.c_void_p]
    L.hgpu_launch_count.restype = ctypes.c_longlong
    L.hgpu_alloc_pinned.argtypes = [ctypes.c_size_t, _P(ctypes.c_void_p)]
    L.hgpu_free_pinned.argtypes = [ctypes.c_void_p]
    L.hgpu_fp64_peak.argtypes = [_dp]
    L.hgpu_create_batch.argtypes = [_P(hgpu_config), ctypes.c_int, _ip, _dp, _dp, _dp, _P(ctypes.c_void_p)]
    L.hgpu_batch_layout.argtypes = [ctypes.c_void_p, _ip]
    L.hgpu_batch_status.argtypes = [ctypes.c_void_p, _dp, _dp, _ip, _ip]
    L.hgpu_batch_set_time.argtypes = [ctypes.c_void_p, _dp, _dp]
    L.hgpu_step_graph.argtypes = [ctypes.c_void_p, ctypes.c_int, _P(hgpu_stats)]
    L.hgpu_autotune.argtypes = [ctypes.c_void_p, _P(hgpu_tuning)]
    L.hgpu_set_tuning.argtypes = [ctypes.c_void_p, _P(hgpu_tuning)]
    L.hgpu_diagnostics.argtypes = [ctypes.c_void_p, _P(hgpu_diag)]
    L.hgpu_download_conserved.argtypes = [ctypes.c_void_p, _dp]
    L.hgpu_download_bsqflags.argtypes = [ctypes.c_void_p, _ip]
    L.hgpu_reconfigure.argtypes = [ctypes.c_void_p, _P(hgpu_config)]
    L.hgpu_upload_conserved.argtypes = [ctypes.c_void_p, _dp]
    L.hgpu_set_bondi_boundaries.argtypes = [ctypes.c_void_p, _dp]
    L.hgpu_upload_active.argtypes = [ctypes.c_void_p, _dp, ctypes.c_double, ctypes.c_double]
    L.hgpu_download_active.argtypes = [ctypes.c_void_p, _dp, _ip, _dp, _dp]
    L.hgpu_download_failfloorcount.argtypes = [ctypes.c_void_p, _P(ctypes.c_longlong), ctypes.c_int]
    L.hgpu_write_rdump.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]
    L.hgpu_read_rdump.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t, ctypes.c_int, ctypes.c_double,
                                  ctypes.c_double]
    L.hgpu_context_bytes.argtypes = [_P(hgpu_config)]
    L.hgpu_context_bytes.restype = ctypes.c_size_t
    L.hgpu_server_create.argtypes = [ctypes.c_size_t, ctypes.c_int, ctypes.c_int, _P(ctypes.c_void_p)]
    L.hgpu_server_destroy.argtypes = [ctypes.c_void_p]
    L.hgpu_server_destroy.restype = None
    L.hgpu_server_submit.argtypes = [ctypes.c_void_p, _P(hgpu_config)] + [_dp] * 7 + [ctypes.c_double,
                                                                                       _P(ctypes.c_longlong)]
    L.hgpu_server_submit_borrowed.argtypes = L.hgpu_server_submit.argtypes
    L.hgpu_server_poll.argtypes = [ctypes.c_void_p, _ip, _ip, _ip]
    L.hgpu_server_result.argtypes = [ctypes.c_void_p, ctypes.c_longlong, _dp, _ip, _dp, _P(ctypes.c_longlong), _dp,
                                     _dp]
    L.hgpu_server_release.argtypes = [ctypes.c_void_p, ctypes.c_longlong]
    L.hgpu_batch_run.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _ip, _P(ctypes.c_float), _ip,
                                 _P(ctypes.c_float)]
    _v = ctypes.c_void_p
    L.hgpu_halo_bytes.argtypes = [_v, _P(ctypes.c_size_t)]
    L.hgpu_halo_pack.argtypes = [_v, ctypes.c_int, ctypes.c_int, ctypes.c_int, _v]
    L.hgpu_halo_unpack.argtypes = [_v, ctypes.c_int, ctypes.c_int, ctypes.c_int, _v]
    L.hgpu_stats_clear.argtypes = [_v]
    L.hgpu_stats_read.argtypes = [_v, _P(hgpu_stats)]
    L.hgpu_stage_advance.argtypes = [_v, ctypes.c_int]
    L.hgpu_stage_fixup.argtypes = [_v, ctypes.c_int]
    L.hgpu_dt_probe.argtypes = [_v]
    L.hgpu_step_end.argtypes = [_v, ctypes.c_int]
    L.hgpu_ndt_pack.argtypes = [_v, _v]
    L.hgpu_ndt_unpack.argtypes = [_v, _v]
    L.hgpu_stream.argtypes = [_v, _P(_v)]
    for name in ("hgpu_init_dt", "hgpu_step_ch_timed", "hgpu_set_profiling", "hgpu_kernel_times", "hgpu_alloc_pinned",
                 "hgpu_free_pinned", "hgpu_fp64_peak"):
        getattr(L, name).restype = ctypes.c_int
    for name in ("hgpu_create", "hgpu_upload_geometry", "hgpu_upload_state", "hgpu_download_state", "hgpu_step_ch",
                 "hgpu_advance_stage", "hgpu_fluxcalc", "hgpu_bound_prim", "hgpu_post_fixup", "hgpu_utoprim_batch", "hgpu_utoprimgen_batch",
                 "hgpu_device_prims", "hgpu_sync", "hgpu_create_batch", "hgpu_batch_layout", "hgpu_batch_status", "hgpu_batch_set_time",
                 "hgpu_step_graph", "hgpu_autotune", "hgpu_set_tuning", "hgpu_batch_run", "hgpu_diagnostics", "hgpu_download_conserved", "hgpu_upload_conserved",
                 "hgpu_write_rdump", "hgpu_read_rdump", "hgpu_download_failfloorcount", "hgpu_set_bondi_boundaries", "hgpu_upload_active", "hgpu_download_active", "hgpu_server_create", "hgpu_server_submit", "hgpu_server_submit_borrowed",
                 "hgpu_server_poll", "hgpu_server_result", "hgpu_server_release", "hgpu_halo_bytes", "hgpu_halo_pack",
                 "hgpu_halo_unpack", "hgpu_stats_clear", "hgpu_stats_read", "hgpu_stage_advance", "hgpu_stage_fixup",
                 "hgpu_dt_probe", "hgpu_step_end", "hgpu_ndt_pack", "hgpu_ndt_unpack", "hgpu_stream"):
        getattr(L, name).restype = ctypes.c_int
    if path == _build.LIB:
        _lib = L
    return L


def set_device(device):
    """hgpu_set_device: the CUDA device the library uses on this thread (its
    runtime is linked statically, so torch.cuda.set_device does not reach
    it); call before creating contexts."""
    L = load_library()
    _check(L, L.hgpu_set_device(int(device)))


def _check(L, rc):
    if rc != 0:
        raise HarmGPUError(rc, L.hgpu_last_error().decode(errors="replace"))


def _ptr(a, ctype=ctypes.c_double):
    if a is None:
        return None
    return a.ctypes.data_as(ctypes.POINTER(ctype))


def _contig(a, dtype):
    a = np.asarray(a)
    if a.dtype != dtype or not a.flags.c_contiguous:
        a = np.ascontiguousarray(a, dtype=dtype)
    return a


class HarmGPU:
    """One device-resident domain (the reference's global state for one run)."""

    def __init__(self, n1, n2, n3, ng, dx, lim="MC", flux="HLL", bc=("OUTFLOW", "OUTFLOW", "POLARAXIS",
                 "POLARAXIS", "PERIODIC", "PERIODIC"), precision="fp64", gam=4.0 / 3.0, cour=0.8, safe=1.3,
                 defcon=1.0, tf=2000.0, rhominlimit=1e-20, uuminlimit=1e-20, gammamax=25.0, gammafail=2500.0,
                 timeorder=2, utoprim="2DFINAL", doenoflux="NOENOFLUX"):
        self.L = load_library()
        c = hgpu_config()
        c.timeorder = int(timeorder)
        c.utoprimversion = UTOPRIM[utoprim] if isinstance(utoprim, str) else int(utoprim)
        c.doenoflux = DOENOFLUX[doenoflux] if isinstance(doenoflux, str) else int(doenoflux)
        c.n1, c.n2, c.n3, c.ng = n1, n2, n3, ng
        c.lim = LIM[lim] if isinstance(lim, str) else int(lim)
        c.fluxmethod = FLUX[flux] if isinstance(flux, str) else int(flux)
        for i, b in enumerate(bc):
            c.bc[i] = BC[b] if isinstance(b, str) else int(b)
        c.precision = PREC[precision] if isinstance(precision, str) else int(precision)
        c.dx[0] = 0.0
        for i in range(3):
            c.dx[i + 1] = float(dx[i])
        c.gam, c.cour, c.safe, c.defcon, c.tf = gam, cour, safe, defcon, tf
        c.rhominlimit, c.uuminlimit, c.gammamax, c.gammafail = rhominlimit, uuminlimit, gammamax, gammafail
        self.cfg = c
        self.n = (n1, n2, n3)
        self.g = tuple(ng if n > 1 else 0 for n in self.n)
        self.s = tuple(1 if n > 1 else 0 for n in self.n)
        self.nt = tuple(n + 2 * g for n, g in zip(self.n, self.g))
        self.gt = (self.nt[0] + self.s[0], self.nt[1] + self.s[1])
        h = ctypes.c_void_p()
        _check(self.L, self.L.hgpu_create(ctypes.byref(c), ctypes.byref(h)))
        self.h = h

    def reconfigure(self, dx=None, gam=None, cour=None, tf=None):
        """hgpu_reconfigure: the same context for another solve of the same
        allocation shape (upload geometry and state afterwards)."""
        c = hgpu_config.from_buffer_copy(self.cfg)
        if dx is not None:
            for i in range(3):
                c.dx[i + 1] = float(dx[i])
        if gam is not None:
            c.gam = float(gam)
        if cour is not None:
            c.cour = float(cour)
        if tf is not None:
            c.tf = float(tf)
        _check(self.L, self.L.hgpu_reconfigure(self.h, ctypes.byref(c)))
        self.cfg = c

    @classmethod
    def from_problem(cls, pr, precision="fp64"):
        """Build from an object with the oracle Problem's attributes."""
        inv_bc = {v: k for k, v in BC.items()}
        o = cls(pr.n[0], pr.n[1], pr.n[2], pr.ng, pr.dx, lim=pr.lim, flux=pr.flux,
                bc=tuple(inv_bc[b] for b in pr.bc), precision=precision, gam=pr.gam, cour=pr.cour, safe=pr.safe,
                defcon=pr.defcon, tf=pr.tf, rhominlimit=pr.rhominlimit, uuminlimit=pr.uuminlimit,
                gammamax=pr.gammamax, gammafail=pr.gammafail, timeorder=getattr(pr, "timeorder", 2),
                utoprim=getattr(pr, "utoprim", "2DFINAL"), doenoflux=getattr(pr, "doenoflux", "NOENOFLUX"))
        o.upload_geometry(pr.gcov, pr.gcon, pr.gcovpert, pr.gdet, pr.conn, pr.floors)
        if getattr(pr, "bondi_bc", None) is not None:
            o.set_bondi_boundaries(pr.bondi_bc)
        o.upload_state(pr.p, pr.pflag, pr.t, pr.dt)
        if getattr(pr, "u", None) is not None and o.cfg.doenoflux == DOENOFLUX["ENOFINITEVOLUME"]:
            o.upload_conserved(pr.u)
        return o

    def close(self):
        if getattr(self, "h", None):
            self.L.hgpu_destroy(self.h)
            self.h = None
        for ptr in getattr(self, "_pinned", []):
            self.L.hgpu_free_pinned(ptr)
        self._pinned = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def upload_geometry(self, gcov, gcon, gcovpert, gdet, conn, floors):
        arrs = [_contig(a, np.float64) for a in (gcov, gcon, gcovpert, gdet, conn, floors)]
        nij = self.gt[0] * self.gt[1]
        expect = [nij * 128, nij * 128, nij * 32, nij * 8, nij * 64, nij * 2]
        for a, e in zip(arrs, expect):
            if a.size != e:
                raise ValueError(f"geometry array has {a.size} values, expected {e}")
        _check(self.L, self.L.hgpu_upload_geometry(self.h, *[_ptr(a) for a in arrs]))

    def upload_state(self, p, pflag=None, t=0.0, dt=0.0):
        p = _contig(p, np.float64)
        if p.size != np.prod(self.nt) * NPR:
            raise ValueError("primitive array has the wrong size")
        pf = None if pflag is None else _contig(pflag, np.int32)
        _check(self.L, self.L.hgpu_upload_state(self.h, _ptr(p), _ptr(pf, ctypes.c_int), float(t), float(dt)))

    def download_state(self, out=None):
        if out is None:
            p = np.empty(self.nt + (NPR,))
            pf = np.empty(self.nt, dtype=np.int32)
        else:
            p, pf = out
        t = ctypes.c_double()
        dt = ctypes.c_double()
        _check(self.L, self.L.hgpu_download_state(self.h, _ptr(p), _ptr(pf, ctypes.c_int), ctypes.byref(t),
                                                  ctypes.byref(dt)))
        return p, pf, t.value, dt.value

    def step_ch(self, nsteps=1, stats=True):
        st = hgpu_stats()
        _check(self.L, self.L.hgpu_step_ch(self.h, int(nsteps), ctypes.byref(st) if stats else None))
        return st

    def upload_conserved(self, u):
        """Set the conserved state unew (restart's unew; evolved by the
        finite-volume scheme, reported until the next step otherwise)."""
        u = _contig(u, np.float64)
        assert u.shape == self.nt + (NPR,)
        _check(self.L, self.L.hgpu_upload_conserved(self.h, _ptr(u)))

    def download_bsqflags(self):
        """hgpu_download_bsqflags: the FLAGBSQORHO and FLAGBSQOU pflag slots,
        int32 [n1+2g][n2+2g][n3+2g][2]."""
        f = np.zeros(self.nt + (2,), dtype=np.int32)
        _check(self.L, self.L.hgpu_download_bsqflags(self.h, _ptr(f, ctypes.c_int)))
        return f

    def upload_active(self, p, t, dt):
        """hgpu_upload_active: active-zone primitives [n1][n2][n3][8]; the
        ghosts by bound_prim on the device."""
        p = _contig(p, np.float64)
        assert p.shape == tuple(self.n) + (NPR,)
        _check(self.L, self.L.hgpu_upload_active(self.h, _ptr(p), float(t), float(dt)))

    def download_active(self, out=None):
        """hgpu_download_active: (p [n1][n2][n3][8], pflag [n1][n2][n3], t, dt)."""
        if out is None:
            out = (np.empty(tuple(self.n) + (NPR,)), np.empty(tuple(self.n), dtype=np.int32))
        p, f = out
        t, dt = ctypes.c_double(), ctypes.c_double()
        _check(self.L, self.L.hgpu_download_active(self.h, _ptr(p), _ptr(f, ctypes.c_int), ctypes.byref(t),
                                                   ctypes.byref(dt)))
        return p, f, t.value, dt.value

    def pinned_active_buffers(self):
        """Page-locked host arrays for the active-zone transfers."""
        n = tuple(self.n)
        return self._pinned_array(n + (NPR,), np.float64), self._pinned_array(n, np.int32)

    def set_bondi_boundaries(self, table):
        """hgpu_set_bondi_boundaries: [2][ng+1][n2][49] coordinate data (r,
        dx/dx', its inverse, the Kerr-Schild metric) of the x1 edge and ghost
        zones, for the Bondi-integral boundaries."""
        table = _contig(table, np.float64)
        g1 = self.g[0]
        assert table.shape == (2, g1 + 1, self.n[1], 49)
        _check(self.L, self.L.hgpu_set_bondi_boundaries(self.h, _ptr(table)))

    def download_failfloorcount(self, clear=False):
        """hgpu_download_failfloorcount: int64 [n1+2g][n2+2g][n3+2g][9], the
        reference's failfloorcount categories per zone."""
        c = np.zeros(self.nt + (9,), dtype=np.int64)
        _check(self.L, self.L.hgpu_download_failfloorcount(self.h, _ptr(c, ctypes.c_longlong), int(bool(clear))))
        return c

    def write_rdump(self, path, header=b"", binary=False):
        """hgpu_write_rdump: the reference's restart dump of the current state
        (header bytes, then p[0..7] and unew[0..7] of every active zone)."""
        header = bytes(header)
        _check(self.L, self.L.hgpu_write_rdump(self.h, os.fsencode(path), header, len(header), int(bool(binary))))

    def read_rdump(self, path, t, dt, header_bytes=0, binary=False):
        """hgpu_read_rdump: state from a restart dump, ghosts by bound_prim."""
        _check(self.L, self.L.hgpu_read_rdump(self.h, os.fsencode(path), int(header_bytes), int(bool(binary)),
                                              float(t), float(dt)))

    def download_conserved(self):
        """The conserved state after the last step (the reference's unew)."""
        u = np.empty(self.nt + (NPR,))
        _check(self.L, self.L.hgpu_download_conserved(self.h, _ptr(u)))
        return u

    def diagnostics(self):
        """hgpu_diagnostics as a dict."""
        dg = hgpu_diag()
        _check(self.L, self.L.hgpu_diagnostics(self.h, ctypes.byref(dg)))
        return {"t": dg.t, "dt": dg.dt, "integral": list(dg.integral), "divb_max": dg.divb_max,
                "divb_avg": dg.divb_avg, "nfail": dg.nfail, "nfloor": dg.nfloor, "nsteps": dg.nsteps,
                "divb_max_interior": dg.divb_max_interior}

    def step_graph(self, nsteps=1, stats=True):
        """step_ch as replays of one captured CUDA graph per time step."""
        st = hgpu_stats()
        _check(self.L, self.L.hgpu_step_graph(self.h, int(nsteps), ctypes.byref(st) if stats else None))
        return st

    def autotune(self):
        """hgpu_autotune: pick the resident-block variant of each heavy FP64
        kernel and the WENO5 tile shape per direction on this state; returns
        {family: {"minb": chosen, "ms": {candidate: ms}}, "weno_tiles": {dir:
        {"lb": cells, "lines": lines, "ms": per launch}}}."""
        tu = hgpu_tuning()
        _check(self.L, self.L.hgpu_autotune(self.h, ctypes.byref(tu)))
        out = {}
        for fam in ("flux", "weno", "update", "invert"):
            cand = list(getattr(tu, fam + "_cand"))
            ms = list(getattr(tu, fam + "_ms"))
            out[fam] = {"minb": getattr(tu, fam + "_minb"), "ms": {str(c): round(m, 4) for c, m in zip(cand, ms)}}
        out["weno_tiles"] = {str(q): {"lb": tu.weno_lb[q], "lines": tu.weno_lines[q],
                                      "ms": round(tu.weno_tile_ms[q], 4)} for q in (1, 2, 3) if tu.weno_lb[q] > 0}
        return out

    def set_tuning(self, minb):
        """hgpu_set_tuning: {"flux": 4, "weno": 3, "update": 3, "invert": 1} (blocks per SM), optionally
        "weno_tiles": {dir: (cells per tile, lines per tile)}."""
        tu = hgpu_tuning()
        tu.flux_minb, tu.weno_minb = int(minb["flux"]), int(minb["weno"])
        tu.update_minb, tu.invert_minb = int(minb["update"]), int(minb["invert"])
        for q, (lb, lines) in (minb.get("weno_tiles") or {}).items():
            tu.weno_lb[int(q)], tu.weno_lines[int(q)] = int(lb), int(lines)
        _check(self.L, self.L.hgpu_set_tuning(self.h, ctypes.byref(tu)))

    def advance_stage(self, timeorder):
        st = hgpu_stats()
        ndt = ctypes.c_double()
        _check(self.L, self.L.hgpu_advance_stage(self.h, int(timeorder), ctypes.byref(ndt), ctypes.byref(st)))
        return ndt.value, st

    def fluxcalc(self, which=0):
        F = [np.zeros(self.nt + (NPR,)) for _ in range(3)]
        nd = [ctypes.c_double() for _ in range(3)]
        _check(self.L, self.L.hgpu_fluxcalc(self.h, int(which), _ptr(F[0]), _ptr(F[1]), _ptr(F[2]),
                                            *[ctypes.byref(x) for x in nd]))
        return F, [x.value for x in nd]

    def init_dt(self):
        dt = ctypes.c_double()
        _check(self.L, self.L.hgpu_init_dt(self.h, ctypes.byref(dt)))
        return dt.value

    def time(self):
        t = ctypes.c_double()
        dt = ctypes.c_double()
        _check(self.L, self.L.hgpu_download_state(self.h, None, None, ctypes.byref(t), ctypes.byref(dt)))
        return t.value, dt.value

    def step_ch_timed(self, nsteps):
        st = hgpu_stats()
        ms = ctypes.c_float()
        _check(self.L, self.L.hgpu_step_ch_timed(self.h, int(nsteps), ctypes.byref(ms), ctypes.byref(st)))
        return ms.value, st

    def set_profiling(self, on):
        _check(self.L, self.L.hgpu_set_profiling(self.h, 1 if on else 0))

    def kernel_times(self):
        n = 32
        names = (ctypes.c_char_p * n)()
        ms = (ctypes.c_double * n)()
        cnt = (ctypes.c_longlong * n)()
        k = self.L.hgpu_kernel_times(self.h, names, ms, cnt, n)
        if k < 0:
            raise HarmGPUError(-k, self.L.hgpu_last_error().decode(errors="replace"))
        return {names[i].decode(): {"ms": ms[i], "launches": cnt[i]} for i in range(k)}

    def launch_count(self):
        return self.L.hgpu_launch_count(self.h)

    def _pinned_array(self, shape, dtype):
        """A page-locked host array owned by this object."""
        nbytes = int(np.prod(shape)) * np.dtype(dtype).itemsize
        ptr = ctypes.c_void_p()
        _check(self.L, self.L.hgpu_alloc_pinned(nbytes, ctypes.byref(ptr)))
        self._pinned = getattr(self, "_pinned", []) + [ptr]
        arr = np.ctypeslib.as_array(ctypes.cast(ptr, ctypes.POINTER(ctypes.c_byte)), shape=(nbytes,))
        return arr.view(dtype).reshape(shape)

    def pinned_state_buffers(self):
        """Primitive and flag arrays in page-locked host memory (owned by this object)."""
        return self._pinned_array(self.nt + (NPR,), np.float64), self._pinned_array(self.nt, np.int32)

    def bound_prim(self, which=0):
        _check(self.L, self.L.hgpu_bound_prim(self.h, int(which)))

    def post_fixup(self, finalstep=1):
        """hgpu_post_fixup: bound_pflag, fixup_checksolution, fixup_utoprim on
        the state and its flags; returns hgpu_stats."""
        st = hgpu_stats()
        _check(self.L, self.L.hgpu_post_fixup(self.h, int(finalstep), ctypes.byref(st)))
        return st

    def sync(self):
        _check(self.L, self.L.hgpu_sync(self.h))

    def active(self, a):
        g = self.g
        return a[g[0]:g[0] + self.n[0], g[1]:g[1] + self.n[1], g[2]:g[2] + self.n[2]]


def utoprim_batch(U, gcov, gcon, gdet, guess, gam, gammafail, version="2DFINAL"):
    """Batched Utoprimgen on the GPU (hgpu_utoprimgen_batch): version
    "2DFINAL" (UTOPRIM2DFINAL) or "JON" (UTOPRIMJONNONRELCOMPAT)."""
    L = load_library()
    U = _contig(U, np.float64)
    gcov = _contig(gcov, np.float64)
    gcon = _contig(gcon, np.float64)
    gdet = _contig(gdet, np.float64)
    pr = np.array(guess, dtype=np.float64, order="C", copy=True)
    n = U.shape[0]
    pflag = np.zeros(n, dtype=np.int32)
    it = ctypes.c_longlong(0)
    _check(L, L.hgpu_utoprimgen_batch(_ptr(U), _ptr(gcov), _ptr(gcon), _ptr(gdet), _ptr(pr),
                                      _ptr(pflag, ctypes.c_int), n, gam, gammafail,
                                      UTOPRIM[version] if isinstance(version, str) else int(version),
                                      ctypes.byref(it)))
    return pr, pflag, it.value


def fp64_peak_tflops():
    """Measured FP64 DMUL/DADD issue rate of the current GPU (hgpu_fp64_peak)."""
    L = load_library()
    v = ctypes.c_double()
    _check(L, L.hgpu_fp64_peak(ctypes.byref(v)))
    return v.value


class HarmBatch(HarmGPU):
    """Many independent 1D problems in one context (hgpu_create_batch): one
    launch of every kernel advances all of them, each with its own gamma, dx,
    t, dt and end time.  The state is one concatenated 1D line; `layout`
    gives each instance's first active zone (relative to the line's first
    active zone) and `split` cuts a line array into per-instance arrays
    with their own ng ghosts."""

    def __init__(self, n1s, dx1s, gams, tfs, ng=3, lim="MC", flux="HLL", precision="fp64", cour=0.5, safe=1.3,
                 defcon=1.0, rhominlimit=1e-20, uuminlimit=1e-20, gammamax=25.0, gammafail=2500.0, utoprim="2DFINAL",
                 timeorder=2):
        self.L = load_library()
        n1s = np.ascontiguousarray(n1s, dtype=np.int32)
        self.ninst = len(n1s)
        c = hgpu_config()
        c.n1, c.n2, c.n3, c.ng = int(n1s.sum() + 2 * ng * (self.ninst - 1)), 1, 1, ng
        c.lim = LIM[lim] if isinstance(lim, str) else int(lim)
        c.fluxmethod = FLUX[flux] if isinstance(flux, str) else int(flux)
        for i, b in enumerate(("OUTFLOW_COPY", "OUTFLOW_COPY", "OUTFLOW", "OUTFLOW", "OUTFLOW", "OUTFLOW")):
            c.bc[i] = BC[b]
        c.precision = PREC[precision] if isinstance(precision, str) else int(precision)
        c.dx[1] = c.dx[2] = c.dx[3] = 1.0
        c.gam, c.cour, c.safe, c.defcon, c.tf = 4.0 / 3.0, cour, safe, defcon, 0.0
        c.rhominlimit, c.uuminlimit, c.gammamax, c.gammafail = rhominlimit, uuminlimit, gammamax, gammafail
        c.utoprimversion = UTOPRIM[utoprim] if isinstance(utoprim, str) else int(utoprim)
        c.timeorder = int(timeorder)
        self.cfg = c
        self.n = (c.n1, 1, 1)
        self.g = (ng, 0, 0)
        self.s = (1, 0, 0)
        self.nt = (c.n1 + 2 * ng, 1, 1)
        self.gt = (self.nt[0] + 1, 1)
        self.n1s = n1s
        self.ng = ng
        h = ctypes.c_void_p()
        _check(self.L, self.L.hgpu_create_batch(ctypes.byref(c), self.ninst, _ptr(n1s, ctypes.c_int),
                                                _ptr(_contig(dx1s, np.float64)), _ptr(_contig(gams, np.float64)),
                                                _ptr(_contig(tfs, np.float64)), ctypes.byref(h)))
        self.h = h
        i0 = np.zeros(self.ninst, dtype=np.int32)
        _check(self.L, self.L.hgpu_batch_layout(self.h, _ptr(i0, ctypes.c_int)))
        self.i0 = i0

    def status(self):
        t = np.zeros(self.ninst)
        dt = np.zeros(self.ninst)
        done = np.zeros(self.ninst, dtype=np.int32)
        nd = ctypes.c_int()
        _check(self.L, self.L.hgpu_batch_status(self.h, _ptr(t), _ptr(dt), _ptr(done, ctypes.c_int),
                                                ctypes.byref(nd)))
        return t, dt, done, nd.value

    def set_time(self, t, dt):
        """hgpu_batch_set_time: every instance's t and dt."""
        _check(self.L, self.L.hgpu_batch_set_time(self.h, _ptr(_contig(t, np.float64)), _ptr(_contig(dt, np.float64))))

    def split(self, line):
        """Per-instance views (own ghosts included) of a line array [nt1, ...]."""
        ng = self.ng
        return [line[ng + i0 - ng: ng + i0 + n + ng] for i0, n in zip(self.i0, self.n1s)]

    def join(self, parts, fill=None):
        """The inverse of split: one line array from per-instance arrays."""
        shape = (self.nt[0],) + parts[0].shape[1:]
        out = np.zeros(shape, dtype=parts[0].dtype) if fill is None else np.full(shape, fill, dtype=parts[0].dtype)
        ng = self.ng
        for part, i0, n in zip(parts, self.i0, self.n1s):
            out[ng + i0 - ng: ng + i0 + n + ng] = part
        return out

    def run(self, check_every=50, max_steps=1_000_000):
        """Advance until every instance has reached its end time (CUDA-graph
        replays).  Returns (batch steps, device ms, steps per instance, ms at
        which each instance was seen finished)."""
        steps = ctypes.c_int()
        ms = ctypes.c_float()
        per = np.zeros(self.ninst, dtype=np.int32)
        fin = np.zeros(self.ninst, dtype=np.float32)
        _check(self.L, self.L.hgpu_batch_run(self.h, int(check_every), int(max_steps), ctypes.byref(steps),
                                             ctypes.byref(ms), _ptr(per, ctypes.c_int), _ptr(fin, ctypes.c_float)))
        return steps.value, ms.value, per, fin


def make_config(n, ng, dx, lim="MC", flux="HLL", bc=("OUTFLOW", "OUTFLOW", "POLARAXIS", "POLARAXIS", "PERIODIC",
                "PERIODIC"), precision="fp64", gam=4.0 / 3.0, cour=0.8, safe=1.3, defcon=1.0, tf=2000.0,
                rhominlimit=1e-20, uuminlimit=1e-20, gammamax=25.0, gammafail=2500.0, timeorder=2,
                utoprim="2DFINAL", doenoflux="NOENOFLUX"):
    c = hgpu_config()
    c.timeorder = int(timeorder)
    c.utoprimversion = UTOPRIM[utoprim] if isinstance(utoprim, str) else int(utoprim)
    c.doenoflux = DOENOFLUX[doenoflux] if isinstance(doenoflux, str) else int(doenoflux)
    c.n1, c.n2, c.n3 = n
    c.ng = ng
    c.lim = LIM[lim] if isinstance(lim, str) else int(lim)
    c.fluxmethod = FLUX[flux] if isinstance(flux, str) else int(flux)
    for i, b in enumerate(bc):
        c.bc[i] = BC[b] if isinstance(b, str) else int(b)
    c.precision = PREC[precision] if isinstance(precision, str) else int(precision)
    for i in range(3):
        c.dx[i + 1] = float(dx[i])
    c.gam, c.cour, c.safe, c.defcon, c.tf = gam, cour, safe, defcon, tf
    c.rhominlimit, c.uuminlimit, c.gammamax, c.gammafail = rhominlimit, uuminlimit, gammamax, gammafail
    return c


def context_bytes(cfg):
    return int(load_library().hgpu_context_bytes(ctypes.byref(cfg)))


class HarmServer:
    """The serving loop (hgpu_server_*): submit solves at any time, call
    poll() repeatedly, collect results of finished solves."""

    def __init__(self, max_device_bytes, max_active=64, steps_per_chunk=8):
        self.L = load_library()
        h = ctypes.c_void_p()
        _check(self.L, self.L.hgpu_server_create(int(max_device_bytes), int(max_active), int(steps_per_chunk),
                                                 ctypes.byref(h)))
        self.h = h
        self.shapes = {}
        self._held = {}

    def submit(self, dom, tf, precision="fp64", borrow=True):
        """dom: an object with the Domain/Problem attributes (n, ng, dx, lim, ...).
        borrow: the server reads dom's arrays at admission instead of copying
        them now (they are held here until the result is released)."""
        inv_bc = {v: k for k, v in BC.items()}
        bc = tuple(inv_bc[b] if not isinstance(b, str) else b for b in dom.bc)
        c = make_config(dom.n, dom.ng, dom.dx, lim=dom.lim, flux=dom.flux, bc=bc, precision=precision, gam=dom.gam,
                        cour=dom.cour, safe=dom.safe, defcon=dom.defcon, tf=tf, rhominlimit=dom.rhominlimit,
                        uuminlimit=dom.uuminlimit, gammamax=dom.gammamax, gammafail=dom.gammafail)
        arrs = [_contig(a, np.float64) for a in (dom.gcov, dom.gcon, dom.gcovpert, dom.gdet, dom.conn, dom.floors,
                                                 dom.p)]
        rid = ctypes.c_longlong()
        fn = self.L.hgpu_server_submit_borrowed if borrow else self.L.hgpu_server_submit
        _check(self.L, fn(self.h, ctypes.byref(c), *[_ptr(a) for a in arrs], float(tf), ctypes.byref(rid)))
        self.shapes[rid.value] = dom.p.shape
        if borrow:
            self._held[rid.value] = arrs
        return rid.value

    def poll(self):
        p, a, f = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _check(self.L, self.L.hgpu_server_poll(self.h, ctypes.byref(p), ctypes.byref(a), ctypes.byref(f)))
        return p.value, a.value, f.value

    def result(self, rid):
        """(p, pflag, t, steps, queue_ms, run_ms) of a finished solve, or None while it runs."""
        shape = self.shapes[rid]
        t, q, r = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        steps = ctypes.c_longlong()
        # a cheap check first: no arrays while the solve runs
        rc = self.L.hgpu_server_result(self.h, rid, None, None, ctypes.byref(t), ctypes.byref(steps),
                                       ctypes.byref(q), ctypes.byref(r))
        if rc == 1:  # HGPU_E_INVALID: not finished
            return None
        _check(self.L, rc)
        p = np.empty(shape)
        pf = np.empty(shape[:-1], dtype=np.int32)
        _check(self.L, self.L.hgpu_server_result(self.h, rid, _ptr(p), _ptr(pf, ctypes.c_int), ctypes.byref(t),
                                                 ctypes.byref(steps), ctypes.byref(q), ctypes.byref(r)))
        return p, pf, t.value, steps.value, q.value, r.value

    def release(self, rid):
        _check(self.L, self.L.hgpu_server_release(self.h, rid))
        self.shapes.pop(rid, None)
        self._held.pop(rid, None)

    def close(self):
        if getattr(self, "h", None):
            self.L.hgpu_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
