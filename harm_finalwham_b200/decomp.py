"""A domain split along x3 over ranks: the reference's MPI decomposition.

The reference places ncpux1 x ncpux2 x ncpux3 ranks on the grid
(init_placeongrid, mpi_init.c:226), fills ghost zones that face another rank
in bound_prim / bound_pflag (bound_mpi boundmpi.c:6-180: pack, Isend/Irecv,
unpack boundmpi.c:185-290; bound_mpi_int boundmpiint.c:4) and takes the
minimum of dt over ranks (mpifmin, step_ch.c:243, mpi_fileio.c:1905).

Here the split is along x3 (the periodic azimuth; the metric does not depend
on it, so every rank uploads the same per-(i,j) geometry).  Each subdomain is
a HarmGPU context driven through the phase entry points of the C ABI
(hgpu_stage_advance / hgpu_stage_fixup / hgpu_step_end); a transport moves
the x3 ghost planes and the per-direction ndt minima between the phases:

* LocalTransport: all subdomains in one process on one device (device
  copies); used to check that a split run reproduces the whole-domain run.
* CollectiveTransport: one subdomain per rank of a torch.distributed process
  group: NCCL point-to-point sends of the packed planes to the x3 neighbours
  and an all-reduce(MIN) of the ndt minima; with the gloo backend and host
  tensors the same code moves planes between CPU ranks.

The minimum over ranks is taken per direction before the three directions
are combined, so a split run takes the whole-domain dt; the reference
combines per rank first (step_ch.c:243) and its split runs can take a
slightly smaller dt than its one-rank runs.
"""
import contextlib
import ctypes
import dataclasses

import numpy as np

from .gpu import HarmGPU, hgpu_stats, _check

NPR = 8


def split_x3(dom, nranks, rank):
    """Rank `rank`'s slab of a domain with the reference's host layouts.

    The slab keeps the full x1/x2 extent (with ghosts) and n3/nranks active
    planes; its x3 ghost planes are the periodic neighbours' planes, as the
    first exchange would fill them.
    """
    n1, n2, n3 = dom.n
    if n3 < 2 or n3 % nranks:
        raise ValueError(f"n3={n3} does not split into {nranks} slabs")
    nl = n3 // nranks
    g3 = dom.g[2]
    if nl < g3:
        raise ValueError(f"slab of {nl} planes is thinner than the {g3} ghost planes")
    k = (rank * nl + np.arange(-g3, nl + g3)) % n3 + g3
    sub = dataclasses.replace(dom, n=(n1, n2, nl))
    for a in ("timeorder", "utoprim", "doenoflux"):  # scheme options set as plain attributes
        if hasattr(dom, a):
            setattr(sub, a, getattr(dom, a))
    sub.p = np.ascontiguousarray(dom.p[:, :, k])
    sub.pflag = None if dom.pflag is None else np.ascontiguousarray(dom.pflag[:, :, k])
    if getattr(dom, "u", None) is not None:
        sub.u = np.ascontiguousarray(dom.u[:, :, k])
    sub.meta = dict(dom.meta, x3_rank=rank, x3_ranks=nranks)
    return sub


def join_x3(parts):
    """Active zones of the whole domain from its slabs' active zones."""
    return np.concatenate(parts, axis=2)


class SlabContext:
    """What a transport needs from one subdomain (a HarmGPU context)."""

    def __init__(self, ctx):
        import torch
        self.ctx = ctx
        L, h = ctx.L, ctx.h
        nb = ctypes.c_size_t()
        _check(L, L.hgpu_halo_bytes(h, ctypes.byref(nb)))
        self.nbytes = nb.value
        s = ctypes.c_void_p()
        _check(L, L.hgpu_stream(h, ctypes.byref(s)))
        self.stream = torch.cuda.ExternalStream(s.value)
        self.device = torch.device("cuda", torch.cuda.current_device())

    def pack(self, stage, side, with_pflag, buf):
        _check(self.ctx.L, self.ctx.L.hgpu_halo_pack(self.ctx.h, stage, side, int(with_pflag), buf.data_ptr()))

    def unpack(self, stage, side, with_pflag, buf):
        _check(self.ctx.L, self.ctx.L.hgpu_halo_unpack(self.ctx.h, stage, side, int(with_pflag), buf.data_ptr()))

    def ndt_pack(self, buf):
        _check(self.ctx.L, self.ctx.L.hgpu_ndt_pack(self.ctx.h, buf.data_ptr()))

    def ndt_unpack(self, buf):
        _check(self.ctx.L, self.ctx.L.hgpu_ndt_unpack(self.ctx.h, buf.data_ptr()))

    def sync(self):
        _check(self.ctx.L, self.ctx.L.hgpu_sync(self.ctx.h))


def _halo_len(sub, with_pflag):
    """Bytes of one face's halo with or without the pflag planes."""
    per_plane_zone = NPR * 8 + 4
    nzones = sub.nbytes // per_plane_zone
    return nzones * (NPR * 8 + (4 if with_pflag else 0))


class LocalTransport:
    """All slabs in this process on one device; slab r's x3 neighbours are
    r-1 and r+1 (mod the slab count).  Between the packs and the unpacks every
    slab's stream is synchronised, so the slabs never wait on one another
    inside a kernel."""

    def __init__(self, subs):
        import torch
        self.subs = subs
        self.lo = [torch.empty(s.nbytes, dtype=torch.uint8, device=s.device) for s in subs]
        self.hi = [torch.empty(s.nbytes, dtype=torch.uint8, device=s.device) for s in subs]
        self.ndt = [torch.empty(3, dtype=torch.int64, device=s.device) for s in subs]

    def exchange(self, stage, with_pflag):
        n = len(self.subs)
        for r, s in enumerate(self.subs):
            s.pack(stage, 0, with_pflag, self.lo[r])
            s.pack(stage, 1, with_pflag, self.hi[r])
        for s in self.subs:
            s.sync()
        for r, s in enumerate(self.subs):
            s.unpack(stage, 0, with_pflag, self.hi[(r - 1) % n])
            s.unpack(stage, 1, with_pflag, self.lo[(r + 1) % n])
        for s in self.subs:
            s.sync()

    def ndt_min(self):
        import torch
        for r, s in enumerate(self.subs):
            s.ndt_pack(self.ndt[r])
        for s in self.subs:
            s.sync()
        m = self.ndt[0].clone()
        for b in self.ndt[1:]:
            m = torch.minimum(m, b)
        torch.cuda.synchronize()
        for s in self.subs:
            s.ndt_unpack(m)
        for s in self.subs:
            s.sync()


class CollectiveTransport:
    """One slab per rank of the default torch.distributed group.

    Rank r sends its upper edge planes to rank r+1 and its lower edge planes
    to rank r-1 (mod the world size) and receives the matching ghosts, all in
    one batch of point-to-point operations; with one rank the planes wrap
    onto itself.  The ndt minima are reduced with all_reduce(MIN) on their
    order-preserving 64-bit patterns.  On a GPU the operations are issued on
    the context's stream, so they follow the pack and precede the unpack
    without a host synchronisation.
    """

    def __init__(self, sub, group=None, host_staging=None):
        import torch
        import torch.distributed as dist
        self.dist = dist
        self.sub = sub
        self.group = group
        # without a process group the one slab's planes wrap onto itself
        up = dist.is_available() and dist.is_initialized()
        self.rank = dist.get_rank(group) if up else 0
        self.world = dist.get_world_size(group) if up else 1
        dev = getattr(sub, "device", torch.device("cpu"))
        self.send_lo = torch.empty(sub.nbytes, dtype=torch.uint8, device=dev)
        self.send_hi = torch.empty_like(self.send_lo)
        self.recv_lo = torch.empty_like(self.send_lo)
        self.recv_hi = torch.empty_like(self.send_lo)
        self.ndt = torch.empty(3, dtype=torch.int64, device=dev)
        # a backend that cannot move device memory (gloo) gets the planes
        # through host copies, as a non-CUDA-aware MPI would (blocking copies
        # on the context's stream; pageable buffers, so that no host-allocator
        # events outlive the context)
        if host_staging is None:
            host_staging = up and dev.type == "cuda" and dist.get_backend(group) != "nccl"
        self.staged = bool(host_staging)
        if self.staged:
            self.h = {k: torch.empty(sub.nbytes, dtype=torch.uint8) for k in ("send_lo", "send_hi", "recv_lo",
                                                                               "recv_hi")}
            self.h_ndt = torch.empty(3, dtype=torch.int64)

    def _on_stream(self):
        import torch
        st = getattr(self.sub, "stream", None)
        return torch.cuda.stream(st) if st is not None else contextlib.nullcontext()

    def _peer(self, r):
        return self.dist.get_global_rank(self.group, r) if self.group is not None else r

    def exchange(self, stage, with_pflag):
        dist, s = self.dist, self.sub
        nb = _halo_len(s, with_pflag)
        with self._on_stream():
            s.pack(stage, 0, with_pflag, self.send_lo)
            s.pack(stage, 1, with_pflag, self.send_hi)
            if self.world == 1:
                s.unpack(stage, 0, with_pflag, self.send_hi)
                s.unpack(stage, 1, with_pflag, self.send_lo)
                return
            left = self._peer((self.rank - 1) % self.world)
            right = self._peer((self.rank + 1) % self.world)
            # tag 0: a rank's lower edge, received as its left neighbour's
            # upper ghosts; tag 1: its upper edge, the right neighbour's lower
            # ghosts.  The issue order is the same on every rank, which is
            # what NCCL matches sends and receives by.
            if self.staged:
                h = self.h
                h["send_lo"][:nb].copy_(self.send_lo[:nb])
                h["send_hi"][:nb].copy_(self.send_hi[:nb])
                bufs = (h["send_lo"], h["recv_hi"], h["send_hi"], h["recv_lo"])
            else:
                bufs = (self.send_lo, self.recv_hi, self.send_hi, self.recv_lo)
            ops = [dist.P2POp(dist.isend, bufs[0][:nb], left, self.group, 0),
                   dist.P2POp(dist.irecv, bufs[1][:nb], right, self.group, 0),
                   dist.P2POp(dist.isend, bufs[2][:nb], right, self.group, 1),
                   dist.P2POp(dist.irecv, bufs[3][:nb], left, self.group, 1)]
            for w in dist.batch_isend_irecv(ops):
                w.wait()
            if self.staged:
                self.recv_lo[:nb].copy_(self.h["recv_lo"][:nb])
                self.recv_hi[:nb].copy_(self.h["recv_hi"][:nb])
            s.unpack(stage, 0, with_pflag, self.recv_lo)
            s.unpack(stage, 1, with_pflag, self.recv_hi)

    def ndt_min(self):
        with self._on_stream():
            self.sub.ndt_pack(self.ndt)
            if self.world > 1 and self.staged:
                self.h_ndt.copy_(self.ndt)
                self.dist.all_reduce(self.h_ndt, op=self.dist.ReduceOp.MIN, group=self.group)
                self.ndt.copy_(self.h_ndt)
            elif self.world > 1:
                self.dist.all_reduce(self.ndt, op=self.dist.ReduceOp.MIN, group=self.group)
            self.sub.ndt_unpack(self.ndt)


class SplitRun:
    """Drive the slabs of one split domain through whole time steps.

    `ctxs` are this process's slab contexts (all of them for a
    LocalTransport, one for a CollectiveTransport) and `transport` moves the
    planes between them.
    """

    def __init__(self, ctxs, transport):
        self.ctxs = list(ctxs)
        self.t = transport
        self.norders = self.ctxs[0].cfg.timeorder or 2

    @classmethod
    def local(cls, dom, nslabs, precision="fp64", init_dt=False):
        """All `nslabs` slabs of `dom` as contexts on the current device."""
        ctxs = [HarmGPU.from_problem(split_x3(dom, nslabs, r), precision=precision) for r in range(nslabs)]
        run = cls(ctxs, LocalTransport([SlabContext(c) for c in ctxs]))
        run.start(init_dt=init_dt)
        return run

    def start(self, init_dt=False):
        """bound_prim after the upload, as the reference's init does before
        the first step (the physical boundaries, then the x3 ghost planes of
        p and pflag from the neighbours), and optionally the start-up dt from
        the fluxes of the whole domain."""
        self._all("hgpu_bound_prim", 0)
        self.t.exchange(-1, True)
        if init_dt:
            for c in self.ctxs:
                _check(c.L, c.L.hgpu_dt_probe(c.h))
            self.t.ndt_min()
            for c in self.ctxs:
                _check(c.L, c.L.hgpu_step_end(c.h, 0))

    def _all(self, fn, *a):
        for c in self.ctxs:
            _check(c.L, getattr(c.L, fn)(c.h, *a))

    def step(self, nsteps=1, stats=True):
        """`nsteps` time steps of every slab; returns the summed statistics."""
        self._all("hgpu_stats_clear")
        for _ in range(nsteps):
            for s in range(self.norders):
                self._all("hgpu_stage_advance", s)
                self.t.exchange(s, True)
                self._all("hgpu_stage_fixup", s)
                self.t.exchange(s, False)
            self.t.ndt_min()
            self._all("hgpu_step_end", 1)
        return self.stats() if stats else None

    def stats(self):
        """Statistics since the last step call, summed over the slabs held here
        (synchronises)."""
        tot = hgpu_stats()
        for c in self.ctxs:
            st = hgpu_stats()
            _check(c.L, c.L.hgpu_stats_read(c.h, ctypes.byref(st)))
            tot.newton_iters += st.newton_iters
            tot.err |= st.err
            tot.nfail += st.nfail
            tot.nfixed += st.nfixed
        return tot

    def download(self):
        """(active primitives, active pflag, t, dt) of the slabs held here,
        joined along x3."""
        ps, fs, t, dt = [], [], None, None
        for c in self.ctxs:
            p, f, t, dt = c.download_state()
            ps.append(c.active(p))
            fs.append(c.active(f))
        return join_x3(ps), join_x3(fs), t, dt

    def close(self):
        for c in self.ctxs:
            c.close()
        self.ctxs = []
