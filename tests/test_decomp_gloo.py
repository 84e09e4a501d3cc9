"""The x3 split's host side on CPU: slabs cover the domain, and the
collective transport (the torch.distributed point-to-point exchange of the
x3 ghost planes and the all-reduce(MIN) of the ndt minima) fills every
rank's ghost planes with its periodic neighbours' edge planes, on 1, 2 and 3
gloo ranks.  The subdomain here is a host array with the device halo
buffer's layout ([8 primitives][i][j][plane] doubles, then [i][j][plane]
pflag ints)."""
import datetime
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from harm_finalwham_b200.decomp import split_x3
from harm_finalwham_b200.torus import fm_torus

NT1, NT2, G3, NL = 5, 4, 3, 4


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _global(world):
    rng = np.random.default_rng(11)
    n3 = NL * world
    return rng.random((8, NT1, NT2, n3)), rng.integers(-5, 100, (NT1, NT2, n3)).astype(np.int32)


class HostSlab:
    """A slab of a global array, laid out as a context's state (SoA, k fastest)."""

    def __init__(self, rank, world):
        gp, gf = _global(world)
        self.p = np.full((8, NT1, NT2, NL + 2 * G3), np.nan)
        self.f = np.full((NT1, NT2, NL + 2 * G3), -999, dtype=np.int32)
        self.p[..., G3:G3 + NL] = gp[..., rank * NL:(rank + 1) * NL]
        self.f[..., G3:G3 + NL] = gf[..., rank * NL:(rank + 1) * NL]
        self.nbytes = NT1 * NT2 * G3 * (8 * 8 + 4)
        self.ndt_bits = torch.tensor(np.array([1.0 + rank, 3.0 - rank, 0.5 + 0.25 * rank]).view(np.int64))

    def _planes(self, side, unpack):
        if unpack:
            return slice(0, G3) if side == 0 else slice(NL + G3, NL + 2 * G3)
        return slice(G3, 2 * G3) if side == 0 else slice(NL, NL + G3)

    def pack(self, stage, side, with_pflag, buf):
        ks = self._planes(side, False)
        b = buf.numpy()
        nd = 8 * NT1 * NT2 * G3
        b[:nd * 8] = np.ascontiguousarray(self.p[..., ks]).reshape(-1).view(np.uint8)
        if with_pflag:
            b[nd * 8:] = np.ascontiguousarray(self.f[..., ks]).reshape(-1).view(np.uint8)

    def unpack(self, stage, side, with_pflag, buf):
        ks = self._planes(side, True)
        b = buf.numpy()
        nd = 8 * NT1 * NT2 * G3
        self.p[..., ks] = b[:nd * 8].view(np.float64).reshape(8, NT1, NT2, G3)
        if with_pflag:
            self.f[..., ks] = b[nd * 8:self.nbytes].view(np.int32).reshape(NT1, NT2, G3)

    def ndt_pack(self, buf):
        buf.copy_(self.ndt_bits)

    def ndt_unpack(self, buf):
        self.ndt_bits = buf.clone()


def _rank(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        from harm_finalwham_b200.decomp import CollectiveTransport
        slab = HostSlab(rank, world)
        tr = CollectiveTransport(slab)
        tr.exchange(-1, False)
        flags_before = slab.f.copy()
        tr.exchange(0, True)
        tr.ndt_min()
        out[rank] = (slab.p.copy(), slab.f.copy(), flags_before, slab.ndt_bits.numpy().copy())
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [1, 2, 3])
def test_collective_exchange_fills_periodic_neighbour_planes(world):
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    gp, gf = _global(world)
    n3 = NL * world
    for r in range(world):
        p, f, f_before, ndt = out[r]
        k = (r * NL + np.arange(-G3, NL + G3)) % n3
        assert np.array_equal(p, gp[..., k])
        assert np.array_equal(f, gf[..., k])
        # the exchange without pflag leaves the ghost flags alone
        assert (f_before[..., :G3] == -999).all() and (f_before[..., NL + G3:] == -999).all()
        want = np.array([min(1.0 + q for q in range(world)), min(3.0 - q for q in range(world)),
                         min(0.5 + 0.25 * q for q in range(world))])
        assert np.array_equal(ndt.view(np.float64), want)


def test_slabs_cover_the_domain():
    dom = fm_torus(16, 8, 12, ng=3)
    g = dom.g
    parts = [split_x3(dom, 3, r) for r in range(3)]
    act = np.concatenate([pa.p[g[0]:g[0] + 16, g[1]:g[1] + 8, g[2]:g[2] + 4] for pa in parts], axis=2)
    assert np.array_equal(act.view(np.uint8), dom.active(dom.p).view(np.uint8))
    # ghost planes of slab 0 are the periodic images of the last planes
    assert np.array_equal(parts[0].p[:, :, :g[2]], dom.p[:, :, g[2] + 12 - g[2]:g[2] + 12])
    with pytest.raises(ValueError):
        split_x3(dom, 5, 0)
    with pytest.raises(ValueError):
        split_x3(dom, 6, 0)
