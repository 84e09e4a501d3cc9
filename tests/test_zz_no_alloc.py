"""hgpu_utoprim_batch_noalloc: the batched con-to-prim inversion for callers
that cannot allocate device memory (their device memory is held by another
allocator's pool, or they invert small batches so often -- as the reference
calls Utoprimgen zone by zone -- that cudaMalloc/cudaFree would dominate).

Checked through the C ABI against the allocating entry point
hgpu_utoprim_batch on two calls in a row (the second call must not see the
first call's leftovers in the shared scratch array), with the exact equality
the other parity tests use.  This file is collected last on purpose."""
import ctypes

import numpy as np
import pytest

from harm_finalwham_b200.gpu import load_library, utoprim_batch
from tests.fixtures import load

pytestmark = pytest.mark.gpu

HGPU_E_INVALID = 1
MAX_ZONES = 16384

_dp = ctypes.POINTER(ctypes.c_double)


def _ptr(a, t=ctypes.c_double):
    return a.ctypes.data_as(ctypes.POINTER(t))


def noalloc(U, gcov, gcon, gdet, guess, gam, gammafail):
    L = load_library()
    f = L.hgpu_utoprim_batch_noalloc
    f.argtypes = [_dp, _dp, _dp, _dp, _dp, ctypes.POINTER(ctypes.c_int), ctypes.c_longlong, ctypes.c_double,
                  ctypes.c_double, ctypes.POINTER(ctypes.c_longlong)]
    f.restype = ctypes.c_int
    pr = np.array(guess, dtype=np.float64, order="C", copy=True)
    n = U.shape[0]
    pflag = np.full(n, -7, dtype=np.int32)
    it = ctypes.c_longlong(-1)
    rc = f(_ptr(U), _ptr(gcov), _ptr(gcon), _ptr(gdet), _ptr(pr), _ptr(pflag, ctypes.c_int), n, gam, gammafail,
           ctypes.byref(it))
    return rc, pr, pflag, it.value


def inputs(seed, scale):
    """Inversion inputs from the 3D torus fixture: CENT metrics and perturbed
    conserved vectors from the reference state."""
    pr, ref = load("torus3d_12x12x6_mc_laxf")
    g0 = pr.g
    p = ref[10]["p"][g0[0]:g0[0] + pr.n[0], g0[1]:g0[1] + pr.n[1], g0[2]:g0[2] + pr.n[2]].reshape(-1, 8)
    ii, jj = np.meshgrid(np.arange(pr.n[0]), np.arange(pr.n[1]), indexing="ij")
    gi = (ii + g0[0]).ravel().repeat(pr.n[2])
    gj = (jj + g0[1]).ravel().repeat(pr.n[2])
    gcov = np.ascontiguousarray(pr.gcov[gi, gj, 7].reshape(-1, 16))
    gcon = np.ascontiguousarray(pr.gcon[gi, gj, 7].reshape(-1, 16))
    gdet = np.ascontiguousarray(pr.gdet[gi, gj, 7])
    rng = np.random.default_rng(seed)
    U = p * gdet[:, None] * (1.0 + scale * rng.standard_normal(p.shape))
    U[:, 1] = -np.abs(U[:, 1]) - U[:, 0]
    guess = p * (1.0 + 0.01 * rng.standard_normal(p.shape))
    return np.ascontiguousarray(U), gcov, gcon, gdet, np.ascontiguousarray(guess), pr.gam, pr.gammafail


def test_noalloc_matches_allocating_entry_point_twice():
    for call, (seed, scale) in enumerate([(11, 0.05), (12, 0.2)]):
        U, gcov, gcon, gdet, guess, gam, gfail = inputs(seed, scale)
        if call == 1:  # a smaller second batch: stale tail entries must not matter
            U, gcov, gcon, gdet, guess = U[:500], gcov[:500], gcon[:500], gdet[:500], guess[:500]
        rc, a, fa, ia = noalloc(U, gcov, gcon, gdet, guess, gam, gfail)
        assert rc == 0, load_library().hgpu_last_error()
        b, fb, ib = utoprim_batch(U, gcov, gcon, gdet, guess, gam, gfail)
        assert np.array_equal(fa, fb), f"pflag differs on call {call}"
        same = (a == b) | (np.isnan(a) & np.isnan(b))
        assert same.all(), f"{np.count_nonzero(~same)} values differ on call {call}"
        assert ia == ib


def test_noalloc_takes_no_device_memory():
    # the device's free memory is the same before and after further calls
    # (the first call, which looks up the scratch array, comes first)
    import torch
    U, gcov, gcon, gdet, guess, gam, gfail = inputs(13, 0.1)
    rc, *_ = noalloc(U, gcov, gcon, gdet, guess, gam, gfail)
    assert rc == 0, load_library().hgpu_last_error()
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(3):
        rc, *_ = noalloc(U, gcov, gcon, gdet, guess, gam, gfail)
        assert rc == 0, load_library().hgpu_last_error()
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0


def test_noalloc_rejects_oversized_batch():
    n = MAX_ZONES + 1
    z = np.zeros((n, 8))
    g = np.zeros((n, 16))
    d = np.ones(n)
    rc, _, _, _ = noalloc(z, g, g, d, z, 4.0 / 3.0, 2500.0)
    assert rc == HGPU_E_INVALID
    assert b"HGPU_NOALLOC_MAX_ZONES" in load_library().hgpu_last_error()
