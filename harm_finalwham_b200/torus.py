"""Synthetic initial data: Fishbone-Moncrief torus around a Kerr hole in
modified Kerr-Schild coordinates, the workload of the per-zone update.

Host-side input generation only (the reference does this once at init:
set_grid.c:7-151, init.fishmon.c:364-680, initbase.c:558-590); nothing here
runs per step.  The arrays follow include/harmgpu.h.  The reference's
geometry is reproduced by the same formulas (MKS map coord.c:389-420,
dxdxp coord.c:611-631, KS metric metric.c:697-760, numerical connection
metric.c:1388-1472); the generator is checked against the reference's own
dumps in tests/test_torus_generator.py.

Seeded randomness (NumPy PCG64) replaces the reference's glibc-seeded ranc():
the 4% internal-energy noise and, for 3D, the density perturbation
drho/rho = 0.02 sum_{m=1..4} A_m cos(m phi + phi_m).
"""
from dataclasses import dataclass, field

import numpy as np

NPR = 8
RHO, UU, U1, U2, U3, B1, B2, B3 = range(8)
# reference grid locations (global.h:948-955)
FACE1, FACE2, FACE3, CORN1, CORN2, CORN3, CORNT, CENT = range(8)
LOC_OFFSETS = {FACE1: (0.0, 0.5, 0.5), FACE2: (0.5, 0.0, 0.5), FACE3: (0.5, 0.5, 0.0), CORN1: (0.5, 0.0, 0.0),
               CORN2: (0.0, 0.5, 0.0), CORN3: (0.0, 0.0, 0.5), CORNT: (0.0, 0.0, 0.0), CENT: (0.5, 0.5, 0.5)}
SINGSMALL = 1e-14  # init.fishmon.h:204 (COORDSINGFIX)


@dataclass
class Domain:
    """Everything one solve needs: options, geometry, state (reference layouts)."""
    n: tuple
    ng: int
    dx: tuple
    lim: str = "MC"
    flux: str = "HLL"
    bc: tuple = (0, 0, 4, 4, 7, 7)  # X1UP,X1DN,X2UP,X2DN,X3UP,X3DN: OUTFLOW, POLARAXIS, PERIODIC
    gam: float = 4.0 / 3.0
    cour: float = 0.8
    safe: float = 1.3
    defcon: float = 1.0
    tf: float = 2000.0
    rhominlimit: float = 1e-20
    uuminlimit: float = 1e-20
    gammamax: float = 25.0
    gammafail: float = 2500.0
    gcov: np.ndarray = None
    gcon: np.ndarray = None
    gcovpert: np.ndarray = None
    gdet: np.ndarray = None
    conn: np.ndarray = None
    floors: np.ndarray = None
    p: np.ndarray = None
    pflag: np.ndarray = None
    t: float = 0.0
    dt: float = 0.0
    meta: dict = field(default_factory=dict)

    @property
    def g(self):
        return tuple(self.ng if n > 1 else 0 for n in self.n)

    @property
    def s(self):
        return tuple(1 if n > 1 else 0 for n in self.n)

    @property
    def nt(self):
        return tuple(n + 2 * g for n, g in zip(self.n, self.g))

    @property
    def gt(self):
        nt, s = self.nt, self.s
        return (nt[0] + s[0], nt[1] + s[1])

    def active(self, a):
        g = self.g
        return a[g[0]:g[0] + self.n[0], g[1]:g[1] + self.n[1], g[2]:g[2] + self.n[2]]


def rhor(a):
    return 1.0 + np.sqrt(1.0 - a * a)


def set_rin(n1, a, rout, r0=0.0):
    """setRin(setihor()) (coord.c:1079-1104): horizon at FACE1 of i=ihor+0.25."""
    ihor = 10 if n1 * 0.1 > 10 else int(n1 * 0.1)
    ftemp = (ihor + 0.25) / n1
    return r0 + ((rhor(a) - r0) / (rout - r0) ** ftemp) ** (1.0 / (1.0 - ftemp))


def _theta(x2, hslope):
    return np.where(x2 < 0.5, np.pi * x2 + ((1.0 - hslope) / 2.0) * np.sin(2.0 * np.pi * x2),
                    np.pi - (np.pi * (1.0 - x2)) + ((1.0 - hslope) / 2.0) * (-np.sin(2.0 * np.pi * (1.0 - x2))))


def _dthdx2(x2, hslope):
    return np.where(x2 < 0.5, np.pi + (1.0 - hslope) * np.pi * np.cos(2.0 * np.pi * x2),
                    np.pi + (1.0 - hslope) * np.pi * np.cos(2.0 * np.pi * (1.0 - x2)))


def gcov_mks(x1, x2, a, hslope, r0=0.0):
    """KS metric in MKS coordinates; returns (gcov[...,4,4], gcovpert_tt)."""
    r = r0 + np.exp(x1)
    th = _theta(x2, hslope)
    # keep the polar axis off exact zero (COORDSINGFIX, coord.c:571-580)
    th = np.where(np.abs(th) < SINGSMALL, np.where(th >= 0, SINGSMALL, -SINGSMALL), th)
    th = np.where(np.abs(np.pi - th) < SINGSMALL, np.where(th >= np.pi, np.pi + SINGSMALL, np.pi - SINGSMALL), th)
    s, c = np.sin(th), np.cos(th)
    s2 = s * s
    sig = r * r + a * a * c * c
    two_r = 2.0 * r / sig
    g = np.zeros(np.broadcast(x1, x2).shape + (4, 4))
    g[..., 0, 0] = -(1.0 - two_r)
    g[..., 0, 1] = g[..., 1, 0] = two_r
    g[..., 0, 3] = g[..., 3, 0] = -two_r * a * s2
    g[..., 1, 1] = 1.0 + two_r
    g[..., 1, 3] = g[..., 3, 1] = -a * s2 * (1.0 + two_r)
    g[..., 2, 2] = sig
    g[..., 3, 3] = s2 * (sig + a * a * s2 * (1.0 + two_r))
    d = np.zeros_like(g[..., 0, :])
    d[..., 0] = 1.0
    d[..., 1] = r - r0
    d[..., 2] = _dthdx2(x2, hslope)
    d[..., 3] = 2.0 * np.pi
    gm = g * d[..., :, None] * d[..., None, :]
    pert_tt = two_r  # 1 + g_tt
    return gm, pert_tt


def geometry(n1, n2, ng, a, hslope, rin, rout, x1s, dx1, dx2, dconn=1e-5):
    """gcov/gcon/gcovpert/gdet at the 8 locations and conn at CENT per (i,j)."""
    s1, s2 = int(n1 > 1), int(n2 > 1)
    g1, g2 = (ng if n1 > 1 else 0), (ng if n2 > 1 else 0)
    gt1, gt2 = n1 + 2 * g1 + s1, n2 + 2 * g2 + s2
    ii = np.arange(gt1) - g1
    jj = np.arange(gt2) - g2
    I, J = np.meshgrid(ii, jj, indexing="ij")
    gcov = np.zeros((gt1, gt2, 8, 4, 4))
    gcon = np.zeros_like(gcov)
    gcovpert = np.zeros((gt1, gt2, 8, 4))
    gdet = np.zeros((gt1, gt2, 8))
    for loc, (o1, o2, _o3) in LOC_OFFSETS.items():
        x1 = x1s + (I + o1) * dx1
        x2 = 0.0 + (J + o2) * dx2
        gm, pert = gcov_mks(x1, x2, a, hslope)
        gcov[:, :, loc] = gm
        gcon[:, :, loc] = np.linalg.inv(gm)
        gdet[:, :, loc] = np.sqrt(np.abs(np.linalg.det(gm)))
        gcovpert[:, :, loc, 0] = pert
        for q in (1, 2, 3):
            gcovpert[:, :, loc, q] = gm[..., q, q] - 1.0
    # numerical connection at CENT (metric.c:1388-1472): dg_{ij}/dX^k, then raise
    x1 = x1s + (I + 0.5) * dx1
    x2 = 0.0 + (J + 0.5) * dx2
    dg = np.zeros((gt1, gt2, 4, 4, 4))  # [i][j][k] = d g_ij / dX^k
    gh, _ = gcov_mks(x1 + dconn, x2, a, hslope)
    gl, _ = gcov_mks(x1 - dconn, x2, a, hslope)
    dg[..., 1] = (gh - gl) / (2 * dconn)
    gh, _ = gcov_mks(x1, x2 + dconn, a, hslope)
    gl, _ = gcov_mks(x1, x2 - dconn, a, hslope)
    dg[..., 2] = (gh - gl) / (2 * dconn)
    low = 0.5 * (np.einsum("...jik->...ijk", dg) + np.einsum("...kij->...ijk", dg) - np.einsum("...kji->...ijk", dg))
    conn = np.einsum("...il,...ljk->...ijk", gcon[:, :, CENT], low)
    return gcov, gcon, gcovpert, gdet, conn


def _lfish(a, r):
    return (((a ** 2 - 2.0 * a * np.sqrt(r) + r ** 2) *
             ((-2.0 * a * r * (a ** 2 - 2.0 * a * np.sqrt(r) + r ** 2)) / np.sqrt(2.0 * a * np.sqrt(r) + (-3.0 + r) * r) +
              ((a + (-2.0 + r) * np.sqrt(r)) * (r ** 3 + a ** 2 * (2.0 + r))) /
              np.sqrt(1 + (2.0 * a) / r ** 1.5 - 3.0 / r))) /
            (r ** 3 * np.sqrt(2.0 * a * np.sqrt(r) + (-3.0 + r) * r) * (a ** 2 + (-2.0 + r) * r)))


def fm_torus(n1, n2, n3, ng=3, a=0.9375, hslope=0.3, rout=40.0, rin_torus=6.0, rmax=12.0, kappa=1e-3, beta=100.0,
             gam=4.0 / 3.0, noise=0.04, phi_modes=0.02, seed=7, lim="MC", flux="HLL", cour=0.8, rhomin=1e-4,
             uumin=1e-6):
    """FM torus (init.fishmon.c:364-680) on an MKS grid (LOGRSINTH)."""
    rng = np.random.default_rng(seed)
    rin = set_rin(n1, a, rout)
    x1s = np.log(rin)
    dx1 = np.log(rout / rin) / n1
    dx2 = 1.0 / n2
    dx3 = 1.0 / n3
    dom = Domain(n=(n1, n2, n3), ng=ng, dx=(dx1, dx2, dx3), lim=lim, flux=flux, gam=gam, cour=cour)
    dom.gcov, dom.gcon, dom.gcovpert, dom.gdet, dom.conn = geometry(n1, n2, ng, a, hslope, rin, rout, x1s, dx1, dx2)
    g1, g2, g3 = dom.g
    nt = dom.nt
    gt = dom.gt
    # floors at CENT: rescaletype 0 (fixup.c:1566-1570)
    I, J = np.meshgrid(np.arange(gt[0]) - g1, np.arange(gt[1]) - g2, indexing="ij")
    rc = np.exp(x1s + (I + 0.5) * dx1)
    dom.floors = np.stack([rhomin * rc ** -1.5, uumin * rc ** -2.5], axis=-1)
    # zone centres
    i = np.arange(nt[0]) - g1
    j = np.arange(nt[1]) - g2
    k = np.arange(nt[2]) - g3
    r = np.exp(x1s + (i + 0.5) * dx1)[:, None, None] * np.ones((1, nt[1], nt[2]))
    th = _theta((j + 0.5) * dx2, hslope)[None, :, None] * np.ones((nt[0], 1, nt[2]))
    ph = (2 * np.pi * (k + 0.5) * dx3)[None, None, :] * np.ones((nt[0], nt[1], 1))
    sth, cth = np.sin(th), np.cos(th)
    l = _lfish(a, rmax)
    DD = r * r - 2.0 * r + a * a
    AA = (r * r + a * a) ** 2 - DD * a * a * sth * sth
    SS = r * r + a * a * cth * cth
    DDin = rin_torus ** 2 - 2.0 * rin_torus + a * a
    AAin = (rin_torus ** 2 + a * a) ** 2 - DDin * a * a
    SSin = rin_torus ** 2
    with np.errstate(invalid="ignore", divide="ignore"):
        lnh = (0.5 * np.log((1.0 + np.sqrt(1.0 + 4.0 * (l * l * SS * SS) * DD / (AA * sth * AA * sth))) / (SS * DD / AA))
               - 0.5 * np.sqrt(1.0 + 4.0 * (l * l * SS * SS) * DD / (AA * AA * sth * sth)) - 2.0 * a * r * l / AA
               - (0.5 * np.log((1.0 + np.sqrt(1.0 + 4.0 * (l * l * SSin * SSin) * DDin / (AAin * AAin))) /
                               (SSin * DDin / AAin))
                  - 0.5 * np.sqrt(1.0 + 4.0 * (l * l * SSin * SSin) * DDin / (AAin * AAin)) - 2.0 * a * rin_torus * l / AAin))
    lnh = np.where(r >= rin_torus, lnh, 1.0)
    intorus = (lnh >= 0.0) & (r >= rin_torus)
    hm1 = np.exp(np.where(intorus, lnh, 0.0)) - 1.0
    rho = np.where(intorus, (hm1 * (gam - 1.0) / (kappa * gam)) ** (1.0 / (gam - 1.0)), 0.0)
    u = kappa * rho ** gam / (gam - 1.0)
    if noise:
        u = u * (1.0 + noise * (rng.random(u.shape) - 0.5))
    if n3 > 1 and phi_modes:
        Am = rng.random(4)
        phm = rng.random(4) * 2 * np.pi
        pert = sum(Am[m] * np.cos((m + 1) * ph + phm[m]) for m in range(4))
        rho = rho * (1.0 + phi_modes * pert)
    # BL u^phi of the FM solution, then u^t from normalisation in BL
    with np.errstate(invalid="ignore", divide="ignore"):
        expm2chi = SS * SS * DD / (AA * AA * sth * sth)
        up1 = np.sqrt((-1.0 + np.sqrt(1.0 + 4.0 * l * l * expm2chi)) / 2.0)
        up = 2.0 * a * r * np.sqrt(1.0 + up1 * up1) / np.sqrt(AA * SS * DD) + np.sqrt(SS / AA) * up1 / sth
        gtt = -(1.0 - 2.0 * r / SS)
        gtp = -2.0 * a * r * sth * sth / SS
        gpp = AA * sth * sth / SS
        # gtt ut^2 + 2 gtp ut up + gpp up^2 = -1
        Aq, Bq, Cq = gtt, 2.0 * gtp * up, gpp * up * up + 1.0
        ut = (-Bq - np.sqrt(Bq * Bq - 4.0 * Aq * Cq)) / (2.0 * Aq)
    # BL -> KS with u^r = 0 leaves u^t, u^phi; KS -> MKS: u^X3 = u^phi / (2 pi)
    ucon = np.zeros(nt + (4,))
    ucon[..., 0] = np.where(intorus, ut, 1.0)
    ucon[..., 3] = np.where(intorus, up / (2 * np.pi), 0.0)
    # relative 4-velocity u~^i = u^i - u^t g^{ti}/g^{tt} with the CENT metric
    gconc = dom.gcon[:nt[0], :nt[1], CENT][:, :, None]
    p = np.zeros(nt + (NPR,))
    for q in (1, 2, 3):
        p[..., U1 + q - 1] = np.where(intorus, ucon[..., q] - ucon[..., 0] * gconc[..., 0, q] / gconc[..., 0, 0], 0.0)
    p[..., RHO] = rho
    p[..., UU] = u
    # normalise densities to rho_max = 1 over active zones (init.fishmon.c:566-593)
    act = (slice(g1, g1 + n1), slice(g2, g2 + n2), slice(g3, g3 + n3))
    rhomax = p[act][..., RHO].max()
    umax = np.where(r[act] > rin_torus, p[act][..., UU], 0.0).max()
    p[..., RHO] /= rhomax
    p[..., UU] /= rhomax
    umax /= rhomax
    # atmosphere (set_atmosphere fixup.c:1665-1720, VELREL4: zero velocity)
    ratm = rhomin * r ** -1.5
    uatm = uumin * r ** -2.5
    low = p[..., RHO] < ratm
    p[..., RHO] = np.where(low, ratm, p[..., RHO])
    p[..., UU] = np.where(low, uatm, p[..., UU])
    for q in (U1, U2, U3):
        p[..., q] = np.where(low, 0.0, p[..., q])
    # vector potential A_phi at CORN3 from the averaged density (init.fishmon.c:483-540)
    rp = np.pad(p[..., RHO], ((1, 1), (1, 1), (0, 0)), mode="edge")
    ravg = 0.25 * (rp[1:-1, 1:-1] + rp[:-2, 1:-1] + rp[1:-1, :-2] + rp[:-2, :-2])  # corner (i-1/2, j-1/2)
    A3 = np.maximum(ravg - 0.2, 0.0)
    A3 = np.concatenate([A3, A3[-1:]], axis=0)
    A3 = np.concatenate([A3, A3[:, -1:]], axis=1)  # (nt1+1, nt2+1, nt3)
    # vpot2field (initbase.c:558-590): B^1 = dA3/dX2 / gdet, B^2 = -dA3/dX1 / gdet
    gdc = dom.gdet[:nt[0], :nt[1], CENT][:, :, None]
    avg1 = lambda A, jo: 0.5 * (A[1:, jo:jo + nt[1]] + A[:-1, jo:jo + nt[1]])  # noqa: E731
    avg2 = lambda A, io: 0.5 * (A[io:io + nt[0], 1:] + A[io:io + nt[0], :-1])  # noqa: E731
    p[..., B1] = (avg1(A3, 1) - avg1(A3, 0)) / (gdc * dx2)
    p[..., B2] = -(avg2(A3, 1) - avg2(A3, 0)) / (gdc * dx1)
    p[..., B3] = 0.0
    # normalise to plasma beta (init.fishmon.c:597-660)
    bsq = _bsq(p, dom.gcov[:nt[0], :nt[1], CENT][:, :, None], gconc)
    bsq_max = bsq[act].max()
    beta_act = (gam - 1.0) * umax / (0.5 * bsq_max)
    norm = np.sqrt(beta_act / beta)
    p[..., B1:B3 + 1] *= norm
    dom.p = np.ascontiguousarray(p)
    dom.pflag = np.zeros(nt, dtype=np.int32)
    dom.meta = dict(a=a, hslope=hslope, rin=rin, rout=rout, x1s=x1s, rhomax=rhomax, beta=beta, seed=seed)
    return dom


def _bsq(p, gcov, gcon):
    """b^2 from primitives (get_state phys.c:849 + bsq_calc phys.c:755)."""
    alpha = 1.0 / np.sqrt(-gcon[..., 0, 0])
    ut = p[..., U1:U3 + 1]
    qsq = np.einsum("...i,...ij,...j->...", ut, gcov[..., 1:, 1:], ut)
    gamma = np.sqrt(1.0 + np.maximum(qsq, 0.0))
    ucon = np.zeros(p.shape[:-1] + (4,))
    ucon[..., 0] = gamma / alpha
    for q in (1, 2, 3):
        ucon[..., q] = ut[..., q - 1] - ucon[..., 0] * gcon[..., 0, q] * alpha * alpha
    ucov = np.einsum("...ij,...j->...i", gcov, ucon)
    B = p[..., B1:B3 + 1]
    bt = np.einsum("...i,...i->...", B, ucov[..., 1:])
    bcon = np.zeros_like(ucon)
    bcon[..., 0] = bt
    for q in (1, 2, 3):
        bcon[..., q] = (B[..., q - 1] + bt * ucon[..., q]) / ucon[..., 0]
    bcov = np.einsum("...ij,...j->...i", gcov, bcon)
    return np.einsum("...i,...i->...", bcon, bcov)
