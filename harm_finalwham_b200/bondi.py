"""Spherical (Michel) accretion onto a Schwarzschild hole on the MKS grid.

The reference's Bondi problem reads tabulated solutions (bondigrid*.dat via
readin_bondi_solution, init.c:350).  Here the same transonic solution is
computed directly: polytrope p = K rho^Gamma, sonic point r_s (in M), with
the relativistic Bernoulli constant h^2 (1 - 2/r + u^2) and the mass flux
rho u r^2 fixed by the sonic conditions u_s^2 = 1/(2 r_s),
c_s^2 = u_s^2 / (1 - 3 u_s^2); the branch is subsonic outside r_s and
supersonic inside.  The radial 4-velocity is transformed to Kerr-Schild
(t_KS = t_BL + 2 ln|r/2 - 1|) and MKS, the field is a monopole with gdet B^1
constant, normalised to a plasma beta at r_s, and u carries seeded noise.
"""
import numpy as np

from . import torus

NPR = 8
CENT = torus.CENT


def _sonic(gam, rs, K=1.0):
    us2 = 0.5 / rs
    cs2 = us2 / (1.0 - 3.0 * us2)
    th = cs2 / (gam * (1.0 - cs2 / (gam - 1.0)))       # theta = p / rho
    rho = (th / K) ** (1.0 / (gam - 1.0))
    h = 1.0 + gam / (gam - 1.0) * th
    mdot = rs * rs * rho * np.sqrt(us2)                 # rho u r^2
    C2 = h * h * (1.0 - 2.0 / rs + us2)
    return mdot, C2


def solution(r, gam=4.0 / 3.0, rs=8.0, K=1.0):
    """rho(r), u(r) = |u^r| of the transonic Bondi flow."""
    mdot, C2 = _sonic(gam, rs, K)

    def F(lth, rr):
        th = np.exp(lth)
        rho = (th / K) ** (1.0 / (gam - 1.0))
        u = mdot / (rr * rr * rho)
        h = 1.0 + gam / (gam - 1.0) * th
        return h * h * (1.0 - 2.0 / rr + u * u) - C2

    r = np.asarray(r, dtype=float)
    rho = np.zeros_like(r)
    uu = np.zeros_like(r)
    lo_all, hi_all = np.log(1e-12), np.log(1e3)
    for idx, rr in np.ndenumerate(r):
        # the minimum of F over log theta separates the two branches
        a, b = lo_all, hi_all
        for _ in range(200):
            m1, m2 = a + (b - a) * 0.382, a + (b - a) * 0.618
            if F(m1, rr) < F(m2, rr):
                b = m2
            else:
                a = m1
        lc = 0.5 * (a + b)
        if F(lc, rr) >= 0.0:
            # at the sonic radius the branches touch
            th = np.exp(lc)
            rho[idx] = (th / K) ** (1.0 / (gam - 1.0))
            uu[idx] = mdot / (rr * rr * rho[idx])
            continue
        if rr >= rs:
            a, b = lc, hi_all        # subsonic: hotter, denser
        else:
            a, b = lo_all, lc        # supersonic
        fa = F(a, rr)
        for _ in range(200):
            mid = 0.5 * (a + b)
            fm = F(mid, rr)
            if (fm > 0) == (fa > 0):
                a, fa = mid, fm
            else:
                b = mid
        th = np.exp(0.5 * (a + b))
        rho[idx] = (th / K) ** (1.0 / (gam - 1.0))
        uu[idx] = mdot / (rr * rr * rho[idx])
    return rho, uu


def bondi(n1, n2, ng=3, hslope=0.3, rout=40.0, rs=8.0, beta=100.0, gam=4.0 / 3.0, noise=0.04, seed=7, lim="MC",
          flux="HLL", cour=0.8, rhomin=1e-4, uumin=1e-6):
    """2D Bondi flow (a = 0) on an n1 x n2 MKS grid; returns a torus.Domain."""
    rng = np.random.default_rng(seed)
    a = 0.0
    rin = torus.set_rin(n1, a, rout)
    x1s = np.log(rin)
    dx1 = np.log(rout / rin) / n1
    dx2 = 1.0 / n2
    dom = torus.Domain(n=(n1, n2, 1), ng=ng, dx=(dx1, dx2, 1.0), lim=lim, flux=flux, gam=gam, cour=cour,
                       bc=(1000, 1000, 4, 4, 7, 7))
    dom.gcov, dom.gcon, dom.gcovpert, dom.gdet, dom.conn = torus.geometry(n1, n2, ng, a, hslope, rin, rout, x1s,
                                                                          dx1, dx2)
    g1, g2, _ = dom.g
    nt, gt = dom.nt, dom.gt
    I, J = np.meshgrid(np.arange(gt[0]) - g1, np.arange(gt[1]) - g2, indexing="ij")
    rc = np.exp(x1s + (I + 0.5) * dx1)
    dom.floors = np.stack([rhomin * rc ** -1.5, uumin * rc ** -2.5], axis=-1)
    i = np.arange(nt[0]) - g1
    r1 = np.exp(x1s + (i + 0.5) * dx1)
    rho1, u1 = solution(r1, gam, rs)
    # rescale to rho(r_s) = 1 (rho -> lambda rho, u -> lambda u keeps a
    # polytropic solution with K -> K lambda^(1 - Gamma))
    lam = 1.0 / solution(np.array([rs]), gam, rs)[0][0]
    # BL: u^t from normalisation with u^r = -u; KS: u^t += 2/(r - 2) u^r; MKS: u^X1 = u^r / r
    ur = -u1
    f = 1.0 - 2.0 / r1
    ut_bl = np.sqrt(ur * ur + f) / f
    ut = ut_bl + 2.0 / (r1 - 2.0) * ur
    ucon = np.zeros((nt[0], nt[1], 4))
    ucon[..., 0] = ut[:, None]
    ucon[..., 1] = (ur / r1)[:, None]
    gconc = dom.gcon[:nt[0], :nt[1], CENT]
    gcovc = dom.gcov[:nt[0], :nt[1], CENT]
    p = np.zeros(nt + (NPR,))
    p[..., 0] = (lam * rho1)[:, None, None]
    p[..., 1] = (lam * rho1 ** gam / (gam - 1.0))[:, None, None]
    for q in (1, 2, 3):
        p[..., 1 + q] = (ucon[..., q] - ucon[..., 0] * gconc[..., 0, q] / gconc[..., 0, 0])[..., None]
    if noise:
        p[..., 1] *= 1.0 + noise * (rng.random(p[..., 1].shape) - 0.5)
    # monopole: gdet B^1 constant, scaled to beta at r_s on the equator
    gdc = dom.gdet[:nt[0], :nt[1], CENT]
    B1 = 1.0 / gdc
    ucov = np.einsum("...ij,...j->...i", gcovc, ucon)
    bt = B1 * ucov[..., 1]
    bcon = np.zeros_like(ucon)
    bcon[..., 0] = bt
    bcon[..., 1] = (B1 + bt * ucon[..., 1]) / ucon[..., 0]
    for q in (2, 3):
        bcon[..., q] = bt * ucon[..., q] / ucon[..., 0]
    bsq = np.einsum("...i,...ij,...j->...", bcon, gcovc, bcon)
    ir = int(np.argmin(np.abs(r1 - rs)))
    jr = nt[1] // 2
    pg = (gam - 1.0) * p[ir, jr, 0, 1]
    scale = np.sqrt(2.0 * pg / (beta * bsq[ir, jr]))
    p[..., 5] = (B1 * scale)[..., None]
    dom.p = p
    dom.pflag = np.zeros(nt, dtype=np.int32)
    dom.meta = {"problem": "bondi", "rs": rs, "beta": beta}
    return dom
