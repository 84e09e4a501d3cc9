"""Seeded 1D relativistic-MHD Riemann problems in Minkowski space.

The reference sets up its 1D Riemann tests in init.c (REL1DRIEMANNTEST,
init.c:3057-3110): Cartesian Minkowski metric (CARTMINKMETRIC), x in
[-0.5, 0.5] with the interface at x0 = 0, left/right states of rho, p, v,
B, outflow boundaries (bounds.c OUTFLOW: plain copy).  This module draws
many such problems from one seed with the distributions

    N      ~ U{nmin..nmax} zones
    rho    ~ logU[0.1, 10],  p ~ logU[0.01, 100]  (each side)
    v_i    ~ U(-0.9, 0.9), rescaled so that |v| <= 0.95   (each side)
    B_x    ~ U(-2, 2) shared by both sides, B_y, B_z ~ U(-5, 5) (each side)
    Gamma  in {4/3, 5/3}

and builds the reference-layout arrays of one problem (primitives rho, u,
u~^i (relative 4-velocity, = gamma v^i in Minkowski space), B^i; geometry at
the 8 grid locations).
"""
from dataclasses import dataclass

import numpy as np

NPR = 8
LOCS = 8


@dataclass
class RiemannProblem:
    n: int
    gam: float
    left: np.ndarray    # rho, p, vx, vy, vz, Bx, By, Bz
    right: np.ndarray
    x0: float = 0.0
    xmin: float = -0.5
    xmax: float = 0.5

    @property
    def dx(self):
        return (self.xmax - self.xmin) / self.n


def draw(count, seed=2024, nmin=200, nmax=2000):
    """`count` problems from one seed."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n = int(rng.integers(nmin, nmax + 1))
        gam = float(rng.choice([4.0 / 3.0, 5.0 / 3.0]))
        bx = rng.uniform(-2.0, 2.0)
        sides = []
        for _side in range(2):
            rho = 10.0 ** rng.uniform(-1.0, 1.0)
            p = 10.0 ** rng.uniform(-2.0, 2.0)
            v = rng.uniform(-0.9, 0.9, 3)
            vm = np.sqrt(np.sum(v * v))
            if vm > 0.95:
                v *= 0.95 / vm
            by, bz = rng.uniform(-5.0, 5.0, 2)
            sides.append(np.array([rho, p, v[0], v[1], v[2], bx, by, bz]))
        out.append(RiemannProblem(n, gam, sides[0], sides[1]))
    return out


def primitives(prob, ng):
    """Reference-layout primitives [n + 2 ng][1][1][8] of one problem (ghosts
    filled with the outflow copy of the edge zones)."""
    n = prob.n
    x = prob.xmin + (np.arange(-ng, n + ng) + 0.5) * prob.dx
    p = np.zeros((n + 2 * ng, 1, 1, NPR))
    for side, mask in ((prob.left, x < prob.x0), (prob.right, x >= prob.x0)):
        rho, pres, vx, vy, vz, bx, by, bz = side
        gamma = 1.0 / np.sqrt(1.0 - (vx * vx + vy * vy + vz * vz))
        p[mask, 0, 0] = [rho, pres / (prob.gam - 1.0), gamma * vx, gamma * vy, gamma * vz, bx, by, bz]
    p[:ng] = p[ng]
    p[n + ng:] = p[n + ng - 1]
    return p


def minkowski_geometry(nt1):
    """Geometry arrays of a 1D line of nt1 zones (ghosts included): the
    Minkowski metric at every location, gdet = 1, no connection, zero floors
    (the density floors then come from rhominlimit/uuminlimit)."""
    gt1 = nt1 + 1
    eta = np.diag([-1.0, 1.0, 1.0, 1.0])
    gcov = np.broadcast_to(eta, (gt1, 1, LOCS, 4, 4)).copy()
    gcon = gcov.copy()
    gcovpert = np.zeros((gt1, 1, LOCS, 4))   # g_mu mu - eta_mu mu
    gdet = np.ones((gt1, 1, LOCS))
    conn = np.zeros((gt1, 1, 4, 4, 4))
    floors = np.zeros((gt1, 1, 2))
    return gcov, gcon, gcovpert, gdet, conn, floors


def domain(prob, ng=3, cour=0.5):
    """One problem as a single-solve domain (the reference's own 1D run:
    MC + HLL, bounds.c OUTFLOW copies at both ends), with the attributes the
    context and the serving loop read."""
    from .torus import Domain
    n = prob.n
    dom = Domain(n=(n, 1, 1), ng=ng, dx=(prob.dx, 1.0, 1.0), lim="MC", flux="HLL",
                 bc=(1000, 1000, 0, 0, 0, 0), gam=prob.gam, cour=cour)
    dom.gcov, dom.gcon, dom.gcovpert, dom.gdet, dom.conn, dom.floors = minkowski_geometry(n + 2 * ng)
    dom.p = primitives(prob, ng)
    dom.meta = dict(kind="shock tube", n=n, gam=prob.gam)
    return dom


def _main(argv=None):
    """Advance a seeded batch of problems on the GPU as one batch context:
    `python -m harm_finalwham_b200.riemann --count 256 --steps 20` (steps of
    the shared step graph; 0 runs every instance to tf)."""
    import argparse
    from .gpu import HarmBatch
    ap = argparse.ArgumentParser()
    ap.add_argument("--count", type=int, default=256)
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--tf", type=float, default=0.4)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--ng", type=int, default=3)
    args = ap.parse_args(argv)
    probs = draw(args.count, seed=args.seed)
    b = HarmBatch([p.n for p in probs], [p.dx for p in probs], [p.gam for p in probs], [args.tf] * len(probs),
                  ng=args.ng, lim="MC", flux="HLL", cour=0.5)
    try:
        b.upload_geometry(*minkowski_geometry(b.nt[0]))
        b.upload_state(b.join([primitives(p, args.ng) for p in probs]), None, 0.0, 0.0)
        b.init_dt()
        if args.steps > 0:
            b.step_ch(args.steps)
        else:
            b.run()
        b.sync()
        print(f"{args.count} problems, {sum(p.n for p in probs)} zones: ok")
    finally:
        b.close()


if __name__ == "__main__":
    _main()
