"""Corner-centred div B of the flux-CT scheme (the reference's DIVBFLUXCT,
global.h:1586-1645): B*gdet at cell centres averaged onto cell corners, then
differenced, normalised by max(dx) / (|sum of the averages| * gdet_corner / 3)."""
import numpy as np

SMALL = 1e-50


def divb_max(p, gdet, ng, dx, n):
    """max |div B| over the interior corners of primitives p [nt1][nt2][nt3][8]
    with gdet [gt1][gt2][8] (CENT=7, CORNT=6): x1 corners 1..n1-1, all x3
    corners, x2 corners 2..n2-2 -- the polar boundary (POLEDEATH,
    bounds.fishmon.c) resets B2 in the first and last active rows, so the
    corners next to them are not constrained by flux-CT."""
    n1, n2, n3 = n
    g1, g2, g3 = (ng if n1 > 1 else 0), (ng if n2 > 1 else 0), (ng if n3 > 1 else 0)
    gc = gdet[:p.shape[0], :p.shape[1], 7][:, :, None]
    Fg = p[..., 5:8] * gc[..., None]
    i = np.arange(1, n1) + g1
    j = np.arange(2, n2 - 1) + g2
    k = (np.arange(0, n3) if n3 > 1 else np.array([0])) + g3
    I, J, K = np.meshgrid(i, j, k, indexing="ij")
    km = K - (1 if n3 > 1 else 0)

    def F(a, b, c, q):
        return Fg[a, b, c, q]

    def for1(a):  # B1 averaged over (j-1..j, k-1..k) at x1 index a
        return 0.5 * (0.5 * (F(a, J, K, 0) + F(a, J - 1, K, 0)) + 0.5 * (F(a, J, km, 0) + F(a, J - 1, km, 0)))

    def for2(b):
        return 0.5 * (0.5 * (F(I, b, K, 1) + F(I - 1, b, K, 1)) + 0.5 * (F(I, b, km, 1) + F(I - 1, b, km, 1)))

    def for3(c):
        return 0.5 * (0.5 * (F(I, J, c, 2) + F(I, J - 1, c, 2)) + 0.5 * (F(I - 1, J, c, 2) + F(I - 1, J - 1, c, 2)))

    dxs = (dx[0] if n1 > 1 else 1.0, dx[1] if n2 > 1 else 1.0, dx[2] if n3 > 1 else 1.0)
    diff = (for1(I) - for1(I - 1)) / dxs[0] + (for2(J) - for2(J - 1)) / dxs[1]
    norm = for1(I) + for1(I - 1) + for2(J) + for2(J - 1)
    if n3 > 1:
        diff = diff + (for3(K) - for3(km)) / dxs[2]
        norm = norm + for3(K) + for3(km)
    gcorn = gdet[I, J, 6]
    dmax = max(dx[0], dx[1], dx[2] if n3 > 1 else 0.0)
    d = diff * (dmax / ((1.0 / 3.0) * gcorn * np.abs(norm) + SMALL))
    return float(np.max(np.abs(d)))


def divb_maxavg(p, gdet, ng, dx, n, interior=False):
    """The reference's divbmaxavg (dump_ener.c:482-520): max and mean over all
    active zones of |DIVBFLUXCT| at the zone's lower corner (dims of size 1
    use the same zone on both sides); gdet at the corner from CORN3 (=CORNT,
    the metric does not depend on x3).  interior: the max over the corners
    flux-CT constrains only (x1 corners 1..n1-1, x2 corners 2..n2-2)."""
    n1, n2, n3 = n
    s1, s2, s3 = int(n1 > 1), int(n2 > 1), int(n3 > 1)
    g1, g2, g3 = ng * s1, ng * s2, ng * s3
    gc = gdet[:p.shape[0], :p.shape[1], 7][:, :, None]
    Fg = p[..., 5:8] * gc[..., None]
    I, J, K = np.meshgrid(np.arange(n1) + g1, np.arange(n2) + g2, np.arange(n3) + g3, indexing="ij")

    def avg1(a, b, c, q):
        return 0.5 * (Fg[a, b, c, q] + Fg[a - s1, b, c, q])

    def avg2(a, b, c, q):
        return 0.5 * (Fg[a, b, c, q] + Fg[a, b - s2, c, q])

    def for1(a, b, c):
        return 0.5 * (avg2(a, b, c, 0) + avg2(a, b, c - s3, 0))

    def for2(a, b, c):
        return 0.5 * (avg1(a, b, c, 1) + avg1(a, b, c - s3, 1))

    def for3(a, b, c):
        return 0.5 * (avg2(a, b, c, 2) + avg2(a - s1, b, c, 2))

    dfx = for1(I, J, K) - for1(I - s1, J, K)
    dfy = for2(I, J, K) - for2(I, J - s2, K)
    dfz = for3(I, J, K) - for3(I, J, K - s3)
    nx = for1(I, J, K) + for1(I - s1, J, K)
    ny = for2(I, J, K) + for2(I, J - s2, K)
    nz = for3(I, J, K) + for3(I, J, K - s3)
    mx = max(max(dx[0], dx[1]), dx[2])
    norm = mx / ((1.0 / 3.0) * gdet[I, J, 5] * np.abs(nx + ny + nz) + SMALL)
    d = np.abs((dfx / dx[0] + dfy / dx[1] + dfz / dx[2]) * norm)
    if interior:
        m = np.ones(d.shape, dtype=bool)
        if s1:
            m &= (I - g1 >= 1) & (I - g1 <= n1 - 1)
        if s2:
            m &= (J - g2 >= 2) & (J - g2 <= n2 - 2)
        return float(d[m].max())
    return float(d.max()), float(d.mean())


def divb_scaled_max(p, gdet, ng, dx, n):
    """The flux-CT corner divergence of divb_max without the local
    normalisation (which divides by the signed sum of the corner averages and
    spikes where that sum nearly cancels): max |div(gdet B)| times max(dx)
    over max |gdet B| on the grid, a round-off measure that does not depend
    on the grid size."""
    n1, n2, n3 = n
    g1, g2, g3 = (ng if n1 > 1 else 0), (ng if n2 > 1 else 0), (ng if n3 > 1 else 0)
    gc = gdet[:p.shape[0], :p.shape[1], 7][:, :, None]
    Fg = p[..., 5:8] * gc[..., None]
    i = np.arange(1, n1) + g1
    j = np.arange(2, n2 - 1) + g2
    k = (np.arange(0, n3) if n3 > 1 else np.array([0])) + g3
    I, J, K = np.meshgrid(i, j, k, indexing="ij")
    km = K - (1 if n3 > 1 else 0)

    def for1(a):
        return 0.5 * (0.5 * (Fg[a, J, K, 0] + Fg[a, J - 1, K, 0]) + 0.5 * (Fg[a, J, km, 0] + Fg[a, J - 1, km, 0]))

    def for2(b):
        return 0.5 * (0.5 * (Fg[I, b, K, 1] + Fg[I - 1, b, K, 1]) + 0.5 * (Fg[I, b, km, 1] + Fg[I - 1, b, km, 1]))

    def for3(c):
        return 0.5 * (0.5 * (Fg[I, J, c, 2] + Fg[I, J - 1, c, 2]) + 0.5 * (Fg[I - 1, J, c, 2] + Fg[I - 1, J - 1, c, 2]))

    dxs = (dx[0] if n1 > 1 else 1.0, dx[1] if n2 > 1 else 1.0, dx[2] if n3 > 1 else 1.0)
    diff = (for1(I) - for1(I - 1)) / dxs[0] + (for2(J) - for2(J - 1)) / dxs[1]
    if n3 > 1:
        diff = diff + (for3(K) - for3(km)) / dxs[2]
    dmax = max(dx[0], dx[1], dx[2] if n3 > 1 else 0.0)
    return float(np.max(np.abs(diff)) * dmax / (np.max(np.abs(Fg)) + SMALL))
