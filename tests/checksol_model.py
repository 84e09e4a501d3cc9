"""fixup_checksolution (fixup.c:460-560) restated two ways, for the tests.

`sequential` is the reference's loop: candidates (active zones with gamma >=
2) visited in (i, j, k) order, each reading the flags earlier visits wrote.
`device_scheme` is the formulation of the device kernels (checksol_map /
prep / resolve / apply): per candidate the 16 vote bits, the "fixed and not
failed" and "earlier candidate" neighbour masks; every candidate whose vote
its earlier candidate neighbours cannot change is final at once; the others
iterate to a fixpoint in an arbitrary order.  Both work on padded arrays
(zone layout with ghosts) of flags, gamma and u.  `craft` draws states rich
in candidates on a fixture's grid."""
import numpy as np

from oracle.pyoracle import CENT

RHO, UU, U1 = 0, 1, 2
GAMMAPERCDIFFMAX, UPERCDIFFMAX = 2.0, 10.0
GAMMAPERC, UPERC = 12, 13
# failure codes drawn into crafted states: every code the reference's
# fixup_utoprim accepts (fixup.c:1346-1425) ...
REF_FAIL_CODES = [1, 1, 1, 2, 5, 8, 9, 10, 11, 12, 13, 14, 15, 101]
# ... and the set the GPU test draws, which adds -1 (UTOPRIMFAILFIXED, a code
# fixup_utoprim writes but rejects on input) to compare the device's
# handling of it with the oracle's
FAIL_CODES = [1, 1, 1, 9, 10, 11, 12, 13, 14, 15, -1]


def neighbours(z, s):
    """The 8 neighbours of fixup.c:508-526, in its order (k fixed)."""
    i, j, k = z
    return [(i, j + s[1], k), (i, j - s[1], k), (i + s[0], j, k), (i - s[0], j, k), (i + s[0], j + s[1], k),
            (i + s[0], j - s[1], k), (i + s[0], j + s[1], k), (i - s[0], j - s[1], k)]


def _ratio_bits(gam, uu, z, nbs):
    gc, uc = gam[z], uu[z]
    with np.errstate(all="ignore"):
        pd = [np.float64(gam[nb]) / np.float64(gc) for nb in nbs]
        pd2 = [np.float64(uu[nb]) / np.float64(uc) for nb in nbs]
    v0 = [bool(abs(x) > GAMMAPERCDIFFMAX or abs(x) < 1.0 / GAMMAPERCDIFFMAX) for x in pd]
    v1 = [bool(abs(x) > UPERCDIFFMAX or abs(x) < 1.0 / UPERCDIFFMAX) for x in pd2]
    return pd, v0, v1


def _active(n, g):
    for i in range(n[0]):
        for j in range(n[1]):
            for k in range(n[2]):
                yield (i + g[0], j + g[1], k + g[2])


def sequential(flags, gam, uu, n, g, s, order_free=False):
    """order_free: every visit reads the original flags instead (not the
    reference's semantics; shows where the order matters)."""
    out = flags.copy()
    for z in _active(n, g):
        if not (gam[z] >= 2.0):
            continue
        nbs = neighbours(z, s)
        ok = [(flags if order_free else out)[nb] <= 0 for nb in nbs]
        pd, v0, v1 = _ratio_bits(gam, uu, z, nbs)
        # a failed neighbour's ratio is -1: no vote, and no votes at all when
        # it is neighbour 0
        vote0 = vote1 = numvotes = 0
        if ok[0] and pd[0] >= 0.0:
            vote0 = sum(1 for q in range(8) if ok[q] and v0[q])
            vote1 = sum(1 for q in range(8) if ok[q] and v1[q])
            numvotes = 8
        if vote0 > numvotes * 0.5:
            out[z] = GAMMAPERC
        if vote1 > numvotes * 0.5:
            out[z] = UPERC
    return out


def _vote(v0, v1, ok):
    if not ok & 1:
        return 0
    c0 = bin(ok & v0).count("1")
    c1 = bin(ok & v1).count("1")
    v = 0
    if c0 > 4:
        v = 1
    if c1 > 4:
        v = 2
    return v


def device_scheme(flags, gam, uu, n, g, s, rng, jacobi=False):
    """The device's four-kernel formulation; candidates listed in a random
    order (the device appends them with atomics), the dependent ones swept
    in a random order each sweep (in place), or all from the previous
    sweep's values (jacobi=True)."""
    cand = [z for z in _active(n, g) if gam[z] >= 2.0]
    rng.shuffle(cand)
    candmap = {z: a for a, z in enumerate(cand)}
    orig = [int(flags[z]) for z in cand]
    codes = [0, GAMMAPERC, UPERC]
    dec, bits, deplist = [0] * len(cand), [None] * len(cand), []
    for a, z in enumerate(cand):
        nbs = neighbours(z, s)
        pd, v0l, v1l = _ratio_bits(gam, uu, z, nbs)
        v0 = sum(1 << q for q in range(8) if v0l[q])
        v1 = sum(1 << q for q in range(8) if v1l[q])
        if not pd[0] >= 0.0:
            v0 = v1 = 0
        okfix = earlier = 0
        for q, nb in enumerate(nbs):
            if nb < z and nb in candmap:
                earlier |= 1 << q
            elif flags[nb] <= 0:
                okfix |= 1 << q
        bits[a] = (v0, v1, okfix, earlier)
        vlo = _vote(v0, v1, okfix)
        if earlier and ((earlier & 1) or vlo != _vote(v0, v1, okfix | earlier)):
            dec[a] = orig[a]
            deplist.append(a)
        else:
            dec[a] = codes[vlo] if vlo else orig[a]
    rng.shuffle(deplist)
    for _sweep in range(len(deplist) + 1):
        src = list(dec) if jacobi else dec
        changed = False
        for a in deplist:
            v0, v1, okfix, earlier = bits[a]
            ok = okfix
            nbs = neighbours(cand[a], s)
            for q in range(8):
                if (earlier >> q) & 1 and src[candmap[nbs[q]]] <= 0:
                    ok |= 1 << q
            v = _vote(v0, v1, ok)
            nd = codes[v] if v else orig[a]
            if nd != dec[a]:
                dec[a] = nd
                changed = True
        if not changed:
            break
    out = flags.copy()
    for a, z in enumerate(cand):
        out[z] = dec[a]
    return out, len(deplist)


def craft(pr, seed, codes=FAIL_CODES):
    """Overwrite pr.p / pr.pflag with a seeded state rich in candidates:
    Lorentz factors from 1.1 to 9 (u~^1 alone, sized by g_11 at the zone
    centre), internal energies over four decades, failure codes on a quarter
    of the zones."""
    rng = np.random.default_rng(seed)
    nt = pr.nt
    g11 = pr.gcov[:nt[0], :nt[1], CENT, 1, 1][:, :, None]
    target = rng.choice([1.1, 1.6, 2.1, 2.6, 3.5, 5.0, 9.0], size=nt, p=[.1, .1, .2, .2, .15, .15, .1])
    sign = rng.choice([-1.0, 1.0], size=nt)
    pr.p[..., U1] = sign * np.sqrt(target * target - 1.0) / np.sqrt(g11)
    pr.p[..., U1 + 1] = 0.0
    pr.p[..., U1 + 2] = 0.0
    pr.p[..., RHO] = 10.0 ** rng.uniform(-2.0, 0.0, size=nt)
    pr.p[..., UU] = pr.p[..., RHO] * 10.0 ** rng.uniform(-4.0, 0.0, size=nt)
    fail = rng.random(nt) < 0.25
    pr.pflag[...] = np.where(fail, rng.choice(codes, size=nt), 0).astype(np.int32)
    pr.p = np.ascontiguousarray(pr.p)
    pr.pflag = np.ascontiguousarray(pr.pflag)
