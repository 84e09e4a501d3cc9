"""CPU restatement of the reference's Bondi-integral radial boundaries.

Test infrastructure only (the oracle): used to pin the restatement against
the ghost zones the reference build itself writes, and by the GPU tests as
the checker.  Follows bounds.c:
  * BONDIINTOUTFLOW at the inner x1 boundary (bounds.c:140-156): the
    integrals C1, C2, K of the first active zone (bondi_compute_integrals,
    bounds.c:788-836) carried to every ghost zone (interpn of order
    BONDIEXTRAPORDER = 1 returns the first value, init.c:3449-3500);
  * BONDIMDOTOUTFLOW at the outer x1 boundary (bounds.c:295-308): C1 of the
    last active zone with the tabulated C2 = 1.373125 and K = 1
    (bounds.c:48-49);
  * each ghost zone's primitives from the integrals (bondi_generate_solution,
    bounds.c:839-888, with bondi_invert_integrals, bounds.c:1013-1083):
    the temperature by fixed-point iteration at the ghost's Boyer-Lindquist
    radius, rho, u and u^r in Kerr-Schild coordinates, u^t from the
    Kerr-Schild metric (pr2ucon VEL4, phys.c:1192-1260), to the internal
    coordinates with the inverse Jacobian (mettometpface, bounds.c:937-970)
    and to the relative 4-velocity of the internal metric (ucon2pr VELREL4,
    transforms.c:330-347); the field is zero.
The edge zone's u^r comes from metp2met2bl(VEL4, KSCOORDS) (transforms.c:51-84):
the relative 4-velocity to u^mu (ucon_calc_rel4vel, phys.c:983-1019) and
u^j = sum_k dxdxp[j][k] u^k (metptomet, transforms.c:310-328).

Inputs per zone: the primitives, the internal metric (gcov, gcon at CENT)
and the coordinate data of the harness's --bcgeom dump: r, dxdxp, its
inverse and the Kerr-Schild metric.  math.pow and math.sqrt are the C
library's, as in the reference build.
"""
import math

RHO, UU, U1, U2, U3, B1, B2, B3 = range(8)
C2X, KX = 1.373125, 1.0  # bounds.c:48-49 (bondigrid4acc.nb)


def ucon_rel4vel(pr, gcov, gcon):
    """ucon_calc_rel4vel (phys.c:983-1019); gcov, gcon 4x4 nested lists."""
    alpha = 1. / math.sqrt(-gcon[0][0])
    beta = [0.0] + [gcon[0][j] * alpha * alpha for j in (1, 2, 3)]
    u1, u2, u3 = pr[U1], pr[U2], pr[U3]
    qsq = (gcov[1][1] * u1 * u1 + gcov[2][2] * u2 * u2 + gcov[3][3] * u3 * u3
           + 2. * (gcov[1][2] * u1 * u2 + gcov[1][3] * u1 * u3 + gcov[2][3] * u2 * u3))
    gamma = math.sqrt(1. + qsq)
    u0 = gamma / alpha
    return [u0, u1 - u0 * beta[1], u2 - u0 * beta[2], u3 - u0 * beta[3]]


def mat_vec(M, u):
    """tmp[j] = sum_k M[j][k] u[k], accumulated from k = 0 (transforms.c:322-325)."""
    out = []
    for j in range(4):
        t = 0.
        for k in range(4):
            t += M[j][k] * u[k]
        out.append(t)
    return out


def integrals(pr, gcov, gcon, dxdxp, r, gam):
    """bondi_compute_integrals (bounds.c:788-836): C1, C2, K of a zone."""
    n = 1 / (gam - 1)
    ucon = mat_vec(dxdxp, ucon_rel4vel(pr, gcov, gcon))
    p = (gam - 1) * pr[UU]
    rho = pr[RHO]
    uu1 = ucon[1]
    T = p / rho
    C1 = math.pow(T, n) * uu1 * r * r
    C2 = math.pow(1 + (1 + n) * T, 2.) * (1 - 2. / r + uu1 * uu1)
    K = p / math.pow(rho, gam)
    return C1, C2, K


def invert_integrals(n, C1, C2, K, acc, r):
    """bondi_invert_integrals (bounds.c:1013-1083): rho, u, u^r."""
    T0, T1 = 0.2, 0.1
    it = 0
    if 0.35 < r < 2.5:
        while it < 250 and math.fabs((T0 - T1) / T1) > acc:
            T0 = T1
            u1 = C1 / (r * r * math.pow(T0, n))
            T1 = T0 + 0.02 * (T0 - (math.sqrt(C2 / (1 - 2 / r + u1 * u1)) - 1) / (1 + n))
            it += 1
    elif r > 9:
        while it < 250 and (T0 - T1) / T1 > acc:
            T0 = T1
            u1 = C1 / (r * r * math.pow(T0, n))
            T1 = (math.sqrt(C2 / (1 - 2 / r + u1 * u1)) - 1) / (1 + n)
            it += 1
        if T1 > T0:
            raise ValueError("Bondi integrals: temperature not decreasing")
    else:
        raise ValueError(f"Bondi integrals: radius {r} outside the supported ranges")
    rho = math.pow(T1 / K, n)
    return rho, rho * T1 * n, C1 / (math.pow(T1, n) * r * r)


def generate(C1, C2, K, gam, r, idxdxp, gks, gcon):
    """bondi_generate_solution (bounds.c:839-888) at a zone centre: the
    primitives (relative 4-velocity of the internal coordinates)."""
    n = 1 / (gam - 1)
    rho, u, ur = invert_integrals(n, C1, C2, K, 1.0e-15, r)
    # pr2ucon(VEL4) in Kerr-Schild coordinates (get_4velterms, phys.c:1236-1262)
    uc = [0., ur, 0., 0.]
    AA = gks[0][0]
    BB = 2. * (gks[0][1] * uc[1] + gks[0][2] * uc[2] + gks[0][3] * uc[3])
    CCM1 = (gks[1][1] * uc[1] * uc[1] + gks[2][2] * uc[2] * uc[2] + gks[3][3] * uc[3] * uc[3]
            + 2. * (gks[1][2] * uc[1] * uc[2] + gks[1][3] * uc[1] * uc[3] + gks[2][3] * uc[2] * uc[3]))
    CC = CCM1 + 1.0
    discr = BB * BB - 4. * AA * CC
    uc[0] = (-BB - math.sqrt(discr)) / (2. * AA)
    uc = mat_vec(idxdxp, uc)
    # ucon2pr(VELREL4) with the internal metric
    alphasq = 1. / (-gcon[0][0])
    gammaoalpha = uc[0]
    pr = [0.0] * 8
    pr[RHO], pr[UU] = rho, u
    for j in (1, 2, 3):
        pr[U1 + j - 1] = uc[j] + (alphasq * gcon[0][j]) * gammaoalpha
    return pr
