/*
 * harm_oracle.c -- CPU restatement of HARM's per-zone conservative update.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity checker for the CUDA
 * path in harm_finalwham_b200/csrc.  Only tests/, __graft_entry__.smoke() and
 * bench.py's cpu_baseline leg may load it, and only to check or to time the
 * CPU baseline; the product never links it.
 *
 * It restates, in the reference's own floating-point operation order (so
 * that with gcc -O2 -ffp-contract=off results are bit-identical to the
 * reference build in oracle/_ref), the path
 *
 *   step_ch_simplempi (step_ch.c:35-252, midpoint RK2 tables :504-524)
 *     pre_fixup          (fixup.c:25; flags only, no effect on state here)
 *     advance_standard   (advance.c:58-238)
 *       fluxcalc         (flux.c:7-318), fluxcalc_standard (flux.c:469-680)
 *         MC slopes      (interppoint.c:387-397, getp2interplr flux.c:753-810)
 *         p2SFUevolve    (fluxcompute.c:57-65), get_wavespeeds (wavespeeds.c:12)
 *         vchar/simplefast (vchar.c:37-312), cminmax_calc (wavespeeds.c:325)
 *         HLL / LAXF     (fluxcompute.c:75-78, :223-264)
 *       flux_ct          (fluxct.c:10-844, FLUXCTTOTH, CORNGDETVERSION=1)
 *       per zone: primtoU, source_conn (phys.c:578-752), flux2dUavg + dUtoU
 *                 (advance.c:741-949), Utoprimgen (utoprimgen.c:23-436) ->
 *                 Utoprim_2d_final (utoprim_2d_final.c:34-1278), fixup1zone
 *                 (fixup.c:341-447) on the final substep
 *     bound_prim         (bounds.fishmon.c:29-345 with inflow_check_rel4vel
 *                         fixup.c:2271 and limit_gamma fixup.c:1859)
 *     post_fixup         (fixup.c:37-96: bound_pflag boundsint.c:6,
 *                         fixup_checksolution fixup.c:460, fixup_utoprim
 *                         fixup.c:669-1470)
 *     dt update          (advance.c:231, step_ch.c:236-247)
 *
 * for the build options of the FM-torus configuration: WHICHVEL=VELREL4,
 * REMOVERESTMASSFROMUU=2, WHICHEOM=WITHGDET, EOMTYPE=EOMGRMHD, ideal gas,
 * DOENOFLUX=NOENOFLUX, FLUXB=FLUXCTTOTH, UTOPRIMVERSION=UTOPRIM2DFINAL,
 * TIMEORDER=2, LIMADJUST/FLUXADJUST fixed, STEPOVERNEG*=-1, CHECKSOLUTION=1,
 * UTOPRIMADJUST=UTOPRIMAVG, BDIRCONT=1, EVOLVECHECKS=0.
 *
 * Geometry (gcov/gcon/gcovpert/gdet at the 8 grid locations, conn at CENT)
 * and the density floors are inputs: the reference computes them once on the
 * host (set_grid.c:7-151, fixup.c:1542-1654) and they carry no per-step work.
 * The metric is stored per (i,j): it does not depend on x3.
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <stdio.h>

#include "harm_oracle.h"

#define NPR 8
#define NDIM 4
#define RHO 0
#define UU 1
#define U1 2
#define U2 3
#define U3 4
#define B1 5
#define B2 6
#define B3 7
#define TT 0

/* grid locations (global.h:948-955) */
#define FACE1 0
#define FACE2 1
#define FACE3 2
#define CORN1 3
#define CORN2 4
#define CORN3 5
#define CORNT 6
#define CENT 7

/* failure codes (global.h:782-799) */
#define UTOPRIMFAILFIXED -1
#define UTOPRIMNOFAIL 0
#define UTOPRIMFAILCONV 1
#define UTOPRIMFAILCONVW 2
#define UTOPRIMFAILCONVUTSQ 3
#define UTOPRIMFAILCONVGUESSUTSQ 4
#define UTOPRIMFAILCONVUTSQVERYBAD 5
#define UTOPRIMFAILCONVBADINVERTCOMPARE 6
#define UTOPRIMFAILNANGUESS 7
#define UTOPRIMFAILNANRESULT 8
#define UTOPRIMFAILRHONEG 9
#define UTOPRIMFAILUNEG 10
#define UTOPRIMFAILRHOUNEG 11
#define UTOPRIMFAILGAMMAPERC 12
#define UTOPRIMFAILUPERC 13
#define UTOPRIMFAILU2AVG1 14
#define UTOPRIMFAILU2AVG2 15
#define UTOPRIMFAILCONVRET 101

#define NUMEPSILON (2.2204460492503131e-16)
#define BIG (1.e+50)
#define SMALL (1.e-50) /* global.h:1041 */

/* u2p_defs.h (PRECISEINVERSION=1, NEWCONVERGE=1, OPTIMIZED=1) */
#define MAX_NEWT_ITER 200
#define NEWT_TOL (1E3 * NUMEPSILON)
#define MIN_NEWT_TOL (1E-6)
#define EXTRA_NEWT_ITER 0
#define MAXNEGUTSQ (1E-10)
#define MAXNEGVSQ (1.0 - 1.0 / (MAXNEGUTSQ + 1.0))
#define FAIL_VAL 1.e30

/* fixup.c:447-460,484 */
#define GAMMAPERCDIFFMAX 2.0
#define UPERCDIFFMAX 10.0
#define MAXVOTES 8

typedef struct {
  const double *gcov; /* [4][4] */
  const double *gcon; /* [4][4] */
  const double *gcovpert; /* [4] */
  double g;
} geomref;

typedef struct {
  double ucon[NDIM], ucov[NDIM], bcon[NDIM], bcov[NDIM];
} zstate;

#define GCOV(g, a, b) ((g)->gcov[(a) * 4 + (b)])
#define GCON(g, a, b) ((g)->gcon[(a) * 4 + (b)])

/* error bits reported to the caller (the reference calls fail()/myexit()) */
#define ERR_UTCALC_DISCR 1
#define ERR_COEFF_NEG 2
#define ERR_COEFF_SUP 4
#define ERR_VCHAR_DISCR 8
#define ERR_VSQ_NEG 16
#define ERR_NONFINITE_SPEED 32
#define ERR_PREF_NEG 64

/* ------------------------------------------------------------------ */
/* domain bookkeeping                                                  */
/* ------------------------------------------------------------------ */
typedef struct {
  const hgo_config *c;
  int n[4];      /* active sizes, index 1..3 */
  int ng[4];     /* ghost widths */
  int nt[4];     /* totals with ghosts */
  int sh[4];     /* SHIFTd = (n>1) */
  int gt[3];     /* geometry totals per (i,j): nt+sh */
  const double *gcov, *gcon, *gcovpert, *gdet, *conn, *floors;
  int err;
} dom;

static inline long zidx(const dom *d, int i, int j, int k)
{
  return ((long)(i + d->ng[1]) * d->nt[2] + (j + d->ng[2])) * d->nt[3] + (k + d->ng[3]);
}

static inline long gidx(const dom *d, int i, int j)
{
  return (long)(i + d->ng[1]) * d->gt[2] + (j + d->ng[2]);
}

static void get_geometry(const dom *d, int i, int j, int loc, geomref *g)
{
  long q = gidx(d, i, j) * 8 + loc;
  g->gcov = d->gcov + q * 16;
  g->gcon = d->gcon + q * 16;
  g->gcovpert = d->gcovpert + q * 4;
  g->g = d->gdet[q];
}

/* ------------------------------------------------------------------ */
/* per-zone physics (phys.c)                                           */
/* ------------------------------------------------------------------ */

/* lower_vec (phys.c:766-787): upper-triangle gcov entries */
static void lower_vec(const double *ucon, const geomref *g, double *ucov)
{
  ucov[0] = GCOV(g, 0, 0) * ucon[0] + GCOV(g, 0, 1) * ucon[1] + GCOV(g, 0, 2) * ucon[2] + GCOV(g, 0, 3) * ucon[3];
  ucov[1] = GCOV(g, 0, 1) * ucon[0] + GCOV(g, 1, 1) * ucon[1] + GCOV(g, 1, 2) * ucon[2] + GCOV(g, 1, 3) * ucon[3];
  ucov[2] = GCOV(g, 0, 2) * ucon[0] + GCOV(g, 1, 2) * ucon[1] + GCOV(g, 2, 2) * ucon[2] + GCOV(g, 2, 3) * ucon[3];
  ucov[3] = GCOV(g, 0, 3) * ucon[0] + GCOV(g, 1, 3) * ucon[1] + GCOV(g, 2, 3) * ucon[2] + GCOV(g, 3, 3) * ucon[3];
}

/* raise_vec (phys.c:826-846) */
static void raise_vec(const double *ucov, const geomref *g, double *ucon)
{
  ucon[0] = GCON(g, 0, 0) * ucov[0] + GCON(g, 0, 1) * ucov[1] + GCON(g, 0, 2) * ucov[2] + GCON(g, 0, 3) * ucov[3];
  ucon[1] = GCON(g, 0, 1) * ucov[0] + GCON(g, 1, 1) * ucov[1] + GCON(g, 1, 2) * ucov[2] + GCON(g, 1, 3) * ucov[3];
  ucon[2] = GCON(g, 0, 2) * ucov[0] + GCON(g, 1, 2) * ucov[1] + GCON(g, 2, 2) * ucov[2] + GCON(g, 2, 3) * ucov[3];
  ucon[3] = GCON(g, 0, 3) * ucov[0] + GCON(g, 1, 3) * ucov[1] + GCON(g, 2, 3) * ucov[2] + GCON(g, 3, 3) * ucov[3];
}

static inline double dot4(const double *a, const double *b)
{
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2] + a[3] * b[3];
}

/* qsq_calc (phys.c:1077-1090) */
static double qsq_calc(const double *u, const geomref *g)
{
  return +GCOV(g, 1, 1) * u[1] * u[1] + GCOV(g, 2, 2) * u[2] * u[2] + GCOV(g, 3, 3) * u[3] * u[3] +
         2. * (GCOV(g, 1, 2) * u[1] * u[2] + GCOV(g, 1, 3) * u[1] * u[3] + GCOV(g, 2, 3) * u[2] * u[3]);
}

/* gamma_calc_fromuconrel (phys.c:1047-1074) */
static int gamma_calc_fromuconrel(const double *uconrel, const geomref *g, double *gamma)
{
  double qsq = qsq_calc(uconrel, g);
  if (qsq < 0.0) {
    if (qsq > -NUMEPSILON * 100) qsq = 0.0;
    else return 1;
  }
  *gamma = sqrt(1. + qsq);
  return 0;
}

/* gamma_calc (phys.c:1022-1044) */
static int gamma_calc(const double *pr, const geomref *g, double *gamma)
{
  double u[NDIM];
  u[0] = 0;
  u[1] = pr[U1];
  u[2] = pr[U2];
  u[3] = pr[U3];
  return gamma_calc_fromuconrel(u, g, gamma);
}

/* ucon_calc_rel4vel (phys.c:983-1019) */
static int ucon_calc(const double *pr, const geomref *g, double *ucon)
{
  double alpha, gamma, beta[NDIM], u[NDIM];
  int j;
  u[0] = 0;
  u[1] = pr[U1];
  u[2] = pr[U2];
  u[3] = pr[U3];
  alpha = 1. / sqrt(-GCON(g, TT, TT));
  for (j = 1; j < NDIM; j++) beta[j] = GCON(g, TT, j) * alpha * alpha;
  if (gamma_calc_fromuconrel(u, g, &gamma)) return 1;
  ucon[TT] = gamma / alpha;
  for (j = 1; j < NDIM; j++) ucon[j] = u[j] - ucon[TT] * beta[j];
  return 0;
}

/* bcon_calc (phys.c:309-318) */
static void bcon_calc(const double *pr, const double *ucon, const double *ucov, double *bcon)
{
  int j;
  bcon[TT] = pr[B1] * ucov[1] + pr[B2] * ucov[2] + pr[B3] * ucov[3];
  for (j = 1; j <= 3; j++) bcon[j] = (pr[B1 - 1 + j] + bcon[TT] * ucon[j]) / ucon[TT];
}

/* get_state (phys.c:849-859) */
static int get_state(const double *pr, const geomref *g, zstate *q)
{
  if (ucon_calc(pr, g, q->ucon)) return 1;
  lower_vec(q->ucon, g, q->ucov);
  bcon_calc(pr, q->ucon, q->ucov, q->bcon);
  lower_vec(q->bcon, g, q->bcov);
  return 0;
}

/* Mcon_calc, PRIMMAXWELL (phys.c:178-210) */
static void mcon_calc(const double *pr, const zstate *q, double M[NDIM][NDIM])
{
  int j, k;
  for (j = 0; j < NDIM; j++) M[j][j] = 0.0;
  for (k = 1; k < NDIM; k++) {
    M[k][0] = pr[B1 + k - 1];
    M[0][k] = -M[k][0];
  }
  for (j = 1; j < NDIM; j++)
    for (k = 1; k < NDIM; k++) M[j][k] = (pr[B1 + j - 1] * q->ucon[k] - pr[B1 + k - 1] * q->ucon[j]) / q->ucon[0];
}

/* lower_A (phys.ffde.c:1707-1735) */
static void lower_A(double Acon[NDIM][NDIM], const geomref *g, double Acov[NDIM][NDIM])
{
  int j, k;
  for (j = 0; j < NDIM; j++)
    for (k = 0; k < NDIM; k++) Acov[j][k] = 0.;
  for (j = 0; j < NDIM; j++)
    for (k = 0; k < NDIM; k++) {
      Acov[0][1] += (GCOV(g, 0, j)) * (GCOV(g, 1, k)) * Acon[j][k];
      Acov[0][2] += (GCOV(g, 0, j)) * (GCOV(g, 2, k)) * Acon[j][k];
      Acov[0][3] += (GCOV(g, 0, j)) * (GCOV(g, 3, k)) * Acon[j][k];
      Acov[1][2] += (GCOV(g, 1, j)) * (GCOV(g, 2, k)) * Acon[j][k];
      Acov[2][3] += (GCOV(g, 2, j)) * (GCOV(g, 3, k)) * Acon[j][k];
      Acov[3][1] += (GCOV(g, 3, j)) * (GCOV(g, 1, k)) * Acon[j][k];
    }
  Acov[1][0] = -Acov[0][1];
  Acov[2][0] = -Acov[0][2];
  Acov[3][0] = -Acov[0][3];
  Acov[2][1] = -Acov[1][2];
  Acov[3][2] = -Acov[2][3];
  Acov[1][3] = -Acov[3][1];
}

/* compute_1plusud0 (phys.c:541-575) */
static double compute_1plusud0(const geomref *g, const zstate *q)
{
  int j, k;
  double plus1gv00, vsq, gvtt, alpha, uu0, vcon[NDIM];
  for (j = 1; j < NDIM; j++) vcon[j] = q->ucon[j] / q->ucon[TT];
  plus1gv00 = g->gcovpert[TT];
  vsq = g->gcovpert[TT];
  for (j = 1; j < NDIM; j++) vsq += 2.0 * GCOV(g, TT, j) * vcon[j];
  for (j = 1; j < NDIM; j++)
    for (k = 1; k < NDIM; k++) vsq += GCOV(g, j, k) * vcon[j] * vcon[k];
  gvtt = GCOV(g, TT, TT);
  alpha = 0.0;
  for (j = 1; j < NDIM; j++) alpha += GCOV(g, j, TT) * q->ucon[j];
  uu0 = q->ucon[TT];
  return alpha + ((1.0 - gvtt) * plus1gv00 - uu0 * uu0 * vsq * gvtt * gvtt) / (1.0 - gvtt * uu0);
}

/* Per-state electromagnetic pieces that mhd_calc_norestmass recomputes on
   every call (Mcon_calc, lower_A, Msq, 1+u_t); computing them once per state
   gives the same bits. */
typedef struct {
  double Mcon[NDIM][NDIM], Mcov[NDIM][NDIM], Msq, plus1ud0;
} emstate;

static void em_prepare(const double *pr, const geomref *g, const zstate *q, emstate *e)
{
  int j, k;
  mcon_calc(pr, q, e->Mcon);
  lower_A(e->Mcon, g, e->Mcov);
  e->Msq = 0.;
  for (j = 0; j < NDIM; j++)
    for (k = 0; k < NDIM; k++) e->Msq += e->Mcov[j][k] * e->Mcon[j][k];
  e->plus1ud0 = compute_1plusud0(g, q);
}

/* mhd_calc_norestmass (phys.c:442-506) + ffdestresstensor_dir
   (phys.ffde.c:1483-1515): T^dir_mu without rest mass */
static void mhd_calc(const double *pr, int dir, const double gam, const zstate *q, const emstate *e, double *mhd)
{
  int j, i;
  double rho = pr[RHO], u = pr[UU];
  double P = (gam - 1.) * u;
  double w = P + rho + u;
  double eta = w, ptot = P;
  double TEM[NDIM];
  j = 0;
  mhd[j] = (P + u) * q->ucon[dir] * q->ucov[j] + rho * q->ucon[dir] * e->plus1ud0 + ptot * ((dir == j) ? 1. : 0.);
  for (j = 1; j < NDIM; j++) mhd[j] = eta * q->ucon[dir] * q->ucov[j] + ptot * ((dir == j) ? 1. : 0.);
  for (j = 0; j < NDIM; j++) TEM[j] = 0.;
  for (j = 0; j < NDIM; j++)
    for (i = 0; i < NDIM; i++) TEM[j] += e->Mcon[dir][i] * e->Mcov[j][i];
  TEM[dir] -= 0.25 * e->Msq;
  for (j = 0; j < NDIM; j++) mhd[j] += TEM[j];
}

/* primtoflux (phys.c:16-55) with UEVOLVE; WITHGDET so every EOM factor is gdet */
static void primtoflux(const double *pr, const zstate *q, const emstate *e, int dir, const geomref *g, double gam,
                       double *flux)
{
  double fin[NPR];
  fin[RHO] = pr[RHO] * q->ucon[dir];
  mhd_calc(pr, dir, gam, q, e, &fin[UU]);
  if (dir > 0) {
    fin[B1] = (pr[B1] * q->ucon[dir] - pr[B1 + dir - 1] * q->ucon[1]) / q->ucon[0];
    fin[B2] = (pr[B2] * q->ucon[dir] - pr[B1 + dir - 1] * q->ucon[2]) / q->ucon[0];
    fin[B3] = (pr[B3] * q->ucon[dir] - pr[B1 + dir - 1] * q->ucon[3]) / q->ucon[0];
  } else {
    fin[B1] = pr[B1];
    fin[B2] = pr[B2];
    fin[B3] = pr[B3];
  }
  for (int pl = 0; pl < NPR; pl++) flux[pl] = fin[pl] * g->g;
}

/* ------------------------------------------------------------------ */
/* wave speeds (vchar.c, wavespeeds.c)                                 */
/* ------------------------------------------------------------------ */

/* simplefast (vchar.c:213-312) */
static int simplefast(int dir, const geomref *g, const zstate *q, double cms2, double *vmin, double *vmax)
{
  double discr, Acov[NDIM], Bcov[NDIM], Acon[NDIM], Bcon[NDIM];
  double Asq, Bsq, Au, Bu, AB, Au2, Bu2, AuBu, A, B, vm, vp;
  int j;
  for (j = 0; j < NDIM; j++) Acov[j] = 0.;
  Acov[dir] = 1.;
  raise_vec(Acov, g, Acon);
  for (j = 0; j < NDIM; j++) Bcov[j] = 0.;
  Bcov[TT] = 1.;
  raise_vec(Bcov, g, Bcon);
  Asq = dot4(Acon, Acov);
  Bsq = dot4(Bcon, Bcov);
  Au = dot4(Acov, q->ucon);
  Bu = dot4(Bcov, q->ucon);
  AB = dot4(Acon, Bcov);
  Au2 = Au * Au;
  Bu2 = Bu * Bu;
  AuBu = Au * Bu;
  A = Bu2 * (1.0 - cms2) - Bsq * cms2;
  B = 2. * (AuBu * (1.0 - cms2) - AB * cms2);
  discr = 4.0 * cms2 * ((AB * AB - Asq * Bsq) * cms2 + (2.0 * AB * Au * Bu - Asq * Bu2 - Bsq * Au2) * (cms2 - 1.0));
  if ((discr < 0.0) && (discr > -1E-10)) discr = 0.0;
  else if (discr < 0.0) return ERR_VCHAR_DISCR;
  discr = sqrt(discr);
  vm = -(-B + discr) / (2. * A);
  vp = -(-B - discr) / (2. * A);
  if ((!isfinite(vm)) || (!isfinite(vp))) return ERR_NONFINITE_SPEED;
  if (vp < vm) {
    *vmax = vm;
    *vmin = vp;
  } else {
    *vmax = vp;
    *vmin = vm;
  }
  return 0;
}

/* vchar (vchar.c:37-171), TRUEFAST=0 */
static int vchar(const double *pr, const zstate *q, int dir, const geomref *g, double gam, double *vmax,
                 double *vmin)
{
  double bsq, WW, EF, va2, cs2, cms2, rho, u, P;
  bsq = dot4(q->bcon, q->bcov);
  rho = pr[RHO];
  u = pr[UU];
  if (u < 0) u = 0;
  if (rho < 0) rho = 0;
  P = (gam - 1.) * u;
  WW = rho + u + P;
  if (WW > 0.0) {
    double pressure = (gam - 1.) * u;
    double h = rho + u + pressure;
    cs2 = gam * pressure / h;
  } else WW = cs2 = 0.0;
  if (cs2 >= 1.0) cs2 = 1.0 - 1e-9;
  else if (cs2 <= 0.0) cs2 = 0.0;
  EF = bsq + WW;
  if (EF > 0.0) va2 = bsq / EF;
  else EF = va2 = 0.0;
  cms2 = cs2 + va2 - cs2 * va2;
  if (cms2 < 0.0) {
    if (cms2 / (cs2 + va2) > -NUMEPSILON * 100.0) cms2 = 0.0;
    else return ERR_COEFF_NEG;
  }
  if (cms2 > 1.) {
    if (cms2 < 1.0 + NUMEPSILON * 100.0) cms2 = 1.0;
    else if (rho < 0.0) cms2 = 1.0;
    else return ERR_COEFF_SUP;
  }
  return simplefast(dir, g, q, cms2, vmin, vmax);
}

static inline double fmax_ref(double a, double b) { return (a > b) ? a : b; } /* phys.c:1797 */
static inline double fmin_ref(double a, double b) { return (a > b) ? b : a; } /* phys.c:1804 */
static inline double fmin_macro(double a, double b) { return ((a) < (b)) ? (a) : (b); } /* MIN, global.h:751 */

/* ------------------------------------------------------------------ */
/* slopes and face fluxes (interppoint.c, flux.c, fluxcompute.c)       */
/* ------------------------------------------------------------------ */

#define MINMODB(a, b) ((fabs(a) < fabs(b)) ? (a) : (b))
#define MINMOD(a, b) (((a) * (b) <= 0) ? 0.0 : MINMODB(a, b))

/* slope_lim_3points (interppoint.c:387-443) */
static double slope3(int lim, double yl, double yc, double yr)
{
  double Dqm, Dqp, Dqc, s;
  if (lim == HGO_LIM_MC) {
    Dqm = 2.0 * (yc - yl);
    Dqp = 2.0 * (yr - yc);
    Dqc = 0.5 * (yr - yl);
    return MINMOD(Dqc, MINMOD(Dqm, Dqp));
  } else if (lim == HGO_LIM_VANL) {
    Dqm = (yc - yl);
    Dqp = (yr - yc);
    s = Dqm * Dqp;
    if (s <= 0.) return 0.;
    return (2.0 * s / (Dqm + Dqp));
  } else if (lim == HGO_LIM_MINM) {
    Dqm = 1.0 * (yc - yl);
    Dqp = 1.0 * (yr - yc);
    Dqc = 0.5 * (yr - yl);
    return MINMOD(MINMOD(Dqm, Dqc), Dqp);
  }
  return 0.0; /* DONOR */
}

/* para4 (interppoint.c:736-869) with PARA2LIM=MC (global.h:425-427, the
   "Xiaoyue" branch) and JONPARAREDUCE=0: left/right face values of the cell
   at y[0] from y[-2..2]; min/max are the functions of phys.c:1797-1812 */
static void para4(const double *y, double *lout, double *rout)
{
  double dq0[3], *dq = dq0 + 1, Dqm, Dqp, Dqc, aDqm, aDqp, aDqc, s, l, r, qa, qd, qe;
  int mm;
  for (mm = -1; mm <= 1; mm++) {
    Dqm = 2.0 * (y[mm] - y[mm - 1]);
    Dqp = 2.0 * (y[mm + 1] - y[mm]);
    Dqc = 0.5 * (y[mm + 1] - y[mm - 1]);
    aDqm = fabs(Dqm);
    aDqp = fabs(Dqp);
    aDqc = fabs(Dqc);
    s = Dqm * Dqp;
    if (s <= 0.) dq[mm] = 0.;
    else dq[mm] = fmin_ref(aDqc, fmin_ref(aDqm, aDqp)) * ((Dqc > 0.0) ? 1.0 : ((Dqc < 0.0) ? -1.0 : 0.0));
  }
  l = 0.5 * (y[0] + y[-1]) - (dq[0] - dq[-1]) / 8.0;
  r = 0.5 * (y[1] + y[0]) - (dq[1] - dq[0]) / 8.0;
  l = fmax_ref(fmin_ref(y[0], y[-1]), l);
  l = fmin_ref(fmax_ref(y[0], y[-1]), l);
  r = fmax_ref(fmin_ref(y[0], y[1]), r);
  r = fmin_ref(fmax_ref(y[0], y[1]), r);
  qa = (r - y[0]) * (y[0] - l);
  qd = (r - l);
  qe = 6.0 * (y[0] - 0.5 * (l + r));
  if (qa <= 0.) {
    l = y[0];
    r = y[0];
  } else {
    if (qd * (qd - qe) < 0.0) l = 3.0 * y[0] - 2.0 * r;
    if (qd * (qd + qe) < 0.0) r = 3.0 * y[0] - 2.0 * l;
  }
  *lout = l;
  *rout = r;
}

/* ------------------------------------------------------------------ */
/* WENO5 centre-to-edge line reconstruction (lim = WENO5)              */
/*                                                                     */
/* slope_lim_linetype_c2e (interpline.c:517-678) with the options of   */
/* the torus build: VARTOINTERP=PRIMTOINTERP, COMPUTEDRHODP=1, SMONO   */
/* (DOMONOINTERP=SMONOINTERP, SMONO_DO_SMOOTH_TRANSITION=1), stencil   */
/* reduction "AND" (DO_OR_STENCIL_REDUCTION=0), post/pre-shock dP/P    */
/* reduction, DO_SMOOTH_ADJUSTMENT_UNOPTIMIZED_WEIGHTS=1, no stencil   */
/* shift (STOREWAVESPEEDS=0), WENO_REDUCE_TYPE_DEFAULT.  The shock     */
/* indicator (get_shock_indicator, interpline.c:2025) is computed by   */
/* the reference but only read by the PPM-type reduction, so it has no */
/* effect here and is not computed.                                    */
/*                                                                     */
/* One output cell c reads the line from c-5 to c+5: unoptimised       */
/* weights and SMONO indicators at c-3..c+3 (each from c-2..c+2 of the */
/* line), weight ratios at c-1..c+1, dP/P at c (from c-1..c+1).  The   */
/* reference feeds the whole line including MAXBND ghosts; with its    */
/* default MAXBND=11 no stencil of an output cell -1..N reaches the    */
/* ends of the line, so every boundary-truncation branch of            */
/* compute_cf_stencil_weights / compute_weights_ratios is dead and     */
/* only ghost cells up to depth 6 are read.                            */
/* ------------------------------------------------------------------ */

#define WENO_EPS 1.e-26     /* WENO_EPSILON = REDUCEEPSILON (reconstructeno.h:195-200) */
#define SMONO_EPS 1.e-13    /* SMONO_EPSILON = SQRT_WENO_EPSILON (reconstructeno.h:73,196) */
#define W_MIN_RAT 1.3       /* MIN_TRANSITION_RATIO, AND reduction (reconstructeno.h:175-176) */
#define W_MAX_RAT 1.6
#define W_DP_FRAC (0.5)     /* REDUCE_DP_FRACTION (reconstructeno.h:96) */
#define W_BIG (1.e+50)      /* BIG (global.h:1040) */
#define W_MIN(a, b) (((a) < (b)) ? (a) : (b)) /* global.h:750-751 */
#define W_MAX(a, b) (((a) > (b)) ? (a) : (b))

/* sign (phys.c:1778-1783) */
static inline double w_sign(double a) { return (a > 0.0) ? 1.0 : ((a < 0.0) ? -1.0 : 0.0); }

/* get_sum_of_elements with SYMMETRIZE_WENO (reconstructeno.c:1920-1946):
   pairs a[i] with a[n-1-i], then adds the middle element times (n odd) */
static double w_sum(int n, const double *a)
{
  double s = 0.0;
  int i, h = n / 2;
  for (i = 0; i < h; i++) s += a[i] + a[n - 1 - i];
  s += a[i] * (double)(n % 2);
  return s;
}

/* normalize_array (reconstructeno.c:1948-1960) */
static double w_normalize(int n, double eps, double *a)
{
  double s = w_sum(n, a);
  int i;
  for (i = 0; i < n; i++) a[i] /= (s + eps);
  return s;
}

/* check_for_cusp_new (smonointerp.c:439-476) at line cell y[0] */
static int w_cusp(const double *y)
{
  double df[4], ddf[3], norm, f1a, f1, f2, f3, f3a, f4, f4a, f5a, f5, f6, f7, f7a, f8, f8a;
  double *dfp = df + 1, *ddfp = ddf + 1;
  int k;
  for (k = -1; k <= 2; k++) dfp[k] = y[k] - y[k - 1];
  for (k = -1; k <= 1; k++) ddfp[k] = dfp[k + 1] - dfp[k];
  norm = (fabs(y[-2]) + fabs(y[-1]) + fabs(y[0]) + fabs(y[1]) + fabs(y[2]) + SMALL);
  norm = norm * SMONO_EPS;
  f1a = fabs(dfp[0]) - norm;
  f1 = ddfp[-1] * w_sign(dfp[0]) - norm;
  f2 = -ddfp[0] * w_sign(dfp[0]) - norm;
  f3 = -dfp[2] * w_sign(dfp[0]) - norm;
  f3a = fabs(-dfp[2] - dfp[0]) - 0.25 * (fabs(dfp[2]) + fabs(dfp[0]));
  f4 = -dfp[1] * w_sign(dfp[0]) - norm;
  f4a = fabs(-dfp[1] - dfp[0]) - 0.25 * (fabs(dfp[1]) + fabs(dfp[0]));
  if (f1a > 0 && f1 > 0 && f2 > 0 && ((f3 > 0 && f3a > 0) || (f4 > 0 && f4a > 0))) return 1;
  f5a = fabs(dfp[1]) - norm;
  f5 = -ddfp[1] * w_sign(dfp[1]) - norm;
  f6 = ddfp[0] * w_sign(dfp[1]) - norm;
  f7 = -dfp[-1] * w_sign(dfp[1]) - norm;
  f7a = fabs(-dfp[-1] - dfp[1]) - 0.25 * (fabs(dfp[-1]) + fabs(dfp[1]));
  f8 = -dfp[0] * w_sign(dfp[1]) - norm;
  f8a = fabs(-dfp[0] - dfp[1]) - 0.25 * (fabs(dfp[0]) + fabs(dfp[1]));
  if (f5a > 0 && f5 > 0 && f6 > 0 && ((f7 > 0 && f7a > 0) || (f8 > 0 && f8a > 0))) return 1;
  return 0;
}

/* compute_mono_indicator_point_eno5 (smonointerp.c:296-425) with
   DO_MONO_1ST_DERIVATIVE=1, DO_3RD_DER=1, and transition_function
   (smonointerp.c:428-437): derivatives of the 5-point polynomial at -1 and +1 */
static double w_mono(const double *y)
{
  double ld[4], rd[4], mm, minabs = W_BIG, norm, cut, v;
  int n;
  ld[1] = (((-3 * y[-2] + y[2]) + (-10 * y[-1] - 6 * y[1])) + 18 * y[0]) / 12.;
  ld[2] = (((11 * y[-2] - y[2]) + (-20 * y[-1] + 4 * y[1])) + 6 * y[0]) / 12.;
  ld[3] = (((-3 * y[-2] - y[2]) + (10 * y[-1] + 6 * y[1])) - 12 * y[0]) / 2.;
  rd[1] = (((-y[-2] + 3 * y[2]) + (6 * y[-1] + 10 * y[1])) - 18 * y[0]) / 12.;
  rd[2] = (((-y[-2] + 11 * y[2]) + (4 * y[-1] - 20 * y[1])) + 6 * y[0]) / 12.;
  rd[3] = (((y[-2] + 3 * y[2]) - (6 * y[-1] + 10 * y[1])) + 12 * y[0]) / 2.;
  ld[1] = MINMOD(ld[1], y[-1] - y[-2]);
  rd[1] = MINMOD(rd[1], y[2] - y[1]);
  for (n = 1; n <= 3; n++) {
    mm = MINMOD(ld[n], rd[n]);
    minabs = W_MIN(minabs, fabs(mm));
  }
  norm = fabs(y[0]) + ((fabs(y[-1]) + fabs(y[1])) + (fabs(y[-2]) + fabs(y[2])));
  cut = norm * SMONO_EPS + DBL_MIN;
  v = (minabs - 0.0) / (cut - 0.0);
  return W_MAX(0., W_MIN(1., v));
}

/* c2e_simple_eno(5, ...) (reconstructeno.c:826-901): the central row of the
   5-point centre-to-left / centre-to-right Lagrange matrices */
static double w_eno5(int right, const double *y)
{
  static const double cl[5] = {-5. / 128., 15. / 32., 45. / 64., -5. / 32., 3. / 128.};
  static const double cr[5] = {3. / 128., -5. / 32., 45. / 64., 15. / 32., -5. / 128.};
  const double *c = right ? cr : cl;
  double d[5];
  int k;
  for (k = 0; k < 5; k++) d[k] = c[k] * y[k - 2];
  return w_sum(5, d);
}

/* WENO weight set of one cell: weights[0..order-1] unoptimised,
   [order..2order-1] left-face, [2order..3order-1] right-face optimised
   (weno_weights_s, reconstructeno.h:146-160) */
typedef struct {
  double w[9];
  int order;
  double lof, fordpp;
} wset;

/* optimal centre-to-face weights c2e_optimal_weights_{left,right}face
   (reconstructeno_static.h) for order 2 and 3 */
static const double w_optl[2][3] = {{1. / 4., 3. / 4, 0.0}, {1. / 16., 5. / 8., 5. / 16.}};
static const double w_optr[2][3] = {{3. / 4., 1. / 4., 0.0}, {5. / 16., 5. / 8., 1. / 16.}};

/* compute_cf_stencil_weights (reconstructeno.c:1406-1614) for order 2 or 3
   on a long line, followed for order 3 by mono_adjust_unoptimized_weights
   (reconstructeno.c:702-728); m0 = monoindicator[0], cusp = (m0 == 0 and
   monoindicator[1] != 0) */
static void w_unopt(int order, double m0, int cusp, const double *u, wset *s)
{
  double si[3], fd[3], sd[3], u2[5], normu, e;
  int sh, i;
  s->lof = 0.;
  s->order = order;
  if (m0 == 1) {
    for (i = 0; i < order; i++) s->w[i] = 1.0 / order;
    return;
  } else if (m0 == 0 && cusp) {
    s->lof = 1.0;
  }
  if (order == 2) {
    fd[0] = u[1] - u[0];
    fd[1] = u[0] - u[-1];
    for (sh = 0; sh < 2; sh++) si[sh] = fd[sh] * fd[sh];
  } else {
    fd[0] = -(3 * u[0] + u[2]) + 4 * u[1];
    fd[1] = u[1] - u[-1];
    fd[2] = (3 * u[0] + u[-2]) - 4 * u[-1];
    sd[0] = (u[0] + u[2]) - 2 * u[1];
    sd[1] = (u[-1] + u[1]) - 2 * u[0];
    sd[2] = (u[0] + u[-2]) - 2 * u[-1];
    for (sh = 0; sh < 3; sh++) si[sh] = 13. / 12. * sd[sh] * sd[sh] + 1. / 4. * fd[sh] * fd[sh];
  }
  /* desensitise_smoothness_indicators (reconstructeno.c:1687-1707), USE_NORMU=1 */
  for (i = -order + 1; i < order; i++) u2[i + order - 1] = u[i] * u[i];
  normu = w_sum(2 * order - 1, u2);
  e = normu * WENO_EPS;
  for (sh = 0; sh < order; sh++) si[sh] += e;
  /* DO_NORMALIZE_SMOOTHNESS_INDICATORS=1 */
  w_normalize(order, DBL_MIN, si);
  /* compute_weights_from_smoothness_indicators (reconstructeno.c:1878-1917) */
  for (sh = 0; sh < order; sh++) {
    double t = si[sh] + WENO_EPS / 1.;
    t *= t;
    s->w[sh] = 1. / t;
  }
  w_normalize(order, 0, s->w);
  if (order == 3 && m0 > 0.0 && m0 < 1.0) {
    double simple = 1.0 / (double)order;
    for (i = 0; i < order; i++) s->w[i] = (1.0 - m0) * s->w[i] + m0 * simple;
  }
}

/* compute_optimized_cf_stencil_weights (reconstructeno.c:1617-1683) */
static void w_opt(double m0, wset *s)
{
  int o = s->order, sh;
  if (m0 == 1 || m0 == -1) return;
  for (sh = 0; sh < o; sh++) {
    s->w[o + sh] = s->w[sh] * w_optl[o - 2][sh];
    s->w[2 * o + sh] = s->w[sh] * w_optr[o - 2][sh];
  }
  w_normalize(o, DBL_MIN, &s->w[o]);
  w_normalize(o, DBL_MIN, &s->w[2 * o]);
}

/* eno_cvt (reconstructeno.c:730-823) for CVT_C2L (right=0) / CVT_C2R (right=1)
   with the order-2/3 centre-to-face matrices (reconstructeno_static.h) */
static double w_cvt(const wset *s, int right, const double *u)
{
  static const double l2[2][2] = {{3. / 2., -1. / 2.}, {1. / 2., 1. / 2.}};
  static const double r2[2][2] = {{1. / 2., 1. / 2.}, {-1. / 2., 3. / 2.}};
  static const double l3[3][3] = {{15. / 8., -5. / 4., 3. / 8.}, {3. / 8., 3. / 4., -1. / 8.}, {-1. / 8., 3. / 4., 3. / 8.}};
  static const double r3[3][3] = {{3. / 8., 3. / 4., -1. / 8.}, {-1. / 8., 3. / 4., 3. / 8.}, {3. / 8., -5. / 4., 15. / 8.}};
  int o = s->order, sh, j;
  const double *w = s->w + o * (right ? 2 : 1);
  double pu[3], su[3];
  for (sh = 0; sh < o; sh++) {
    for (j = 0; j < o; j++) pu[j] = (o == 2 ? (right ? r2[sh][j] : l2[sh][j]) : (right ? r3[sh][j] : l3[sh][j])) * u[j - sh];
    su[sh] = 0.0;
    if (w[sh] != 0.0) su[sh] = w[sh] * w_sum(o, pu);
  }
  return w_sum(o, su);
}

/* compute_df_line_new (interpline.c:2148-2222): dP/P-type jump indicator at
   line cell c from the primitives at c-1, c, c+1 and their CENT metrics */
static double w_dp(const double *pm, const double *p0, const double *pp, const geomref *gm, const geomref *g0,
                   const geomref *gp, double gam)
{
  zstate ql, q, qr;
  double a, b, c_, parl, par, parr, uparl, upar, uparr;
  get_state(pm, gm, &ql);
  get_state(p0, g0, &q);
  get_state(pp, gp, &qr);
  a = compute_1plusud0(gm, &ql);
  b = compute_1plusud0(g0, &q);
  c_ = compute_1plusud0(gp, &qr);
  parl = a * (ql.ucon[TT]);
  par = b * (q.ucon[TT]);
  parr = c_ * (qr.ucon[TT]);
  uparl = gam * pm[UU] * (ql.ucon[TT] * ql.ucov[TT]) + (gam - 1.0) * pm[UU];
  upar = gam * p0[UU] * (q.ucon[TT] * q.ucov[TT]) + (gam - 1.0) * p0[UU];
  uparr = gam * pp[UU] * (qr.ucon[TT] * qr.ucov[TT]) + (gam - 1.0) * pp[UU];
  return (fabs(p0[RHO] * (parr - parl)) + fabs(uparr - uparl)) / (fabs(p0[RHO] * par) + fabs(upar) + DBL_MIN);
}

/* eno_line_reconstruct (reconstructeno.c:261-563) for CVT_C2E together with
   compute_smonotonicity_line (smonointerp.c:15-175): y is the line of one
   primitive (valid at -6..n+5), dP the jump indicator (valid at -1..n);
   yl/yr receive the left/right face values of cells -1..n (index +1). */
static void weno5_line(int n, const double *y, const double *dP, double *yl, double *yr, wset *ws, double *m0,
                       int *cusp)
{
  int c;
  /* SMONO indicators and unoptimised weights at -4..n+3 (index +4) */
  for (c = -4; c <= n + 3; c++) {
    int q = c + 4;
    cusp[q] = w_cusp(&y[c]);
    m0[q] = cusp[q] ? 0.0 : w_mono(&y[c]);
    w_unopt(3, m0[q], cusp[q], &y[c], &ws[q]);
  }
  /* compute_weights_ratios (reconstructeno.c:1962-2083) at -2..n+1: both
     neighbours are inside the line, AND reduction, C2E ratios */
  for (c = -2; c <= n + 1; c++) {
    wset *s = &ws[c + 4];
    double wrl, wrr, wr, lof, minr = W_MIN_RAT, maxr = W_MAX_RAT;
    wrl = (s->w[2] + WENO_EPS) / (ws[c + 4 - 2].w[0] + WENO_EPS);
    wrr = (s->w[0] + WENO_EPS) / (ws[c + 4 + 2].w[2] + WENO_EPS);
    wr = W_MIN(wrl, wrr);
    lof = (wr - minr) / (maxr - minr);
    lof = W_MAX(0., W_MIN(lof, 1.0));
    s->lof = W_MAX(lof, s->lof);
    s->fordpp = s->lof;
  }
  /* apply_additional_reduction_to_weights (reconstructeno.c:650-700): post-
     and pre-shock reduction from dP/P; reads fordpp only, so order-free */
  for (c = -1; c <= n; c++) {
    wset *s = &ws[c + 4];
    double ss = W_MIN((fabs(dP[c]) - 0.5 * W_DP_FRAC) / (0.5 * W_DP_FRAC), 1.);
    double lof = s->lof;
    lof = W_MAX(lof, ss * ws[c + 4 + 1].fordpp);
    lof = W_MAX(lof, ss * ws[c + 4 - 1].fordpp);
    s->lof = lof;
  }
  /* optimised weights, choose_weno_order (reconstructeno.c:2087-2247) and
     the output combination (reconstructeno.c:470-545) */
  for (c = -1; c <= n; c++) {
    int q = c + 4, side;
    wset hi = ws[q], lo;
    double lof, mi = m0[q];
    w_opt(mi, &hi);
    lof = hi.lof;
    if (0.0 < lof) {
      int k;
      for (k = 3; k < 9; k++) hi.w[k] *= (1. - lof);
      w_unopt(2, mi, cusp[q], &y[c], &lo);
      w_opt(mi, &lo);
      for (k = 0; k < 6; k++) lo.w[k] *= lof;
    }
    for (side = 0; side < 2; side++) {
      double *out = side ? &yr[c + 1] : &yl[c + 1];
      /* SMONO's 5-point value where its indicator is nonzero (cusps have
         indicator 0); eno_line_reconstruct zeroes the output where it is 0 */
      double prev = (mi != 0.0) ? w_eno5(side, &y[c]) : 0.0;
      if (mi >= 0.0 && mi < 1.0) {
        double v = 0.0;
        v += w_cvt(&hi, side, &y[c]);
        if (0.0 < lof) v += w_cvt(&lo, side, &y[c]);
        prev = (1.0 - mi) * v + mi * prev;
      }
      *out = prev;
    }
  }
}

/* flux_compute_general (fluxcompute.c:12-51) for one face */
static int face_flux(const hgo_config *c, int dir, const geomref *g, double *p_l, double *p_r, double *F, double *ctop)
{
  zstate ql, qr;
  emstate el, er;
  double Fl[NPR], Fr[NPR], Ul[NPR], Ur[NPR];
  double cminl, cmaxl, cminr, cmaxr, lmin, lmax, cmin, cmax;
  int pl, e;
  if (get_state(p_l, g, &ql)) return ERR_UTCALC_DISCR;
  em_prepare(p_l, g, &ql, &el);
  primtoflux(p_l, &ql, &el, dir, g, c->gam, Fl);
  primtoflux(p_l, &ql, &el, TT, g, c->gam, Ul);
  if (get_state(p_r, g, &qr)) return ERR_UTCALC_DISCR;
  em_prepare(p_r, g, &qr, &er);
  primtoflux(p_r, &qr, &er, dir, g, c->gam, Fr);
  primtoflux(p_r, &qr, &er, TT, g, c->gam, Ur);
  if ((e = vchar(p_l, &ql, dir, g, c->gam, &cmaxl, &cminl))) return e;
  if ((e = vchar(p_r, &qr, dir, g, c->gam, &cmaxr, &cminr))) return e;
  /* cminmax_calc (wavespeeds.c:325-385), HYPERHLL=0 */
  lmin = fmin_ref(cminl, cminr);
  lmax = fmax_ref(cmaxl, cmaxr);
  lmin = fabs(fmax_ref(0., -lmin));
  lmax = fabs(fmax_ref(0., lmax));
  cmin = lmin;
  cmax = lmax;
  *ctop = fmax_ref(lmax, lmin);
  if (c->fluxmethod == HGO_FLUX_HLL && (cmax + cmin != 0.0)) {
    for (pl = 0; pl < NPR; pl++) F[pl] = ((cmax * Fl[pl] + cmin * Fr[pl]) - (cmax * cmin) * (Ur[pl] - Ul[pl])) / (cmax + cmin);
  } else {
    for (pl = 0; pl < NPR; pl++) F[pl] = (0.5 * ((Fl[pl] + Fr[pl]) - (*ctop) * (Ur[pl] - Ul[pl])));
  }
  return 0;
}

static long dom_ntot(const dom *d);

/* slope_lim_linetype_c2e (interpline.c:517-678) for the lines along `dir`
   through the transverse ranges of the flux loop: pleft/pright (the
   reference's arrays, AoS with NPR per zone) of the line cells -1..n */
static void weno5_faces(dom *d, const double *pr, int dir, int is, int ie, int js, int je, int ks, int ke,
                        double *pleft, double *pright)
{
  int n = d->n[dir], a, b, c, pl;
  int ta0, ta1, tb0, tb1;
  int L = n + 12; /* line cells -6..n+5 */
  double *y = (double *)malloc(sizeof(double) * L), *dP = (double *)malloc(sizeof(double) * (n + 2));
  double *yl = (double *)malloc(sizeof(double) * (n + 2)), *yr = (double *)malloc(sizeof(double) * (n + 2));
  double *m0 = (double *)malloc(sizeof(double) * (n + 8));
  int *cusp = (int *)malloc(sizeof(int) * (n + 8));
  wset *ws = (wset *)malloc(sizeof(wset) * (n + 8));
  /* transverse ranges: the two directions other than dir */
  if (dir == 1) { ta0 = js; ta1 = je; tb0 = ks; tb1 = ke; }
  else if (dir == 2) { ta0 = is; ta1 = ie; tb0 = ks; tb1 = ke; }
  else { ta0 = is; ta1 = ie; tb0 = js; tb1 = je; }
  for (a = ta0; a <= ta1; a++)
    for (b = tb0; b <= tb1; b++) {
#define CELL(cc) ((dir == 1) ? zidx(d, (cc), a, b) : ((dir == 2) ? zidx(d, a, (cc), b) : zidx(d, a, b, (cc))))
      /* dP/P from the primitives along the line (get_df_line_gen_new, interpline.c:1152-1198) */
      for (c = -1; c <= n; c++) {
        geomref gm, g0, gp;
        int im = (dir == 1) ? c - 1 : a, jm = (dir == 2) ? c - 1 : ((dir == 1) ? a : b);
        int i0 = (dir == 1) ? c : a, j0 = (dir == 2) ? c : ((dir == 1) ? a : b);
        int ip = (dir == 1) ? c + 1 : a, jp = (dir == 2) ? c + 1 : ((dir == 1) ? a : b);
        get_geometry(d, im, jm, CENT, &gm);
        get_geometry(d, i0, j0, CENT, &g0);
        get_geometry(d, ip, jp, CENT, &gp);
        dP[c + 1] = w_dp(&pr[CELL(c - 1) * NPR], &pr[CELL(c) * NPR], &pr[CELL(c + 1) * NPR], &gm, &g0, &gp, d->c->gam);
      }
      for (pl = 0; pl < NPR; pl++) {
        for (c = -6; c <= n + 5; c++) y[c + 6] = pr[CELL(c) * NPR + pl];
        weno5_line(n, y + 6, dP + 1, yl, yr, ws, m0, cusp);
        for (c = -1; c <= n; c++) {
          pleft[CELL(c) * NPR + pl] = yl[c + 1];
          pright[CELL(c) * NPR + pl] = yr[c + 1];
        }
      }
#undef CELL
    }
  free(y); free(dP); free(yl); free(yr); free(m0); free(cusp); free(ws);
}

/* fluxcalc_standard for one direction (flux.c:469-680) with MC-type slopes */
static void fluxcalc_dir(dom *d, const double *pr, int dir, double *F, double *dq, double *ndt)
{
  const hgo_config *c = d->c;
  int is, ie, js, je, ks, ke, i, j, k, pl;
  int di = (dir == 1), dj = (dir == 2), dk = (dir == 3);
  int n1 = d->n[1], n2 = d->n[2], n3 = d->n[3];
  geomref g;
  double p_l[NPR], p_r[NPR], ctop = 0.0, dtij;
  int loc = (dir == 1) ? FACE1 : ((dir == 2) ? FACE2 : FACE3);
  long dofs = (long)di * d->nt[2] * d->nt[3] + (long)dj * d->nt[3] + dk;

  *ndt = BIG;
  if (d->n[dir] == 1) return;

  if (c->doenoflux == HGO_ENOFINITEVOLUME) {
    /* interp_loop_set (initbase.c:952-994), ENOFINITEVOLUME with avgo = 0:
       the faces along dir, every transverse zone including all ghosts
       (INFULL..OUTFULL); the dt minimum runs over all of them */
    is = (dir == 1) ? 0 : -d->ng[1];
    ie = (dir == 1) ? n1 : n1 - 1 + d->ng[1];
    js = (dir == 2) ? 0 : -d->ng[2];
    je = (dir == 2) ? n2 : n2 - 1 + d->ng[2];
    ks = (dir == 3) ? 0 : -d->ng[3];
    ke = (dir == 3) ? n3 : n3 - 1 + d->ng[3];
  } else {
    /* interp_loop_set (initbase.c:1010-1058), NOENOFLUX */
    is = (dir == 1) ? 0 : -d->sh[1];
    ie = (dir == 1) ? n1 - 1 + d->sh[1] : n1 - 1 + d->sh[1];
    js = (dir == 2) ? 0 : -d->sh[2];
    je = (dir == 2) ? n2 - 1 + d->sh[2] : n2 - 1 + d->sh[2];
    ks = (dir == 3) ? 0 : -d->sh[3];
    ke = (dir == 3) ? n3 - 1 + d->sh[3] : n3 - 1 + d->sh[3];
  }

  if (c->lim == HGO_LIM_WENO5) {
    weno5_faces(d, pr, dir, is, ie, js, je, ks, ke, dq, dq + dom_ntot(d) * NPR);
  } else if (c->lim == HGO_LIM_PARA) {
    /* slope_lim_pointtype (interppoint.c:21-151) -> slope_lim_point -> para4
       on the cells the faces read; pleft | pright as for the line methods */
    double *pleft = dq, *pright = dq + dom_ntot(d) * NPR;
    for (i = is - di; i <= ie; i++)
      for (j = js - dj; j <= je; j++)
        for (k = ks - dk; k <= ke; k++) {
          long z = zidx(d, i, j, k);
          for (pl = 0; pl < NPR; pl++) {
            double y[5];
            int l;
            for (l = -2; l <= 2; l++) y[l + 2] = pr[(z + l * dofs) * NPR + pl];
            para4(y + 2, &pleft[z * NPR + pl], &pright[z * NPR + pl]);
          }
        }
  } else {
    /* slopes over the zones the faces read: centers (face-1) and (face) */
    for (i = is - di; i <= ie; i++)
      for (j = js - dj; j <= je; j++)
        for (k = ks - dk; k <= ke; k++) {
          long z = zidx(d, i, j, k);
          for (pl = 0; pl < NPR; pl++)
            dq[z * NPR + pl] = slope3(c->lim, pr[(z - dofs) * NPR + pl], pr[z * NPR + pl], pr[(z + dofs) * NPR + pl]);
        }
  }

  for (i = is; i <= ie; i++)
    for (j = js; j <= je; j++)
      for (k = ks; k <= ke; k++) {
        long z = zidx(d, i, j, k);
        long zm = z - dofs;
        int e;
        /* getp2interplr (flux.c:788-808) */
        if (c->lim == HGO_LIM_WENO5 || c->lim == HGO_LIM_PARA) {
          const double *pleft = dq, *pright = dq + dom_ntot(d) * NPR;
          for (pl = 0; pl < NPR; pl++) {
            p_l[pl] = pright[zm * NPR + pl];
            p_r[pl] = pleft[z * NPR + pl];
          }
        } else {
          for (pl = 0; pl < NPR; pl++) {
            p_l[pl] = pr[zm * NPR + pl] + 0.5 * dq[zm * NPR + pl];
            p_r[pl] = pr[z * NPR + pl] - 0.5 * dq[z * NPR + pl];
          }
        }
        get_geometry(d, i, j, loc, &g);
        /* BDIRCONT (flux.c:629-633) */
        p_l[B1 + dir - 1] = p_r[B1 + dir - 1] = 0.5 * (p_l[B1 + dir - 1] + p_r[B1 + dir - 1]);
        e = face_flux(c, dir, &g, p_l, p_r, &F[z * NPR], &ctop);
        if (e) d->err |= e;
        dtij = c->cour * c->dx[dir] / ctop;
        if (dtij < *ndt) *ndt = dtij;
      }
}

/* flux_ct, FLUXCTTOTH with CORNGDETVERSION=1 (fluxct.c:10-844).
   The reference strips/averages over nearly the whole array; only the faces
   of the flux loops (initbase.c:1010-1058) and the corners that the updated
   faces read matter, and those are the ranges used here. */
static void flux_ct(dom *d, double *F1, double *F2, double *F3, double *emf)
{
  int n1 = d->n[1], n2 = d->n[2], n3 = d->n[3];
  int s1 = d->sh[1], s2 = d->sh[2], s3 = d->sh[3];
  int i, j, k;
  long ntot = (long)d->nt[1] * d->nt[2] * d->nt[3];
  long o1 = (long)d->nt[2] * d->nt[3], o2 = d->nt[3], o3 = 1;
  double coef1, coef2, coef3;
  double *e1 = emf, *e2 = emf + ntot, *e3 = emf + 2 * ntot;
  geomref g;

  /* strip gdet (fluxct.c:74-96) on the flux-loop faces */
  if (n1 > 1)
    for (i = 0; i <= n1; i++)
      for (j = -s2; j <= n2 - 1 + s2; j++)
        for (k = -s3; k <= n3 - 1 + s3; k++) {
          long z = zidx(d, i, j, k);
          get_geometry(d, i, j, FACE1, &g);
          F1[z * NPR + B1] /= g.g;
          F1[z * NPR + B2] /= g.g;
          F1[z * NPR + B3] /= g.g;
        }
  if (n2 > 1)
    for (i = -s1; i <= n1 - 1 + s1; i++)
      for (j = 0; j <= n2; j++)
        for (k = -s3; k <= n3 - 1 + s3; k++) {
          long z = zidx(d, i, j, k);
          get_geometry(d, i, j, FACE2, &g);
          F2[z * NPR + B1] /= g.g;
          F2[z * NPR + B2] /= g.g;
          F2[z * NPR + B3] /= g.g;
        }
  if (n3 > 1)
    for (i = -s1; i <= n1 - 1 + s1; i++)
      for (j = -s2; j <= n2 - 1 + s2; j++)
        for (k = 0; k <= n3; k++) {
          long z = zidx(d, i, j, k);
          get_geometry(d, i, j, FACE3, &g);
          F3[z * NPR + B1] /= g.g;
          F3[z * NPR + B2] /= g.g;
          F3[z * NPR + B3] /= g.g;
        }

  coef1 = ((n2 > 1) && (n3 > 1)) ? 0.25 : 0.5;
  coef2 = ((n1 > 1) && (n3 > 1)) ? 0.25 : 0.5;
  coef3 = ((n1 > 1) && (n2 > 1)) ? 0.25 : 0.5;

  /* emf1 (fluxct.c:148-161) on i=0..n1-1, j=0..n2-1+s2, k=0..n3-1+s3; x CORN1 gdet */
  for (i = 0; i <= n1 - 1; i++)
    for (j = 0; j <= n2 - 1 + s2; j++)
      for (k = 0; k <= n3 - 1 + s3; k++) {
        long z = zidx(d, i, j, k);
        double v;
        if (n2 > 1 && n3 > 1)
          v = coef1 * (+F2[z * NPR + B3] + F2[(z - s3 * o3) * NPR + B3] - F3[z * NPR + B2] - F3[(z - s2 * o2) * NPR + B2]);
        else if (n2 > 1)
          v = coef1 * (+F2[z * NPR + B3] + F2[(z - s3 * o3) * NPR + B3]);
        else if (n3 > 1)
          v = coef1 * (-F3[z * NPR + B2] - F3[(z - s2 * o2) * NPR + B2]);
        else
          v = 0.0;
        get_geometry(d, i, j, CORN1, &g);
        e1[z] = v * g.g;
      }
  /* emf2 (fluxct.c:166-179) on i=0..n1-1+s1, j=0..n2-1, k=0..n3-1+s3; x CORN2 gdet */
  for (i = 0; i <= n1 - 1 + s1; i++)
    for (j = 0; j <= n2 - 1; j++)
      for (k = 0; k <= n3 - 1 + s3; k++) {
        long z = zidx(d, i, j, k);
        double v;
        if (n1 > 1 && n3 > 1)
          v = coef2 * (+F3[z * NPR + B1] + F3[(z - s1 * o1) * NPR + B1] - F1[z * NPR + B3] - F1[(z - s3 * o3) * NPR + B3]);
        else if (n3 > 1)
          v = coef2 * (+F3[z * NPR + B1] + F3[(z - s1 * o1) * NPR + B1]);
        else if (n1 > 1)
          v = coef2 * (-F1[z * NPR + B3] - F1[(z - s3 * o3) * NPR + B3]);
        else
          v = 0.0;
        get_geometry(d, i, j, CORN2, &g);
        e2[z] = v * g.g;
      }
  /* emf3 (fluxct.c:184-197) on i=0..n1-1+s1, j=0..n2-1+s2, k=0..n3-1; x CORN3 gdet */
  for (i = 0; i <= n1 - 1 + s1; i++)
    for (j = 0; j <= n2 - 1 + s2; j++)
      for (k = 0; k <= n3 - 1; k++) {
        long z = zidx(d, i, j, k);
        double v;
        if (n1 > 1 && n2 > 1)
          v = coef3 * (+F1[z * NPR + B2] + F1[(z - s2 * o2) * NPR + B2] - F2[z * NPR + B1] - F2[(z - s1 * o1) * NPR + B1]);
        else if (n1 > 1)
          v = coef3 * (+F1[z * NPR + B2] + F1[(z - s2 * o2) * NPR + B2]);
        else if (n2 > 1)
          v = coef3 * (-F2[z * NPR + B1] - F2[(z - s1 * o1) * NPR + B1]);
        else
          v = 0.0;
        get_geometry(d, i, j, CORN3, &g);
        e3[z] = v * g.g;
      }

  /* B fluxes from EMFs on the faces read by the update (fluxct.c:724-781) */
  if (n1 > 1)
    for (i = 0; i <= n1; i++)
      for (j = 0; j <= n2 - 1; j++)
        for (k = 0; k <= n3 - 1; k++) {
          long z = zidx(d, i, j, k);
          F1[z * NPR + B1] = 0.;
          F1[z * NPR + B2] = 0.5 * (e3[z] + e3[z + s2 * o2]);
          F1[z * NPR + B3] = -0.5 * (e2[z] + e2[z + s3 * o3]);
        }
  if (n2 > 1)
    for (i = 0; i <= n1 - 1; i++)
      for (j = 0; j <= n2; j++)
        for (k = 0; k <= n3 - 1; k++) {
          long z = zidx(d, i, j, k);
          F2[z * NPR + B1] = -0.5 * (e3[z] + e3[z + s1 * o1]);
          F2[z * NPR + B2] = 0.;
          F2[z * NPR + B3] = 0.5 * (e1[z] + e1[z + s3 * o3]);
        }
  if (n3 > 1)
    for (i = 0; i <= n1 - 1; i++)
      for (j = 0; j <= n2 - 1; j++)
        for (k = 0; k <= n3; k++) {
          long z = zidx(d, i, j, k);
          F3[z * NPR + B1] = 0.5 * (e2[z] + e2[z + s1 * o1]);
          F3[z * NPR + B2] = -0.5 * (e1[z] + e1[z + s2 * o2]);
          F3[z * NPR + B3] = 0.;
        }
}

/* ------------------------------------------------------------------ */
/* con-to-prim: Utoprim_2d_final (utoprim_2d_final.c)                   */
/* ------------------------------------------------------------------ */
typedef struct {
  double Bsq, QdotBsq, Qtsq, Qdotn, D, wglobal, gam, gammasq_too_big, vsq_too_big;
  int iters;
} u2pctx;

/* vsq_calc (utoprim_2d_final.c:457-470) */
static double vsq_calc(const u2pctx *c, double W)
{
  double Wsq = W * W;
  double Xsq = (c->Bsq + W) * (c->Bsq + W);
  return ((Wsq * c->Qtsq + c->QdotBsq * (c->Bsq + 2. * W)) / (Wsq * Xsq));
}

/* EOS pieces (utoprim_jon_eos.c:83-108, :214-247, :316-345, :433-437; eos.c:178-194) */
static double wmrho0_compute_vsq(double Wp, double D, double vsq, double gamma, double gammasq)
{
  return (Wp / gammasq - D * vsq / (1.0 + gamma));
}

static double pressure_W_vsq(const u2pctx *c, double W, double D, double vsq)
{
  double Wp = W - D;
  double gamma = 1.0 / sqrt(1.0 - vsq);
  double gammasq = gamma * gamma;
  double wmrho0 = wmrho0_compute_vsq(Wp, D, vsq, gamma, gammasq);
  return ((c->gam - 1.0) / c->gam) * wmrho0; /* pressure_wmrho0_grmhd: IGAMMAR*wmrho0 */
}

static double dpdW_calc_vsq(const u2pctx *c, double W, double D, double vsq)
{
  double Wp = W - D;
  double gamma = 1.0 / sqrt(1.0 - vsq);
  double gammasq = gamma * gamma;
  double idwmrho0dp, dwmrho0dW, drho0dW, idrho0dp;
  (void)wmrho0_compute_vsq(Wp, D, vsq, gamma, gammasq);
  idwmrho0dp = (c->gam - 1.0) / c->gam; /* compute_idwmrho0dp_grmhd: GAMMAM1/GAMMA */
  dwmrho0dW = 1.0 - vsq;
  drho0dW = 0.0;
  idrho0dp = 0.0; /* compute_idrho0dp_grmhd */
  return drho0dW * idrho0dp + dwmrho0dW * idwmrho0dp;
}

static double dpdvsq_calc(const u2pctx *c, double W, double D, double vsq)
{
  double Wp = W - D;
  double gamma = 1.0 / sqrt(1.0 - vsq);
  double idwmrho0dp, dwmrho0dvsq, drho0dvsq, idrho0dp;
  idwmrho0dp = (c->gam - 1.0) / c->gam;
  dwmrho0dvsq = (D * (gamma * 0.5 - 1.0) - Wp);
  drho0dvsq = -D * gamma * 0.5;
  idrho0dp = 0.0;
  return drho0dvsq * idrho0dp + dwmrho0dvsq * idwmrho0dp;
}

/* func_vsq2 (utoprim_2d_final.c:1189-1278) */
static void func_vsq2(const u2pctx *c, const double x[2], double dx[2], double *f, double *df)
{
  double W = x[0], vsq = x[1], Wsq = W * W;
  double p_tmp = pressure_W_vsq(c, W, c->D, vsq);
  double dPdW = dpdW_calc_vsq(c, W, c->D, vsq);
  double dPdvsq = dpdvsq_calc(c, W, c->D, vsq);
  double t2, t3, t4, t9, t11, t16, t18, t21, t23, t24, t25, t35, t36, t40;
  double Bsq = c->Bsq, QdotBsq = c->QdotBsq, Qtsq = c->Qtsq, Qdotn = c->Qdotn;
  double resid0, resid1;
  t2 = -0.5 * Bsq + dPdvsq;
  t3 = Bsq + W;
  t4 = t3 * t3;
  t9 = 1 / Wsq;
  t11 = Qtsq - vsq * t4 + QdotBsq * (Bsq + 2.0 * W) * t9;
  t16 = QdotBsq * t9;
  t18 = -Qdotn - 0.5 * Bsq * (1.0 + vsq) + 0.5 * t16 - W + p_tmp;
  t21 = 1 / t3;
  t23 = 1 / W;
  t24 = t16 * t23;
  t25 = -1.0 + dPdW - t24;
  t35 = t25 * t3 + (Bsq - 2.0 * dPdvsq) * (QdotBsq + vsq * Wsq * W) * t9 * t23;
  t36 = 1 / t35;
  dx[0] = -(t2 * t11 + t4 * t18) * t21 * t36;
  t40 = (vsq + t24) * t3;
  dx[1] = -(-t25 * t11 - 2.0 * t40 * t18) * t21 * t36;
  resid0 = t11;
  resid1 = t18;
  *df = -resid0 * resid0 - resid1 * resid1;
  *f = -0.5 * (*df);
}

/* general_newton_raphson with do_line_search = USE_LINE_SEARCH = -2
   (utoprim_2d_final.c:736-1119): plain Newton steps */
static int general_newton_raphson(u2pctx *c, double x[2])
{
  double f, df, dx[2], x_old[2], errx;
  int n_iter = 0, keep_iterating = 1, id, doing_extra = 0, i_extra = 0;
  errx = 1.;
  df = f = 1.;
  for (id = 0; id < 2; id++) x_old[id] = x[id];
  while (keep_iterating) {
    c->iters++;
    func_vsq2(c, x, dx, &f, &df);
    errx = 0.;
    for (id = 0; id < 2; id++) x_old[id] = x[id];
    for (id = 0; id < 2; id++) x[id] += dx[id];
    errx = (x[0] == 0.) ? fabs(dx[0]) : fabs(dx[0] / x[0]);
    /* validate_x (utoprim_2d_final.c:708-728) */
    x[0] = fabs(x[0]);
    x[0] = (x[0] / c->wglobal > c->gammasq_too_big) ? x_old[0] : x[0];
    x[1] = (x[1] > 1.) ? c->vsq_too_big : x[1];
    if ((fabs(errx) <= NEWT_TOL) && (doing_extra == 0) && (EXTRA_NEWT_ITER > 0)) doing_extra = 1;
    if (doing_extra == 1) i_extra++;
    if (((fabs(errx) <= NEWT_TOL) && (doing_extra == 0)) || (i_extra > EXTRA_NEWT_ITER) || (n_iter >= (MAX_NEWT_ITER - 1)))
      keep_iterating = 0;
    n_iter++;
  }
  if ((isfinite(f) == 0) || (isfinite(df) == 0) || (isfinite(x[0]) == 0) || (isfinite(x[1]) == 0)) return 1;
  if (fabs(errx) > MIN_NEWT_TOL) return 1;
  return 0;
}

/* Utoprim_2d_final + Utoprim_new_body.  U is the geometry-free conserved
   vector with rest mass included in U[UU] (utoprimgen.c:76-85); prim holds
   the guess on input.  Returns the pflag code. */
static int utoprim_2d_final(const double *U, const geomref *g, const hgo_config *cfg, double *prim, int *iters)
{
  double U_tmp[NPR], prim_tmp[NPR], alpha;
  double Bcon[4], Bcov[4], Qcov[4], Qcon[4], ncov[4], ncon[4], Qtcon[4];
  double QdotB, Qsq, rho0, u, p, w, gammasq, gamma, gtmp, W_last, W, utsq, vsq, Wtest;
  int i, j, retval, i_increase, lpflag;
  u2pctx c;
  double x[2];

  c.gam = cfg->gam;
  c.gammasq_too_big = cfg->gammafail * cfg->gammafail;
  c.vsq_too_big = (c.gammasq_too_big - 1.0) / (c.gammasq_too_big);
  c.iters = 0;

  for (i = B1; i <= B3; i++) prim[i] = U[i];
  alpha = 1.0 / sqrt(-GCON(g, 0, 0));
  for (i = RHO; i <= B3; i++) U_tmp[i] = alpha * U[i];
  for (i = 0; i < B1; i++) prim_tmp[i] = prim[i];
  for (i = B1; i <= B3; i++) prim_tmp[i] = alpha * prim[i];

  /* Utoprim_new_body (utoprim_2d_final.c:152-453) */
  lpflag = UTOPRIMNOFAIL;
  for (i = B1; i <= B3; i++) prim_tmp[i] = U_tmp[i];
  Bcon[0] = 0.;
  for (i = 1; i < 4; i++) Bcon[i] = U_tmp[B1 + i - 1];
  /* lower_g / raise_g (u2p_util.c:120-143): full-matrix sums starting from 0 */
  for (i = 0; i < 4; i++) {
    Bcov[i] = 0.;
    for (j = 0; j < 4; j++) Bcov[i] += GCOV(g, i, j) * Bcon[j];
  }
  for (i = 0; i < 4; i++) Qcov[i] = U_tmp[UU + i];
  for (i = 0; i < 4; i++) {
    Qcon[i] = 0.;
    for (j = 0; j < 4; j++) Qcon[i] += GCON(g, i, j) * Qcov[j];
  }
  c.Bsq = 0.;
  for (i = 1; i < 4; i++) c.Bsq += Bcon[i] * Bcov[i];
  QdotB = 0.;
  for (i = 0; i < 4; i++) QdotB += Qcov[i] * Bcon[i];
  c.QdotBsq = QdotB * QdotB;
  {
    /* ncov_calc (u2p_util.c:146-157) */
    double lapse = sqrt(-1. / GCON(g, 0, 0));
    ncov[0] = -lapse;
    ncov[1] = 0.;
    ncov[2] = 0.;
    ncov[3] = 0.;
  }
  for (i = 0; i < 4; i++) {
    ncon[i] = 0.;
    for (j = 0; j < 4; j++) ncon[i] += GCON(g, i, j) * ncov[j];
  }
  c.Qdotn = Qcon[0] * ncov[0];
  Qsq = 0.;
  for (i = 0; i < 4; i++) Qsq += Qcov[i] * Qcon[i];
  c.Qtsq = Qsq + c.Qdotn * c.Qdotn;
  c.D = U_tmp[RHO];

  utsq = 0.;
  for (i = 1; i < 4; i++)
    for (j = 1; j < 4; j++) utsq += GCOV(g, i, j) * prim_tmp[U1 + i - 1] * prim_tmp[U1 + j - 1];
  if ((utsq < 0.) && (fabs(utsq) < MAXNEGUTSQ)) utsq = 0.0;
  if (utsq < 0. || utsq > ((cfg->gammafail - 1.0) * (cfg->gammafail - 1.0))) {
    *iters = c.iters;
    return UTOPRIMFAILCONVGUESSUTSQ;
  }
  gammasq = 1. + utsq;
  gamma = sqrt(gammasq);
  rho0 = c.D / gamma;
  u = prim_tmp[UU];
  p = (cfg->gam - 1.) * u;
  w = rho0 + u + p;
  W_last = w * gammasq;
  i_increase = 0;
  while (((W_last * W_last * W_last * (W_last + 2. * c.Bsq) - c.QdotBsq * (2. * W_last + c.Bsq)) <=
          W_last * W_last * (c.Qtsq - c.Bsq * c.Bsq)) &&
         (i_increase < 10)) {
    W_last *= 10.;
    i_increase++;
  }
  c.wglobal = w;
  /* find_root_2D_gen (utoprim_2d_final.c:573-644), MAX_NEWT_RETRIES=0 */
  x[0] = fabs(W_last);
  {
    double vs = vsq_calc(&c, W_last);
    x[1] = (vs > 1.) ? c.vsq_too_big : vs;
  }
  retval = general_newton_raphson(&c, x);
  W = x[0];
  *iters = c.iters;
  if ((retval != 0) || (W == FAIL_VAL)) {
    return retval * 100 + 1;
  } else {
    Wtest = W / c.wglobal;
    if (Wtest <= 0. || Wtest > c.gammasq_too_big) return UTOPRIMFAILCONVW;
  }
  vsq = vsq_calc(&c, W);
  if ((vsq < 0.) && (fabs(vsq) < MAXNEGVSQ)) vsq = 0.0;
  if ((vsq > c.vsq_too_big) || (vsq < 0.0)) return UTOPRIMFAILCONVUTSQ;
  gtmp = sqrt(1. - vsq);
  gamma = 1. / gtmp;
  rho0 = c.D * gtmp;
  w = W * (1. - vsq);
  {
    double wmrho0 = w - rho0; /* pressure_rho0_w (eos.c:550-558) */
    p = ((cfg->gam - 1.0) / cfg->gam) * wmrho0;
  }
  u = w - (rho0 + p);
  if ((rho0 <= 0.) || (u < 0.)) {
    if ((rho0 <= 0.) && (u >= 0.)) lpflag = UTOPRIMFAILRHONEG;
    if ((rho0 > 0.) && (u < 0.)) lpflag = UTOPRIMFAILUNEG;
    if ((rho0 <= 0.) && (u < 0.)) lpflag = UTOPRIMFAILRHOUNEG;
    /* UTOPRIMFAILRETURNTYPE==UTOPRIMRETURNADJUSTED: assign anyway */
  }
  prim_tmp[RHO] = rho0;
  prim_tmp[UU] = u;
  for (i = 1; i < 4; i++) Qtcon[i] = Qcon[i] + ncon[i] * c.Qdotn;
  for (i = 1; i < 4; i++) prim_tmp[U1 + i - 1] = gamma / (W + c.Bsq) * (Qtcon[i] + QdotB * Bcon[i] / W);
  for (i = B1; i <= B3; i++) prim_tmp[i] = U_tmp[i];
  /* back in Utoprim_2d_final: ret == retval == 0 here */
  for (i = 0; i < B1; i++) prim[i] = prim_tmp[i];
  return lpflag;
}

/* ------------------------------------------------------------------ */
/* con-to-prim: Utoprim_jon_nonrelcompat_inputnorestmass (utoprim_jon.c) */
/* 1-D E'(W') Newton solve in W' = W - D (WHICHHOTINVERTER 3,             */
/* PRIMFROMVSQ 0, USE_LINE_SEARCH -2, JONGENNEWTSTUFF 1; u2p_defs.h with   */
/* PRECISEINVERSION 1 and OPTIMIZED 1), hot GRMHD, ideal-gas EOS.          */
/* ------------------------------------------------------------------ */
#define GAMMASQCHECKRESID (1e2)              /* u2p_defs.h:21 */
#define NEWT_TOL_ULTRAREL (NUMEPSILON)       /* u2p_defs.h:29 */
#define EXTRA_NEWT_ITER_ULTRAREL 2           /* u2p_defs.h:67 */

typedef struct {
  double Bsq, QdotB, QdotBsq, Qtsq, Qdotnp, D, wglobal, igammar, gammasq_too_big;
  int iters;
} jonctx;

static inline double jon_sign(double a) { return (a > 0.0) ? 1.0 : ((a < 0.0) ? -1.0 : 0.0); } /* phys.c:1778 */
static inline double jon_max(double a, double b) { return ((a) > (b)) ? (a) : (b); }           /* global.h:750 */

/* utsq_calc (utoprim_jon.c:1294-1315) */
static double jon_utsq(const jonctx *c, double W)
{
  double SoW = c->QdotB / W;
  double top = c->Qtsq + (c->Bsq + 2.0 * W) * SoW * SoW;
  double bottom = (c->Bsq * c->Bsq - c->Qtsq) + 2.0 * c->Bsq * W + W * W - SoW * SoW * (c->Bsq + 2.0 * W);
  return top / bottom;
}

/* dvsq_dW (utoprim_jon.c:1378-1398) */
static double jon_dvsq_dW(const jonctx *c, double W)
{
  double X = c->Bsq + W;
  double Wsq = W * W;
  double W3 = Wsq * W;
  double X3 = X * X * X;
  return (-2. * (c->Qtsq / X3 + c->QdotBsq * (3.0 * W * X + c->Bsq * c->Bsq) / (W3 * X3)));
}

/* wmrho0_compute_utsq (utoprim_jon_eos.c:474-478) */
static inline double jon_wmrho0(double Wp, double D, double utsq, double gamma, double gammasq)
{
  return ((Wp - D * utsq / (1.0 + gamma)) / gammasq);
}

/* pressure_Wp_utsq (utoprim_jon_eos.c:134-152) with pressure_wmrho0_grmhd (eos.c:178-181) */
static double jon_pressure(const jonctx *c, double Wp, double D, double utsq)
{
  double gammasq = 1.0 + utsq;
  double gamma = sqrt(gammasq);
  double wmrho0 = jon_wmrho0(Wp, D, utsq, gamma, gammasq);
  return c->igammar * wmrho0;
}

/* Eprime_Wp (utoprim_jon.c:1529-1554) */
static double jon_Eprime(const jonctx *c, double Wp)
{
  double W = Wp + c->D;
  double X = c->Bsq + W + SMALL;
  double X2 = X * X;
  double utsq = jon_utsq(c, W);
  double p_tmp;
  if (utsq < -0.1) utsq = 0.0;
  p_tmp = jon_pressure(c, Wp, c->D, utsq);
  return c->Qdotnp + Wp - p_tmp + 0.5 * c->Bsq + 0.5 * (c->Bsq * c->Qtsq - c->QdotBsq) / X2;
}

/* dEprimedWp (utoprim_jon.c:1558-1587) with dpdWp_calc_utsq / dpdvsq_calc2_Wp
   (utoprim_jon_eos.c:262-290, 391-426) and the ideal-gas derivatives
   compute_idwmrho0dp_grmhd = (gam-1)/gam, compute_idrho0dp_grmhd = 0
   (eos.c:184-194) */
static double jon_dEprime(const jonctx *c, double Wp)
{
  double D = c->D;
  double W = Wp + D;
  double X = c->Bsq + W + SMALL;
  double X3 = X * X * X;
  double utsq = jon_utsq(c, W);
  double dvsq, dp1, dp2, dpdWp, gammasq, gamma;
  if (utsq < -0.1) utsq = 0.0;
  dvsq = jon_dvsq_dW(c, W);
  gammasq = 1.0 + utsq;
  gamma = sqrt(gammasq);
  dp1 = 0.0 * 0.0 + (1.0 / gammasq) * c->igammar;
  dp2 = (-D * gamma * 0.5) * 0.0 + (D * (gamma * 0.5 - 1.0) - Wp) * c->igammar;
  dpdWp = dp1 + dp2 * dvsq;
  return (1.0 - dpdWp) - (c->Bsq * c->Qtsq - c->QdotBsq) / X3;
}

/* coldgrhd (utoprim_jon.c:1402-1425) */
static int jon_coldgrhd(double Qtsq, double D, double *Wp)
{
  double det = D * D + Qtsq;
  if (det < 0.0) return 1;
  if (D > 0.0) *Wp = Qtsq / (D + sqrt(det));
  else *Wp = Qtsq / (D - sqrt(det));
  return 0;
}

/* validate_Wp (utoprim_jon.c:1726-1758).  The reference leaves Wp unset
   when coldgrhd finds no root (D^2 + Qtsq < 0, which needs Qtsq < -D^2 < 0);
   here the step is then left as it is. */
static void jon_validate(const jonctx *c, double Wpold, double *Wpnew)
{
  double Wp;
  if (*Wpnew < -c->D && c->D > 0.0) {
    if (!jon_coldgrhd(c->Qtsq, c->D, &Wp)) *Wpnew = Wp * 10.0;
  }
  *Wpnew = (fabs(*Wpnew / c->wglobal) > c->gammasq_too_big) ? 0.5 * (Wpold + *Wpnew) : *Wpnew;
}

/* newt_errorcheck / newt_extracheck (utoprim_jon.c:3430-3458) */
static int jon_ultrarel(double x0, double wglobal)
{
  return (fabs(wglobal) > fabs(GAMMASQCHECKRESID)) || (fabs(x0) > fabs(GAMMASQCHECKRESID));
}
static int jon_errorcheck(double errx, double x0, double wglobal)
{
  return jon_ultrarel(x0, wglobal) ? (fabs(errx) <= NEWT_TOL_ULTRAREL) : (fabs(errx) <= NEWT_TOL);
}
static int jon_extracheck(double x0, double wglobal)
{
  return jon_ultrarel(x0, wglobal) ? EXTRA_NEWT_ITER_ULTRAREL : EXTRA_NEWT_ITER;
}

/* general_newton_raphson (utoprim_jon.c:2896-3424) for n = 1 with func_Eprime
   (utoprim_jon.c:2258-2281) and no line search: the step is damped by half and
   restarted from the previous iterate when the residual changed sign against
   the first one in the ultrarelativistic regime; errx is the relative size of
   the previous step (the last evaluation only checks), and the returned root is
   the last evaluated iterate.  The reference's final finite() test also reads
   x[1] of a one-element array; only x[0] is tested here. */
static int jon_newton(jonctx *c, double *xio)
{
  double x = *xio, x_old = x, x_older = x, dx = 0., dx_old = 1E30 * x;
  double f = 1., df = 1., errx = 1., resid, drdW;
  double xold0 = 0., residold = 0., damp = 1.0;
  int n_iter = 0, keep_iterating = 1, doing_extra = 0, i_extra = 0;
  while (keep_iterating) {
    c->iters++;
    resid = jon_Eprime(c, x);
    drdW = jon_dEprime(c, x);
    dx = -resid / drdW;
    f = 0.5 * resid * resid;
    df = -2. * f;
    x_older = x_old;
    x_old = x;
    if (n_iter == 0) {
      xold0 = x;
      residold = resid;
    } else if (jon_sign(residold) != jon_sign(resid)) {
      if (fabs(xold0) > GAMMASQCHECKRESID || fabs(x_old) > GAMMASQCHECKRESID) {
        damp = 0.5 * damp;
        x = x_older;
        dx = dx_old;
      }
    }
    x += damp * dx;
    errx = (c->wglobal == 0.) ? fabs(dx_old) : fabs(dx_old / jon_max(fabs(c->wglobal), fabs(x)));
    jon_validate(c, x_old, &x);
    dx_old = dx;
    if (jon_errorcheck(errx, x, c->wglobal) && (doing_extra == 0) && (jon_extracheck(x, c->wglobal) > 0))
      doing_extra = 1;
    if (doing_extra == 1) i_extra++;
    if ((jon_errorcheck(errx, x, c->wglobal) && (doing_extra == 0)) || (i_extra > jon_extracheck(x, c->wglobal)) ||
        (n_iter >= (MAX_NEWT_ITER - 1)))
      keep_iterating = 0;
    n_iter++;
  }
  if ((isfinite(f) == 0) || (isfinite(df) == 0) || (isfinite(x) == 0)) {
    *xio = x;
    return 1;
  }
  x = x_old;
  *xio = x;
  if (jon_errorcheck(errx, x, c->wglobal)) return 0;
  if (fabs(errx) <= MIN_NEWT_TOL) return 0;
  return 1;
}

/* Utoprim_jon_nonrelcompat_inputnorestmass (utoprim_jon.c:65-205) with
   Utoprim_new_body (:209-488), compute_setup_quantities (:494-636),
   set_guess_Wp + verify_Wlast (:640-812), check_Wp (:819-903) and Wp2prim
   (:949-1165).  U is geometry-free with no rest mass in U[UU]; prim holds
   the guess on input.  Returns the pflag code.  The reference returns 0 and
   reports through the flag; the non-B primitives are replaced whenever the
   Newton solve returned 0, so a flag of UTOPRIMFAILCONVW, a negative density
   or energy, or a flag of 1 (a root equal to FAIL_VAL) comes with new
   primitives, while UTOPRIMFAILCONVRET leaves the guess.  When the guess has
   u~^2 < -MAXNEGUTSQ or u~^2 > UTSQ_TOO_BIG the reference carries on with an
   unset W' guess (its return value is ignored, utoprim_jon.c:281), and when
   get_state fails on the guess its bsq_calc leaves b^2 unset; here the zone
   then keeps its guess with flag UTOPRIMFAILCONVGUESSUTSQ. */
static int utoprim_jon(const double *U, const geomref *g, const hgo_config *cfg, double *prim, int *iters)
{
  double U_tmp[NPR], prim_tmp[NPR], pr0[NPR], alpha;
  double Bcon[4], Bcov[4], ncov[4], ncon[4], Qcovp[4], Qconp[4], Qcov[4], Qcon[4], Qtcon[4], Qtcov[4];
  double utsq, gammasq, gamma, rho0, u, p, w, bsq, Wp_last, W_last, Wp, W, wmrho0, Wtest, lapse;
  int i, j, lpflag, retval, i_increase;
  jonctx c;

  c.igammar = (cfg->gam - 1.0) / cfg->gam; /* IGAMMAR = GAMMAM1/GAMMA (eos.c:50-54) */
  c.gammasq_too_big = cfg->gammafail * cfg->gammafail;
  c.iters = 0;
  *iters = 0;

  for (i = B1; i <= B3; i++) prim[i] = U[i];
  alpha = 1.0 / sqrt(-GCON(g, 0, 0));
  for (i = RHO; i <= B3; i++) U_tmp[i] = alpha * U[i];
  for (i = 0; i < B1; i++) prim_tmp[i] = prim[i];
  for (i = B1; i <= B3; i++) prim_tmp[i] = alpha * prim[i];

  lpflag = UTOPRIMNOFAIL;
  /* compute_setup_quantities */
  c.D = U_tmp[RHO];
  for (i = B1; i <= B3; i++) prim_tmp[i] = U_tmp[i];
  Bcon[0] = 0.;
  for (i = 1; i < 4; i++) Bcon[i] = U_tmp[B1 + i - 1];
  for (i = 0; i < 4; i++) {
    Bcov[i] = 0.;
    for (j = 0; j < 4; j++) Bcov[i] += GCOV(g, i, j) * Bcon[j];
  }
  c.Bsq = 0.;
  for (i = 1; i < 4; i++) c.Bsq += Bcon[i] * Bcov[i];
  lapse = sqrt(-1. / GCON(g, 0, 0));
  ncov[0] = -lapse;
  ncov[1] = 0.;
  ncov[2] = 0.;
  ncov[3] = 0.;
  for (i = 0; i < 4; i++) {
    ncon[i] = 0.;
    for (j = 0; j < 4; j++) ncon[i] += GCON(g, i, j) * ncov[j];
  }
  for (i = 0; i < 4; i++) Qcovp[i] = U_tmp[UU + i];
  for (i = 0; i < 4; i++) {
    Qconp[i] = 0.;
    for (j = 0; j < 4; j++) Qconp[i] += GCON(g, i, j) * Qcovp[j];
  }
  for (j = 0; j < 4; j++) Qtcon[j] = 0.0;
  for (j = 1; j < 4; j++)
    for (i = 1; i < 4; i++) Qtcon[j] += U_tmp[UU + i] * (GCON(g, i, j) + ncon[i] * ncon[j]);
  for (i = 0; i < 4; i++) {
    Qtcov[i] = 0.;
    for (j = 0; j < 4; j++) Qtcov[i] += GCOV(g, i, j) * Qtcon[j];
  }
  c.Qtsq = 0.;
  for (i = 0; i < 4; i++) c.Qtsq += Qtcov[i] * Qtcon[i];
  for (i = 0; i < 4; i++) Qcov[i] = (i == 0) ? Qcovp[i] - c.D : Qcovp[i];
  for (i = 0; i < 4; i++) {
    Qcon[i] = 0.;
    for (j = 0; j < 4; j++) Qcon[i] += GCON(g, i, j) * Qcov[j];
  }
  c.QdotB = 0.;
  for (i = 1; i < 4; i++) c.QdotB += Qcov[i] * Bcon[i];
  c.QdotBsq = c.QdotB * c.QdotB;
  c.Qdotnp = Qconp[0] * ncov[0] + c.D * (1.0 - 1.0 / fabs(ncov[TT]));

  /* set_guess_Wp */
  utsq = 0.;
  for (i = 1; i < 4; i++)
    for (j = 1; j < 4; j++) utsq += GCOV(g, i, j) * prim_tmp[U1 + i - 1] * prim_tmp[U1 + j - 1];
  if ((utsq < 0.) && (fabs(utsq) < MAXNEGUTSQ)) utsq = 0.0;
  if (utsq < 0. || utsq > ((cfg->gammafail - 1.0) * (cfg->gammafail - 1.0))) return UTOPRIMFAILCONVGUESSUTSQ;
  gammasq = 1. + utsq;
  gamma = sqrt(gammasq);
  rho0 = c.D / gamma;
  u = prim_tmp[UU];
  p = (cfg->gam - 1.) * u; /* pressure_rho0_u_grmhd (eos.c:58-65) */
  w = rho0 + u + p;
  {
    /* bsq_calc (phys.c:755-763) on the guess with B^i -> alpha B^i */
    zstate q;
    if (get_state(prim_tmp, g, &q)) return UTOPRIMFAILCONVGUESSUTSQ;
    bsq = dot4(q.bcon, q.bcov);
  }
  Wp_last = c.D * utsq / (1.0 + gamma) + (u + p) * gammasq;
  W_last = Wp_last + c.D;
  if ((w + bsq) * gammasq >= GAMMASQCHECKRESID) {
    double Wpcoldhd;
    if (jon_coldgrhd(c.Qtsq, c.D, &Wpcoldhd)) Wpcoldhd = Wp_last;
    c.wglobal = 1E-5 * jon_max(jon_max(Wpcoldhd, Wp_last), w + bsq);
    Wp_last = jon_max(jon_max(2.0 * Wpcoldhd, Wp_last), w + bsq);
  } else {
    c.wglobal = w + bsq;
  }
  /* verify_Wlast */
  if (W_last < -c.D || Wp_last < 0) {
    W_last = -c.D;
    Wp_last = 0;
  }
  i_increase = 0;
  while ((W_last * W_last * W_last * (W_last + 2. * c.Bsq) - c.QdotBsq * (2. * W_last + c.Bsq) <=
          W_last * W_last * (c.Qtsq - c.Bsq * c.Bsq)) &&
         (i_increase < 10)) {
    Wp_last *= 10.;
    W_last = Wp_last + c.D;
    i_increase++;
  }

  /* find_root_1D_gen_Eprime (utoprim_jon.c:2704-2726) */
  Wp = Wp_last;
  retval = jon_newton(&c, &Wp);
  *iters = c.iters;

  /* check_Wp */
  if ((retval != 0) || (Wp == FAIL_VAL)) {
    lpflag = retval * 100 + 1;
    if (retval != 0) return lpflag; /* Utoprim_new_body returns, guess kept */
  } else {
    Wtest = Wp / c.wglobal;
    if (Wtest <= 0.0) {
      /* check_Wp sets its own copy of Wp to SMALL and returns 0 */
    } else if (Wtest > c.gammasq_too_big) {
      lpflag = UTOPRIMFAILCONVW;
    }
  }

  /* Wp2prim, PRIMFROMVSQ 0 */
  for (i = B1; i <= B3; i++) prim_tmp[i] = U_tmp[i];
  for (i = 0; i < NPR; i++) pr0[i] = prim_tmp[i];
  W = Wp + c.D;
  utsq = jon_utsq(&c, W);
  gammasq = 1.0 + utsq;
  gamma = sqrt(gammasq);
  wmrho0 = jon_wmrho0(Wp, c.D, utsq, gamma, gammasq);
  rho0 = c.D / gamma;
  p = c.igammar * wmrho0; /* pressure_wmrho0_grmhd */
  u = wmrho0 - p;
  if ((rho0 <= 0.) || (u < 0.)) {
    if ((rho0 <= 0.) && (u >= 0.)) lpflag = UTOPRIMFAILRHONEG;
    if ((rho0 > 0.) && (u < 0.)) lpflag = UTOPRIMFAILUNEG;
    if ((rho0 <= 0.) && (u < 0.)) lpflag = UTOPRIMFAILRHOUNEG;
    /* UTOPRIMFAILRETURNTYPE==UTOPRIMRETURNADJUSTED: assign anyway */
  }
  prim_tmp[RHO] = rho0;
  prim_tmp[UU] = u;
  for (i = 1; i < 4; i++) prim_tmp[U1 + i - 1] = gamma / (W + c.Bsq) * (Qtcon[i] + c.QdotB * Bcon[i] / W);
  for (i = 0; i < NPR; i++)
    if (!isfinite(prim_tmp[i])) {
      prim_tmp[i] = pr0[i];
      lpflag = UTOPRIMFAILNANRESULT;
    }
  for (i = 0; i < B1; i++) prim[i] = prim_tmp[i];
  return lpflag;
}

/* Utoprimgen (utoprimgen.c:23-436): geometry-free U, rest mass, inversion.
   U is the evolved conserved vector (with gdet).  Returns pflag.  The 2D
   inverter wants the rest mass in U[UU] (utoprimgen.c:76-85); the Jon
   inverter takes U[UU] without it, as evolved with REMOVERESTMASSFROMUU 2. */
static int utoprimgen(const double *U, const geomref *g, const hgo_config *cfg, double *pr, int *iters)
{
  double Ugf[NPR];
  int pl;
  for (pl = 0; pl < NPR; pl++) Ugf[pl] = U[pl] / g->g; /* UtoU UEVOLVE->UNOTHING */
  if (cfg->utoprimversion == HGO_UTOPRIMJONNONRELCOMPAT) return utoprim_jon(Ugf, g, cfg, pr, iters);
  Ugf[UU] -= Ugf[RHO];
  return utoprim_2d_final(Ugf, g, cfg, pr, iters);
}

/* ------------------------------------------------------------------ */
/* fixups (fixup.c)                                                    */
/* ------------------------------------------------------------------ */

/* limit_gamma (fixup.c:1859-1905) */
static int limit_gamma(double gammamax, double *pr, const geomref *g, int *err)
{
  double f, gamma, pref;
  if (gammamax <= 1.0) return 0;
  if (gamma_calc(pr, g, &gamma)) {
    *err |= ERR_UTCALC_DISCR;
    return 1;
  }
  if ((gamma > gammamax && (gamma != 1.0))) {
    pref = (gammamax * gammamax - 1.) / (gamma * gamma - 1.);
    if (pref < 0.0) {
      *err |= ERR_PREF_NEG;
      return 1;
    }
    f = sqrt(pref);
    pr[U1] *= f;
    pr[U2] *= f;
    pr[U3] *= f;
    return -1;
  }
  return 0;
}

/* fixup1zone (fixup.c:341-447) with floors precomputed per zone; returns
   whether it changed the primitives (didchangeprim), 0 when limit_gamma
   failed (the reference returns through FAILSTATEMENT before diag_fixup) */
static int fixup1zone(double *pr, const geomref *g, const double *floor2, const hgo_config *c, int *err)
{
  double prfloor[2];
  int changed = 0, r;
  prfloor[RHO] = floor2[0];
  prfloor[UU] = floor2[1];
  if (prfloor[RHO] < c->rhominlimit) prfloor[RHO] = c->rhominlimit;
  if (prfloor[UU] < c->uuminlimit) prfloor[UU] = c->uuminlimit;
  if (prfloor[RHO] > pr[RHO]) {
    pr[RHO] = prfloor[RHO];
    changed = 1;
  }
  if (prfloor[UU] > pr[UU]) {
    pr[UU] = prfloor[UU];
    changed = 1;
  }
  r = limit_gamma(c->gammamax, pr, g, err);
  if (r >= 1) return 0;
  if (r == -1) changed = 1;
  return changed;
}

/* diag_fixup's correction of the evolved conserved state for
   ENOFINITEVOLUME with DOENOFLUXMEMORY (fixup.c:196-252), on the final
   substep: unew += UtoU(UDIAG->UEVOLVE, U(pr)) - UtoU(UDIAG->UEVOLVE, U(pr0))
   with U = primtoU(UDIAG) (phys.c:225, UtoU phys.c:243-285: divide by gdet,
   multiply by e = gdet).  It runs once per energy region (ENERREGIONLOOP,
   NUMENERREGIONS = 3 with DOJETDIAG, global.h:435-439): the correctable
   region (Uconsloop = the active zones for avgo = 0) holds in each, so an
   active zone gets the difference added three times. */
static void fv_diag_fixup(dom *d, const double *pr0, const double *pr, const geomref *g, double *unew)
{
  zstate q;
  emstate e;
  double Ui[NPR], Uf[NPR], Upre[NPR], Upost[NPR];
  int pl, region;
  if (get_state(pr0, g, &q)) {
    d->err |= ERR_UTCALC_DISCR;
    return;
  }
  em_prepare(pr0, g, &q, &e);
  primtoflux(pr0, &q, &e, TT, g, d->c->gam, Ui);
  if (get_state(pr, g, &q)) {
    d->err |= ERR_UTCALC_DISCR;
    return;
  }
  em_prepare(pr, g, &q, &e);
  primtoflux(pr, &q, &e, TT, g, d->c->gam, Uf);
  for (pl = 0; pl < NPR; pl++) {
    Upre[pl] = (Ui[pl] / g->g) * g->g;
    Upost[pl] = (Uf[pl] / g->g) * g->g;
  }
  for (region = 0; region < 3; region++)
    for (pl = 0; pl < NPR; pl++) unew[pl] += Upost[pl] - Upre[pl];
}

/* inflow_check_rel4vel for dir 1 at a CENT ghost zone (fixup.c:2271-2400) */
static void inflow_check_x1(const dom *d, int i, double *pr, const geomref *g, int *err)
{
  double ucon[NDIM], gamma, alpha, betacon, vsq;
  int dofix = 0, j, k;
  if (ucon_calc(pr, g, ucon)) {
    *err |= ERR_UTCALC_DISCR;
    return;
  }
  if (((i <= -1) && (d->c->bc[HGO_X1DN] == HGO_BC_OUTFLOW) && (ucon[1] > 0.)) ||
      ((i >= d->n[1]) && (d->c->bc[HGO_X1UP] == HGO_BC_OUTFLOW) && (ucon[1] < 0.)))
    dofix = 1;
  if (!dofix) return;
  if (gamma_calc(pr, g, &gamma)) {
    *err |= ERR_UTCALC_DISCR;
    return;
  }
  pr[U1] /= gamma;
  pr[U2] /= gamma;
  pr[U3] /= gamma;
  alpha = 1. / sqrt(-GCON(g, 0, 0));
  betacon = GCON(g, 0, 1) * alpha * alpha;
  pr[U1] = betacon / alpha;
  vsq = 0.;
  for (j = 1; j < NDIM; j++)
    for (k = 1; k < NDIM; k++) vsq += GCOV(g, j, k) * pr[U1 + j - 1] * pr[U1 + k - 1];
  if (vsq < 0.0) {
    if (vsq > -NUMEPSILON * 100.0) vsq = 0.0;
    else {
      *err |= ERR_VSQ_NEG;
      return;
    }
  }
  if (vsq >= 1.0) vsq = 1.0 - 1.0 / (d->c->gammamax * d->c->gammamax);
  gamma = 1. / sqrt(1. - vsq);
  pr[U1] *= gamma;
  pr[U2] *= gamma;
  pr[U3] *= gamma;
}

/* bound_prim_user (bounds.fishmon.c:29-345): x1 OUTFLOW with inflow check
   and gamma limit, x2 POLARAXIS (POSDEFMETRIC=0, POLEDEATH=1), x3 PERIODIC;
   and the plain x1 OUTFLOW copy of bounds.c (HGO_BC_OUTFLOW_COPY) */
static void bound_prim(dom *d, double *p)
{
  int n1 = d->n[1], n2 = d->n[2], n3 = d->n[3];
  int g1 = d->ng[1], g2 = d->ng[2], g3 = d->ng[3];
  int i, j, k, pl;
  geomref g;
  const hgo_config *c = d->c;
  if (n1 > 1) {
    if (c->bc[HGO_X1DN] == HGO_BC_OUTFLOW_COPY)
      for (j = 0; j < n2; j++)
        for (k = 0; k < n3; k++)
          for (i = -g1; i <= -1; i++)
            for (pl = 0; pl < NPR; pl++) p[zidx(d, i, j, k) * NPR + pl] = p[zidx(d, 0, j, k) * NPR + pl];
    if (c->bc[HGO_X1UP] == HGO_BC_OUTFLOW_COPY)
      for (j = 0; j < n2; j++)
        for (k = 0; k < n3; k++)
          for (i = n1; i <= n1 + g1 - 1; i++)
            for (pl = 0; pl < NPR; pl++) p[zidx(d, i, j, k) * NPR + pl] = p[zidx(d, n1 - 1, j, k) * NPR + pl];
    if (c->bc[HGO_X1DN] == HGO_BC_OUTFLOW) {
      for (j = 0; j < n2; j++)
        for (k = 0; k < n3; k++) {
          for (i = -g1; i <= -1; i++)
            for (pl = 0; pl < NPR; pl++) p[zidx(d, i, j, k) * NPR + pl] = p[zidx(d, 0, j, k) * NPR + pl];
          for (i = -g1; i <= -1; i++) {
            double *pr = &p[zidx(d, i, j, k) * NPR];
            get_geometry(d, i, j, CENT, &g);
            inflow_check_x1(d, i, pr, &g, &d->err);
            limit_gamma(c->gammamax, pr, &g, &d->err);
          }
        }
    }
    if (c->bc[HGO_X1UP] == HGO_BC_OUTFLOW) {
      for (j = 0; j < n2; j++)
        for (k = 0; k < n3; k++) {
          for (i = n1; i <= n1 + g1 - 1; i++)
            for (pl = 0; pl < NPR; pl++) p[zidx(d, i, j, k) * NPR + pl] = p[zidx(d, n1 - 1, j, k) * NPR + pl];
          for (i = n1; i <= n1 + g1 - 1; i++) {
            double *pr = &p[zidx(d, i, j, k) * NPR];
            get_geometry(d, i, j, CENT, &g);
            inflow_check_x1(d, i, pr, &g, &d->err);
            limit_gamma(c->gammamax, pr, &g, &d->err);
          }
        }
    }
  }
  if (n2 > 1) {
    if (c->bc[HGO_X2DN] == HGO_BC_POLARAXIS) {
      for (i = -g1; i <= n1 - 1 + g1; i++)
        for (k = 0; k < n3; k++)
          for (j = -g2; j <= -1; j++)
            for (pl = 0; pl < NPR; pl++) p[zidx(d, i, j, k) * NPR + pl] = p[zidx(d, i, -j - 1, k) * NPR + pl];
      /* antisymmetry factors are 1 for POSDEFMETRIC=0; POLEDEATH zeroes U2,B2 */
      for (i = -g1; i <= n1 - 1 + g1; i++)
        for (k = 0; k < n3; k++)
          for (j = -g2; j < 0 + 1; j++) {
            p[zidx(d, i, j, k) * NPR + U2] *= 0;
            p[zidx(d, i, j, k) * NPR + B2] *= 0.;
          }
    }
    if (c->bc[HGO_X2UP] == HGO_BC_POLARAXIS) {
      for (i = -g1; i <= n1 - 1 + g1; i++)
        for (k = 0; k < n3; k++)
          for (j = n2; j <= n2 + g2 - 1; j++)
            for (pl = 0; pl < NPR; pl++)
              p[zidx(d, i, j, k) * NPR + pl] = p[zidx(d, i, (n2 - 1) + ((n2 - 1) - j + 1), k) * NPR + pl];
      for (i = -g1; i <= n1 - 1 + g1; i++)
        for (k = 0; k < n3; k++)
          for (j = n2 - 1; j <= n2 - 1 + g2; j++) {
            p[zidx(d, i, j, k) * NPR + U2] *= 0;
            p[zidx(d, i, j, k) * NPR + B2] *= 0.;
          }
    }
  }
  if (n3 > 1 && c->bc[HGO_X3DN] == HGO_BC_PERIODIC && c->bc[HGO_X3UP] == HGO_BC_PERIODIC) {
    for (i = -g1; i <= n1 - 1 + g1; i++)
      for (j = -g2; j <= n2 - 1 + g2; j++) {
        for (k = -g3; k <= -1; k++)
          for (pl = 0; pl < NPR; pl++) p[zidx(d, i, j, k) * NPR + pl] = p[zidx(d, i, j, n3 + k) * NPR + pl];
        for (k = n3; k <= n3 + g3 - 1; k++)
          for (pl = 0; pl < NPR; pl++) p[zidx(d, i, j, k) * NPR + pl] = p[zidx(d, i, j, k - n3) * NPR + pl];
      }
  }
}

/* bound_pflag_user (boundsint.c:6-266), FLAGUTOPRIMFAIL only */
static void bound_pflag(dom *d, int *pf)
{
  int n1 = d->n[1], n2 = d->n[2], n3 = d->n[3];
  int g1 = d->ng[1], g2 = d->ng[2], g3 = d->ng[3];
  int i, j, k;
  const hgo_config *c = d->c;
  if (n3 > 1 && c->bc[HGO_X3DN] == HGO_BC_PERIODIC && c->bc[HGO_X3UP] == HGO_BC_PERIODIC) {
    for (i = -g1; i <= n1 - 1 + g1; i++)
      for (j = -g2; j <= n2 - 1 + g2; j++) {
        for (k = -g3; k <= -1; k++) pf[zidx(d, i, j, k)] = pf[zidx(d, i, j, n3 + k)];
        for (k = n3; k <= n3 + g3 - 1; k++) pf[zidx(d, i, j, k)] = pf[zidx(d, i, j, k - n3)];
      }
  }
  if (n1 > 1 && (c->bc[HGO_X1DN] == HGO_BC_OUTFLOW || c->bc[HGO_X1DN] == HGO_BC_OUTFLOW_COPY))
    for (j = -g2; j <= n2 - 1 + g2; j++)
      for (k = -g3; k <= n3 - 1 + g3; k++)
        for (i = -g1; i <= -1; i++) pf[zidx(d, i, j, k)] = pf[zidx(d, 0, j, k)];
  if (n1 > 1 && (c->bc[HGO_X1UP] == HGO_BC_OUTFLOW || c->bc[HGO_X1UP] == HGO_BC_OUTFLOW_COPY))
    for (j = -g2; j <= n2 - 1 + g2; j++)
      for (k = -g3; k <= n3 - 1 + g3; k++)
        for (i = n1; i <= n1 + g1 - 1; i++) pf[zidx(d, i, j, k)] = pf[zidx(d, n1 - 1, j, k)];
  if (n2 > 1 && c->bc[HGO_X2DN] == HGO_BC_POLARAXIS)
    for (i = -g1; i <= n1 - 1 + g1; i++)
      for (k = -g3; k <= n3 - 1 + g3; k++)
        for (j = -g2; j <= -1; j++) pf[zidx(d, i, j, k)] = pf[zidx(d, i, -j - 1, k)];
  if (n2 > 1 && c->bc[HGO_X2UP] == HGO_BC_POLARAXIS)
    for (i = -g1; i <= n1 - 1 + g1; i++)
      for (k = -g3; k <= n3 - 1 + g3; k++)
        for (j = n2; j <= n2 + g2 - 1; j++) pf[zidx(d, i, j, k)] = pf[zidx(d, i, (n2 - 1) + ((n2 - 1) - j + 1), k)];
}

/* fixup_checksolution (fixup.c:460-560) */
static void fixup_checksolution(dom *d, const double *pv, int *pf, double *gammacheck)
{
  int n1 = d->n[1], n2 = d->n[2], n3 = d->n[3];
  int s1 = d->sh[1], s2 = d->sh[2], s3 = d->sh[3];
  int i, j, k, l;
  geomref g;
  /* gammacheck stored on the zone grid at the zone's own index */
  for (i = -s1; i <= n1 - 1 + s1; i++)
    for (j = -s2; j <= n2 - 1 + s2; j++)
      for (k = -s3; k <= n3 - 1 + s3; k++) {
        long z = zidx(d, i, j, k);
        get_geometry(d, i, j, CENT, &g);
        if (gamma_calc(&pv[z * NPR], &g, &gammacheck[z])) d->err |= ERR_UTCALC_DISCR;
      }
  for (i = 0; i < n1; i++)
    for (j = 0; j < n2; j++)
      for (k = 0; k < n3; k++) {
        long z = zidx(d, i, j, k);
        double percdiff[8], percdiff2[8], gc = gammacheck[z], uc = pv[z * NPR + UU];
        int vote0 = 0, vote1 = 0, numvotes = 0;
        int im = i - s1, ip = i + s1, jm = j - s2, jp = j + s2;
        if (!(gc >= 2.0)) continue;
#define NB(ii, jj) zidx(d, ii, jj, k)
#define PD(idx, ii, jj)                                                                         \
  percdiff[idx] = (pf[NB(ii, jj)] <= UTOPRIMNOFAIL) ? (gammacheck[NB(ii, jj)] / gc) : -1;        \
  percdiff2[idx] = (pf[NB(ii, jj)] <= UTOPRIMNOFAIL) ? (pv[NB(ii, jj) * NPR + UU] / uc) : -1;
        PD(0, i, jp);
        PD(1, i, jm);
        PD(2, ip, j);
        PD(3, im, j);
        PD(4, ip, jp);
        PD(5, ip, jm);
        PD(6, ip, jp);
        PD(7, im, jm);
#undef PD
#undef NB
        for (l = 0; l < MAXVOTES; l++) {
          if (percdiff[0] >= 0.0) {
            if ((fabs(percdiff[l]) > GAMMAPERCDIFFMAX) || (fabs(percdiff[l]) < 1.0 / GAMMAPERCDIFFMAX)) vote0++;
            if (((fabs(percdiff2[l]) > UPERCDIFFMAX) || (fabs(percdiff2[l]) < 1.0 / UPERCDIFFMAX))) vote1++;
            numvotes++;
          }
        }
        if (vote0 > numvotes * 0.5) pf[z] = UTOPRIMFAILGAMMAPERC;
        if (vote1 > numvotes * 0.5) pf[z] = UTOPRIMFAILUPERC;
      }
}

/* fixup_utoprim (fixup.c:669-1470), GENERALAVERAGE=1, ORDERINDEPENDENT=1,
   HOWTOAVG_WHEN_U2AVG=MAXUPOSAVG, CAUSALAVG=0, TODONOGOOD=NOGOODAVERAGE,
   STEPOVERNEG*=-1, DOCOUNTNEG*=1, ADJUSTCONSERVEDQUANTITY=0 */
static void fixup_utoprim(dom *d, double *pv, double *ptoavg, int *pf, int finalstep, double *unew)
{
  int n1 = d->n[1], n2 = d->n[2], n3 = d->n[3];
  int s1 = d->sh[1], s2 = d->sh[2], s3 = d->sh[3];
  long ntot = (long)d->nt[1] * d->nt[2] * d->nt[3];
  int i, j, k, pl, qq;
  int rnx = (s1 == 1) ? 3 * s1 : 1, rny = (s2 == 1) ? 3 * s2 : 1;
  int numupairs = (int)(pow(3, s1 + s2 + s3) - 1) / 2;
  geomref g;
  memcpy(ptoavg, pv, sizeof(double) * NPR * ntot);
  for (i = 0; i < n1; i++)
    for (j = 0; j < n2; j++)
      for (k = 0; k < n3; k++) {
        long z = zidx(d, i, j, k);
        int mypflag = pf[z], fixed = 0, failtype;
        if (mypflag != 0) {
          get_geometry(d, i, j, CENT, &g);
          if (mypflag == UTOPRIMFAILUNEG || mypflag == UTOPRIMFAILRHONEG || mypflag == UTOPRIMFAILRHOUNEG) fixed = 1;
          if (fixed == 0) {
            double gamma = 1.0, mysum[2][NPR], lastmin[NPR], avganswer0[NPR], avganswer1[NPR];
            int startpl, endpl, failavglooptype, numavg, numavg0 = 0, numavg1 = 0;
            if (gamma_calc(&ptoavg[z * NPR], &g, &gamma)) d->err |= ERR_UTCALC_DISCR;
            if (gamma > d->c->gammamax) gamma = d->c->gammamax;
            if (mypflag == UTOPRIMFAILU2AVG1 || mypflag == UTOPRIMFAILU2AVG2) {
              startpl = UU;
              endpl = UU;
              failavglooptype = 1;
            } else {
              startpl = RHO;
              endpl = U3;
              failavglooptype = 0;
            }
            for (pl = startpl; pl <= endpl; pl++) {
              mysum[0][pl] = 0.0;
              mysum[1][pl] = 0.0;
              lastmin[pl] = 1E50;
            }
            for (qq = 0; qq < numupairs; qq++) {
              int ii = (int)(qq % rnx) - s1;
              int jj = (int)((qq % (rnx * rny)) / rnx) - s2;
              int kk = (int)(qq / (rnx * rny)) - s3;
              long za = zidx(d, i + ii, j + jj, k + kk), zb = zidx(d, i - ii, j - jj, k - kk);
              int thisnotfail = pf[za] <= UTOPRIMNOFAIL;
              int thatnotfail = pf[zb] <= UTOPRIMNOFAIL;
              numavg1 += (ptoavg[za * NPR + UU] > 0.0);
              numavg1 += (ptoavg[zb * NPR + UU] > 0.0);
              numavg0 += thisnotfail + thatnotfail;
              if (failavglooptype == 0) {
                for (pl = startpl; pl <= endpl; pl++)
                  mysum[qq % 2][pl] += ptoavg[za * NPR + pl] * thisnotfail + ptoavg[zb * NPR + pl] * thatnotfail;
              } else {
                for (pl = startpl; pl <= endpl; pl++) {
                  double ftemp = ptoavg[za * NPR + pl];
                  if (ftemp >= 0.0) lastmin[pl] = fmin_macro(lastmin[pl], ftemp);
                  ftemp = ptoavg[zb * NPR + pl];
                  if (ftemp >= 0.0) lastmin[pl] = fmin_macro(lastmin[pl], ftemp);
                }
              }
            }
            if (failavglooptype == 0) {
              if (numavg0 != 0)
                for (pl = startpl; pl <= endpl; pl++) avganswer0[pl] = (mysum[0][pl] + mysum[1][pl]) / ((double)(numavg0));
              if (numavg0 != 0)
                for (pl = startpl; pl <= endpl; pl++) pv[z * NPR + pl] = avganswer0[pl];
              numavg = numavg0;
            } else {
              for (pl = startpl; pl <= endpl; pl++) avganswer1[pl] = lastmin[pl];
              if (numavg1 != 0)
                for (pl = startpl; pl <= endpl; pl++) pv[z * NPR + pl] = avganswer1[pl];
              numavg = numavg1;
            }
            if (mypflag == UTOPRIMFAILU2AVG2) numavg++;
            if (numavg == 0) {
              /* NOGOODAVERAGE: 0.5*(AVG4_1 + AVG4_2) of ptoavg (fixup.c:562-566) */
              for (pl = startpl; pl <= endpl; pl++) {
                double a41 = (0.25 * ((ptoavg[zidx(d, i, j + s2, k) * NPR + pl] + ptoavg[zidx(d, i, j - s2, k) * NPR + pl]) +
                                      (ptoavg[zidx(d, i - s1, j, k) * NPR + pl] + ptoavg[zidx(d, i + s1, j, k) * NPR + pl])));
                double a42 = (0.25 * ((ptoavg[zidx(d, i + s1, j + s2, k) * NPR + pl] + ptoavg[zidx(d, i + s1, j - s2, k) * NPR + pl]) +
                                      (ptoavg[zidx(d, i - s1, j + s2, k) * NPR + pl] + ptoavg[zidx(d, i - s1, j - s2, k) * NPR + pl])));
                pv[z * NPR + pl] = 0.5 * (a41 + a42);
              }
            }
            limit_gamma(gamma, &pv[z * NPR], &g, &d->err);
          }
        }
        /* accounting: which failures get reset to UTOPRIMFAILFIXED */
        if (mypflag == UTOPRIMNOFAIL) failtype = -1;
        else if (mypflag == UTOPRIMFAILRHONEG || mypflag == UTOPRIMFAILUNEG || mypflag == UTOPRIMFAILU2AVG1 ||
                 mypflag == UTOPRIMFAILU2AVG2 || mypflag == UTOPRIMFAILRHOUNEG)
          failtype = finalstep ? 1 : -1;
        else failtype = 1;
        if (failtype != -1) {
          /* diag_fixup(pr0 = ptoavg, pv) (fixup.c:1428); pr0 is the zone's
             pre-fixup state */
          if (unew && finalstep) {
            get_geometry(d, i, j, CENT, &g);
            fv_diag_fixup(d, &ptoavg[z * NPR], &pv[z * NPR], &g, &unew[z * NPR]);
          }
          pf[z] = UTOPRIMFAILFIXED;
        }
      }
}

/* ------------------------------------------------------------------ */
/* drivers                                                             */
/* ------------------------------------------------------------------ */

static void dom_init(dom *d, const hgo_config *c, const hgo_geometry *g)
{
  int dd;
  d->c = c;
  d->n[1] = c->n1;
  d->n[2] = c->n2;
  d->n[3] = c->n3;
  for (dd = 1; dd <= 3; dd++) {
    d->sh[dd] = d->n[dd] > 1;
    d->ng[dd] = d->sh[dd] ? c->ng : 0;
    d->nt[dd] = d->n[dd] + 2 * d->ng[dd];
  }
  d->gt[1] = d->nt[1] + d->sh[1];
  d->gt[2] = d->nt[2] + d->sh[2];
  d->gcov = g->gcov;
  d->gcon = g->gcon;
  d->gcovpert = g->gcovpert;
  d->gdet = g->gdet;
  d->conn = g->conn;
  d->floors = g->floors;
  d->err = 0;
}

static long dom_ntot(const dom *d) { return (long)d->nt[1] * d->nt[2] * d->nt[3]; }

/* source() + source_conn() at CENT (phys.c:578-752); cooling=0 so the
   physics sources are zero and only the connection term contributes */
static int source_conn(const dom *d, int i, int j, const double *pr, const geomref *g, double *dU)
{
  zstate q;
  emstate e;
  double mhd[NDIM][NDIM], dUconn[NPR];
  const double *conn = d->conn + gidx(d, i, j) * 64;
  int jj, kk, l, pl;
  if (get_state(pr, g, &q)) return ERR_UTCALC_DISCR;
  em_prepare(pr, g, &q, &e);
  for (jj = 0; jj < NDIM; jj++) mhd_calc(pr, jj, d->c->gam, &q, &e, mhd[jj]);
  for (pl = 0; pl < NPR; pl++) dUconn[pl] = 0;
  for (l = 0; l < NDIM; l++)
    for (jj = 0; jj < NDIM; jj++)
      for (kk = 0; kk < NDIM; kk++) dUconn[UU + l] += mhd[jj][kk] * conn[(kk * 4 + l) * 4 + jj];
  for (l = 0; l < NDIM; l++)
    for (jj = 0; jj < NDIM; jj++) dUconn[UU + l] += -pr[RHO] * q.ucon[jj] * conn[(TT * 4 + l) * 4 + jj];
  /* dU = sum over the NUMSOURCES components; only GEOMSOURCE is nonzero:
     dUcomp[0] = 0 + g*dUconn, the other six components are 0 */
  for (pl = 0; pl < NPR; pl++) {
    double comp0 = 0. + g->g * dUconn[pl];
    double acc = 0.;
    acc += comp0;
    for (l = 1; l < 7; l++) acc += 0.0;
    dU[pl] = acc;
  }
  return 0;
}

typedef struct {
  double CUf[4], Cunew[4];
} rkstage;

/* midpoint method tables (step_ch.c:504-524) */
/* setup_rktimestep (step_ch.c:442-562): CUf (Ui, ulast, dU) and Cunew (Ui,
   dU, Uf) of stage `timeorder` of the TIMEORDER=`norders` method */
static void rk_stage(int norders, int timeorder, rkstage *s)
{
  static const double cuf4[4][3] = {{1.0, 0.0, 0.5}, {1.0, 0.0, 0.5}, {1.0, 0.0, 1.0}, {1.0, 0.0, 1.0}};
  static const double cun4[4][3] = {{1.0, 1.0 / 6.0, 0.0}, {0.0, 1.0 / 3.0, 0.0}, {0.0, 1.0 / 3.0, 0.0},
                                    {0.0, 1.0 / 6.0, 0.0}};
  static const double cuf3[3][3] = {{1.0, 0.0, 1.0}, {3.0 / 4.0, 1.0 / 4.0, 1.0 / 4.0}, {1.0 / 3.0, 2.0 / 3.0, 2.0 / 3.0}};
  static const double cun3[3][3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}, {0.0, 0.0, 1.0}};
  static const double cuf2[2][3] = {{1.0, 0.0, 0.5}, {1.0, 0.0, 1.0}};
  static const double cun2[2][3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 1.0}};
  static const double cuf1[1][3] = {{1.0, 0.0, 1.0}};
  static const double cun1[1][3] = {{0.0, 0.0, 1.0}};
  const double(*cuf)[3] = norders == 4 ? cuf4 : norders == 3 ? cuf3 : norders == 2 ? cuf2 : cuf1;
  const double(*cun)[3] = norders == 4 ? cun4 : norders == 3 ? cun3 : norders == 2 ? cun2 : cun1;
  int q;
  for (q = 0; q < 3; q++) {
    s->CUf[q] = cuf[timeorder][q];
    s->Cunew[q] = cun[timeorder][q];
  }
  s->CUf[3] = 0.0;
  s->Cunew[3] = 0.0;
}

typedef struct {
  double *dq, *emf, *ptoavg, *gammacheck;
} scratch;

/* advance_standard (advance.c:58-238) for the midpoint RK2 stage `timeorder` */
static void advance(dom *d, const double *pi, const double *pb, double *pf, double *uf, double *ucum, double *F1,
                    double *F2, double *F3, int *pflag, double dt, int timeorder, int numtimeorders, double *ndt,
                    scratch *sc, long *iters, const double *ui)
{
  const hgo_config *c = d->c;
  double ndt1, ndt2, ndt3;
  rkstage rk;
  int i, j, k, pl;
  double idx1 = 1.0 / c->dx[1], idx2 = 1.0 / c->dx[2], idx3 = 1.0 / c->dx[3];
  long o1 = (long)d->nt[2] * d->nt[3], o2 = d->nt[3], o3 = 1;
  int finalstep = (timeorder == numtimeorders - 1);
  rk_stage(numtimeorders, timeorder, &rk);

  fluxcalc_dir(d, pb, 1, F1, sc->dq, &ndt1);
  fluxcalc_dir(d, pb, 2, F2, sc->dq, &ndt2);
  fluxcalc_dir(d, pb, 3, F3, sc->dq, &ndt3);
  flux_ct(d, F1, F2, F3, sc->emf);

  for (i = 0; i < d->n[1]; i++)
    for (j = 0; j < d->n[2]; j++)
      for (k = 0; k < d->n[3]; k++) {
        long z = zidx(d, i, j, k);
        geomref g;
        zstate q;
        emstate e;
        double Ui[NPR], dUgeom[NPR], dU1[NPR], dU2[NPR], dU3[NPR], dUr[NPR], Uf[NPR];
        int it = 0, r;
        if (timeorder == 0)
          for (pl = 0; pl < NPR; pl++) uf[z * NPR + pl] = ucum[z * NPR + pl] = 0.0;
        get_geometry(d, i, j, CENT, &g);
        if (ui) {
          /* advance_finitevolume (advance.c:245-501): Ui is the stored
             conserved state (ui = ucum of the last step, advance.c:330-343) */
          for (pl = 0; pl < NPR; pl++) Ui[pl] = ui[z * NPR + pl];
        } else {
          if (get_state(&pi[z * NPR], &g, &q)) d->err |= ERR_UTCALC_DISCR;
          em_prepare(&pi[z * NPR], &g, &q, &e);
          primtoflux(&pi[z * NPR], &q, &e, TT, &g, c->gam, Ui);
        }
        if ((r = source_conn(d, i, j, &pb[z * NPR], &g, dUgeom))) d->err |= r;
        /* flux2dUavg (advance.c:741-914) */
        for (pl = 0; pl < NPR; pl++) {
          dU1[pl] = 0;
          dU2[pl] = 0;
          dU3[pl] = 0;
          if (d->n[1] > 1) dU1[pl] = (-(F1[(z + o1) * NPR + pl] - F1[z * NPR + pl]) * idx1);
          if (d->n[2] > 1) dU2[pl] = (-(F2[(z + o2) * NPR + pl] - F2[z * NPR + pl]) * idx2);
          if (d->n[3] > 1) dU3[pl] = (-(F3[(z + o3) * NPR + pl] - F3[z * NPR + pl]) * idx3);
          dUr[pl] = dU1[pl] + dU2[pl] + dU3[pl];
        }
        /* dUtoU (advance.c:922-949) */
        for (pl = 0; pl < NPR; pl++)
          uf[z * NPR + pl] = Uf[pl] =
              rk.CUf[0] * Ui[pl] + rk.CUf[1] * uf[z * NPR + pl] + rk.CUf[2] * dt * (dUr[pl] + dUgeom[pl]);
        for (pl = 0; pl < NPR; pl++)
          ucum[z * NPR + pl] += rk.Cunew[0] * Ui[pl] + rk.Cunew[1] * dt * (dUr[pl] + dUgeom[pl]) + rk.Cunew[2] * Uf[pl];
        for (pl = 0; pl < NPR; pl++) pf[z * NPR + pl] = pb[z * NPR + pl];
        if (finalstep) pflag[z] = utoprimgen(&ucum[z * NPR], &g, c, &pf[z * NPR], &it);
        else pflag[z] = utoprimgen(Uf, &g, c, &pf[z * NPR], &it);
        *iters += it;
        if (finalstep) {
          double pr0[NPR];
          for (pl = 0; pl < NPR; pl++) pr0[pl] = pf[z * NPR + pl];
          if (fixup1zone(&pf[z * NPR], &g, &d->floors[gidx(d, i, j) * 2], c, &d->err) && ui)
            fv_diag_fixup(d, pr0, &pf[z * NPR], &g, &ucum[z * NPR]); /* diag_fixup, fixup.c:443 */
        }
      }
  *ndt = c->defcon * 1. / (1. / ndt1 + 1. / ndt2 + 1. / ndt3);
}

static int alloc_scratch(const dom *d, scratch *sc)
{
  long n = dom_ntot(d);
  sc->dq = (double *)calloc((size_t)n * NPR * 2, sizeof(double)); /* MC slopes, or WENO5 pleft|pright */
  sc->emf = (double *)calloc((size_t)n * 3, sizeof(double));
  sc->ptoavg = (double *)calloc((size_t)n * NPR, sizeof(double));
  sc->gammacheck = (double *)calloc((size_t)n, sizeof(double));
  return (sc->dq && sc->emf && sc->ptoavg && sc->gammacheck) ? 0 : -1;
}

static void free_scratch(scratch *sc)
{
  free(sc->dq);
  free(sc->emf);
  free(sc->ptoavg);
  free(sc->gammacheck);
}

/* one RK stage with its boundary/fixup sequence (step_ch.c:94-186) */
static void stage_with_fixups(dom *d, const double *pi, const double *pb, double *pf, double *uf, double *ucum,
                              double *F1, double *F2, double *F3, int *pflag, double dt, int timeorder,
                              int numtimeorders, double *ndt, scratch *sc, long *iters, const double *ui)
{
  int finalstep = (timeorder == numtimeorders - 1);
  /* pre_fixup: b^2 flags only (LIMADJUST=FLUXADJUST=0), no state change */
  advance(d, pi, pb, pf, uf, ucum, F1, F2, F3, pflag, dt, timeorder, numtimeorders, ndt, sc, iters, ui);
  bound_prim(d, pf);
  bound_pflag(d, pflag);
  fixup_checksolution(d, pf, pflag, sc->gammacheck);
  fixup_utoprim(d, pf, sc->ptoavg, pflag, finalstep, ui ? ucum : NULL);
  bound_prim(d, pf);
}

int hgo_substep(const hgo_config *c, const hgo_geometry *g, const double *pi, const double *pb, double *pf,
                double *uf, double *ucum, double *F1, double *F2, double *F3, int *pflag, double dt, int timeorder,
                double *ndt, hgo_stats *st)
{
  dom d;
  scratch sc;
  long iters = 0;
  dom_init(&d, c, g);
  if (alloc_scratch(&d, &sc)) return -1;
  stage_with_fixups(&d, pi, pb, pf, uf, ucum, F1, F2, F3, pflag, dt, timeorder, c->timeorder ? c->timeorder : 2,
                    ndt, &sc, &iters, NULL);
  free_scratch(&sc);
  if (st) {
    st->newton_iters = iters;
    st->err = d.err;
  }
  return d.err;
}

/* pi2Uavg (initbase.c:1833-1880), avgscheme=DONOR: U(p) over FULLLOOP */
static void pi2u(dom *d, const double *p, double *u)
{
  int i, j, k;
  for (i = -d->ng[1]; i < d->n[1] + d->ng[1]; i++)
    for (j = -d->ng[2]; j < d->n[2] + d->ng[2]; j++)
      for (k = -d->ng[3]; k < d->n[3] + d->ng[3]; k++) {
        long z = zidx(d, i, j, k);
        geomref g;
        zstate q;
        emstate e;
        get_geometry(d, i, j, CENT, &g);
        if (get_state(&p[z * NPR], &g, &q)) {
          d->err |= ERR_UTCALC_DISCR;
          continue;
        }
        em_prepare(&p[z * NPR], &g, &q, &e);
        primtoflux(&p[z * NPR], &q, &e, TT, &g, d->c->gam, &u[z * NPR]);
      }
}

int hgo_pi2u(const hgo_config *c, const hgo_geometry *g, const double *p, double *u)
{
  dom d;
  dom_init(&d, c, g);
  pi2u(&d, p, u);
  return d.err;
}

int hgo_step(const hgo_config *c, const hgo_geometry *g, double *p, int *pflag, double *t, double *dt, int nsteps,
             hgo_stats *st)
{
  return hgo_step_u(c, g, p, pflag, NULL, t, dt, nsteps, st);
}

int hgo_step_u(const hgo_config *c, const hgo_geometry *g, double *p, int *pflag, double *u, double *t, double *dt,
               int nsteps, hgo_stats *st)
{
  dom d;
  scratch sc;
  long n, iters = 0;
  double *pk, *pk1, *uf, *ucum, *F1, *F2, *F3, *ui = NULL, *uown = NULL;
  int s, z, nf = 0, norders = c->timeorder ? c->timeorder : 2, o;
  int fv = (c->doenoflux == HGO_ENOFINITEVOLUME);
  dom_init(&d, c, g);
  n = dom_ntot(&d);
  if (alloc_scratch(&d, &sc)) return -1;
  pk = (double *)calloc((size_t)n * NPR, sizeof(double));
  pk1 = (double *)calloc((size_t)n * NPR, sizeof(double));
  uf = (double *)calloc((size_t)n * NPR, sizeof(double));
  F1 = (double *)calloc((size_t)n * NPR, sizeof(double));
  F2 = (double *)calloc((size_t)n * NPR, sizeof(double));
  F3 = (double *)calloc((size_t)n * NPR, sizeof(double));
  if (fv) {
    /* unew is the evolved state; ui receives it at the start of each step
       (advance.c:330-343; at the first call uinitial = unew = U(p) from
       init_conservatives, initbase.c:146-153) */
    ui = (double *)calloc((size_t)n * NPR, sizeof(double));
    if (!u) {
      u = uown = (double *)calloc((size_t)n * NPR, sizeof(double));
      if (uown) pi2u(&d, p, u);
    }
    ucum = u;
  } else {
    ucum = (double *)calloc((size_t)n * NPR, sizeof(double));
  }
  if (!pk || !pk1 || !uf || !ucum || !F1 || !F2 || !F3 || (fv && !ui)) return -1;
  for (s = 0; s < nsteps; s++) {
    double ndt;
    /* pii/pbb/pff of setup_rktimestep (step_ch.c:442-562): pi = p always;
       (pb, pf): Euler (p,p); midpoint (p,pk0) (pk0,p); RK3 (p,pk0) (pk0,pk1)
       (pk1,p); RK4 (p,pk0) (pk0,pk1) (pk1,pk0) (pk0,p) */
    double *pb4[4] = {p, pk, pk1, pk}, *pf4[4] = {pk, pk1, pk, p};
    double *pb3[3] = {p, pk, pk1}, *pf3[3] = {pk, pk1, p};
    double *pb2[2] = {p, pk}, *pf2[2] = {pk, p};
    double *pb1[1] = {p}, *pf1[1] = {p};
    double **pbs = norders == 4 ? pb4 : norders == 3 ? pb3 : norders == 2 ? pb2 : pb1;
    double **pfs = norders == 4 ? pf4 : norders == 3 ? pf3 : norders == 2 ? pf2 : pf1;
    memcpy(pk, p, sizeof(double) * NPR * n);
    if (fv) memcpy(ui, ucum, sizeof(double) * NPR * n);
    for (o = 0; o < norders; o++)
      stage_with_fixups(&d, p, pbs[o], pfs[o], uf, ucum, F1, F2, F3, pflag, *dt, o, norders, &ndt, &sc, &iters, ui);
    /* step_ch.c:236-247 */
    *t += *dt;
    if (ndt > c->safe * (*dt)) ndt = c->safe * (*dt);
    *dt = ndt;
    if (*t + *dt > c->tf) *dt = c->tf - *t;
  }
  for (z = 0; z < n; z++) nf += (pflag[z] != 0);
  free(pk);
  free(pk1);
  free(uf);
  if (!fv) free(ucum);
  free(ui);
  free(uown);
  free(F1);
  free(F2);
  free(F3);
  free_scratch(&sc);
  if (st) {
    st->newton_iters = iters;
    st->err = d.err;
    st->nfail_final = nf;
  }
  return d.err;
}

/* post_fixup (fixup.c:37-96) on its own: bound_pflag, fixup_checksolution,
   fixup_utoprim; unew (may be NULL) receives the finite-volume scheme's
   diag_fixup corrections on a final step */
int hgo_post_fixup(const hgo_config *c, const hgo_geometry *g, double *p, int *pflag, int finalstep, double *unew)
{
  dom d;
  scratch sc;
  dom_init(&d, c, g);
  if (alloc_scratch(&d, &sc)) return -1;
  bound_pflag(&d, pflag);
  fixup_checksolution(&d, p, pflag, sc.gammacheck);
  fixup_utoprim(&d, p, sc.ptoavg, pflag, finalstep, unew);
  free_scratch(&sc);
  return d.err;
}

/* fluxcalc (flux.c:7-318) with flux_ct (fluxct.c:10) on p: F1..F3 receive
   the face fluxes the update reads (others untouched), ndt[0..2] the three
   directions' dt estimates */
int hgo_fluxcalc(const hgo_config *c, const hgo_geometry *g, const double *p, double *F1, double *F2, double *F3,
                 double *ndt)
{
  dom d;
  scratch sc;
  dom_init(&d, c, g);
  if (alloc_scratch(&d, &sc)) return -1;
  fluxcalc_dir(&d, p, 1, F1, sc.dq, &ndt[0]);
  fluxcalc_dir(&d, p, 2, F2, sc.dq, &ndt[1]);
  fluxcalc_dir(&d, p, 3, F3, sc.dq, &ndt[2]);
  flux_ct(&d, F1, F2, F3, sc.emf);
  free_scratch(&sc);
  return d.err;
}

/* fixup_checksolution (fixup.c:460-560) alone on p and pflag; gammacheck
   (may be NULL) receives the Lorentz factors it compares, zone layout */
int hgo_checksolution(const hgo_config *c, const hgo_geometry *g, const double *p, int *pflag, double *gammacheck)
{
  dom d;
  scratch sc;
  dom_init(&d, c, g);
  if (alloc_scratch(&d, &sc)) return -1;
  fixup_checksolution(&d, p, pflag, sc.gammacheck);
  if (gammacheck) memcpy(gammacheck, sc.gammacheck, sizeof(double) * dom_ntot(&d));
  free_scratch(&sc);
  return d.err;
}

int hgo_bound_prim(const hgo_config *c, const hgo_geometry *g, double *p)
{
  dom d;
  dom_init(&d, c, g);
  bound_prim(&d, p);
  return d.err;
}

int hgo_utoprim_batch(const double *U, const double *gcov, const double *gcon, const double *gdet, double *pr,
                      int *pflag, long n, double gam, double gammafail, long *iters)
{
  return hgo_utoprim_batch_v(U, gcov, gcon, gdet, pr, pflag, n, gam, gammafail, HGO_UTOPRIM2DFINAL, iters);
}

int hgo_utoprim_batch_v(const double *U, const double *gcov, const double *gcon, const double *gdet, double *pr,
                        int *pflag, long n, double gam, double gammafail, int utoprimversion, long *iters)
{
  hgo_config c;
  long z;
  long tot = 0;
  memset(&c, 0, sizeof(c));
  c.gam = gam;
  c.gammafail = gammafail;
  c.utoprimversion = utoprimversion;
  for (z = 0; z < n; z++) {
    geomref g;
    int it = 0;
    g.gcov = gcov + z * 16;
    g.gcon = gcon + z * 16;
    g.gcovpert = NULL;
    g.g = gdet[z];
    pflag[z] = utoprimgen(&U[z * NPR], &g, &c, &pr[z * NPR], &it);
    tot += it;
  }
  if (iters) *iters = tot;
  return 0;
}

int hgo_abi_version(void) { return 3; }
