/*
 * harm_oracle.h -- interface of the CPU restatement used as parity checker.
 * TEST INFRASTRUCTURE ONLY (see harm_oracle.c).
 *
 * Array layout (all row-major, ghosts included):
 *   zone arrays   [n1+2g1][n2+2g2][n3+2g3]            (x1 slowest, x3 fastest)
 *     primitives  [..][8]   rho,u,u~1,u~2,u~3,B1,B2,B3 (global.h:916-923)
 *     pflag       [..]      FLAGUTOPRIMFAIL codes (global.h:782-799)
 *   geometry      [n1+2g1+s1][n2+2g2+s2] per (i,j) -- independent of x3
 *     gcov, gcon  [..][8 locations][4][4]
 *     gcovpert    [..][8][4]
 *     gdet        [..][8]
 *     conn        [..][4][4][4]   at CENT, conn[k][l][j] as the reference
 *     floors      [..][2]         rho/u floor at CENT (set_density_floors)
 *   where gd = (nd>1) ? ng : 0 and sd = (nd>1).
 */
#ifndef HARM_ORACLE_H
#define HARM_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* limiter ids as global.h:297-314 */
#define HGO_LIM_DONOR 0
#define HGO_LIM_VANL 1
#define HGO_LIM_MINM 2
#define HGO_LIM_MC 3
#define HGO_LIM_PARA 4
#define HGO_LIM_WENO5 9
/* flux ids as global.h:247-251 */
#define HGO_FLUX_LAXF 0
#define HGO_FLUX_HLL 1
/* boundary ids as definit.h:300-310 */
#define HGO_BC_OUTFLOW 0
#define HGO_BC_POLARAXIS 4
#define HGO_BC_PERIODIC 7
/* x1 OUTFLOW of the general bounds.c (bounds.c:84-135, 218-292): a plain
   zero-gradient copy, without the inflow check and gamma limit that
   bounds.fishmon.c applies to OUTFLOW (own id: the reference reuses 0) */
#define HGO_BC_OUTFLOW_COPY 1000
/* face ids as global.h:467-472 */
#define HGO_X1UP 0
#define HGO_X1DN 1
#define HGO_X2UP 2
#define HGO_X2DN 3
#define HGO_X3UP 4
#define HGO_X3DN 5

typedef struct {
  int n1, n2, n3, ng;
  int lim, fluxmethod;
  int bc[6];
  double dx[4];
  double gam, cour, safe, defcon, tf;
  double rhominlimit, uuminlimit, gammamax, gammafail;
  int timeorder;   /* TIMEORDER: 1 Euler, 2 midpoint, 3 TVD RK3, 4 RK4 (0 = 2) */
  int utoprimversion; /* UTOPRIMVERSION: HGO_UTOPRIM2DFINAL (0 also) or HGO_UTOPRIMJONNONRELCOMPAT */
  int doenoflux;      /* DOENOFLUX: HGO_NOENOFLUX (advance_standard) or HGO_ENOFINITEVOLUME
                         (advance_finitevolume with avgscheme=DONOR, the FM torus setting) */
} hgo_config;

/* DOENOFLUX choices (global.h:188-191) */
#define HGO_NOENOFLUX 0
#define HGO_ENOFINITEVOLUME 3

/* inverter choices, numbered as global.h:283-287 */
#define HGO_UTOPRIM2DFINAL 6
#define HGO_UTOPRIMJONNONRELCOMPAT 8

typedef struct {
  const double *gcov, *gcon, *gcovpert, *gdet, *conn, *floors;
} hgo_geometry;

typedef struct {
  long newton_iters;   /* total Newton iterations (the reference's nstroke) */
  int err;             /* bitmask of conditions where the reference calls fail()/myexit() */
  int nfail_final;     /* zones with nonzero FLAGUTOPRIMFAIL after the last substep */
} hgo_stats;

/* Advance nsteps full time steps (step_ch).  p/pflag hold the full arrays with
   ghosts; t/dt are updated as step_ch.c:236-247 does.  Returns 0 or the
   error bitmask. */
int hgo_step(const hgo_config *c, const hgo_geometry *g, double *p, int *pflag, double *t, double *dt, int nsteps,
             hgo_stats *st);

/* hgo_step with the evolved conserved state u (the reference's unew, same
   layout as p).  With DOENOFLUX = ENOFINITEVOLUME the scheme evolves u
   itself (each step starts from ui = unew) and u is read and written; NULL
   starts from U(p) as after init.  Ignored (may be NULL) otherwise. */
int hgo_step_u(const hgo_config *c, const hgo_geometry *g, double *p, int *pflag, double *u, double *t, double *dt,
               int nsteps, hgo_stats *st);

/* pi2Uavg (initbase.c:1833) with avgscheme=DONOR: u = U(p) in every zone,
   ghosts included. */
int hgo_pi2u(const hgo_config *c, const hgo_geometry *g, const double *p, double *u);

/* One substep of advance_standard() + bound_prim + post_fixup + bound_prim
   for RK stage `timeorder` of the midpoint method (for debugging/parity of
   intermediate states).  pb is read, pi read, pf written; uf/ucum are the
   conserved accumulators; F1..F3 receive the face fluxes after flux_ct;
   ndt receives the new dt estimate. */
int hgo_substep(const hgo_config *c, const hgo_geometry *g, const double *pi, const double *pb, double *pf,
                double *uf, double *ucum, double *F1, double *F2, double *F3, int *pflag, double dt, int timeorder,
                double *ndt, hgo_stats *st);

/* Batched con-to-prim: Utoprimgen (utoprimgen.c:23) for n zones given the
   evolved conserved vector U (with gdet) and the per-zone metric at CENT;
   pr holds the guess on input and the solution on output. */
int hgo_utoprim_batch(const double *U, const double *gcov, const double *gcon, const double *gdet, double *pr,
                      int *pflag, long n, double gam, double gammafail, long *iters);

/* The same with the inverter chosen (HGO_UTOPRIM2DFINAL or
   HGO_UTOPRIMJONNONRELCOMPAT). */
int hgo_utoprim_batch_v(const double *U, const double *gcov, const double *gcon, const double *gdet, double *pr,
                        int *pflag, long n, double gam, double gammafail, int utoprimversion, long *iters);

/* post_fixup (fixup.c:37-96) on p and pflag in place: bound_pflag,
   fixup_checksolution, fixup_utoprim (the bound_prim that follows it in
   step_ch is not part of it).  unew may be NULL; with the finite-volume
   scheme on a final step it receives the diag_fixup corrections. */
int hgo_post_fixup(const hgo_config *c, const hgo_geometry *g, double *p, int *pflag, int finalstep, double *unew);

/* fluxcalc (flux.c:7-318) including flux_ct (fluxct.c:10) on p: F1..F3
   (zone layout x NPR) receive the face fluxes the update reads, the others
   are left as they were; ndt[0..2] the per-direction dt estimates. */
int hgo_fluxcalc(const hgo_config *c, const hgo_geometry *g, const double *p, double *F1, double *F2, double *F3,
                 double *ndt);

/* fixup_checksolution (fixup.c:460-560) alone: pflag in place; gammacheck
   (may be NULL, else zone layout) receives the Lorentz factors compared. */
int hgo_checksolution(const hgo_config *c, const hgo_geometry *g, const double *p, int *pflag, double *gammacheck);

/* Bound the primitives in place (bound_prim). */
int hgo_bound_prim(const hgo_config *c, const hgo_geometry *g, double *p);

int hgo_abi_version(void);

#ifdef __cplusplus
}
#endif
#endif
