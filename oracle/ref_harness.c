/*
 * Test harness main() for the reference HARM build (oracle/_ref).
 *
 * This file is NOT part of the product.  It is compiled by oracle/build_ref.py
 * together with the reference's own sources (copied to a scratch directory,
 * never into this repository) in place of the reference main.c
 * (main.c:5-98).  It runs the reference's init() and step_ch() exactly as the
 * reference main loop does (main.c:33-49: nstroke=0; step_ch(); nstep++),
 * skipping only the diagnostics/dump cadence (diag(), postdt()), and writes the
 * reference's own arrays to raw binary files so that the CPU restatement
 * (oracle/harm_oracle.c) and the CUDA path can be pinned against them.
 *
 * usage: harm_ref <outdir|-> <nsteps> [dumpstep ...]
 *   writes <outdir>/init_*  (geometry, floors, initial primitives/flags, meta)
 *          <outdir>/s<step>_* after each listed step (and always after nsteps)
 *   and prints the CLOCK_MONOTONIC start/end of every step to stderr (the
 *   CPU baseline's step-loop timing).  "-" as outdir writes no files.
 *
 * options (before <outdir>):
 *   --phimodes <seed>  multiplies rho of every active zone by
 *                      1 + 0.02 sum_{m=1..4} A_m cos(m phi + phi_m), A_m ~ U(0,1),
 *                      phi_m ~ U(0,2pi) drawn from <seed> (splitmix64), after
 *                      the reference's init() and before its first step, then
 *                      repeats init's own closing sequence on the perturbed
 *                      state (initbase.c:107-160: fixup, bound_prim,
 *                      pre_fixup, set_dt, init_conservatives).  phi is the
 *                      reference's own Boyer-Lindquist azimuth of the zone
 *                      centre (coord + bl_coord, coord.c:1195, :389).
 *   --geomplane        writes the geometry of the first x3 plane only (the
 *                      metric does not depend on x3): keeps the init dump of
 *                      large 3D grids small.
 *   --ener             calls the reference's own dump_ener (dump_ener.c:3)
 *                      after init and after every dumped step, which appends
 *                      a line to ener.out in the working directory (t,
 *                      realnstep, the conserved integrals, ..., divbmax,
 *                      divbavg).
 *   --ffc              with every state dump also writes the reference's
 *                      failure and floor counters per zone (failfloorcount
 *                      of the first time scale, fixup.c:206; all zones with
 *                      ghosts, 9 categories, doubles as CTYPE is).
 *   --bcgeom           writes init_bcgeom.bin: per (i,j) of the first x3
 *                      plane, all zones with ghosts, at CENT, 49 doubles:
 *                      the Boyer-Lindquist r (coord + bl_coord, coord.c:1195,
 *                      389), dx/dx' (dxdxprim, coord.c:596), its inverse
 *                      (matrix_inverse, metric.c:1346) and the Kerr-Schild
 *                      metric g_{mu nu} (gcov_func(0, KSCOORDS), metric.c:11):
 *                      what the Bondi-integral boundaries use (bounds.c:788-1000).
 *   --rdump            calls the reference's own restart_write(0)
 *                      (restart.c:206) after the last step, which writes
 *                      dumps/rdump-0 in the working directory (its header,
 *                      then p and unew of every active zone).
 *
 * usage: harm_ref --invert <infile> <outfile>
 *   runs the reference's Utoprimgen() (utoprimgen.c:20) zone by zone on
 *   the records of <infile> (int64 n, then n x 49 doubles: evolved U[8]
 *   with gdet, gcov[16], gcon[16], gdet, guess primitives[8]) after init(),
 *   and writes <outfile>: n x 8 doubles (primitives), n int32 FLAGUTOPRIMFAIL
 *   flags, n int32 Newton iteration counts (nstroke per zone).
 *
 * usage: harm_ref --postfixup <infile> <outfile> <finalstep>
 *   after init(), replaces the primitives and the FLAGUTOPRIMFAIL flags by
 *   those of <infile> (the bytes of the reference's p array, N1M x N2M x N3M
 *   x NPR doubles with its MAXBND ghosts, then N1M x N2M x N3M int32 flags in
 *   the same zone order), runs the reference's own post_fixup(STAGEM1, p, p,
 *   finalstep) (fixup.c:37-96: bound_pflag, fixup_checksolution,
 *   fixup_utoprim) and writes the two arrays back to <outfile> in the same
 *   form.
 *
 * usage: harm_ref --boundprim <infile> <outfile>
 *   the same for the reference's own bound_prim(STAGEM1, p) (the problem
 *   file's boundaries, e.g. bounds.fishmon.c:29-345 with the inflow check
 *   of fixup.c:2271); <infile> and <outfile> hold the p array only.
 *
 * usage: harm_ref --fluxcalc <infile> <outfile>
 *   the reference's own fluxcalc(STAGEM1, p, F1, F2, F3, 1.0, &ndt1, &ndt2,
 *   &ndt3) (flux.c:7: reconstruction, wave speeds, Riemann fluxes and
 *   flux_ct) on the p of <infile>; <outfile>: F1, F2, F3 (each N1M x N2M x
 *   N3M x NPR doubles, zeros for a direction of one zone) then ndt1..3.
 */
#include "defs.h"  /* defines the reference globals, as the reference main.c does */
#include <sys/stat.h>
#include <time.h>

extern int init(int argc, char *argv[]);
extern int step_ch(void);
extern int error_check(int wherefrom);
extern int set_density_floors(struct of_geom *ptrgeom, FTYPE *pr, FTYPE *prfloor);

static char outdir[1024];
static int geomplane = 0;
static int do_ener = 0;
static int do_rdump = 0;
static int do_ffc = 0;
static int do_bcgeom = 0;
extern void dxdxprim(FTYPE *X, FTYPE *V, FTYPE (*dxdxp)[NDIM]);
extern void matrix_inverse(FTYPE gcov[][NDIM], FTYPE gcon[][NDIM]);
extern void gcov_func(int getprim, int whichcoord, FTYPE *X, FTYPE gcov[][NDIM], FTYPE *gcovpert);
extern int restart_write(long dump_cnt);
extern int dump_ener(int doener, int dordump, int call_code);

/* splitmix64 (Steele, Lea and Flood, OOPSLA 2014): a small seeded generator
   for the azimuthal mode amplitudes and phases */
static unsigned long long sm_state;
static double sm_uniform(void)
{
  unsigned long long z = (sm_state += 0x9E3779B97F4A7C15ULL);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  z = z ^ (z >> 31);
  return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

extern int fixup(int stage, FTYPE (*pv)[N2M][N3M][NPR], int finalstep);
extern int pre_fixup(int stage, FTYPE (*pv)[N2M][N3M][NPR]);
extern int bound_prim(int boundstage, FTYPE prim[][N2M][N3M][NPR]);
extern int fluxcalc(int stage, FTYPE pr[][N2M][N3M][NPR], FTYPE F1[][N2M][N3M][NPR], FTYPE F2[][N2M][N3M][NPR],
                    FTYPE F3[][N2M][N3M][NPR], FTYPE CUf, FTYPE *ndt1, FTYPE *ndt2, FTYPE *ndt3);
extern int set_dt(FTYPE (*prim)[N2M][N3M][NPR], SFTYPE *dt);
extern int init_conservatives(FTYPE p[][N2M][N3M][NPR], FTYPE Utemp[][N2M][N3M][NPR], FTYPE U[][N2M][N3M][NPR]);
extern void coord(int i, int j, int k, int loc, FTYPE *X);
extern void bl_coord(FTYPE *X, FTYPE *V);

/* density modes along the azimuth on top of the reference's initial data,
   then init's closing sequence again (initbase.c:107-160) */
static int apply_phi_modes(unsigned long long seed, double amp)
{
  double Am[4], phm[4];
  int i, j, k, m;
  sm_state = seed;
  for (m = 0; m < 4; m++) Am[m] = sm_uniform();
  for (m = 0; m < 4; m++) phm[m] = 2.0 * M_PI * sm_uniform();
  ZLOOP {
    FTYPE X[NDIM], V[NDIM];
    double pert = 0.0;
    coord(i, j, k, CENT, X);
    bl_coord(X, V);
    for (m = 0; m < 4; m++) pert += Am[m] * cos((m + 1) * V[3] + phm[m]);
    p[i][j][k][RHO] *= 1.0 + amp * pert;
  }
#if(FIXUPAFTERINIT)
  if (fixup(STAGEM1, p, 0) >= 1) return 1;
#endif
  if (bound_prim(STAGEM1, p) >= 1) return 1;
  if (pre_fixup(STAGEM1, p) >= 1) return 1;
  set_dt(p, &dt);
  if (DOENOFLUXMEMORY) init_conservatives(p, ulast, uinitial);
  else init_conservatives(p, ulast, unew);
  return 0;
}

static void wbin(const char *tag, const char *name, const void *ptr, size_t nbytes)
{
  char fn[2048];
  FILE *f;
  snprintf(fn, sizeof(fn), "%s/%s_%s.bin", outdir, tag, name);
  f = fopen(fn, "wb");
  if (!f) { fprintf(stderr, "harness: cannot write %s\n", fn); exit(3); }
  if (fwrite(ptr, 1, nbytes, f) != nbytes) { fprintf(stderr, "harness: short write %s\n", fn); exit(3); }
  fclose(f);
}

static void write_meta(const char *tag)
{
  char fn[2048];
  FILE *f;
  int pl;
  snprintf(fn, sizeof(fn), "%s/%s_meta.txt", outdir, tag);
  f = fopen(fn, "w");
  if (!f) { fprintf(stderr, "harness: cannot write %s\n", fn); exit(3); }
  fprintf(f, "N1 %d\nN2 %d\nN3 %d\nMAXBND %d\nNPR %d\nNPG %d\nNUMPFLAGS %d\n",
          N1, N2, N3, MAXBND, NPR, NPG, NUMPFLAGS);
  fprintf(f, "SHIFT1 %d\nSHIFT2 %d\nSHIFT3 %d\n", SHIFT1, SHIFT2, SHIFT3);
  fprintf(f, "t %.17g\ndt %.17g\nnstep %ld\nrealnstep %ld\n", (double)t, (double)dt, nstep, realnstep);
  fprintf(f, "gam %.17g\ncour %.17g\nSAFE %.17g\ndefcon %.17g\ntf %.17g\n",
          (double)gam, (double)cour, (double)SAFE, (double)defcon, (double)tf);
  fprintf(f, "dx1 %.17g\ndx2 %.17g\ndx3 %.17g\n", (double)dx[1], (double)dx[2], (double)dx[3]);
  fprintf(f, "startx1 %.17g\nstartx2 %.17g\nstartx3 %.17g\n",
          (double)startx[1], (double)startx[2], (double)startx[3]);
  fprintf(f, "RHOMIN %.17g\nUUMIN %.17g\nRHOMINLIMIT %.17g\nUUMINLIMIT %.17g\n",
          (double)RHOMIN, (double)UUMIN, (double)RHOMINLIMIT, (double)UUMINLIMIT);
  fprintf(f, "GAMMAMAX %.17g\nGAMMAFAIL %.17g\n", (double)GAMMAMAX, (double)GAMMAFAIL);
  fprintf(f, "a %.17g\nhslope %.17g\nRin %.17g\nRout %.17g\nR0 %.17g\n",
          (double)a, (double)hslope, (double)Rin, (double)Rout, (double)R0);
  fprintf(f, "lim %d\nfluxmethod %d\nFLUXB %d\nUTOPRIMVERSION %d\nTIMEORDER %d\nDOENOFLUX %d\n",
          lim, fluxmethod, FLUXB, UTOPRIMVERSION, TIMEORDER, DOENOFLUX);
  fprintf(f, "rescaletype %d\ndefcoord %d\n", rescaletype, defcoord);
  for (pl = 0; pl < 6; pl++) fprintf(f, "BCtype%d %d\n", pl, BCtype[pl]);
  fprintf(f, "failed %d\nnstroke %.17g\n", failed, (double)nstroke);
  fprintf(f, "GEOMPLANE %d\n", geomplane);
  fclose(f);
}

static void dump_state(const char *tag, int with_fluxes)
{
  write_meta(tag);
  wbin(tag, "p", a_p, sizeof(a_p));
  wbin(tag, "pflag", a_pflag, sizeof(a_pflag));
  if (do_ffc) {
    /* time scale 0 of failfloorcount[N1M][N2M][N3M][NUMTSCALES][NUMFAILFLOORFLAGS] */
    const size_t nzone = (size_t)N1M * N2M * N3M;
    double *buf = (double *)malloc(sizeof(double) * NUMFAILFLOORFLAGS * nzone);
    const CTYPE *src = &a_failfloorcount[0][0][0][0][0];
    size_t z;
    int c;
    for (z = 0; z < nzone; z++)
      for (c = 0; c < NUMFAILFLOORFLAGS; c++) buf[z * NUMFAILFLOORFLAGS + c] = (double)src[z * NUMTSCALES * NUMFAILFLOORFLAGS + c];
    wbin(tag, "ffc", buf, sizeof(double) * NUMFAILFLOORFLAGS * nzone);
    free(buf);
  }
  if (!with_fluxes) wbin(tag, "unew", a_unew, sizeof(a_unew)); /* the conserved state after init */
  if (with_fluxes) {
    wbin(tag, "pk", a_pk, sizeof(a_pk));
    wbin(tag, "unew", a_unew, sizeof(a_unew));
#if(N1>1)
    wbin(tag, "F1", a_F1, sizeof(a_F1));
#endif
#if(N2>1)
    wbin(tag, "F2", a_F2, sizeof(a_F2));
#endif
#if(N3>1)
    wbin(tag, "F3", a_F3, sizeof(a_F3));
#endif
    wbin(tag, "emf", a_emf, sizeof(a_emf));
  }
}

static void dump_geometry(void)
{
  /* floors as the reference's fixup1zone() computes them at CENT
     (fixup.c:341-447 via set_density_floors fixup.c:1542) */
  static FTYPE floors[N1M][N2M][N3M][2];
  struct of_geom geom;
  FTYPE prfloor[NPR];
  int i, j, k;
  FULLLOOP {
    get_geometry(i, j, k, CENT, &geom);
    set_density_floors(&geom, p[i][j][k], prfloor);
    floors[i + N1BND][j + N2BND][k + N3BND][0] = prfloor[RHO];
    floors[i + N1BND][j + N2BND][k + N3BND][1] = prfloor[UU];
  }
  if (!geomplane) {
    wbin("init", "floors", floors, sizeof(floors));
    wbin("init", "gcov", a_gcov, sizeof(a_gcov));
    wbin("init", "gcon", a_gcon, sizeof(a_gcon));
    wbin("init", "gcovpert", a_gcovpert, sizeof(a_gcovpert));
    wbin("init", "gdet", a_gdet, sizeof(a_gdet));
    wbin("init", "conn", a_conn, sizeof(a_conn));
    return;
  }
  /* first x3 plane of every array, same element order with the x3 extent 1 */
  {
    const int n1 = N1M + SHIFT1, n2 = N2M + SHIFT2, n3 = N3M + SHIFT3;
    int ii, jj;
#define PLANE(arr, name, n1_, n2_, n3_)                                                        \
    do {                                                                                        \
      size_t per = sizeof(arr) / ((size_t)(n1_) * (n2_) * (n3_));                                \
      char *buf = (char *)malloc(per * (size_t)(n1_) * (n2_));                                   \
      for (ii = 0; ii < (n1_); ii++)                                                             \
        for (jj = 0; jj < (n2_); jj++)                                                           \
          memcpy(buf + per * ((size_t)ii * (n2_) + jj),                                          \
                 (char *)(arr) + per * (((size_t)ii * (n2_) + jj) * (n3_)), per);                 \
      wbin("init", name, buf, per * (size_t)(n1_) * (n2_));                                     \
      free(buf);                                                                                \
    } while (0)
    PLANE(floors, "floors", N1M, N2M, N3M);
    PLANE(a_gcov, "gcov", n1, n2, n3);
    PLANE(a_gcon, "gcon", n1, n2, n3);
    PLANE(a_gcovpert, "gcovpert", n1, n2, n3);
    PLANE(a_gdet, "gdet", n1, n2, n3);
    PLANE(a_conn, "conn", N1M, N2M, N3M);
#undef PLANE
  }
}

/* coordinate data of the Bondi-integral boundaries, first x3 plane */
static void dump_bcgeom(void)
{
  const int n1 = N1M, n2 = N2M;
  double *buf = (double *)malloc(sizeof(double) * 49 * (size_t)n1 * n2);
  int i, j, a, b;
  for (i = -N1BND; i < N1 + N1BND; i++)
    for (j = -N2BND; j < N2 + N2BND; j++) {
      double *o = buf + 49 * ((size_t)(i + N1BND) * n2 + (j + N2BND));
      FTYPE X[NDIM], V[NDIM], dxdxp[NDIM][NDIM], idxdxp[NDIM][NDIM], gks[NDIM][NDIM], gpert[NDIM];
      coord(i, j, 0, CENT, X);
      bl_coord(X, V);
      dxdxprim(X, V, dxdxp);
      matrix_inverse(dxdxp, idxdxp);
      gcov_func(0, KSCOORDS, X, gks, gpert);
      o[0] = V[1];
      for (a = 0; a < NDIM; a++)
        for (b = 0; b < NDIM; b++) {
          o[1 + 4 * a + b] = dxdxp[a][b];
          o[17 + 4 * a + b] = idxdxp[a][b];
          o[33 + 4 * a + b] = gks[a][b];
        }
    }
  wbin("init", "bcgeom", buf, sizeof(double) * 49 * (size_t)n1 * n2);
  free(buf);
}

extern int Utoprimgen(int evolvetype, int inputtype, FTYPE *U, struct of_geom *ptrgeom, FTYPE *pr);

static int invert_file(const char *in, const char *out)
{
  FILE *f = fopen(in, "rb");
  long long n, z;
  double *rec, *pout;
  int *fout, *iout;
  if (!f || fread(&n, sizeof(n), 1, f) != 1 || n < 0) { fprintf(stderr, "harness: bad %s\n", in); return 3; }
  rec = (double *)malloc(sizeof(double) * 49 * (n > 0 ? n : 1));
  pout = (double *)malloc(sizeof(double) * 8 * (n > 0 ? n : 1));
  fout = (int *)malloc(sizeof(int) * (n > 0 ? n : 1));
  iout = (int *)malloc(sizeof(int) * (n > 0 ? n : 1));
  if (fread(rec, sizeof(double) * 49, (size_t)n, f) != (size_t)n) { fprintf(stderr, "harness: short %s\n", in); return 3; }
  fclose(f);
  for (z = 0; z < n; z++) {
    const double *r = rec + 49 * z;
    FTYPE U[NPR], pr[NPR], gcov[NDIM][NDIM], gcon[NDIM][NDIM], gcovpert[NDIM];
    struct of_geom geom;
    int a, b, pl;
    for (pl = 0; pl < NPR; pl++) U[pl] = r[pl];
    for (a = 0; a < NDIM; a++)
      for (b = 0; b < NDIM; b++) {
        gcov[a][b] = r[8 + 4 * a + b];
        gcon[a][b] = r[24 + 4 * a + b];
      }
    for (a = 0; a < NDIM; a++) gcovpert[a] = 0.0;
    for (pl = 0; pl < NPR; pl++) pr[pl] = r[41 + pl];
    geom.gcov = gcov;
    geom.gcon = gcon;
    geom.gcovpert = gcovpert;
    geom.g = r[40];
    for (pl = 0; pl < NPR; pl++) geom.e[pl] = r[40]; /* WHICHEOM == WITHGDET */
    geom.i = geom.j = geom.k = 0;
    geom.p = CENT;
    nstroke = 0;
    Utoprimgen(EVOLVENOENTROPY, UEVOLVE, U, &geom, pr);
    for (pl = 0; pl < NPR; pl++) pout[8 * z + pl] = pr[pl];
    fout[z] = pflag[0][0][0][FLAGUTOPRIMFAIL];
    iout[z] = nstroke;
  }
  f = fopen(out, "wb");
  if (!f) { fprintf(stderr, "harness: cannot write %s\n", out); return 3; }
  fwrite(pout, sizeof(double) * 8, (size_t)n, f);
  fwrite(fout, sizeof(int), (size_t)n, f);
  fwrite(iout, sizeof(int), (size_t)n, f);
  fclose(f);
  free(rec); free(pout); free(fout); free(iout);
  return 0;
}

static int postfixup_file(const char *in, const char *out, int finalstep)
{
  const size_t nzone = (size_t)N1M * N2M * N3M;
  int *fl = (int *)malloc(sizeof(int) * nzone);
  int *pf = &a_pflag[0][0][0][0];
  size_t z;
  FILE *f = fopen(in, "rb");
  if (!fl || !f || fread(a_p, sizeof(a_p), 1, f) != 1 || fread(fl, sizeof(int), nzone, f) != nzone) {
    fprintf(stderr, "harness: bad %s\n", in);
    return 3;
  }
  fclose(f);
  for (z = 0; z < nzone; z++) pf[z * NUMPFLAGS + FLAGUTOPRIMFAIL] = fl[z];
  post_fixup(STAGEM1, p, p, finalstep);
  for (z = 0; z < nzone; z++) fl[z] = pf[z * NUMPFLAGS + FLAGUTOPRIMFAIL];
  f = fopen(out, "wb");
  if (!f || fwrite(a_p, sizeof(a_p), 1, f) != 1 || fwrite(fl, sizeof(int), nzone, f) != nzone) {
    fprintf(stderr, "harness: cannot write %s\n", out);
    return 3;
  }
  fclose(f);
  free(fl);
  return 0;
}

static int boundprim_file(const char *in, const char *out)
{
  FILE *f = fopen(in, "rb");
  if (!f || fread(a_p, sizeof(a_p), 1, f) != 1) {
    fprintf(stderr, "harness: bad %s\n", in);
    return 3;
  }
  fclose(f);
  bound_prim(STAGEM1, p);
  f = fopen(out, "wb");
  if (!f || fwrite(a_p, sizeof(a_p), 1, f) != 1) {
    fprintf(stderr, "harness: cannot write %s\n", out);
    return 3;
  }
  fclose(f);
  return 0;
}

static int fluxcalc_file(const char *in, const char *out)
{
  const size_t nf = (size_t)N1M * N2M * N3M * NPR;
  double *zero = (double *)calloc(nf, sizeof(double));
  FTYPE ndt[3] = {0.0, 0.0, 0.0};
  FILE *f = fopen(in, "rb");
  if (!zero || !f || fread(a_p, sizeof(a_p), 1, f) != 1) {
    fprintf(stderr, "harness: bad %s\n", in);
    return 3;
  }
  fclose(f);
  fluxcalc(STAGEM1, p, F1, F2, F3, 1.0, &ndt[0], &ndt[1], &ndt[2]);
  f = fopen(out, "wb");
  if (!f) {
    fprintf(stderr, "harness: cannot write %s\n", out);
    return 3;
  }
#if(N1>1)
  fwrite(a_F1, sizeof(a_F1), 1, f);
#else
  fwrite(zero, sizeof(double), nf, f);
#endif
#if(N2>1)
  fwrite(a_F2, sizeof(a_F2), 1, f);
#else
  fwrite(zero, sizeof(double), nf, f);
#endif
#if(N3>1)
  fwrite(a_F3, sizeof(a_F3), 1, f);
#else
  fwrite(zero, sizeof(double), nf, f);
#endif
  fwrite(ndt, sizeof(FTYPE), 3, f);
  fclose(f);
  free(zero);
  return 0;
}

int main(int argc, char *argv[])
{
  char *fakeargv[2];
  int nsteps, s, d, ndump = 0, nodump = 0;
  long long phiseed = -1;
  int dumps[64];

  if (argc == 4 && strcmp(argv[1], "--invert") == 0) {
    fakeargv[0] = argv[0];
    fakeargv[1] = NULL;
    if (init(1, fakeargv) >= 1) {
      fprintf(stderr, "harness: init failed\n");
      return 1;
    }
    return invert_file(argv[2], argv[3]);
  }
  if (argc == 5 && strcmp(argv[1], "--postfixup") == 0) {
    fakeargv[0] = argv[0];
    fakeargv[1] = NULL;
    if (init(1, fakeargv) >= 1) {
      fprintf(stderr, "harness: init failed\n");
      return 1;
    }
    return postfixup_file(argv[2], argv[3], atoi(argv[4]));
  }
  if (argc == 4 && strcmp(argv[1], "--boundprim") == 0) {
    fakeargv[0] = argv[0];
    fakeargv[1] = NULL;
    if (init(1, fakeargv) >= 1) {
      fprintf(stderr, "harness: init failed\n");
      return 1;
    }
    return boundprim_file(argv[2], argv[3]);
  }
  if (argc == 4 && strcmp(argv[1], "--fluxcalc") == 0) {
    fakeargv[0] = argv[0];
    fakeargv[1] = NULL;
    if (init(1, fakeargv) >= 1) {
      fprintf(stderr, "harness: init failed\n");
      return 1;
    }
    return fluxcalc_file(argv[2], argv[3]);
  }

  while (argc >= 2 && strncmp(argv[1], "--", 2) == 0) {
    if (strcmp(argv[1], "--phimodes") == 0 && argc >= 3) {
      phiseed = strtoll(argv[2], NULL, 10);
      argv += 2;
      argc -= 2;
    } else if (strcmp(argv[1], "--geomplane") == 0) {
      geomplane = 1;
      argv += 1;
      argc -= 1;
    } else if (strcmp(argv[1], "--ener") == 0) {
      do_ener = 1;
      argv += 1;
      argc -= 1;
    } else if (strcmp(argv[1], "--bcgeom") == 0) {
      do_bcgeom = 1;
      argv += 1;
      argc -= 1;
    } else if (strcmp(argv[1], "--ffc") == 0) {
      do_ffc = 1;
      argv += 1;
      argc -= 1;
    } else if (strcmp(argv[1], "--rdump") == 0) {
      do_rdump = 1;
      argv += 1;
      argc -= 1;
    } else {
      fprintf(stderr, "harness: unknown option %s\n", argv[1]);
      return 2;
    }
  }
  if (argc < 3) {
    fprintf(stderr, "usage: %s [--phimodes seed] [--geomplane] [--ener] [--rdump] [--ffc] [--bcgeom] <outdir|-> <nsteps> [dumpstep ...]\n", argv[0]);
    return 2;
  }
  /* outdir "-" runs the steps for timing only and writes nothing */
  nodump = (strcmp(argv[1], "-") == 0);
  snprintf(outdir, sizeof(outdir), "%s", argv[1]);
  if (!nodump) mkdir(outdir, 0755);
  nsteps = atoi(argv[2]);
  for (d = 3; d < argc && ndump < 64; d++) dumps[ndump++] = atoi(argv[d]);

  fakeargv[0] = argv[0];
  fakeargv[1] = NULL;
  if (init(1, fakeargv) >= 1) {
    fprintf(stderr, "harness: init failed\n");
    return 1;
  }
  if (phiseed >= 0 && apply_phi_modes((unsigned long long)phiseed, 0.02)) {
    fprintf(stderr, "harness: init after the azimuthal modes failed\n");
    return 1;
  }
  if (!nodump) {
    dump_geometry();
    if (do_bcgeom) dump_bcgeom();
    dump_state("init", 0);
  }
  if (do_ener && dump_ener(1, 0, INIT_OUT) >= 1) {
    fprintf(stderr, "harness: dump_ener failed at init\n");
    return 1;
  }

  for (s = 1; s <= nsteps; s++) {
    char tag[64];
    int want = (s == nsteps) && !nodump;
    struct timespec ts;
    nstroke = 0;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    fprintf(stderr, "harness: step %d start %.9f\n", s, ts.tv_sec + 1e-9 * ts.tv_nsec);
    if (step_ch() != 0) { fprintf(stderr, "harness: step_ch failed at step %d\n", s); return 1; }
    if (error_check(2)) { fprintf(stderr, "harness: error_check failed at step %d\n", s); return 1; }
    nstep++;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    fprintf(stderr, "harness: step %d end %.9f\n", s, ts.tv_sec + 1e-9 * ts.tv_nsec);
    for (d = 0; d < ndump; d++) if (dumps[d] == s) want = 1;
    if (want) {
      snprintf(tag, sizeof(tag), "s%d", s);
      /* dump_ener reads the state and the counters and writes ener.out only */
      if (do_ener && dump_ener(1, 0, DUMP_OUT) >= 1) {
        fprintf(stderr, "harness: dump_ener failed at step %d\n", s);
        return 1;
      }
      dump_state(tag, 1);
    }
  }
  if (do_rdump) {
    mkdir("dumps", 0755);
    if (restart_write(0) != 0) { fprintf(stderr, "harness: restart_write failed\n"); return 1; }
  }
  fprintf(stderr, "harness: done %d steps t=%.17g dt=%.17g\n", nsteps, (double)t, (double)dt);
  return 0;
}
