/*
 * step_ch_gpu.c -- drop-in GPU step_ch() for the reference HARM build.
 *
 * Linked into the reference's own C program in place of its CPU step_ch
 * (step_ch.c:16), this file makes the unmodified host loop (main.c:33-84:
 * nstroke = 0; step_ch(); error_check; diag; nstep++) advance the grid on
 * the B200 through the C ABI of include/harmgpu.h.  The reference keeps
 * owning every array: each call copies the primitives (and, with the
 * finite-volume scheme, the evolved conserved state unew) of its static
 * arrays onto the device, runs one full time step there (hgpu_step_ch:
 * advance, fluxcalc + flux_ct, Utoprimgen, fixups, bound_prim, the dt
 * update) and copies the result back into the same arrays, so diag(),
 * dumps and restarts read the state exactly as after a CPU step.
 *
 * Build (oracle/build_ref.py --gpu-shim does this): compile the reference's
 * sources with its own step_ch renamed to harm_cpu_step_ch (a one-token
 * change of step_ch.c:16; the reference never calls step_ch from anywhere
 * but main.c), add this file, -I include/ and link libharmgpu.so:
 *     gcc ... step_ch.c(renamed) ... step_ch_gpu.c -Iinclude -Lharm_finalwham_b200/lib -lharmgpu -lm
 *
 * Set-up happens on the first call, from the reference's globals after
 * init(): grid size and ghosts (N1..N3, MAXBND), options (lim, fluxmethod,
 * BCtype, TIMEORDER, UTOPRIMVERSION, DOENOFLUX), scalars (gam, cour, SAFE,
 * defcon, tf, RHOMINLIMIT, UUMINLIMIT, GAMMAMAX, GAMMAFAIL, dx) and the
 * geometry arrays (gcov, gcon, gcovpert, gdet at the 8 locations, conn at
 * CENT, the density floors of set_density_floors at CENT) of the first x3
 * plane: the metric does not depend on x3.
 *
 * The device keeps the ghost zones the scheme reads (MC 3, PARA 3, WENO5 6;
 * the finite-volume scheme all MAXBND: its flux and dt loops cover every
 * transverse ghost); the reference's ghost zones beyond those are left as
 * they were.  Of pflag, the slots FLAGUTOPRIMFAIL (the inversion and
 * fixups) and FLAGBSQORHO / FLAGBSQOU (pre_fixup's b^2 flags) are produced.
 *
 * Boundary meanings: the FM torus file's bounds.fishmon.c is the default.
 * Built with -DHARMGPU_GENERIC_BOUNDS (the reference's generic bounds.c, as
 * its test problems use), OUTFLOW is the plain copy (HGPU_BC_OUTFLOW_COPY)
 * and POLARAXIS the reflection with u~2 and B2 negated
 * (HGPU_BC_POLARAXIS_FLIP); with the Bondi-integral x1 boundaries
 * (BONDIINTOUTFLOW / BONDIMDOTOUTFLOW, bounds.c:140-156, 295-308) the
 * coordinate data they need comes from the reference's own coord,
 * bl_coord, dxdxprim, matrix_inverse and gcov_func(KSCOORDS).
 *
 * Environment:
 *   HARMGPU_PRECISION=mixed   the mixed-precision path instead of FP64
 *   HARMGPU_RESIDENT=1        upload the state on the first call only and
 *                             keep it on the device across steps (for host
 *                             loops that never modify p between steps);
 *                             results are still copied back every step
 *
 * Restart dumps and diagnostics: the reference's restart_write
 * (restart.c:206), diag (diag.c:9) and dump_ener (dump_ener.c:3) are kept as
 * harm_cpu_restart_write, harm_cpu_diag and harm_cpu_dump_ener (one-token
 * renames, done by the same build step) and wrapped below.  Before any of
 * them runs, the device's failure and floor counters since the last call
 * are added to the reference's failfloorcount (every time scale, as
 * diag_fixup increments them, fixup.c:206), and restart_write first copies
 * unew from the device (the host arrays do not receive it after every step
 * for the non-finite-volume schemes), so dumps, ener.out's counters and
 * the restart file hold what a CPU run writes.
 *
 * Errors: a failing hgpu_* call prints hgpu_last_error() to the reference's
 * fail_file and step_ch returns 1, which the reference's MYFUN/error_check
 * turn into its own failure path.  HGPU_E_PHYSICS marks the conditions where
 * the CPU step would have called fail() or myexit().
 */
#include "decs.h"
#include "harmgpu.h"

extern int set_density_floors(struct of_geom *ptrgeom, FTYPE *pr, FTYPE *prfloor);

static hgpu_ctx *g_ctx;
static int g_ng, g_g[4], g_nt[4], g_gt[3];
static double *g_p, *g_u;
static int *g_pflag, *g_bsq;
static long long *g_ffc;
static int g_resident, g_uploaded;

#define CHECK(call)                                                                            \
  do {                                                                                         \
    int rc_ = (call);                                                                          \
    if (rc_ != HGPU_OK) {                                                                      \
      dualfprintf(fail_file, "step_ch_gpu: %s failed (%d): %s\n", #call, rc_, hgpu_last_error()); \
      return 1;                                                                                \
    }                                                                                          \
  } while (0)

/* ghost zones the device keeps for the reference's scheme */
static int device_ghosts(void)
{
  if (DOENOFLUX == ENOFINITEVOLUME) return MAXBND;
  if (lim == WENO5) return 6;
  return 3;
}

static long long zone_index(int i, int j, int k)
{
  return ((long long)(i + g_g[1]) * g_nt[2] + (j + g_g[2])) * g_nt[3] + (k + g_g[3]);
}

/* copy the device-layout window of a reference zone array (ghosts cropped to
   g_ng) to or from the reference array */
static void window(FTYPE (*a)[N2M][N3M][NPR], double *w, int to_ref)
{
  int i, j, k, pl;
  for (i = -g_g[1]; i < N1 + g_g[1]; i++)
    for (j = -g_g[2]; j < N2 + g_g[2]; j++)
      for (k = -g_g[3]; k < N3 + g_g[3]; k++) {
        double *z = w + NPR * zone_index(i, j, k);
        if (to_ref)
          for (pl = 0; pl < NPR; pl++) a[i][j][k][pl] = z[pl];
        else
          for (pl = 0; pl < NPR; pl++) z[pl] = a[i][j][k][pl];
      }
}

static void flag_window(int to_ref)
{
  int i, j, k;
  for (i = -g_g[1]; i < N1 + g_g[1]; i++)
    for (j = -g_g[2]; j < N2 + g_g[2]; j++)
      for (k = -g_g[3]; k < N3 + g_g[3]; k++) {
        if (to_ref) pflag[i][j][k][FLAGUTOPRIMFAIL] = g_pflag[zone_index(i, j, k)];
        else g_pflag[zone_index(i, j, k)] = pflag[i][j][k][FLAGUTOPRIMFAIL];
      }
}

/* index of a zone in the reference's metric arrays: a constant metric
   (CARTMINKMETRIC) is stored once (defs.h:214, get_geometry phys.c:869-877) */
#if(MCOORD!=CARTMINKMETRIC)
#define MIDX(a) (a)
#else
#define MIDX(a) 0
#endif

/* geometry of the first x3 plane, per (i,j), in the C ABI's layout */
static int upload_geometry(void)
{
  const long long nij = (long long)g_gt[1] * g_gt[2];
  double *gcv = (double *)calloc((size_t)nij * NPG * 16, sizeof(double));
  double *gcn = (double *)calloc((size_t)nij * NPG * 16, sizeof(double));
  double *gpt = (double *)calloc((size_t)nij * NPG * 4, sizeof(double));
  double *gdt = (double *)calloc((size_t)nij * NPG, sizeof(double));
  double *cnn = (double *)calloc((size_t)nij * 64, sizeof(double));
  double *flr = (double *)calloc((size_t)nij * 2, sizeof(double));
  int i, j, loc, a, b, c, rc;
  const int k = 0;
  if (!gcv || !gcn || !gpt || !gdt || !cnn || !flr) {
    dualfprintf(fail_file, "step_ch_gpu: out of host memory for the geometry\n");
    free(gcv); free(gcn); free(gpt); free(gdt); free(cnn); free(flr);
    return 1;
  }
  for (i = -g_g[1]; i < N1 + g_g[1] + (N1 > 1); i++)
    for (j = -g_g[2]; j < N2 + g_g[2] + (N2 > 1); j++) {
      const long long ij = (long long)(i + g_g[1]) * g_gt[2] + (j + g_g[2]);
      /* face/corner locations reach one zone beyond the cell arrays */
      const int in_cells = (i < N1 + N1BND) && (j < N2 + N2BND);
      for (loc = 0; loc < NPG; loc++) {
        for (a = 0; a < NDIM; a++) {
          for (b = 0; b < NDIM; b++) {
            gcv[(ij * NPG + loc) * 16 + 4 * a + b] = gcov[MIDX(i)][MIDX(j)][MIDX(k)][loc][a][b];
            gcn[(ij * NPG + loc) * 16 + 4 * a + b] = gcon[MIDX(i)][MIDX(j)][MIDX(k)][loc][a][b];
          }
          gpt[(ij * NPG + loc) * 4 + a] = gcovpert[MIDX(i)][MIDX(j)][MIDX(k)][loc][a];
        }
        gdt[ij * NPG + loc] = gdet[MIDX(i)][MIDX(j)][MIDX(k)][loc];
      }
      if (in_cells) {
        struct of_geom geom;
        FTYPE prfloor[NPR];
        for (a = 0; a < NDIM; a++)
          for (b = 0; b < NDIM; b++)
            for (c = 0; c < NDIM; c++) cnn[ij * 64 + 16 * a + 4 * b + c] = conn[MIDX(i)][MIDX(j)][MIDX(k)][a][b][c];
        get_geometry(i, j, k, CENT, &geom);
        set_density_floors(&geom, p[i][j][k], prfloor);
        flr[ij * 2 + 0] = prfloor[RHO];
        flr[ij * 2 + 1] = prfloor[UU];
      }
    }
  rc = hgpu_upload_geometry(g_ctx, gcv, gcn, gpt, gdt, cnn, flr);
  free(gcv); free(gcn); free(gpt); free(gdt); free(cnn); free(flr);
  CHECK(rc);
  return 0;
}

extern void dxdxprim(FTYPE *X, FTYPE *V, FTYPE (*dxdxp)[NDIM]);
extern void matrix_inverse(FTYPE gcov[][NDIM], FTYPE gcon[][NDIM]);
extern void gcov_func(int getprim, int whichcoord, FTYPE *X, FTYPE gcov[][NDIM], FTYPE *gcovpert);

/* hgpu_set_bondi_boundaries' table: per x1 side, edge zone and ghost zones,
   active j, at CENT of the first x3 plane: r, dx/dx', its inverse, the
   Kerr-Schild metric */
static int upload_bondi_table(void)
{
  const int nq = g_g[1] + 1;
  double *tab;
  int side, q, j, a, b, rc;
  if (BCtype[X1UP] != HGPU_BC_BONDIMDOTOUTFLOW && BCtype[X1DN] != HGPU_BC_BONDIINTOUTFLOW) return 0;
  tab = (double *)calloc((size_t)2 * nq * N2 * 49, sizeof(double));
  if (!tab) {
    dualfprintf(fail_file, "step_ch_gpu: out of host memory for the Bondi boundary table\n");
    return 1;
  }
  for (side = 0; side < 2; side++)
    for (q = 0; q < nq; q++)
      for (j = 0; j < N2; j++) {
        const int i = side == 0 ? -q : N1 - 1 + q;
        double *o = tab + ((size_t)(side * nq + q) * N2 + j) * 49;
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
  rc = hgpu_set_bondi_boundaries(g_ctx, tab);
  free(tab);
  CHECK(rc);
  return 0;
}

static int setup(void)
{
  hgpu_config cfg;
  const char *prec = getenv("HARMGPU_PRECISION");
  const char *res = getenv("HARMGPU_RESIDENT");
  long long nz;
  int d;
  if (rescaletype != 0) {
    /* the device holds one floor pair per (i,j): the r-only floors of rescaletype 0 */
    dualfprintf(fail_file, "step_ch_gpu: rescaletype %d is not supported (0 only)\n", rescaletype);
    return 1;
  }
  memset(&cfg, 0, sizeof(cfg));
  g_ng = device_ghosts();
  if (g_ng > MAXBND) g_ng = MAXBND;
  cfg.n1 = N1;
  cfg.n2 = N2;
  cfg.n3 = N3;
  cfg.ng = g_ng;
  cfg.lim = lim;
  cfg.fluxmethod = fluxmethod;
  for (d = 0; d < 6; d++) cfg.bc[d] = BCtype[d];
#ifdef HARMGPU_GENERIC_BOUNDS
  for (d = 0; d < 6; d++) {
    if (cfg.bc[d] == POLARAXIS) cfg.bc[d] = HGPU_BC_POLARAXIS_FLIP;  /* bounds.c:477-489 */
    if (cfg.bc[d] == OUTFLOW) cfg.bc[d] = HGPU_BC_OUTFLOW_COPY;      /* bounds.c:84-135 */
  }
#endif
  cfg.precision = (prec && strcmp(prec, "mixed") == 0) ? HGPU_PREC_MIXED : HGPU_PREC_FP64;
  for (d = 1; d <= 3; d++) cfg.dx[d] = dx[d];
  cfg.gam = gam;
  cfg.cour = cour;
  cfg.safe = SAFE;
  cfg.defcon = defcon;
  cfg.tf = tf;
  cfg.rhominlimit = RHOMINLIMIT;
  cfg.uuminlimit = UUMINLIMIT;
  cfg.gammamax = GAMMAMAX;
  cfg.gammafail = GAMMAFAIL;
  cfg.timeorder = TIMEORDER;
  cfg.utoprimversion = UTOPRIMVERSION;
  cfg.doenoflux = DOENOFLUX;
  g_g[1] = N1 > 1 ? g_ng : 0;
  g_g[2] = N2 > 1 ? g_ng : 0;
  g_g[3] = N3 > 1 ? g_ng : 0;
  g_nt[1] = N1 + 2 * g_g[1];
  g_nt[2] = N2 + 2 * g_g[2];
  g_nt[3] = N3 + 2 * g_g[3];
  g_gt[1] = g_nt[1] + (N1 > 1);
  g_gt[2] = g_nt[2] + (N2 > 1);
  nz = (long long)g_nt[1] * g_nt[2] * g_nt[3];
  CHECK(hgpu_create(&cfg, &g_ctx));
  if (hgpu_alloc_pinned((size_t)nz * NPR * sizeof(double), (void **)&g_p) != HGPU_OK ||
      hgpu_alloc_pinned((size_t)nz * sizeof(int), (void **)&g_pflag) != HGPU_OK ||
      hgpu_alloc_pinned((size_t)nz * 2 * sizeof(int), (void **)&g_bsq) != HGPU_OK ||
      (DOENOFLUX == ENOFINITEVOLUME &&
       hgpu_alloc_pinned((size_t)nz * NPR * sizeof(double), (void **)&g_u) != HGPU_OK)) {
    dualfprintf(fail_file, "step_ch_gpu: pinned host buffers: %s\n", hgpu_last_error());
    return 1;
  }
#if(DODEBUG)
  g_ffc = (long long *)malloc(sizeof(long long) * 9 * (size_t)nz);
  if (!g_ffc) {
    dualfprintf(fail_file, "step_ch_gpu: out of host memory for the counters\n");
    return 1;
  }
#endif
  if (upload_geometry()) return 1;
  if (upload_bondi_table()) return 1;
  g_resident = res && atoi(res) != 0;
  trifprintf("step_ch_gpu: %dx%dx%d zones, %d ghosts on the device, %s\n", N1, N2, N3, g_ng,
             cfg.precision == HGPU_PREC_FP64 ? "FP64" : "mixed precision");
  return 0;
}

/* step_ch (step_ch.c:16-252) on the GPU: one full time step of the
   reference's static arrays, t and dt advanced as step_ch_simplempi does
   (step_ch.c:232-247) */
int step_ch(void)
{
  hgpu_stats st;
  double tt, dtt;
  if (!g_ctx && setup()) return 1;
  if (!g_resident || !g_uploaded) {
    window(p, g_p, 0);
    flag_window(0);
    CHECK(hgpu_upload_state(g_ctx, g_p, g_pflag, (double)t, (double)dt));
    if (DOENOFLUX == ENOFINITEVOLUME) {
      window(unew, g_u, 0);
      CHECK(hgpu_upload_conserved(g_ctx, g_u));
    }
    g_uploaded = 1;
  }
  CHECK(hgpu_step_ch(g_ctx, 1, &st));
  CHECK(hgpu_download_state(g_ctx, g_p, g_pflag, &tt, &dtt));
  window(p, g_p, 1);
  flag_window(1);
  CHECK(hgpu_download_bsqflags(g_ctx, g_bsq));
  {
    int i, j, k;
    for (i = -g_g[1]; i < N1 + g_g[1]; i++)
      for (j = -g_g[2]; j < N2 + g_g[2]; j++)
        for (k = -g_g[3]; k < N3 + g_g[3]; k++) {
          pflag[i][j][k][FLAGBSQORHO] = g_bsq[2 * zone_index(i, j, k)];
          pflag[i][j][k][FLAGBSQOU] = g_bsq[2 * zone_index(i, j, k) + 1];
        }
  }
  if (DOENOFLUX == ENOFINITEVOLUME) {
    /* unew is defined on the active zones only */
    int i, j, k, pl;
    CHECK(hgpu_download_conserved(g_ctx, g_u));
    ZLOOP for (pl = 0; pl < NPR; pl++) unew[i][j][k][pl] = g_u[NPR * zone_index(i, j, k) + pl];
  }
  nstroke += st.newton_iters;
  t = tt;
  dt = dtt;
  tstepparti = tsteppartf = t;
  realnstep++;
  return 0;
}

extern int harm_cpu_restart_write(long dump_cnt);
extern int harm_cpu_diag(int call_code);
extern int harm_cpu_dump_ener(int doener, int dordump, int call_code);

/* the device's failure and floor counters since the last call, added to
   failfloorcount of every time scale (the device's categories are the
   reference's, global.h:769-779; active zones) and cleared on the device */
static int sync_counters(void)
{
#if(DODEBUG)
  int i, j, k, c, tscale;
  if (!g_ctx || !g_ffc) return 0;
  CHECK(hgpu_download_failfloorcount(g_ctx, g_ffc, 1));
  ZLOOP {
    const long long *n = g_ffc + 9 * zone_index(i, j, k);
    for (c = 0; c < NUMFAILFLOORFLAGS && c < 9; c++)
      if (n[c]) TSCALELOOP(tscale) failfloorcount[i][j][k][tscale][c] += (CTYPE)n[c];
  }
#endif
  return 0;
}

/* diag (diag.c:9) and dump_ener (dump_ener.c:3) with the device's counters */
int diag(int call_code)
{
  if (sync_counters()) return 1;
  return harm_cpu_diag(call_code);
}

int dump_ener(int doener, int dordump, int call_code)
{
  if (sync_counters()) return 1;
  return harm_cpu_dump_ener(doener, dordump, call_code);
}

/* restart_write (restart.c:206-235) with the device's unew (the conserved
   state after the last step; rdump_content writes p and unew) */
int restart_write(long dump_cnt)
{
  if (sync_counters()) return 1;
  if (g_ctx && DOENOFLUX != ENOFINITEVOLUME) {
    int i, j, k, pl;
    CHECK(hgpu_download_conserved(g_ctx, g_p));
    ZLOOP for (pl = 0; pl < NPR; pl++) unew[i][j][k][pl] = g_p[NPR * zone_index(i, j, k) + pl];
    /* g_p held the primitives of the last step, which p already has */
  }
  return harm_cpu_restart_write(dump_cnt);
}
