/*
 * harmgpu.h -- C ABI of the B200 per-zone conservative update of HARM.
 *
 * Plain C types only (pointers, sizes, ints, doubles).  A caller that can
 * link C (the reference's own C host loop, Python ctypes, cgo, JNI ...)
 * drives the GPU through these entry points.  Each entry point names the
 * reference routine it stands in for.
 *
 * Host array layouts are the reference's (defs.h:27-206 with the pointer
 * shift of set_arrays.c:14-78), restricted to `ng` ghost zones per
 * dimension that has more than one zone:
 *   primitives   double [n1+2g1][n2+2g2][n3+2g3][8]   (rho,u,u~1..3,B1..3)
 *   pflag        int    [n1+2g1][n2+2g2][n3+2g3]      (FLAGUTOPRIMFAIL slot)
 *   geometry     per (i,j) only -- the metric does not depend on x3:
 *     gcov, gcon double [n1+2g1+s1][n2+2g2+s2][8 locations][4][4]
 *     gcovpert   double [..][8][4]
 *     gdet       double [..][8]
 *     conn       double [..][4][4][4]   (CENT; conn[k][l][j] as set_grid.c:118)
 *     floors     double [..][2]         (rho, u floor at CENT: set_density_floors, fixup.c:1542)
 *   with gd = (nd>1 ? ng : 0), sd = (nd>1).
 *
 * Error convention: every entry point returns 0 on success, nonzero on
 * failure (HGPU_E_*), and never aborts the process.  Physical failures are
 * not errors: they are per-zone pflag codes (global.h:782-799) repaired by
 * the fixups, exactly as in the reference.
 */
#ifndef HARMGPU_H
#define HARMGPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HGPU_ABI_VERSION 16

/* return codes */
#define HGPU_OK 0
#define HGPU_E_INVALID 1      /* bad argument or unsupported option */
#define HGPU_E_CUDA 2         /* CUDA runtime error */
#define HGPU_E_PHYSICS 3      /* the reference would have called fail()/myexit() */
#define HGPU_E_NOMEM 4

/* option ids: the reference's own numbering (global.h:247-314, definit.h:300-310) */
#define HGPU_LIM_DONOR 0
#define HGPU_LIM_VANL 1
#define HGPU_LIM_MINM 2
#define HGPU_LIM_MC 3
#define HGPU_LIM_PARA 4
#define HGPU_LIM_WENO5 9
#define HGPU_FLUX_LAXF 0
#define HGPU_FLUX_HLL 1
#define HGPU_BC_OUTFLOW 0
#define HGPU_BC_POLARAXIS 4
#define HGPU_BC_PERIODIC 7
/* x1 OUTFLOW of the reference's general bounds.c (bounds.c:84-135, 218-292):
   a plain zero-gradient copy.  HGPU_BC_OUTFLOW is the OUTFLOW of
   bounds.fishmon.c (copy + inflow check + gamma limit); the reference uses
   id 0 for both, the problem file decides, so the copy gets its own id. */
#define HGPU_BC_OUTFLOW_COPY 1000
/* The generic bounds.c (the reference's test problems) gives POLARAXIS
   another meaning than bounds.fishmon.c: the x2 ghosts mirror the active
   zones with u~2 and B2 negated (bounds.c:477-489, POLEDEATH 0), where the
   FM torus file zeroes them and the first/last active rows.  That variant
   has its own id. */
#define HGPU_BC_POLARAXIS_FLIP 1001
/* Bondi-integral radial boundaries of the generic bounds.c (definit.h:329-330,
   the Bondi flow, init.c's TESTNUMBER 153): each x1 ghost zone holds the
   Bondi solution whose integrals C1 = T^n u^r r^2, C2 = (1 + (1+n) T)^2
   (1 - 2/r + (u^r)^2), K = p / rho^gam (n = 1/(gam-1), T = p/rho, Kerr-Schild
   u^r) are those of the first active zone (inner, BONDIINTOUTFLOW,
   bounds.c:140-156) or C1 of the last active zone with C2 = 1.373125 and
   K = 1 (outer, BONDIMDOTOUTFLOW, bounds.c:295-308); temperature by the
   reference's fixed-point iteration (bounds.c:1013-1083), the field zero.
   They need hgpu_set_bondi_boundaries.  The ghost zones agree with the
   reference's to a few ulp, not bit for bit: the integrals use pow, whose
   CUDA implementation rounds differently from the C library's. */
#define HGPU_BC_BONDIMDOTOUTFLOW 109  /* x1 outer */
#define HGPU_BC_BONDIINTOUTFLOW 110   /* x1 inner */

/* con-to-prim inverters (UTOPRIMVERSION, global.h:283-287) */
#define HGPU_UTOPRIM2DFINAL 6            /* 2D Newton on (W, v^2), utoprim_2d_final.c */
#define HGPU_UTOPRIMJONNONRELCOMPAT 8    /* 1D Newton on E'(W'), utoprim_jon.c; the FM
                                            torus default (init.fishmon.c:46) */

/* DOENOFLUX schemes (global.h:188-191) */
#define HGPU_NOENOFLUX 0                 /* advance_standard (advance.c:58): Ui = U(pi) */
#define HGPU_ENOFINITEVOLUME 3           /* advance_finitevolume (advance.c:245) with
                                            avgscheme=DONOR, the FM torus problem's own
                                            scheme (init.fishmon.c:97, 112): the conserved
                                            state unew is evolved; needs ng = the
                                            reference's MAXBND for its dt */

/* precision modes */
#define HGPU_PREC_FP64 0      /* bit-identical to the reference CPU build */
#define HGPU_PREC_MIXED 1     /* FP32 reconstruction, wave speeds and Riemann flux */

typedef struct {
  int n1, n2, n3;   /* active zones (N1,N2,N3 of the reference) */
  int ng;           /* ghost zones kept on the device (>= 2 for MC, >= 3 for PARA, >= 6 for WENO5) */
  int lim;          /* slope limiter (lim) */
  int fluxmethod;   /* Riemann solver (fluxmethod) */
  int bc[6];        /* BCtype[X1UP,X1DN,X2UP,X2DN,X3UP,X3DN] */
  int precision;    /* HGPU_PREC_* */
  double dx[4];     /* dx[1..3] */
  double gam, cour, safe, defcon, tf;
  double rhominlimit, uuminlimit, gammamax, gammafail;
  int timeorder;    /* TIMEORDER (setup_rktimestep, step_ch.c:442-562): 1 Euler,
                       2 midpoint, 3 TVD RK3, 4 RK4; 0 means 2 */
  int utoprimversion; /* HGPU_UTOPRIM*; 0 means HGPU_UTOPRIM2DFINAL */
  int doenoflux;    /* HGPU_NOENOFLUX or HGPU_ENOFINITEVOLUME */
} hgpu_config;

typedef struct hgpu_ctx hgpu_ctx;

typedef struct {
  long long newton_iters;   /* Newton iterations in the last call (the reference's nstroke) */
  int err;                  /* error bits: conditions where the reference calls fail() */
  int nfail;                /* zones with nonzero FLAGUTOPRIMFAIL after the last substep */
  int nfixed;               /* zones repaired by fixup_utoprim in the last call */
} hgpu_stats;

/* Library/ABI identification. */
int hgpu_abi_version(void);

/* Select the CUDA device that this host thread's later calls use
   (cudaSetDevice in the library's own CUDA runtime, which is linked
   statically, so a device chosen through another runtime, e.g. a Python
   framework's, does not reach it).  One process per GPU calls it with its
   local rank before hgpu_create; contexts keep the device they were created
   on.  HGPU_E_CUDA for a device that does not exist. */
int hgpu_set_device(int device);

/* Create a device context on the current CUDA device (init-time set_arrays.c / set_grid.c
   storage).  Returns HGPU_OK and *out, or an error code. */
int hgpu_create(const hgpu_config *cfg, hgpu_ctx **out);
void hgpu_destroy(hgpu_ctx *ctx);

/* Reuse a context for another solve of the same allocation shape (no
   counterpart in the reference, which runs one problem per process): the
   by-value parameters of cfg (dx, gam, cour, safe, defcon, tf, floor limits,
   gammamax, gammafail, boundary ids) replace the context's; grid size,
   ghosts, scheme, inverter, time order and precision must be unchanged
   (else HGPU_E_INVALID).  Upload the geometry and the state after it.  No
   device memory is allocated or freed, as the serving loop does for its
   idle contexts. */
int hgpu_reconfigure(hgpu_ctx *ctx, const hgpu_config *cfg);

/* Upload the precomputed geometry (set_grid.c:7-151) and floors
   (set_density_floors, fixup.c:1542-1654); host layouts above. */
int hgpu_upload_geometry(hgpu_ctx *ctx, const double *gcov, const double *gcon, const double *gcovpert,
                         const double *gdet, const double *conn, const double *floors);

/* Upload primitives p (and optionally pflag, may be NULL) plus t and dt. */
int hgpu_upload_state(hgpu_ctx *ctx, const double *p, const int *pflag, double t, double dt);
/* Download primitives/pflag (either may be NULL) and t, dt. */
int hgpu_download_state(hgpu_ctx *ctx, double *p, int *pflag, double *t, double *dt);

/* The same for hosts that hold only the active zones: p [n1][n2][n3][8],
   pflag [n1][n2][n3].  The upload fills the ghost zones on the device with
   bound_prim (the reference's step_ch ends with it, step_ch.c:568, so the
   ghosts equal those the host would have sent) and, for the finite-volume
   scheme, sets unew = U(p) as hgpu_upload_state does; pflag keeps the
   device's values (a step writes every flag it reads).  ~20% fewer bytes
   over PCIe than the arrays with ghosts at ng = 6.  Not for batches. */
int hgpu_upload_active(hgpu_ctx *ctx, const double *p, double t, double dt);
int hgpu_download_active(hgpu_ctx *ctx, double *p, int *pflag, double *t, double *dt);

/* step_ch (step_ch.c:16-252): nsteps full midpoint-RK2 steps with
   boundaries, fixups and the dt update.  Asynchronous on the context's stream
   unless stats is non-NULL (then it synchronises and fills stats). */
int hgpu_step_ch(hgpu_ctx *ctx, int nsteps, hgpu_stats *stats);

/* advance (advance.c:16) for RK stage `timeorder` (0 .. TIMEORDER-1),
   followed by the reference's per-stage bound_prim/post_fixup/bound_prim
   sequence (step_ch.c:94-186), with the pi/pb/pf arrays of
   setup_rktimestep.  ndt receives the new dt estimate. */
int hgpu_advance_stage(hgpu_ctx *ctx, int timeorder, double *ndt, hgpu_stats *stats);

/* fluxcalc (flux.c:7-318) including flux_ct (fluxct.c:10), on the current
   primitives (which=0: p, which=1: pk).  Fluxes F1..F3 are returned in the
   reference layout when the pointers are non-NULL (only the faces the update
   reads are defined).  ndt1..3 as fluxcalc. */
int hgpu_fluxcalc(hgpu_ctx *ctx, int which, double *F1, double *F2, double *F3, double *ndt1, double *ndt2,
                  double *ndt3);

/* bound_prim (step_ch.c:568) on p (which=0) or pk (which=1). */
int hgpu_bound_prim(hgpu_ctx *ctx, int which);

/* post_fixup (fixup.c:37-96) on the state p and its flags, as step_ch.c:144
   and :403 call it: bound_pflag, fixup_checksolution, fixup_utoprim
   (finalstep as the reference's argument: fixup_utoprim's final-step
   counting, and with the finite-volume scheme the diag_fixup corrections of
   unew).  The bound_prim that step_ch runs after it is hgpu_bound_prim.
   Synchronises; stats (may be NULL) receives nfixed and the error bits.
   Not for batch contexts, whose fixups run per instance inside a step. */
int hgpu_post_fixup(hgpu_ctx *ctx, int finalstep, hgpu_stats *stats);

/* Utoprimgen (utoprimgen.c:23) for a batch of n zones in host memory:
   U (evolved conserved, with gdet) [n][8], per-zone CENT metric gcov/gcon [n][16],
   gdet [n]; pr holds the guess and receives the result; pflag receives the
   codes.  iters (may be NULL) receives the total Newton iterations. */
int hgpu_utoprim_batch(const double *U, const double *gcov, const double *gcon, const double *gdet, double *pr,
                       int *pflag, long long n, double gam, double gammafail, long long *iters);

/* The same with the inverter chosen: utoprimversion is HGPU_UTOPRIM2DFINAL
   (what hgpu_utoprim_batch runs) or HGPU_UTOPRIMJONNONRELCOMPAT, the
   reference's Utoprimgen_pick(UTOPRIMJONNONRELCOMPAT) (utoprimgen.c:687) ->
   Utoprim_jon_nonrelcompat_inputnorestmass (utoprim_jon.c:65). */
int hgpu_utoprimgen_batch(const double *U, const double *gcov, const double *gcon, const double *gdet, double *pr,
                          int *pflag, long long n, double gam, double gammafail, int utoprimversion,
                          long long *iters);

/* Utoprimgen batch that allocates nothing (no counterpart in the reference).
   Same arguments and results as hgpu_utoprim_batch, for callers that cannot
   call cudaMalloc/cudaFree: a process whose device memory is already held by
   another allocator's pool (cudaMalloc would fail), or a host loop that calls
   the inversion often on small batches -- as the reference calls Utoprimgen
   zone by zone -- where cudaFree's implicit device synchronisation and
   per-call allocation would dominate.  Device scratch is a fixed file-scope
   array in the library: at most HGPU_NOALLOC_MAX_ZONES zones per call (larger
   n is rejected with HGPU_E_INVALID and a message), held by every GPU that
   loads the library until the process exits.  The first call on a device
   looks up the array's device address (cudaGetSymbolAddress) with that device
   current; make that first call before any stream capture.  That address is
   kept for the life of the process: after cudaDeviceReset (or anything else
   that destroys the device's primary context) it is stale, so do not call
   this entry point again in that process.  All calls share the array and
   each call overwrites it, so calls that overlap on the GPU (other host
   threads, other streams) race: serialise them. */
#define HGPU_NOALLOC_MAX_ZONES 16384
int hgpu_utoprim_batch_noalloc(const double *U, const double *gcov, const double *gcon, const double *gdet,
                               double *pr, int *pflag, long long n, double gam, double gammafail, long long *iters);

/* Batch of independent 1D problems in one context (no counterpart in the
   reference, which runs one problem per process): instance b has n1[b]
   active zones, zone size dx1[b], adiabatic index gam[b] and end time tf[b],
   and its own t and dt (step_ch's dt rule per instance; an instance stops
   when its t reaches tf).  The instances are concatenated along x1, each
   with its own cfg->ng ghost zones on both sides, in a line of
   sum(n1[b] + 2 ng) zones that hgpu_upload_state/hgpu_download_state
   exchange as one 1D array; hgpu_batch_layout gives the x1 index of every
   instance's first active zone in that line (relative to the line's first
   active zone).  cfg: n2 = n3 = 1, bc[X1UP] = bc[X1DN] = HGPU_BC_OUTFLOW_COPY;
   cfg->n1, dx, gam and tf are ignored.  Geometry is uploaded per zone of the
   line as for a 1D domain.  Every kernel of a step covers all instances. */
int hgpu_create_batch(const hgpu_config *cfg, int ninst, const int *n1, const double *dx1, const double *gam,
                      const double *tf, hgpu_ctx **out);
int hgpu_batch_layout(hgpu_ctx *ctx, int *i0);
/* per-instance t, dt, done flag (each may be NULL) and the number of finished instances */
int hgpu_batch_status(hgpu_ctx *ctx, double *t, double *dt, int *done, int *ndone);
/* set every instance's t and dt (e.g. an instance's own start-up dt, the
   reference's set_dt of its initial state); an instance with t >= its tf is
   marked done; the per-instance step counts restart from zero */
int hgpu_batch_set_time(hgpu_ctx *ctx, const double *t, const double *dt);

/* Advance a batch until every instance has reached its end time (or
   max_steps batch steps): CUDA-graph replays of check_every steps between
   reads of the instances' done flags.  *steps: batch steps taken; *ms:
   device time of the whole run; steps_per_instance[b]: time steps of
   instance b; done_ms[b]: time at which instance b was seen finished
   (resolution check_every steps; -1 if it did not finish).  Pointers may be
   NULL. */
int hgpu_batch_run(hgpu_ctx *ctx, int check_every, int max_steps, int *steps, float *ms, int *steps_per_instance,
                   float *done_ms);

/* step_ch as nsteps replays of one CUDA graph holding a whole time step
   (captured on the first call; profiling must be off).  Same results as
   hgpu_step_ch. */
int hgpu_step_graph(hgpu_ctx *ctx, int nsteps, hgpu_stats *stats);

/* Autotuner (no counterpart in the reference): for the FP64 flux, WENO5
   reconstruction, update and inversion kernels, times two resident-blocks-per-SM variants
   (registers per thread vs warps per SM) on this context's own state and
   keeps the faster for later steps.  Results do not depend on the choice;
   the state is left as it was (for a batch context, every instance's t,
   dt, done flag and step count too).  *_ms: kernel milliseconds of one step per
   candidate (0 where a family does not apply: weno without WENO5; in the
   mixed-precision mode weno, and flux unless the scheme is WENO5, whose
   Riemann kernel stays FP64). */
typedef struct {
  int flux_minb, weno_minb, update_minb, invert_minb;
  int flux_cand[2], weno_cand[2], update_cand[2], invert_cand[2];
  float flux_ms[2], weno_ms[2], update_ms[2], invert_ms[2];
  /* WENO5 tile shape per direction d = 1..3 (index 0 unused): output cells
     per tile along the direction and lines per tile (a power of two); the
     autotuner times up to four candidate shapes of its cost model per
     direction (weno_tile_ms: the chosen one's time per launch).  In
     hgpu_set_tuning, 0 keeps the current shape. */
  int weno_lb[4], weno_lines[4];
  float weno_tile_ms[4];
} hgpu_tuning;
int hgpu_autotune(hgpu_ctx *ctx, hgpu_tuning *out);
/* Apply a choice found before (the *_minb fields; each must be one of the
   candidates that hgpu_autotune reports), without timing anything. */
int hgpu_set_tuning(hgpu_ctx *ctx, const hgpu_tuning *t);

/* Diagnostics of the current state (the quantities dump_ener.c writes to
   ener.out, computed on the device): integral[pl] = sum over active zones of
   the conserved U (primtoU with gdet, UU without rest mass; the evolved unew
   for HGPU_ENOFINITEVOLUME, as constotal dump_ener.c:596-635) times
   dx1 dx2 dx3; divb_max / divb_avg = max and mean over active zones of the
   flux-CT div B at each zone's lower corner (divbmaxavg, dump_ener.c:482;
   DIVBFLUXCT, global.h:1586-1645); nfail = zones whose last inversion left
   a failure code; nfloor = zone floorings by fixup1zone summed over the last
   stepping call; t, dt, nsteps since the last upload.  divb_max includes
   the axis corners, where gdet vanishes and the reference's normalisation
   divides by ~0; divb_max_interior leaves them out.  Sums are
   deterministic (fixed-order two-pass reduction), not in the reference's
   serial order. */
typedef struct {
  double t, dt;
  double integral[8];
  double divb_max, divb_avg;
  int nfail;
  long long nfloor;
  long long nsteps;
  double divb_max_interior;  /* max over the corners flux-CT constrains (x1 1..n1-1, x2 2..n2-2) */
} hgpu_diag;
int hgpu_diagnostics(hgpu_ctx *ctx, hgpu_diag *out);

/* The conserved state after the last full step (the reference's unew, with
   gdet; defined on active zones), host layout as the primitives: with the
   primitives it is what the reference's restart dump holds
   (rdump_content, restart.c:244-250). */
int hgpu_download_conserved(hgpu_ctx *ctx, double *unew);

/* The pflag slots FLAGBSQORHO and FLAGBSQOU (global.h:867-868) that
   pre_fixup -> get_bsqflags (fixup.c:25, :1751) sets at the start of each RK
   stage (step_ch.c:117-120) from b^2/rho and b^2/u of the stage's input
   state: flags[z][0] = FLAGBSQORHO, flags[z][1] = FLAGBSQOU (0, 1 or 2) per
   zone of the host zone layout, as the last stage of the last step left
   them (0 before the first step).  Not produced for batches of 1D problems. */
int hgpu_download_bsqflags(hgpu_ctx *ctx, int *flags);

/* Coordinate data of the Bondi-integral boundaries (HGPU_BC_BONDI*), which
   the device does not derive from the metric it holds: table[s][q][j][49]
   for side s (0: x1 inner, zones i = 0, -1, ..., -ng; 1: x1 outer,
   i = n1-1, n1, ..., n1-1+ng; q = 0 is the active edge zone), active j
   (the metric does not depend on x3), each at the zone centre: the
   Boyer-Lindquist radius r (coord + bl_coord, coord.c:1195, 389), dx/dx'
   [4][4] (dxdxprim, coord.c:596), its inverse [4][4] (matrix_inverse,
   metric.c:1346) and the Kerr-Schild metric g_{mu nu} [4][4]
   (gcov_func(0, KSCOORDS), metric.c:11).  Copied; a captured step graph is
   dropped (it held the previous table). */
int hgpu_set_bondi_boundaries(hgpu_ctx *ctx, const double *table);

/* Failure and floor counters per zone (the reference's failfloorcount,
   fixup.c:206, incremented by diag_fixup): counts[z*9 + c], zones in the
   primitives' host layout, c the categories COUNTUTOPRIMFAILCONV 0,
   COUNTFLOORACT 1, COUNTLIMITGAMMAACT 2, COUNTINFLOWACT 3,
   COUNTUTOPRIMFAILRHONEG 4, COUNTUTOPRIMFAILUNEG 5, COUNTUTOPRIMFAILRHOUNEG 6,
   COUNTGAMMAPERC 7, COUNTUPERC 8 (global.h:769-779): the number of times
   since hgpu_create / hgpu_reconfigure or the last clearing download
   (uploading a state does not reset them: a host that uploads before every
   step, as the drop-in step_ch does, accumulates them over its steps) that
   fixup1zone
   floored the zone or limited its Lorentz factor (fixup.c:408, 443, 1913),
   that fixup_utoprim limited the averaged state's Lorentz factor
   (fixup.c:1326) and that it reset a failure of each type to fixed
   (fixup.c:1340-1428).  Active zones only: the inflow checks of the
   boundaries (COUNTINFLOWACT) and the limit_gamma there count ghost zones,
   which no output of the reference reads, and are not kept.  clear != 0
   zeroes the counters after the copy. */
int hgpu_download_failfloorcount(hgpu_ctx *ctx, long long *counts, int clear);

/* Set the conserved state unew from the host (same layout), as the
   reference's restart reads unew (restart.c:256-270).  A HGPU_ENOFINITEVOLUME
   context evolves it: the next step starts from it, as the reference copies
   it to uinitial (initbase.c:155-160), and hgpu_upload_state of such a
   context sets it to U(p) in every zone, as init_conservatives/pi2Uavg does
   (initbase.c:146-153, 1833).  Any other context only reports it through
   hgpu_download_conserved until its next step, which rewrites unew without
   reading it (advance_standard, advance.c:58-240).  Not for batches. */
int hgpu_upload_conserved(hgpu_ctx *ctx, const double *unew);

/* The reference's restart dump (restart_write restart.c:206-235, body
   rdump_content :240-245 through dump_gen dumpgen.c:245-283 and myfwrite
   mpi_fileio.c:2073-2150, one process): `header` (header_bytes bytes: the
   caller's write_restart_header output, restart.c:640-800, which holds host
   state such as t, nstep, the options and the cumulative diagnostics; may
   be empty) and then every active zone, k outermost and i fastest
   (DUMPGENLOOP, global.h:1411-1432), as p[0..7] followed by unew[0..7] (the
   context's state after its last step): binary = 0 writes each value as
   "%21.15g " and a newline after each zone (TEXTOUTPUT, the reference's
   format without MPI, initbase.c:237), binary = 1 the 16 doubles of each
   zone in host byte order (BINARYOUTPUT).  HGPU_E_INVALID with a message on
   an I/O error.  Not for batches. */
int hgpu_write_rdump(hgpu_ctx *ctx, const char *path, const void *header, size_t header_bytes, int binary);

/* Reads such a dump (its first header_bytes bytes skipped) into the
   context: the primitives and unew of the active zones, then bound_prim for
   the ghost zones, as restart_init does after restart_read (restart.c:1-150);
   t and dt are the caller's (the header's t; the reference then resets dt
   with set_dt).  pflag is cleared.  HGPU_E_INVALID with a message on a
   missing, short or malformed file. */
int hgpu_read_rdump(hgpu_ctx *ctx, const char *path, size_t header_bytes, int binary, double t, double dt);

/* ---- Domain split along x3 ----------------------------------------------
   The reference decomposes the grid over MPI ranks (ncpux1..3,
   mpi_init.c:226) and fills each rank's ghost zones from its neighbours in
   bound_prim and bound_pflag (bound_mpi boundmpi.c:6-180, bound_mpi_int
   boundmpiint.c:4), and takes the minimum of dt over ranks (mpifmin,
   step_ch.c:243, mpi_fileio.c:1905).  Here a context holds one rank's
   n3 planes of an x3-periodic domain (n3 > 1) and one step runs as phases,
   with the plane exchange and the dt minimum done by the caller between
   them (NCCL send/recv and all-reduce between GPUs, device copies between
   contexts on one GPU):
     hgpu_stats_clear
     for each stage s of TIMEORDER:
       hgpu_stage_advance(s)   advance + bound_prim + bound_pflag
       exchange: hgpu_halo_pack(s, side, 1) -> neighbour -> hgpu_halo_unpack
       hgpu_stage_fixup(s)     post_fixup + bound_prim
       exchange: the same with with_pflag = 0
     ndt: hgpu_ndt_pack -> elementwise minimum over ranks -> hgpu_ndt_unpack
     hgpu_step_end(1); hgpu_stats_read
   The minimum is taken per direction before the three are combined, so a
   split run reproduces the whole-domain dt (the reference combines per rank
   first, step_ch.c:243).  Start-up dt: hgpu_dt_probe, the ndt exchange,
   hgpu_step_end(0).  All calls are asynchronous on the context's stream
   (hgpu_stream) except hgpu_stats_read.
   Halo buffers live in device memory; side 0 is the lower x3 face, 1 the
   upper.  Pack side 1 of rank r is unpacked as side 0 of rank r+1 (mod P),
   and pack side 0 of rank r as side 1 of rank r-1.  stage -1 names the
   state itself (the exchange after an upload, before the first step). */
int hgpu_halo_bytes(hgpu_ctx *ctx, size_t *bytes);
int hgpu_halo_pack(hgpu_ctx *ctx, int stage, int side, int with_pflag, void *dev_buf);
int hgpu_halo_unpack(hgpu_ctx *ctx, int stage, int side, int with_pflag, const void *dev_buf);
int hgpu_stats_clear(hgpu_ctx *ctx);
int hgpu_stats_read(hgpu_ctx *ctx, hgpu_stats *stats);
int hgpu_stage_advance(hgpu_ctx *ctx, int stage);
int hgpu_stage_fixup(hgpu_ctx *ctx, int stage);
int hgpu_dt_probe(hgpu_ctx *ctx);
int hgpu_step_end(hgpu_ctx *ctx, int advance_time);
int hgpu_ndt_pack(hgpu_ctx *ctx, unsigned long long *dev3);
int hgpu_ndt_unpack(hgpu_ctx *ctx, const unsigned long long *dev3);
int hgpu_stream(hgpu_ctx *ctx, void **stream);

/* Device bytes a context of this configuration allocates (0 if invalid). */
size_t hgpu_context_bytes(const hgpu_config *cfg);

/* Serving loop (no counterpart in the reference, which runs one problem per
   process).  Solves arrive at any time (hgpu_server_submit copies their
   inputs); hgpu_server_poll is the request loop: it admits pending solves
   first-fit in arrival order while their device footprint fits
   max_device_bytes and fewer than max_active run, keeps steps_per_chunk
   time steps in flight per running solve on its own CUDA stream (the work
   of all running solves overlaps on the device), retires a solve when its t
   has reached tf (cfg->tf is replaced by tf) and frees its memory for the
   next admission.  Poll never blocks on running work.  A solve's result is
   what running it alone gives.  Times are host wall-clock: queue_ms from
   submit to admission, run_ms from admission to retirement. */
typedef struct hgpu_server hgpu_server;
int hgpu_server_create(size_t max_device_bytes, int max_active, int steps_per_chunk, hgpu_server **out);
void hgpu_server_destroy(hgpu_server *srv);
int hgpu_server_submit(hgpu_server *srv, const hgpu_config *cfg, const double *gcov, const double *gcon,
                       const double *gcovpert, const double *gdet, const double *conn, const double *floors,
                       const double *p, double tf, long long *id);
/* The same without copying: the server reads the caller's arrays when it
   admits the solve, so they must stay valid and unchanged until
   hgpu_server_poll no longer counts the solve as pending. */
int hgpu_server_submit_borrowed(hgpu_server *srv, const hgpu_config *cfg, const double *gcov, const double *gcon,
                                const double *gcovpert, const double *gdet, const double *conn,
                                const double *floors, const double *p, double tf, long long *id);
int hgpu_server_poll(hgpu_server *srv, int *pending, int *active, int *finished);
/* result of a finished solve (HGPU_E_INVALID while it runs); arrays in the layouts above */
int hgpu_server_result(hgpu_server *srv, long long id, double *p, int *pflag, double *t, long long *steps,
                       double *queue_ms, double *run_ms);
int hgpu_server_release(hgpu_server *srv, long long id);

/* Raw device pointers of the resident state for callers that keep data on
   the GPU (e.g. a graph-captured serving loop): primitive planes
   [8][nt1][nt2][nt3] of p (which=0) or pk (which=1). */
int hgpu_device_prims(hgpu_ctx *ctx, int which, double **dptr);

/* Set dt from the face wave speeds of the current primitives: the ndt of
   advance.c:231 evaluated on p (the reference's init uses set_dt,
   advance.c:957, with zone-centre speeds).  *dt (may be NULL) receives it. */
int hgpu_init_dt(hgpu_ctx *ctx, double *dt);

/* step_ch for nsteps with CUDA events recorded on the context's stream
   around the launches; *ms receives the device time. */
int hgpu_step_ch_timed(hgpu_ctx *ctx, int nsteps, float *ms, hgpu_stats *stats);

/* Per-kernel CUDA-event timing (off by default).  While on, every launch
   is bracketed by events on the launching stream.  hgpu_kernel_times fills
   up to n entries: names[i] (static strings), ms[i] total device time and
   launches[i]; returns the number of kernel kinds or a negative error. */
int hgpu_set_profiling(hgpu_ctx *ctx, int on);
int hgpu_kernel_times(hgpu_ctx *ctx, const char **names, double *ms, long long *launches, int n);

/* Number of kernels this context has launched since creation. */
long long hgpu_launch_count(hgpu_ctx *ctx);

/* Page-locked host buffers for fast host<->device copies. */
int hgpu_alloc_pinned(size_t bytes, void **ptr);
int hgpu_free_pinned(void *ptr);

/* FP64 issue-rate probe of the current device: separate DMUL and DADD
   (no FMA), the instruction mix of the bit-identical FP64 path.  Returns the
   measured rate in TFLOP/s (one multiply or add = one flop). */
int hgpu_fp64_peak(double *tflops);

/* Synchronise the context's stream and report pending CUDA errors. */
int hgpu_sync(hgpu_ctx *ctx);

/* Human-readable text of the last error on this thread. */
const char *hgpu_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
